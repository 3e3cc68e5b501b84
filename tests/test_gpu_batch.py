"""Batches of independent RVEs of uneven size: one assembly launch per kernel
kind for all of them, per-RVE CG (block Jacobi or the union multigrid
cycle), each RVE's stiffness and displacement against the oracle."""
import ctypes as C

import numpy as np
import pytest

import oracle
import pigfem_assignment_b200.problem as pb
from helpers import bsr_to_csr, rel_fro
from pigfem_assignment_b200 import _lib
from pigfem_assignment_b200.rve import RVE, rsa_circles

pytestmark = pytest.mark.gpu

K_TOL = 1e-12
U_TOL = 1e-8


def uneven_rves():
    out = []
    for k, (side, n_inc, E_inc) in enumerate([(16, 1, 70000.0), (24, 3, 20000.0), (40, 5, 45000.0), (20, 2, 100000.0),
                                              (48, 8, 30000.0), (32, 4, 85000.0)]):
        circ = rsa_circles(1000 + k, n_inc, 0.05, 0.15, 0.03)
        out.append(RVE(nx=side, ny=side, inclusions=[(x, y, r, 1) for x, y, r in circ],
                       materials=[(3000.0, 0.35), (E_inc, 0.2)], strain=0.01, seed=1000 + k))
    return out


class Batch:
    def __init__(self, rves):
        self.meshes = [pb.Mesh(r) for r in rves]
        arr = (C.c_void_p * len(rves))(*[m.handle.value for m in self.meshes])
        h = C.c_void_p()
        _lib.check(_lib.lib.pg_batch_create(arr, len(rves), 0, C.byref(h)), "pg_batch_create")
        self.h = h
        self.ctx = _lib.lib.pg_batch_context(h)
        n = len(rves)
        self.noff = np.zeros(n + 1, np.int32)
        self.depth = np.zeros(n, np.int32)
        _lib.check(_lib.lib.pg_batch_info(h, _lib.iptr(self.noff), None, _lib.iptr(self.depth)))

    def close(self):
        _lib.lib.pg_batch_destroy(self.h)


def test_batch_assembly_matches_each_rve():
    rves = uneven_rves()
    b = Batch(rves)
    _lib.check(_lib.lib.pg_assemble_linear(b.ctx, None))
    _lib.check(_lib.lib.pg_ctx_sync(b.ctx))
    exports = [m.export() for m in b.meshes]
    nblk = sum(int(e["row_ptr"][-1]) for e in exports)
    K = np.zeros(4 * nblk)
    _lib.check(_lib.lib.pg_get_matrix(b.ctx, _lib.dptr(K)))
    boff = 0
    for r, (rve, e) in enumerate(zip(rves, exports)):
        nb_r = int(e["row_ptr"][-1])
        Kr = bsr_to_csr(e["row_ptr"], e["col"], K[4 * boff:4 * (boff + nb_r)])
        boff += nb_r
        Ko, _, _ = oracle.from_product(e, pb.template_table(), rve).assemble()
        assert rel_fro(Kr, Ko) <= K_TOL, r
    b.close()


@pytest.mark.parametrize("precond,precision", [(_lib.PG_PREC_MG, _lib.PG_PRECISION_FP64),
                                               (_lib.PG_PREC_MG, _lib.PG_PRECISION_MIXED),
                                               (_lib.PG_PREC_BLOCK_JACOBI, _lib.PG_PRECISION_FP64)])
def test_batch_solve_matches_direct_solve_per_rve(precond, precision):
    rves = uneven_rves()
    b = Batch(rves)
    assert len(set(b.depth.tolist())) > 1  # the batch mixes hierarchy depths
    cfg = _lib.SolverCfg()
    _lib.lib.pg_solver_cfg_default(C.byref(cfg))
    cfg.precond, cfg.precision, cfg.rtol, cfg.max_iter = precond, precision, 1e-12, 100000
    per = (_lib.SolveStats * len(rves))()
    tot = _lib.SolveStats()
    _lib.check(_lib.lib.pg_batch_solve(b.h, C.byref(cfg), per, C.byref(tot)), "pg_batch_solve")
    its = [per[r].iterations for r in range(len(rves))]
    assert len(set(its)) > 1  # every RVE stops on its own
    for r, (rve, m) in enumerate(zip(rves, b.meshes)):
        assert per[r].status == 0 and per[r].rel_residual <= 4e-12, (r, per[r].rel_residual)
        e = m.export()
        u = np.zeros(2 * m.info["n_nodes"])
        _lib.check(_lib.lib.pg_batch_get_solution(b.h, r, _lib.dptr(u)))
        Ko, _, _ = oracle.from_product(e, pb.template_table(), rve).assemble()
        uo = oracle.solve_linear(Ko, e["fixed"], e["ubar"])
        assert np.linalg.norm(u - uo) / np.linalg.norm(uo) <= U_TOL, r
    b.close()
