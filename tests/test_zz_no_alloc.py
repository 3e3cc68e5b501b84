"""pg_pcg_solve_static: the PCG entry point that allocates no device memory
(its Krylov vectors live in a fixed array of the library's device image),
against the context solver pg_solve_linear on the same assembled system.

Collected last on purpose: it must give the same answers whether the shared
scratch array is fresh (test run alone) or holds an earlier call's contents.
"""
import ctypes as C

import numpy as np
import pytest

import pigfem_assignment_b200.problem as pb
from helpers import bsr_to_csr
from pigfem_assignment_b200 import _lib
from pigfem_assignment_b200.rve import config0

U_TOL = 1e-8


def test_static_solve_rejects_sizes_beyond_the_scratch():
    st = _lib.SolveStats()
    rc = _lib.lib.pg_pcg_solve_static(_lib.PG_STATIC_MAX_NODES + 1, None, None, None, None, None, None, 1e-8, 10,
                                      None, C.byref(st))
    assert rc == _lib.PG_ERR_LIMIT
    assert b"exceed" in _lib.lib.pg_last_error()
    # the early return still describes this call in stats
    assert st.status == _lib.PG_ERR_LIMIT and st.iterations == 0


@pytest.mark.gpu
def test_static_solve_matches_context_solver_on_two_calls():
    torch = pytest.importorskip("torch")
    prob = pb.ProblemLinearElasticity(config0())
    prob.init()
    prob.get_solver().configure(rtol=1e-12)
    st_ctx = prob.solve_problem()
    assert st_ctx.status == 0
    U = prob.get_solution()
    e = prob.mesh.export()
    n_nodes = prob.mesh.info["n_nodes"]
    assert n_nodes <= _lib.PG_STATIC_MAX_NODES
    fixed = np.asarray(e["fixed"], bool)
    free = ~fixed
    Kv = prob.ctx.matrix_values()
    # the context solve's right-hand side: b = mask(-K U_p)
    Kc = bsr_to_csr(e["row_ptr"], e["col"], Kv)
    Up = np.where(fixed, e["ubar"], 0.0)
    b = -(Kc @ Up)
    b[fixed] = 0.0

    dev = torch.device("cuda:0")
    row_ptr = torch.as_tensor(np.asarray(e["row_ptr"], np.int32), device=dev)
    col = torch.as_tensor(np.asarray(e["col"], np.int32), device=dev)
    K = torch.as_tensor(Kv, device=dev)
    fx = torch.as_tensor(fixed.astype(np.uint8), device=dev)
    bd = torch.as_tensor(b, device=dev)
    x = torch.empty(2 * n_nodes, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    ref = U[free]
    for call in range(2):
        x.fill_(123.0)  # the entry point must overwrite every value
        torch.cuda.synchronize()
        # the module (and its scratch array) is loaded before the second call:
        # from then on the call must leave the device's free memory unchanged
        free_before = torch.cuda.mem_get_info(dev)[0]
        st = _lib.SolveStats()
        rc = _lib.lib.pg_pcg_solve_static(n_nodes, row_ptr.data_ptr(), col.data_ptr(), K.data_ptr(), fx.data_ptr(),
                                          bd.data_ptr(), x.data_ptr(), 1e-12, 200000, None, C.byref(st))
        torch.cuda.synchronize()
        free_after = torch.cuda.mem_get_info(dev)[0]
        assert rc == 0, (call, rc, _lib.lib.pg_last_error())
        if call == 1:
            assert free_after == free_before, (free_before, free_after)
        assert st.status == 0 and st.rel_residual <= 4e-12, (call, st.rel_residual)
        xh = x.cpu().numpy()
        assert np.all(xh[fixed] == 0.0)
        assert np.linalg.norm(xh[free] - ref) / np.linalg.norm(ref) <= U_TOL, call

    # a free node whose diagonal block is zero: reported as a singular block,
    # with stats describing this call
    Ks = Kv.copy()
    i = int(np.flatnonzero(~fixed.reshape(-1, 2).any(axis=1))[0])
    rp = np.asarray(e["row_ptr"])
    cl = np.asarray(e["col"])
    q = rp[i] + int(np.flatnonzero(cl[rp[i]:rp[i + 1]] == i)[0])
    Ks[4 * q:4 * q + 4] = 0.0
    K.copy_(torch.as_tensor(Ks, device=dev))
    st = _lib.SolveStats()
    st.status = 77
    st.iterations = 999
    rc = _lib.lib.pg_pcg_solve_static(n_nodes, row_ptr.data_ptr(), col.data_ptr(), K.data_ptr(), fx.data_ptr(),
                                      bd.data_ptr(), x.data_ptr(), 1e-12, 100, None, C.byref(st))
    assert rc == _lib.PG_ERR_BREAKDOWN and b"singular" in _lib.lib.pg_last_error()
    assert st.status == rc and st.iterations == 0
    prob.ctx.close()
