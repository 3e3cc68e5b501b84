"""Adjoint shape sensitivity dC_11/dr_i of a bonded RVE against central
finite differences of C_11 from re-meshed, re-solved RVEs."""
import ctypes as C
import dataclasses

import numpy as np
import pytest

import pigfem_assignment_b200.problem as pb
from pigfem_assignment_b200 import _lib
from pigfem_assignment_b200.rve import RVE

pytestmark = pytest.mark.gpu


def solver_cfg(rtol=1e-12):
    cfg = _lib.SolverCfg()
    _lib.lib.pg_solver_cfg_default(C.byref(cfg))
    cfg.precond, cfg.rtol, cfg.max_iter = _lib.PG_PREC_MG, rtol, 100000
    return cfg


def c11_and_sens(rve, with_sens=True):
    prob = pb.ProblemLinearElasticity(rve)
    prob.init()
    prob.get_solver().configure(precond=_lib.PG_PREC_MG, rtol=1e-12)
    st = prob.solve_problem()
    assert st.status == 0
    c11 = C.c_double()
    sens = np.zeros(max(1, len(rve.inclusions)))
    ast = _lib.SolveStats()
    _lib.check(_lib.lib.pg_sensitivity_c11(prob.ctx.handle, C.byref(solver_cfg()), 1e-5, C.byref(c11),
                                           _lib.dptr(sens) if with_sens else None, C.byref(ast)),
               "pg_sensitivity_c11")
    prob.ctx.close()
    return c11.value, sens[:len(rve.inclusions)]


def moved(rve, i, dr):
    inc = list(rve.inclusions)
    x, y, r, m = inc[i]
    inc[i] = (x, y, r + dr, m)
    return dataclasses.replace(rve, inclusions=inc)


def test_adjoint_sensitivity_matches_finite_differences():
    rve = RVE(nx=64, ny=64, inclusions=[(0.3, 0.35, 0.16, 1), (0.7, 0.4, 0.13, 1), (0.45, 0.75, 0.15, 1)],
              strain=0.01)
    c11, sens = c11_and_sens(rve)
    assert c11 > 3000.0  # stiffer than the matrix alone (E 3 GPa, plane strain)
    h = 1e-5
    for i in range(len(rve.inclusions)):
        cp, _ = c11_and_sens(moved(rve, i, +h), with_sens=False)
        cm, _ = c11_and_sens(moved(rve, i, -h), with_sens=False)
        fd = (cp - cm) / (2 * h)
        assert abs(sens[i] - fd) <= 1e-4 * abs(fd) + 1e-6 * abs(c11), (i, sens[i], fd)
        # a stiffer inclusion that grows stiffens the RVE
        assert sens[i] > 0.0
