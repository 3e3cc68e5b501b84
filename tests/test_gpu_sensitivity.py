"""Adjoint shape sensitivity of a bonded RVE's right-edge load: against the
reference's own SensitivityAdjoint + SensitivityRightLoad for every centre
coordinate and radius (golden fixtures made by oracle/ref_driver.cpp; the
reference's values agree with its own re-meshed central differences to
~1e-7), and dC_11/dr_i against central finite differences of C_11 from
re-meshed, re-solved RVEs.

Tolerances: f within 1e-10; df/dd within 1e-8 of the largest derivative of
the fixture (both sides solve to ~1e-12; the analytic element derivative
leaves only rounding)."""
import ctypes as C
import dataclasses

import numpy as np
import pytest

import pigfem_assignment_b200.problem as pb
from pigfem_assignment_b200 import _lib
from helpers import golden, rve_from_golden
from pigfem_assignment_b200.rve import RVE

pytestmark = pytest.mark.gpu


def solver_cfg(rtol=1e-12):
    cfg = _lib.SolverCfg()
    _lib.lib.pg_solver_cfg_default(C.byref(cfg))
    cfg.precond, cfg.rtol, cfg.max_iter = _lib.PG_PREC_MG, rtol, 100000
    return cfg


def c11_and_sens(rve, with_sens=True, h_rel=0.0):
    prob = pb.ProblemLinearElasticity(rve)
    prob.init()
    prob.get_solver().configure(precond=_lib.PG_PREC_MG, rtol=1e-12)
    st = prob.solve_problem()
    assert st.status == 0
    c11 = C.c_double()
    sens = np.zeros(max(1, len(rve.inclusions)))
    ast = _lib.SolveStats()
    _lib.check(_lib.lib.pg_sensitivity_c11(prob.ctx.handle, C.byref(solver_cfg()), h_rel, C.byref(c11),
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


def _solved(rve):
    prob = pb.ProblemLinearElasticity(rve)
    prob.init()
    prob.get_solver().configure(precond=_lib.PG_PREC_MG, rtol=1e-13)
    st = prob.solve_problem()
    assert st.status == 0
    return prob


@pytest.mark.parametrize("name", ["sensitivity_3inc.npz", "sensitivity_close.npz"])
def test_shape_sensitivity_matches_reference_adjoint(name):
    g = golden(name)
    prob = _solved(rve_from_golden(g))
    inc = np.ascontiguousarray(g["cfg.sens_inc"], np.int32)
    kind = np.ascontiguousarray(g["cfg.sens_kind"], np.int32)
    n = inc.size
    f = C.c_double()
    dfdp = np.zeros(n)
    st = _lib.SolveStats()
    _lib.check(_lib.lib.pg_sensitivity_shape(prob.ctx.handle, C.byref(solver_cfg()), n, _lib.iptr(inc), _lib.iptr(kind),
                                             C.byref(f), _lib.dptr(dfdp), C.byref(st)), "pg_sensitivity_shape")
    ref_f = float(g["sens.f"][0])
    ref = g["sens.dfdp"]
    assert abs(f.value - ref_f) <= 1e-10 * abs(ref_f)
    np.testing.assert_allclose(dfdp, ref, rtol=0, atol=1e-8 * np.abs(ref).max())
    # the same radii through the C_11 entry point
    c11 = C.c_double()
    sens = np.zeros(len(prob.rve.inclusions))
    _lib.check(_lib.lib.pg_sensitivity_c11(prob.ctx.handle, C.byref(solver_cfg()), 0.0, C.byref(c11),
                                           _lib.dptr(sens), None))
    strain = prob.rve.strain
    np.testing.assert_allclose(sens * strain, ref[kind == _lib.PG_SHAPE_R], rtol=0, atol=1e-8 * np.abs(ref).max())
    prob.ctx.close()


def test_element_central_difference_converges_to_the_analytic_derivative():
    g = golden("sensitivity_close.npz")
    prob = _solved(rve_from_golden(g))
    out = {}
    for h_rel in (0.0, 1e-4, 1e-5, 1e-6):
        sens = np.zeros(len(prob.rve.inclusions))
        _lib.check(_lib.lib.pg_sensitivity_c11(prob.ctx.handle, C.byref(solver_cfg()), h_rel, None,
                                               _lib.dptr(sens), None))
        out[h_rel] = sens
    err = {h: np.abs(out[h] - out[0.0]).max() / np.abs(out[0.0]).max() for h in (1e-4, 1e-5, 1e-6)}
    print("element central difference vs analytic:", err)
    # the central difference converges to the analytic derivative as h shrinks
    assert err[1e-6] <= 1e-5 and err[1e-6] < err[1e-4]
    prob.ctx.close()


def test_shape_sensitivity_rejects_an_unknown_parameter():
    prob = _solved(RVE(nx=16, ny=16, inclusions=[(0.5, 0.5, 0.25, 1)], strain=0.01))
    for inc, kind in ((1, _lib.PG_SHAPE_R), (0, 3), (-1, _lib.PG_SHAPE_X)):
        i = np.array([inc], np.int32)
        k = np.array([kind], np.int32)
        rc = _lib.lib.pg_sensitivity_shape(prob.ctx.handle, C.byref(solver_cfg()), 1, _lib.iptr(i), _lib.iptr(k),
                                           None, None, None)
        assert rc == _lib.PG_ERR_ARG
    prob.ctx.close()
