"""Pins the CPU oracle (oracle/igfem_oracle.c) to the reference's own outputs.

The golden fixtures were produced by running the reference itself (built
from its sources, oracle/Makefile.ref) through its Problem API
(tests/golden/make_golden.py).
"""
import numpy as np
import pytest
import scipy.sparse.linalg as sla

import oracle
from helpers import golden, permute_to_ref, ref_full_K, rel_fro

LINEAR = ["linear_8x8.npz", "linear_cfg0.npz", "linear_3inc.npz"]


@pytest.mark.parametrize("name", LINEAR)
def test_oracle_K_matches_reference(name):
    g = golden(name)
    om = oracle.from_reference(g)
    K, _, _ = om.assemble()
    err = rel_fro(permute_to_ref(K, om.ref_dof), ref_full_K(g))
    # FP64 path tolerance: relative Frobenius error <= 1e-12
    assert err <= 1e-12, err


@pytest.mark.parametrize("name", LINEAR)
def test_oracle_solution_matches_reference(name):
    g = golden(name)
    om = oracle.from_reference(g)
    K, _, _ = om.assemble()
    n = K.shape[0]
    nf = om.n_free
    inv = np.empty(n, np.int64)
    inv[om.ref_dof] = np.arange(n)
    fixed = np.zeros(n, bool)
    fixed[inv[nf:]] = True
    ubar = np.zeros(n)
    ubar[inv[nf:]] = g["U.p"]
    u = oracle.solve_linear(K, fixed, ubar)
    uref = np.concatenate([g["U.f"], g["U.p"]])
    # displacement relative error target <= 1e-8 (both are direct solves)
    assert np.linalg.norm(u[inv] - uref) / np.linalg.norm(uref) <= 1e-8


def test_oracle_cohesive_history_matches_reference():
    g = golden("cohesive_16x16.npz")
    coh = tuple(float(v) for v in g["cfg.coh"])
    om = oracle.from_reference(g, coh_law=0, coh_p=coh)
    n = 2 * om.n_nodes
    inv = np.empty(n, np.int64)
    inv[om.ref_dof] = np.arange(n)
    dt = float(g["cfg.dt"][0])
    isv_c = np.zeros(om.n_coh_qp)
    for k in range(1, int(g["cfg.nsteps"][0]) + 1):
        U = np.zeros(n)
        U[inv] = np.concatenate([g[f"step{k}.U.f"], g[f"step{k}.U.p"]])
        _, f, isv_t = om.assemble(u=U, dt=dt, isv_c=isv_c, want_K=False, want_f=True)
        pref = np.concatenate([g[f"step{k}.Pint.f"], g[f"step{k}.Pint.p"]])
        assert np.linalg.norm(f[inv] - pref) / np.linalg.norm(pref) <= 1e-11
        np.testing.assert_allclose(isv_t, g[f"step{k}.isv.delta_max"], rtol=1e-12, atol=0)
        isv_c = g[f"step{k}.isv.delta_max"]


def test_oracle_patch_test_uniform_strain():
    """Homogeneous material, affine displacement: interior residual vanishes
    (the reference's Analytical_x_tension patch test, Tests/IGFEM_test8.cpp:144-162)."""
    import pigfem_assignment_b200.problem as pb
    from pigfem_assignment_b200.rve import RVE
    rve = RVE(nx=6, ny=5, inclusions=[], strain=0.01)
    m = pb.Mesh(rve)
    e = m.export()
    om = oracle.from_product(e, pb.template_table(), rve)
    K, _, _ = om.assemble()
    xy = e["xy"]
    u = np.zeros(K.shape[0])
    u[0::2] = 0.01 * xy[:, 0] - 0.003 * xy[:, 1]
    u[1::2] = 0.002 * xy[:, 0] + 0.004 * xy[:, 1]
    r = K @ u
    bnd = (np.isclose(xy[:, 0], 0) | np.isclose(xy[:, 0], 1) | np.isclose(xy[:, 1], 0) | np.isclose(xy[:, 1], 1))
    interior = np.repeat(~bnd, 2)
    assert np.abs(r[interior]).max() <= 1e-9 * np.abs(r).max()


def test_oracle_tri3_element_known_answer():
    """K_e of the unit right triangle, plane strain: closed form A * B^T D B."""
    E, nu = 210.0, 0.3
    Ke = oracle.tri3_K([0, 0, 1, 0, 0, 1], E, nu)
    coef = E / ((1 + nu) * (1 - 2 * nu))
    D = coef * np.array([[1 - nu, nu, 0], [nu, 1 - nu, 0], [0, 0, (1 - 2 * nu) / 2]])
    B = np.array([[-1, 0, 1, 0, 0, 0], [0, -1, 0, 0, 0, 1], [-1, -1, 0, 1, 1, 0]], float)
    np.testing.assert_allclose(Ke, 0.5 * B.T @ D @ B, rtol=1e-13, atol=1e-12)
    # symmetric, rigid-body modes in the null space
    np.testing.assert_allclose(Ke, Ke.T, atol=1e-12)
    for mode in ([1, 0, 1, 0, 1, 0], [0, 1, 0, 1, 0, 1], [0, 0, 0, 1, -1, 0]):
        assert np.abs(Ke @ np.array(mode, float)).max() <= 1e-11


def test_op_cohesive_law_finite_difference_tangent():
    """The OP tangent is the derivative of the traction (loading branch)."""
    p = (10.0, 1.5e-4, 1.0, 0.5)
    for delta in ([2e-5, 8e-5], [-3e-5, 2e-4], [1e-4, -5e-5]):
        t, D, _ = oracle.cohesive_law(0, p, 0.1, 0.0, np.array(delta))
        h = 1e-10
        for k in range(2):
            dp = np.array(delta, float)
            dp[k] += h
            tp, _, _ = oracle.cohesive_law(0, p, 0.1, 0.0, dp)
            dm = np.array(delta, float)
            dm[k] -= h
            tm, _, _ = oracle.cohesive_law(0, p, 0.1, 0.0, dm)
            np.testing.assert_allclose((tp - tm) / (2 * h), D[:, k], rtol=1e-5, atol=1e-3)


def test_bilinear_law_envelope():
    """Bilinear law: elastic up to sigma_c at delta_0 = sigma_c/K_p, linear
    softening to zero at delta_f = 2 G_c / sigma_c, unloading to the origin."""
    sc, Gc, Kp = 30.0, 0.01, 1.0e6
    p = (sc, Gc, Kp, 1.0)
    d0, df = sc / Kp, 2 * Gc / sc
    t, D, dm = oracle.cohesive_law(1, p, 0.02, 0.0, np.array([0.0, 0.5 * d0]))
    assert abs(t[1] - Kp * 0.5 * d0) <= 1e-9 * sc and abs(dm - 0.5 * d0) < 1e-20
    t, D, dm = oracle.cohesive_law(1, p, 0.02, 0.0, np.array([0.0, 0.5 * (d0 + df)]))
    assert abs(t[1] - 0.5 * sc) <= 1e-9 * sc
    t, D, dm = oracle.cohesive_law(1, p, 0.02, 0.0, np.array([0.0, 1.5 * df]))
    assert abs(t[1]) <= 1e-12
    # unloading from delta_max back towards zero: secant to the origin
    dmax = 0.5 * (d0 + df)
    t, D, dm2 = oracle.cohesive_law(1, p, 0.02, dmax, np.array([0.0, 0.25 * dmax]))
    assert dm2 == dmax and abs(t[1] - 0.5 * sc * 0.25) <= 1e-9 * sc
    # compression: penalty
    t, D, _ = oracle.cohesive_law(1, p, 0.02, 0.0, np.array([0.0, -1e-6]))
    assert abs(t[1] + Kp * 1e-6) <= 1e-9


def test_bilinear_law_viscous_regularisation():
    """eta adds eta (delta_eff - delta_max) / dt to the loading traction and
    eta / dt to its slope; the tangent stays the derivative of the traction."""
    sc, Gc, Kp, eta, dt = 30.0, 0.01, 1.0e6, 500.0, 0.02
    d0 = sc / Kp
    dmax = 0.8 * d0
    delta = np.array([0.0, 2.0 * d0])
    t0, _, _ = oracle.cohesive_law(1, (sc, Gc, Kp, 1.0, 0.0), dt, dmax, delta)
    t1, D1, dm = oracle.cohesive_law(1, (sc, Gc, Kp, 1.0, eta), dt, dmax, delta)
    assert abs((t1[1] - t0[1]) - eta * (2.0 * d0 - dmax) / dt) <= 1e-9 * sc
    assert dm == 2.0 * d0
    # unloading is rate independent
    tu0, _, _ = oracle.cohesive_law(1, (sc, Gc, Kp, 1.0, 0.0), dt, 3.0 * d0, delta)
    tu1, _, _ = oracle.cohesive_law(1, (sc, Gc, Kp, 1.0, eta), dt, 3.0 * d0, delta)
    assert np.array_equal(tu0, tu1)
    # mixed-mode loading: central differences of the traction
    delta = np.array([1.0e-5, 5.0e-5])
    _, D, _ = oracle.cohesive_law(1, (sc, Gc, Kp, 1.0, eta), dt, 2.0e-5, delta)
    h = 1e-12
    for k in range(2):
        dp, dm_ = delta.copy(), delta.copy()
        dp[k] += h
        dm_[k] -= h
        tp, _, _ = oracle.cohesive_law(1, (sc, Gc, Kp, 1.0, eta), dt, 2.0e-5, dp)
        tm, _, _ = oracle.cohesive_law(1, (sc, Gc, Kp, 1.0, eta), dt, 2.0e-5, dm_)
        np.testing.assert_allclose((tp - tm) / (2 * h), D[:, k], rtol=1e-5, atol=1e-3 * np.abs(D).max())
