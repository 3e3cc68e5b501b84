"""GPU Newton load stepping against the reference's own cohesive trajectory
(Ortiz-Pandolfi law) and against the oracle's Newton (bilinear law)."""
import numpy as np
import pytest

import oracle
import pigfem_assignment_b200.problem as pb
from helpers import golden, rve_from_golden
from pigfem_assignment_b200 import _lib
from pigfem_assignment_b200.rve import RVE

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [_lib.PG_PRECISION_FP64, _lib.PG_PRECISION_MIXED])
def test_gpu_newton_follows_reference_trajectory(precision):
    """Four load steps (dt = 0.1, 0.25% strain each) from zero state: the
    converged displacements and delta_max after every step match the
    reference's (its SNES Newton, run to rtol 1e-12 for the fixture) within
    the displacement bound 1e-8, delta_max within 1e-10."""
    g = golden("cohesive_16x16.npz")
    rve = rve_from_golden(g, cohesive=True)
    nsteps = int(g["cfg.nsteps"][0])
    dt = float(g["cfg.dt"][0])
    rve.strain = float(g["cfg.strain_per_step"][0]) * nsteps
    prob = pb.ProblemNonlinearStructural(rve)
    prob.init()
    prob.configure(rtol=1e-12, stol=0.0, precision=precision)
    e = prob.mesh.export()
    ref = e["ref_dof"]
    for k in range(1, nsteps + 1):
        st = prob.load_step(k / nsteps, dt)
        assert st.reason > 0, st.reason
        prob.commit()
        u = prob.get_solution()
        uref = np.concatenate([g[f"step{k}.U.f"], g[f"step{k}.U.p"]])[ref]
        assert np.linalg.norm(u - uref) / np.linalg.norm(uref) <= 1e-8
        np.testing.assert_allclose(prob.ctx.isv(committed=True), g[f"step{k}.isv.delta_max"], rtol=1e-10, atol=1e-18)
    prob.ctx.close()


def test_gpu_newton_bilinear_matches_oracle_newton():
    # G_c = 1 N/mm keeps the softening branch (slope sigma_c^2 / (2 G_c)) below
    # the surrounding matrix stiffness, so the equilibrium path is continuous
    # and the oracle's direct-solve Newton converges quadratically; with
    # G_c = 0.01 N/mm this 24x24 interface snaps back in the fourth step and
    # no Newton method converges there.
    rve = RVE(nx=24, ny=24, inclusions=[(0.5, 0.5, 0.3, 1)], cohesive=True, coh_law=1,
              coh_params=(30.0, 1.0, 1.0e6, 1.0), strain=0.004)
    prob = pb.ProblemNonlinearStructural(rve)
    prob.init()
    prob.configure(rtol=1e-11)
    e = prob.mesh.export()
    om = oracle.from_product(e, pb.template_table(), rve)
    nsteps, dt = 4, 0.25
    U_o = np.zeros(prob.mesh.info["n_dof"])
    isv_o = np.zeros(prob.mesh.info["n_cohesive_qp"])
    for k in range(1, nsteps + 1):
        st = prob.load_step(k / nsteps, dt)
        assert st.reason > 0, (k, st.reason, st.newton_its, st.res0, st.res)
        prob.commit()
        U_o, isv_t, its, r0, rn = oracle.newton_load_step(om, U_o, e["fixed"], e["ubar"], k / nsteps, dt, isv_o,
                                                          rtol=1e-11)
        isv_o = isv_t
        u = prob.get_solution()
        assert np.linalg.norm(u - U_o) / np.linalg.norm(U_o) <= 1e-7
        np.testing.assert_allclose(prob.ctx.isv(committed=True), isv_o, rtol=1e-6, atol=1e-13)
    # the interface has opened past the elastic limit somewhere (damage)
    assert isv_o.max() > 30.0 / 1.0e6
    prob.ctx.close()


def test_gpu_solve_nonlinear_driver_records_steps():
    rve = RVE(nx=16, ny=16, inclusions=[(0.5, 0.5, 0.25, 1)], cohesive=True, coh_law=1,
              coh_params=(30.0, 0.01, 1.0e6, 1.0), strain=0.004)
    prob = pb.ProblemNonlinearStructural(rve)
    prob.init()
    prob.configure(n_steps=5, T_final=1.0, predictor=_lib.PG_PREDICT_LINEAR)
    recs = prob.solve_problem()
    assert len(recs) >= 5
    assert all(r.reason > 0 for r in recs)
    assert abs(sum(r.dt for r in recs) - 1.0) < 1e-12
    prob.ctx.close()


@pytest.mark.parametrize("precision", [_lib.PG_PRECISION_FP64, _lib.PG_PRECISION_MIXED])
def test_cohesive_load_stepping_is_bit_reproducible(precision):
    """The Krylov dot products add their block sums in a fixed order, so a
    softening load path -- where rounding differences grow into different
    Newton and Krylov iteration counts -- is the same on every run, bit for
    bit."""
    from pigfem_assignment_b200.rve import config2
    rve = config2(nx=64, n_inc=8)
    rve.coh_params = tuple(rve.coh_params[:4]) + (200.0,)
    runs = []
    for _ in range(2):
        prob = pb.ProblemNonlinearStructural(rve)
        prob.init()
        prob.configure(n_steps=50, T_final=1.0, t_start=0.0, t_stop=0.4, precision=precision,
                       predictor=_lib.PG_PREDICT_LINEAR, precond=_lib.PG_PREC_MG, stol=0.0,
                       rtol_base=_lib.PG_RTOL_BASE_ZEROTH, lin_max_iter=1000)
        recs = prob.solve_problem()
        runs.append((prob.get_solution(), prob.ctx.isv(committed=True),
                     [(r.newton_its, r.krylov_its, r.repeats) for r in recs]))
        prob.ctx.close()
    assert runs[0][2] == runs[1][2]
    assert np.array_equal(runs[0][0], runs[1][0])
    assert np.array_equal(runs[0][1], runs[1][1])
