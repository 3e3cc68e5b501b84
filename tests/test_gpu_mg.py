"""Multigrid-preconditioned solves (PG_PREC_MG) against the reference's
solution and the oracle's direct solves: FP64 and FP32 V-cycles, CG and
GMRES, linear and cohesive Newton."""
import numpy as np
import pytest

import oracle
import pigfem_assignment_b200.problem as pb
from helpers import golden, rve_from_golden
from pigfem_assignment_b200 import _lib
from pigfem_assignment_b200.rve import RVE, config0, config1, scaled

pytestmark = pytest.mark.gpu

U_TOL = 1e-8


@pytest.mark.parametrize("precision", [_lib.PG_PRECISION_FP64, _lib.PG_PRECISION_MIXED])
def test_mg_cg_matches_reference_solution(precision):
    g = golden("linear_cfg0.npz")
    rve = rve_from_golden(g)
    prob = pb.ProblemLinearElasticity(rve)
    prob.init()
    e = prob.mesh.export()
    prob.get_solver().configure(precision=precision, precond=_lib.PG_PREC_MG, rtol=1e-12)
    st = prob.solve_problem()
    assert st.status == 0 and st.rel_residual <= 4e-12, (st.status, st.rel_residual)
    # a V-cycle preconditioner: tens of iterations, not the hundreds of block Jacobi
    assert st.iterations <= 120, st.iterations
    u = prob.get_solution()
    ur = np.empty(u.size)
    ur[e["ref_dof"]] = u
    uref = np.concatenate([g["U.f"], g["U.p"]])
    assert np.linalg.norm(ur - uref) / np.linalg.norm(uref) <= U_TOL
    prob.ctx.close()


@pytest.mark.parametrize("nx", [20, 96, 128])
def test_mg_cg_on_uneven_grids_matches_direct_solve(nx):
    # 20 -> 10 -> 5 -> 3 and 96 -> 48 -> ... -> 3: odd coarse sizes use the
    # one-cell end spacing of the coarse grid
    rve = scaled(config1(), nx)
    prob = pb.ProblemLinearElasticity(rve)
    prob.init()
    e = prob.mesh.export()
    prob.get_solver().configure(precond=_lib.PG_PREC_MG, rtol=1e-12)
    st = prob.solve_problem()
    assert st.status == 0, (st.status, st.rel_residual)
    Ko, _, _ = oracle.from_product(e, pb.template_table(), rve).assemble()
    uo = oracle.solve_linear(Ko, e["fixed"], e["ubar"])
    u = prob.get_solution()
    assert np.linalg.norm(u - uo) / np.linalg.norm(uo) <= U_TOL
    prob.ctx.close()


def test_mg_gmres_converges_to_the_cg_solution():
    rve = config0()
    sols = []
    for krylov in (_lib.PG_KRYLOV_CG, _lib.PG_KRYLOV_GMRES):
        prob = pb.ProblemLinearElasticity(rve)
        prob.init()
        s = prob.get_solver()
        s.configure(precond=_lib.PG_PREC_MG, rtol=1e-11)
        s.cfg.krylov = krylov
        s.cfg.gmres_restart = 60
        st = prob.solve_problem()
        assert st.status == 0, (krylov, st.status, st.rel_residual)
        sols.append(prob.get_solution())
        prob.ctx.close()
    assert np.linalg.norm(sols[0] - sols[1]) / np.linalg.norm(sols[0]) <= 1e-8


@pytest.mark.parametrize("precision", [_lib.PG_PRECISION_FP64, _lib.PG_PRECISION_MIXED])
def test_mg_newton_follows_reference_trajectory(precision):
    g = golden("cohesive_16x16.npz")
    rve = rve_from_golden(g, cohesive=True)
    nsteps = int(g["cfg.nsteps"][0])
    dt = float(g["cfg.dt"][0])
    rve.strain = float(g["cfg.strain_per_step"][0]) * nsteps
    prob = pb.ProblemNonlinearStructural(rve)
    prob.init()
    prob.configure(rtol=1e-10, precision=precision, precond=_lib.PG_PREC_MG)
    e = prob.mesh.export()
    ref = e["ref_dof"]
    for k in range(1, nsteps + 1):
        st = prob.load_step(k / nsteps, dt)
        assert st.reason > 0, (k, st.reason)
        prob.commit()
        u = prob.get_solution()
        uref = np.concatenate([g[f"step{k}.U.f"], g[f"step{k}.U.p"]])[ref]
        assert np.linalg.norm(u - uref) / np.linalg.norm(uref) <= 1e-6
    prob.ctx.close()


def test_mg_newton_bilinear_matches_oracle_newton():
    rve = RVE(nx=24, ny=24, inclusions=[(0.5, 0.5, 0.3, 1)], cohesive=True, coh_law=1,
              coh_params=(30.0, 1.0, 1.0e6, 1.0), strain=0.004)
    prob = pb.ProblemNonlinearStructural(rve)
    prob.init()
    prob.configure(rtol=1e-11, precision=_lib.PG_PRECISION_MIXED, precond=_lib.PG_PREC_MG)
    e = prob.mesh.export()
    om = oracle.from_product(e, pb.template_table(), rve)
    U_o = np.zeros(prob.mesh.info["n_dof"])
    isv_o = np.zeros(prob.mesh.info["n_cohesive_qp"])
    for k in range(1, 5):
        st = prob.load_step(k / 4, 0.25)
        assert st.reason > 0, (k, st.reason)
        prob.commit()
        U_o, isv_o, its, r0, rn = oracle.newton_load_step(om, U_o, e["fixed"], e["ubar"], k / 4, 0.25, isv_o,
                                                          rtol=1e-11)
        u = prob.get_solution()
        assert np.linalg.norm(u - U_o) / np.linalg.norm(U_o) <= 1e-7
    prob.ctx.close()
