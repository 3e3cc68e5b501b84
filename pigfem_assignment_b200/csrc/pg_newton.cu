// Newton load stepping for cohesive IGFEM RVEs on the GPU.
//
// Reference:
//   SolverNonlinear::solve (load-step loop, dt control)  src/SolverNonlinear.cpp:111-397, 455-491
//   SolverNonlinearSNES::nonlinearStep / formResidual /
//     formJacobian (SNESNEWTONLS)                        src/SolverNonlinearSNES.cpp:45-241
//   InternalVars::copy_data / copy_data_in               src/InternalVars.cpp:43-85
//
// One load step: prescribed displacements at t_frac * ubar, the free DOFs
// start from the predictor (the reference's zeroth-order predictor keeps the
// last converged U_f), then Newton iterations with a backtracking line
// search on the FP64 residual.  Convergence follows SNES's default tests:
// ||r|| < atol, ||r|| <= rtol ||r_0|| (r_0 = residual of the predictor),
// ||step|| < stol ||U||.  The cohesive trial state is rebuilt from the
// committed state at every assembly and committed when the step converges.
// The residual (f_int) and the tangent are FP64; the linear Newton systems
// are solved in FP64 or in FP32 Krylov + FP64 refinement.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <vector>

#include "pg_internal.cuh"
#include "pg_solve_kernels.cuh"

namespace pgb {

namespace {

inline int nblk(int n) { return (n + kThreads - 1) / kThreads; }

// the learned start falls back to the linear one when its residual exceeds
// the linear start's by more than this factor
constexpr double kLearnedResidualGuard = 8.0;

// res = mask(F_int) (no external force on free DOFs); returns ||res||^2
double newton_residual(Ctx& c, const double* U, double dt, cudaStream_t s) {
    cudaMemsetAsync(c.F, 0, (size_t)c.n_dof * sizeof(double), s);
    launch_assemble(c, U, dt, true, false, s);
    k_mask_copy<<<nblk(c.n_dof), kThreads, 0, s>>>(c.n_dof, c.fixed, c.F, c.res);
    return dev_norm2(c, c.res, c.n_dof, s);
}

}  // namespace

double predictor_residual(Ctx& c, const double* U, double dt, cudaStream_t s) { return newton_residual(c, U, dt, s); }

int newton_load_step(Ctx& c, double t_frac, double dt, const pg_newton_cfg& cfg, pg_step_stats& st, cudaStream_t s,
                     double r_base) {
    const int nd = c.n_dof;
    st = pg_step_stats{};
    st.blend = -1.0;
    st.t_frac = t_frac;
    st.dt = dt;
    cudaEventRecord(c.ev0, s);
    set_prescribed(c, t_frac, s);
    double rr = newton_residual(c, c.U, dt, s);
    const double r0 = std::sqrt(rr);
    st.res0 = r0;
    // rtol is relative to r_base when the caller gives one (the zeroth-order
    // predictor's residual), else to the predictor's own residual (SNES)
    const double rb = r_base > 0.0 ? r_base : r0;
    st.res_base = rb;
    double rnorm = r0;
    int reason = 0;
    if (!(r0 == r0)) reason = -4;
    else if (r0 < cfg.atol) reason = 2;
    else if (r_base > 0.0 && r0 <= cfg.rtol * rb) reason = 3;  // the predictor already meets the target
    pg_solver_cfg lin;
    pg_solver_cfg_default(&lin);
    lin.precision = cfg.precision;
    lin.precond = cfg.precond;
    lin.inclusion_modes = cfg.inclusion_modes;
    lin.deterministic = cfg.deterministic;
    lin.krylov = PG_KRYLOV_CG;
    lin.max_iter = cfg.lin_max_iter;
    lin.inner_rtol = cfg.inner_rtol;
    lin.check_every = 32;
    int it = 0;
    for (; reason == 0 && it < cfg.max_it; ++it) {
        // tangent at U
        launch_assemble(c, c.U, dt, false, true, s);
        // solve K d = -res (forcing term: tighter as Newton converges)
        k_scale_copy<<<nblk(nd), kThreads, 0, s>>>(nd, c.res, c.b, -1.0);
        // never tighter than what lands this iteration on the Newton target:
        // ||r_next|| ~ eta ||r|| once the quadratic term is small
        lin.rtol = std::max(cfg.lin_rtol, std::min(1e-2, 1e-3 * rnorm / r0));
        lin.rtol = std::max(lin.rtol, std::min(1e-2, 0.5 * cfg.rtol * rb / rnorm));
        lin.krylov = PG_KRYLOV_CG;
        pg_solve_stats ls{};
        int rc = krylov_solve(c, lin, ls, s);
        if (rc != PG_OK) return rc;
        st.krylov_its += ls.iterations;
        if (ls.status == PG_ERR_BREAKDOWN) {
            // indefinite tangent (cohesive softening): GMRES with the multigrid
            // cycle when multigrid is selected, else symmetric MINRES (whose
            // preconditioner must stay positive definite: |diag| Jacobi)
            lin.krylov = lin.precond == PG_PREC_MG ? PG_KRYLOV_GMRES : PG_KRYLOV_MINRES;
            pg_solve_stats gs{};
            rc = krylov_solve(c, lin, gs, s);
            if (rc != PG_OK) return rc;
            st.krylov_its += gs.iterations;
            ++st.gmres_fallbacks;
        }
        // backtracking line search on 0.5 ||r||^2 (sufficient decrease 1e-4)
        double lambda = 1.0, rr_t = 0.0;
        bool ok = false;
        for (int bt = 0; bt < 12; ++bt) {
            k_axpy_to<<<nblk(nd), kThreads, 0, s>>>(nd, c.fixed, c.U, c.dx, lambda, c.Ut);
            rr_t = newton_residual(c, c.Ut, dt, s);
            if (rr_t == rr_t && rr_t <= (1.0 - 2.0 * 1e-4 * lambda) * rr) { ok = true; break; }
            lambda *= 0.5;
        }
        if (!ok) { reason = (rr_t == rr_t) ? -6 : -4; break; }
        cudaMemcpyAsync(c.U, c.Ut, (size_t)nd * sizeof(double), cudaMemcpyDeviceToDevice, s);
        rr = rr_t;
        rnorm = std::sqrt(rr);
        const double dn = lambda * std::sqrt(dev_norm2(c, c.dx, nd, s));
        const double un = std::sqrt(dev_norm2(c, c.U, nd, s));
        if (rnorm < cfg.atol) reason = 2;
        else if (rnorm <= cfg.rtol * rb) reason = 3;
        else if (dn < cfg.stol * un) reason = 4;
    }
    if (reason == 0) reason = -5;  // iteration budget exhausted
    st.newton_its = it;
    st.res = rnorm;
    st.reason = reason;
    // the trial state of the last residual evaluation is at the accepted U;
    // the caller commits it when the step is accepted
    cudaEventRecord(c.ev1, s);
    PG_CUDA(cudaEventSynchronize(c.ev1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c.ev0, c.ev1);
    st.seconds = ms * 1e-3;
    return PG_OK;
}

}  // namespace pgb

using namespace pgb;

extern "C" {

void pg_newton_cfg_default(pg_newton_cfg* cfg) {
    if (!cfg) return;
    cfg->n_steps = 50;
    cfg->T_final = 1.0;
    cfg->rtol = 1e-8;
    cfg->atol = 1e-50;
    cfg->stol = 1e-8;
    cfg->max_it = 50;
    cfg->precision = PG_PRECISION_FP64;
    cfg->precond = PG_PREC_BLOCK_JACOBI;
    cfg->lin_rtol = 1e-10;
    cfg->inner_rtol = 1e-3;
    cfg->lin_max_iter = 100000;
    cfg->max_repeat = 20;
    cfg->predictor = PG_PREDICT_ZEROTH;
    cfg->rtol_base = PG_RTOL_BASE_PREDICTOR;
    cfg->inclusion_modes = 0;
    cfg->t_start = 0.0;
    cfg->t_stop = 1.0;
    cfg->deterministic = 1;
}

int pg_newton_load_step(pg_ctx* cx, double t_frac, double dt, const pg_newton_cfg* cfg_in, pg_step_stats* stats) {
    if (!cx) { set_error("null context"); return PG_ERR_ARG; }
    Ctx& c = cx->c;
    cudaSetDevice(c.device);
    pg_newton_cfg cfg;
    if (cfg_in) cfg = *cfg_in;
    else pg_newton_cfg_default(&cfg);
    pg_step_stats st{};
    const int rc = newton_load_step(c, t_frac, dt, cfg, st, c.stream);
    if (stats) *stats = st;
    return rc;
}

// SolverNonlinear::solve: equal load steps dt = T_final / n_steps; a failed
// step is repeated with dt *= 0.25 (at most max_repeat times), a step that
// converged at the first try lets dt grow by 1.5 up to the nominal dt.
int pg_solve_nonlinear(pg_ctx* cx, const pg_newton_cfg* cfg_in, pg_step_stats* per_step, int32_t max_records,
                       int32_t* n_records) {
    if (!cx) { set_error("null context"); return PG_ERR_ARG; }
    Ctx& c = cx->c;
    cudaSetDevice(c.device);
    pg_newton_cfg cfg;
    if (cfg_in) cfg = *cfg_in;
    else pg_newton_cfg_default(&cfg);
    if (cfg.n_steps <= 0 || cfg.T_final <= 0) { set_error("pg_solve_nonlinear: bad step count / T_final"); return PG_ERR_ARG; }
    if (!(cfg.t_start >= 0.0 && cfg.t_start < cfg.t_stop && cfg.t_stop <= 1.0)) {
        set_error("pg_solve_nonlinear: need 0 <= t_start < t_stop <= 1");
        return PG_ERR_ARG;
    }
    cudaStream_t s = c.stream;
    const int nd = c.n_dof;
    const double dt_nom = cfg.T_final / cfg.n_steps;
    const double t_end = cfg.t_stop * cfg.T_final;
    double t = cfg.t_start * cfg.T_final, dt = std::min(dt_nom, t_end - t), dt_prev = dt_nom, dt_prev2 = dt_nom;
    int nrec = 0;
    // the previous converged states for predictors / repeats
    cudaMemcpyAsync(c.Uprev, c.U, (size_t)nd * sizeof(double), cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(c.Uold, c.U, (size_t)nd * sizeof(double), cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(c.Uold2, c.U, (size_t)nd * sizeof(double), cudaMemcpyDeviceToDevice, s);
    if (c.n_coh_qp > 0)
        cudaMemcpyAsync(c.isv_prev, c.isv_c, (size_t)c.n_coh_qp * sizeof(double), cudaMemcpyDeviceToDevice, s);
    while (t < t_end - 1e-12 * cfg.T_final) {
        int repeat = 0;
        bool converged = false;
        pg_step_stats st{};
        // the record of a load step counts every attempt (failed ones included)
        // and its wall time from the predictor to the accepted state
        PG_CUDA(cudaStreamSynchronize(s));
        const auto t_step = std::chrono::steady_clock::now();
        int acc_newton = 0, acc_krylov = 0, acc_fallbacks = 0;
        while (!converged) {
            if (repeat >= cfg.max_repeat) {
                set_error("pg_solve_nonlinear: Newton did not converge within the load-step repeat budget");
                if (n_records) *n_records = nrec;
                return PG_ERR_NOT_CONVERGED;
            }
            ++repeat;
            // U holds the last converged solution here (zeroth-order predictor)
            const double tf = (t + dt) / cfg.T_final;
            double r_base = 0.0;
            if (cfg.rtol_base == PG_RTOL_BASE_ZEROTH) {
                set_prescribed(c, tf, s);
                r_base = std::sqrt(predictor_residual(c, c.U, dt, s));
            }
            int used = PG_PREDICT_ZEROTH;
            double res_lin = -1.0, res_mlp = -1.0, blend = -1.0;
            // the learned start needs two steps of history; before that it is the linear one
            if ((cfg.predictor == PG_PREDICT_LINEAR && nrec > 0) || (cfg.predictor == PG_PREDICT_LEARNED && nrec == 1)) {
                k_extrapolate<<<nblk(nd), kThreads, 0, s>>>(nd, c.fixed, c.U, c.Uold, dt / dt_prev);
                used = PG_PREDICT_LINEAR;
            } else if (cfg.predictor == PG_PREDICT_LEARNED && nrec > 1 && c.mlp) {
                pg_pred_history h{};
                h.U_n = c.Uprev;
                h.U_nm1 = c.Uold;
                h.U_nm2 = c.Uold2;
                h.isv_nm1 = c.n_coh_qp > 0 ? c.isv_prev : nullptr;
                h.dt_n = dt_prev;
                h.dt_nm1 = dt_prev2;
                h.dt = dt;
                h.t_frac = tf;
                h.s_inc = predictor_app(c) * dt / cfg.T_final;
                // candidate 1: linear extrapolation (into Ut)
                cudaMemcpyAsync(c.Ut, c.Uprev, (size_t)nd * sizeof(double), cudaMemcpyDeviceToDevice, s);
                int rc = launch_apply(c, h, nullptr, 0.0, c.Ut, s);
                if (rc) return rc;
                k_apply_dirichlet<<<nblk(nd), kThreads, 0, s>>>(nd, c.fixed, c.ubar, tf, c.Ut);
                res_lin = std::sqrt(predictor_residual(c, c.Ut, dt, s));
                // candidate 2: the network's weighting of the curvature term (into U)
                rc = launch_features(c, h, c.featX, s);
                if (rc) return rc;
                rc = pg_mlp_forward(c.mlp, c.featX, c.n_nodes, c.featY, s);
                if (rc) return rc;
                cudaMemcpyAsync(c.U, c.Uprev, (size_t)nd * sizeof(double), cudaMemcpyDeviceToDevice, s);
                rc = launch_apply(c, h, c.featY, 1.0, c.U, s, &blend);
                if (rc) return rc;
                k_apply_dirichlet<<<nblk(nd), kThreads, 0, s>>>(nd, c.fixed, c.ubar, tf, c.U);
                res_mlp = std::sqrt(predictor_residual(c, c.U, dt, s));
                // the learned start is taken unless its residual is far above the
                // linear one (a start's residual is a poor judge of the Newton
                // work it saves -- the penalty stiffness of the interfaces
                // dominates it -- so only a gross miss falls back)
                if (res_mlp == res_mlp && res_mlp <= kLearnedResidualGuard * res_lin) {
                    used = PG_PREDICT_LEARNED;
                } else {
                    cudaMemcpyAsync(c.U, c.Ut, (size_t)nd * sizeof(double), cudaMemcpyDeviceToDevice, s);
                    used = PG_PREDICT_LINEAR;
                }
            }
            const int rc = newton_load_step(c, tf, dt, cfg, st, s, r_base);
            st.predictor_used = used;
            st.res_linear = res_lin;
            st.res_learned = res_mlp;
            st.blend = blend;
            if (rc != PG_OK) return rc;
            converged = st.reason > 0;
            acc_newton += st.newton_its;
            acc_krylov += st.krylov_its;
            acc_fallbacks += st.gmres_fallbacks;
            if (!converged) {
                // restore the last converged solution and cut the step
                cudaMemcpyAsync(c.U, c.Uprev, (size_t)nd * sizeof(double), cudaMemcpyDeviceToDevice, s);
                dt *= 0.25;
            }
        }
        // accept: commit the cohesive state, remember the converged U
        if (c.n_coh_qp > 0) {
            cudaMemcpyAsync(c.isv_prev, c.isv_c, (size_t)c.n_coh_qp * sizeof(double), cudaMemcpyDeviceToDevice, s);
            cudaMemcpyAsync(c.isv_c, c.isv_t, (size_t)c.n_coh_qp * sizeof(double), cudaMemcpyDeviceToDevice, s);
        }
        cudaMemcpyAsync(c.Uold2, c.Uold, (size_t)nd * sizeof(double), cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(c.Uold, c.Uprev, (size_t)nd * sizeof(double), cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(c.Uprev, c.U, (size_t)nd * sizeof(double), cudaMemcpyDeviceToDevice, s);
        t += dt;
        st.repeats = repeat;
        st.newton_its = acc_newton;
        st.krylov_its = acc_krylov;
        st.gmres_fallbacks = acc_fallbacks;
        PG_CUDA(cudaStreamSynchronize(s));
        st.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_step).count();
        if (per_step && nrec < max_records) per_step[nrec] = st;
        ++nrec;
        dt_prev2 = dt_prev;
        dt_prev = dt;
        if (repeat == 1) dt *= 1.5;
        dt = std::min(dt, dt_nom);
        if (dt > t_end - t) dt = t_end - t;
    }
    PG_CUDA(cudaStreamSynchronize(s));
    if (n_records) *n_records = nrec;
    return PG_OK;
}

}  // extern "C"
