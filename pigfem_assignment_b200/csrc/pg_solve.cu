// Krylov solves of the assembled IGFEM system on sm_100a.
//
// Reference: PETScLinearKSPSolver::solve (src/SolverLinear.cpp:91-162) and
// Solver::initKSP (src/Solver.cpp:56-142).  The reference factors K_ff with
// MUMPS Cholesky; its commented-out alternatives are CG/GMRES with Jacobi/SOR.
// Here mask(K) x = b is solved on the full 2x2-block matrix with the
// prescribed DOFs masked out (the masked operator is exactly K_ff on the free
// DOFs), by
//   * plain FP64 PCG;
//   * mixed: FP32 matrix/vectors in the Krylov loop (FP64 accumulation of the
//     dot products) inside FP64 iterative refinement on the FP64 residual;
//   * restarted FP64 GMRES (right preconditioning, classical Gram-Schmidt
//     applied twice) for tangents that CG cannot handle (indefinite under
//     cohesive softening).
// PCG iterations run as CUDA graphs of fixed length whose kernels stop doing
// work once a device flag says the tolerance (or a breakdown) was reached, so
// the host reads one status word per graph launch.
//
// PCG scalar bookkeeping (iteration k, P = k & 1, Q = 1 - P).  Invariant at
// the start of iteration k: rz[Q] = r_k . z_k, pq[P] = 0.
//   spmv(k):    q = A p, pq[P] += p.q; zeroes rz[P], rr[P]
//   update(k):  alpha = rz[Q] / pq[P]; x += alpha p; r -= alpha q; z = M^-1 r;
//               rz[P] += r.z; rr[P] += r.r; zeroes pq[Q]
//   pupdate(k): beta = rz[P] / rz[Q]; p = z + beta p; done if rr[P] <= tol^2
#include <algorithm>
#include <vector>

#include "pg_solve_kernels.cuh"

namespace pgb {

namespace {

inline int nblk(int n) { return (n + kThreads - 1) / kThreads; }

template <typename MT, typename VT, typename PT>
int pcg_run(Ctx& c, cudaStream_t s, const MT* K, VT* x, VT* r, VT* z, VT* p, VT* q, const PT* minv, double tol2,
            int max_iter, int chunk, bool& breakdown, double& rr_final, int& status) {
    const int n = c.n_nodes;
    status = PG_OK;
    breakdown = false;
    cudaMemsetAsync(c.scal, 0, S_NSCAL * sizeof(double), s);
    cudaMemsetAsync(c.iflags, 0, F_NFLAGS * sizeof(int), s);
    cudaMemcpyAsync(c.scal + S_TOL2, &tol2, sizeof(double), cudaMemcpyHostToDevice, s);
    k_cg_init<VT, PT><<<nblk(n), kThreads, 0, s>>>(n, r, z, p, minv, c.scal, c.red_active);
    cudaMemcpyAsync(c.h_scal, c.scal, S_NSCAL * sizeof(double), cudaMemcpyDeviceToHost, s);
    PG_CUDA(cudaStreamSynchronize(s));
    rr_final = c.h_scal[S_RR0 + 1];
    if (rr_final <= tol2 || max_iter <= 0) return 0;
    // a budget below one graph's worth of iterations is honoured exactly
    chunk = std::max(1, std::min(chunk, max_iter));

    cudaGraph_t graph;
    PG_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    for (int it = 0; it < chunk; ++it) {
        const int P = it & 1;
        k_spmv_cg<MT, VT><<<nblk(n), kThreads, 0, s>>>(n, P, c.row_ptr, c.col, K, p, c.fixed, q, c.scal, c.iflags,
                                                          c.red_active);
        k_cg_update<VT, PT><<<nblk(n), kThreads, 0, s>>>(n, P, x, r, z, p, q, minv, c.scal, c.iflags, c.red_active);
        k_cg_pupdate<VT><<<nblk(n), kThreads, 0, s>>>(n, P, z, p, c.scal, c.iflags);
    }
    PG_CUDA(cudaStreamEndCapture(s, &graph));
    cudaGraphExec_t exec = nullptr;
    PG_CUDA(cudaGraphInstantiate(&exec, graph, 0));
    cudaGraphDestroy(graph);

    int iters = 0;
    while (true) {
        cudaGraphLaunch(exec, s);
        cudaMemcpyAsync(c.h_iflags, c.iflags, F_NFLAGS * sizeof(int), cudaMemcpyDeviceToHost, s);
        cudaMemcpyAsync(c.h_scal, c.scal, S_NSCAL * sizeof(double), cudaMemcpyDeviceToHost, s);
        const cudaError_t e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) {
            cudaGraphExecDestroy(exec);
            status = cuda_fail(e, "pcg graph");
            return 0;
        }
        iters = c.h_iflags[F_ITERS];
        if (c.h_iflags[F_DONE] || iters >= max_iter) break;
    }
    cudaGraphExecDestroy(exec);
    breakdown = c.h_iflags[F_BREAKDOWN] != 0;
    rr_final = iters > 0 ? c.h_scal[S_RR0 + ((iters - 1) & 1)] : c.h_scal[S_RR0 + 1];
    if (breakdown) status = PG_ERR_BREAKDOWN;
    else if (!c.h_iflags[F_DONE]) status = PG_ERR_NOT_CONVERGED;
    return iters;
}

// ---------------- GMRES ----------------
int ensure_gmres(Ctx& c, int m) {
    if (c.V && c.gm >= m) return PG_OK;
    if (c.V) cudaFree(c.V);
    c.V = nullptr;
    PG_CUDA(cudaMalloc((void**)&c.V, (size_t)(m + 1) * c.n_dof * sizeof(double)));
    c.gm = m;
    return PG_OK;
}

// right-preconditioned restarted GMRES on mask(K); x += solution; b = c.b
int gmres_solve(Ctx& c, const pg_solver_cfg& cfg, double rtol, int max_iter, pg_solve_stats& st, cudaStream_t s,
                double bnorm) {
    const int n = c.n_nodes, nd = c.n_dof;
    const int m = std::max(4, std::min(cfg.gmres_restart > 0 ? cfg.gmres_restart : 60, 120));
    int rc = ensure_gmres(c, m);
    if (rc) return rc;
    std::vector<double> H((size_t)(m + 1) * m), cs(m), sn(m), g(m + 1), y(m), hcol(m + 1);
    int total = 0;
    double rnorm = 0.0;
    while (total < max_iter) {
        // r = b - K x, v0 = r / |r|
        rnorm = std::sqrt(residual_into(c, s, c.dx, c.b, c.r));
        if (rnorm <= rtol * bnorm) break;
        k_scale_copy<<<nblk(nd), kThreads, 0, s>>>(nd, c.r, c.V, 1.0 / rnorm);
        std::fill(g.begin(), g.end(), 0.0);
        g[0] = rnorm;
        int j = 0;
        bool done = false;
        for (; j < m && total < max_iter; ++j, ++total) {
            double* vj = c.V + (size_t)j * nd;
            double* w = c.V + (size_t)(j + 1) * nd;
            // w = K M^-1 v_j
            if (cfg.precond == PG_PREC_MG)
                mg_precondition(c, cfg.precision == PG_PRECISION_MIXED, s, vj, c.z);
            else
                k_apply_prec_vec<<<nblk(n), kThreads, 0, s>>>(n, c.minv, vj, c.z);
            k_spmv_plain<double, double><<<nblk(n), kThreads, 0, s>>>(n, c.row_ptr, c.col, c.K, c.z, c.fixed, w);
            // classical Gram-Schmidt, twice
            std::fill(hcol.begin(), hcol.end(), 0.0);
            for (int pass = 0; pass < 2; ++pass) {
                cudaMemsetAsync(c.hbuf, 0, (j + 1) * sizeof(double), s);
                k_multidot<<<std::min(nblk(nd), 1184), kThreads, 0, s>>>(nd, j + 1, c.V, w, c.hbuf, c.red_active);
                k_multi_axpy<<<nblk(nd), kThreads, 0, s>>>(nd, j + 1, c.V, c.hbuf, w);
                std::vector<double> hh(j + 1);
                cudaMemcpyAsync(hh.data(), c.hbuf, (j + 1) * sizeof(double), cudaMemcpyDeviceToHost, s);
                PG_CUDA(cudaStreamSynchronize(s));
                for (int i = 0; i <= j; ++i) hcol[i] += hh[i];
            }
            const double hn = std::sqrt(dev_norm2(c, w, nd, s));
            hcol[j + 1] = hn;
            if (hn > 0.0) k_scale_inplace<<<nblk(nd), kThreads, 0, s>>>(nd, w, 1.0 / hn);
            // apply previous rotations, make a new one
            for (int i = 0; i < j; ++i) {
                const double t = cs[i] * hcol[i] + sn[i] * hcol[i + 1];
                hcol[i + 1] = -sn[i] * hcol[i] + cs[i] * hcol[i + 1];
                hcol[i] = t;
            }
            const double den = std::hypot(hcol[j], hcol[j + 1]);
            cs[j] = den > 0 ? hcol[j] / den : 1.0;
            sn[j] = den > 0 ? hcol[j + 1] / den : 0.0;
            hcol[j] = den;
            hcol[j + 1] = 0.0;
            g[j + 1] = -sn[j] * g[j];
            g[j] = cs[j] * g[j];
            for (int i = 0; i <= j; ++i) H[(size_t)i * m + j] = hcol[i];
            if (std::fabs(g[j + 1]) <= rtol * bnorm || hn == 0.0) {
                ++j;
                ++total;
                done = true;
                break;
            }
        }
        // y = H^-1 g (upper triangular j x j); x += M^-1 V y
        for (int i = j - 1; i >= 0; --i) {
            double acc = g[i];
            for (int k = i + 1; k < j; ++k) acc -= H[(size_t)i * m + k] * y[k];
            y[i] = H[(size_t)i * m + i] != 0.0 ? acc / H[(size_t)i * m + i] : 0.0;
        }
        cudaMemcpyAsync(c.hbuf, y.data(), j * sizeof(double), cudaMemcpyHostToDevice, s);
        k_fill<double><<<nblk(nd), kThreads, 0, s>>>(nd, c.q, 0.0);
        k_multi_axpy_add<<<nblk(nd), kThreads, 0, s>>>(nd, j, c.V, c.hbuf, c.q);
        if (cfg.precond == PG_PREC_MG)
            mg_precondition(c, cfg.precision == PG_PRECISION_MIXED, s, c.q, c.z);
        else
            k_apply_prec_vec<<<nblk(n), kThreads, 0, s>>>(n, c.minv, c.q, c.z);
        k_axpy_free<double><<<nblk(nd), kThreads, 0, s>>>(nd, c.fixed, c.dx, c.z, 1.0);
        if (done) {
            rnorm = std::sqrt(residual_into(c, s, c.dx, c.b, c.r));
            if (rnorm <= rtol * bnorm * 1.0001) break;
        }
    }
    st.iterations += total;
    st.rel_residual = rnorm / bnorm;
    st.status = rnorm <= rtol * bnorm * 1.0001 ? PG_OK : PG_ERR_NOT_CONVERGED;
    return PG_OK;
}

// Preconditioned MINRES on mask(K) x = b (b = c.b), x accumulated into c.dx.
int minres_solve(Ctx& c, double rtol, int max_iter, int chunk, pg_solve_stats& st, cudaStream_t s) {
    const int n = c.n_nodes, nd = c.n_dof;
    double* buf[2] = {c.r, c.q};
    double* W[2] = {c.mw, c.mw + nd};
    double* y = c.z;
    double* v = c.p;
    k_prec_absjacobi<<<nblk(n), kThreads, 0, s>>>(n, c.diag, c.K, c.fixed, c.minv);
    k_copy<double><<<nblk(nd), kThreads, 0, s>>>(nd, c.b, buf[0]);
    k_copy<double><<<nblk(nd), kThreads, 0, s>>>(nd, c.b, buf[1]);
    k_apply_prec_vec<<<nblk(n), kThreads, 0, s>>>(n, c.minv, c.b, y);
    cudaMemsetAsync(c.mw, 0, 2 * (size_t)nd * sizeof(double), s);
    // beta1^2 = b . M^-1 b
    cudaMemsetAsync(c.scal + S_AUX, 0, sizeof(double), s);
    k_dot2<<<nblk(nd), kThreads, 0, s>>>(nd, c.b, y, c.scal + S_AUX, c.red_active);
    cudaMemcpyAsync(c.h_scal + S_AUX, c.scal + S_AUX, sizeof(double), cudaMemcpyDeviceToHost, s);
    PG_CUDA(cudaStreamSynchronize(s));
    const double beta1 = std::sqrt(std::max(c.h_scal[S_AUX], 0.0));
    if (beta1 == 0.0) return PG_OK;
    double h[M_NSCAL] = {0};
    h[M_BETA] = beta1;
    h[M_OLDB] = 0.0;
    h[M_PHIBAR] = beta1;
    h[M_CS] = -1.0;
    h[M_SN] = 0.0;
    h[M_BETA1] = beta1;
    h[M_TOL] = rtol;
    cudaMemcpyAsync(c.scal, h, M_NSCAL * sizeof(double), cudaMemcpyHostToDevice, s);
    cudaMemsetAsync(c.iflags, 0, F_NFLAGS * sizeof(int), s);
    const int len = std::max(2, chunk & ~1);
    cudaGraph_t graph;
    PG_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    for (int k = 0; k < len; ++k) {
        const int P = k & 1, Q = 1 - P;
        k_mr_v<<<nblk(nd), kThreads, 0, s>>>(nd, y, v, c.scal, c.iflags);
        k_mr_av<double><<<nblk(n), kThreads, 0, s>>>(n, c.row_ptr, c.col, c.K, v, c.fixed, buf[P], y, c.scal, c.iflags,
                                                       c.red_active);
        k_mr_2<<<nblk(n), kThreads, 0, s>>>(n, y, buf[Q], buf[P], c.minv, c.scal, c.iflags, c.red_active);
        k_mr_scalars<<<1, 1, 0, s>>>(c.scal, c.iflags);
        k_mr_w<<<nblk(nd), kThreads, 0, s>>>(nd, v, W[P], W[Q], c.dx, c.scal, c.iflags);
        k_mr_seal<<<1, 1, 0, s>>>(c.iflags);
    }
    PG_CUDA(cudaStreamEndCapture(s, &graph));
    cudaGraphExec_t exec = nullptr;
    PG_CUDA(cudaGraphInstantiate(&exec, graph, 0));
    cudaGraphDestroy(graph);
    int iters = 0;
    while (true) {
        cudaGraphLaunch(exec, s);
        cudaMemcpyAsync(c.h_iflags, c.iflags, F_NFLAGS * sizeof(int), cudaMemcpyDeviceToHost, s);
        const cudaError_t e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) {
            cudaGraphExecDestroy(exec);
            return cuda_fail(e, "minres graph");
        }
        iters = c.h_iflags[F_ITERS];
        if (c.h_iflags[F_DONE] || iters >= max_iter) break;
    }
    cudaGraphExecDestroy(exec);
    st.iterations += iters;
    return PG_OK;
}

}  // namespace

double residual_into(Ctx& c, cudaStream_t s, const double* x, const double* b, double* out) {
    const int n = c.n_nodes, nd = c.n_dof;
    k_spmv_plain<double, double><<<nblk(n), kThreads, 0, s>>>(n, c.row_ptr, c.col, c.K, x, c.fixed, out);
    k_rhs_minus<<<nblk(nd), kThreads, 0, s>>>(nd, c.fixed, b, out);
    return dev_norm2(c, out, nd, s);
}

double dev_norm2(Ctx& c, const double* v, int n, cudaStream_t s) {
    cudaMemsetAsync(c.scal + S_AUX, 0, sizeof(double), s);
    k_dot_self<<<nblk(n), kThreads, 0, s>>>(n, v, c.scal + S_AUX, c.red_active);
    cudaMemcpyAsync(c.h_scal + S_AUX, c.scal + S_AUX, sizeof(double), cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    return c.h_scal[S_AUX];
}

void set_prescribed(Ctx& c, double t_frac, cudaStream_t s) {
    c.t_frac = t_frac;
    k_apply_dirichlet<<<nblk(c.n_dof), kThreads, 0, s>>>(c.n_dof, c.fixed, c.ubar, t_frac, c.U);
}

int krylov_solve(Ctx& c, const pg_solver_cfg& cfg, pg_solve_stats& st, cudaStream_t s) {
    const int n = c.n_nodes, nd = c.n_dof;
    st.iterations = 0;
    st.refinements = 0;
    st.status = PG_OK;
    st.rel_residual = 0.0;
    c.red_active = cfg.deterministic ? c.red_ws : nullptr;
    const int block = cfg.precond == PG_PREC_BLOCK_JACOBI ? 1 : 0;
    const int ident = cfg.precond == PG_PREC_NONE ? 1 : 0;
    const int chunk = cfg.check_every > 1 ? ((cfg.check_every + 1) & ~1) : 32;
    k_fill<double><<<nblk(nd), kThreads, 0, s>>>(nd, c.dx, 0.0);
    const double bb = dev_norm2(c, c.b, nd, s);
    if (bb == 0.0) return PG_OK;
    const double tol2 = cfg.rtol * cfg.rtol * bb;
    int status = PG_OK;
    double rr = bb;
    if (cfg.krylov == PG_KRYLOV_MINRES) {
        const int rc = minres_solve(c, cfg.rtol, cfg.max_iter, chunk, st, s);
        if (rc != PG_OK) return rc;
        rr = residual_into(c, s, c.dx, c.b, c.r);
        st.rel_residual = std::sqrt(rr / bb);
        // MINRES monitors the M^-1-norm; accept a true residual within a small factor
        st.status = rr <= tol2 * 100.0 ? PG_OK : PG_ERR_NOT_CONVERGED;
        return PG_OK;
    }
    if (cfg.precond == PG_PREC_MG) {
        // one multigrid V-cycle per iteration (FP32 cycle under PG_PRECISION_MIXED)
        if (cfg.krylov == PG_KRYLOV_GMRES) {
            const int rc = mg_prepare(c, cfg.precision == PG_PRECISION_MIXED, cfg.inclusion_modes != 0, s);
            if (rc == PG_ERR_BREAKDOWN) { st.status = rc; return PG_OK; }
            if (rc != PG_OK) return rc;
            return gmres_solve(c, cfg, cfg.rtol, cfg.max_iter, st, s, std::sqrt(bb));
        }
        return mg_pcg_solve(c, cfg, st, s);
    }
    k_prec_setup<double><<<nblk(n), kThreads, 0, s>>>(n, c.diag, c.K, c.fixed, block, ident, c.minv);
    if (cfg.krylov == PG_KRYLOV_GMRES) {
        const int rc = gmres_solve(c, cfg, cfg.rtol, cfg.max_iter, st, s, std::sqrt(bb));
        return rc;
    }
    if (cfg.precision == PG_PRECISION_FP64) {
        k_copy<double><<<nblk(nd), kThreads, 0, s>>>(nd, c.b, c.r);
        bool brk = false;
        double rrf = 0.0;
        st.iterations = pcg_run<double, double, double>(c, s, c.K, c.dx, c.r, c.z, c.p, c.q, c.minv, tol2,
                                                        cfg.max_iter, chunk, brk, rrf, status);
        if (status == PG_ERR_CUDA) return status;
        rr = residual_into(c, s, c.dx, c.b, c.r);
        if (status == PG_OK && rr > tol2 * 4.0) status = PG_ERR_NOT_CONVERGED;
    } else {
        // Krylov on the FP32-stored matrix (FP64 vectors) inside FP64 refinement
        launch_to_fp32(c, s);
        const double inner = cfg.inner_rtol > 0 ? cfg.inner_rtol : 1e-4;
        k_copy<double><<<nblk(nd), kThreads, 0, s>>>(nd, c.b, c.r);
        int total_it = 0, ref = 0;
        while (rr > tol2 && ref < cfg.max_refine && total_it < cfg.max_iter) {
            k_fill<double><<<nblk(nd), kThreads, 0, s>>>(nd, c.xi, 0.0);
            bool brk = false;
            double rrf = 0.0;
            int st_in = PG_OK;
            // stop the inner solve at inner * |r| but never below the outer target
            const double itol2 = std::max(inner * inner * rr, 0.25 * tol2);
            total_it += pcg_run<float, double, double>(c, s, c.Kf, c.xi, c.r, c.z, c.p, c.q, c.minv, itol2,
                                                        cfg.max_iter - total_it, chunk, brk, rrf, st_in);
            if (st_in == PG_ERR_CUDA) return st_in;
            k_axpy_free<double><<<nblk(nd), kThreads, 0, s>>>(nd, c.fixed, c.dx, c.xi, 1.0);
            rr = residual_into(c, s, c.dx, c.b, c.r);
            ++ref;
            if (brk) { status = PG_ERR_BREAKDOWN; break; }
        }
        st.iterations = total_it;
        st.refinements = ref;
        if (status == PG_OK && rr > tol2) status = PG_ERR_NOT_CONVERGED;
    }
    st.rel_residual = std::sqrt(rr / bb);
    st.status = status;
    return PG_OK;
}

int solve_linear_system(Ctx& c, const pg_solver_cfg& cfg, pg_solve_stats& st, cudaStream_t s) {
    const int nd = c.n_dof;
    cudaEventRecord(c.ev0, s);
    // b = mask(0 - K U): the prescribed part of U drives the free DOFs
    residual_into(c, s, c.U, nullptr, c.b);
    int rc = krylov_solve(c, cfg, st, s);
    if (rc != PG_OK) return rc;
    if (st.status == PG_ERR_BREAKDOWN && cfg.krylov == PG_KRYLOV_CG) {
        pg_solver_cfg g = cfg;
        g.krylov = PG_KRYLOV_GMRES;
        const int it0 = st.iterations;
        rc = krylov_solve(c, g, st, s);
        if (rc != PG_OK) return rc;
        st.iterations += it0;
    }
    k_axpy_free<double><<<nblk(nd), kThreads, 0, s>>>(nd, c.fixed, c.U, c.dx, 1.0);
    cudaEventRecord(c.ev1, s);
    PG_CUDA(cudaEventSynchronize(c.ev1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c.ev0, c.ev1);
    st.seconds = ms * 1e-3;
    return PG_OK;
}

}  // namespace pgb
