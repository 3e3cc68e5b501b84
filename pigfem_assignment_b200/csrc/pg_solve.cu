// Krylov solves of the assembled IGFEM system on sm_100a.
//
// Reference: PETScLinearKSPSolver::solve (src/SolverLinear.cpp:91-162) and
// Solver::initKSP (src/Solver.cpp:56-142).  The reference factors K_ff with
// MUMPS Cholesky; its commented-out alternatives are CG/GMRES with Jacobi/SOR.
// Here K_ff u_f = f_f - K_fp u_p is solved by preconditioned CG on the full
// 2x2-block matrix with the prescribed DOFs masked out (the masked operator
// is exactly K_ff on the free DOFs), in two forms:
//   * plain FP64 PCG;
//   * mixed: FP32 matrix/vectors in the Krylov loop (FP64 accumulation of the
//     dot products) inside FP64 iterative refinement on the FP64 residual.
// Iterations run as CUDA graphs of fixed length whose kernels stop doing work
// once a device flag says the tolerance (or a breakdown) was reached, so the
// host reads one status word per graph launch.
//
// Scalar bookkeeping (iteration k, P = k & 1, Q = 1 - P).  Invariant at the
// start of iteration k: rz[Q] = r_k . z_k, pq[P] = 0.
//   spmv(k):    q = A p, pq[P] += p.q; zeroes rz[P], rr[P]
//   update(k):  alpha = rz[Q] / pq[P]; x += alpha p; r -= alpha q; z = M^-1 r;
//               rz[P] += r.z; rr[P] += r.r; zeroes pq[Q]
//   pupdate(k): beta = rz[P] / rz[Q]; p = z + beta p; done if rr[P] <= tol^2
#include "pg_solve_kernels.cuh"

namespace pgb {

namespace {

inline int nblk(int n) { return (n + kThreads - 1) / kThreads; }

// Graphs of `chunk` PCG iterations, keyed by precision.
struct GraphCache {
    cudaGraphExec_t g = nullptr;
    int chunk = 0;
    const void* key = nullptr;
};

template <typename MT, typename VT, typename PT>
int pcg_run(Ctx& c, cudaStream_t s, const MT* K, VT* x, VT* r, VT* z, VT* p, VT* q, const PT* minv, double tol2,
            int max_iter, int chunk, bool& breakdown, double& rr_final, int& status) {
    const int n = c.n_nodes;
    status = PG_OK;
    cudaMemsetAsync(c.scal, 0, S_NSCAL * sizeof(double), s);
    cudaMemsetAsync(c.iflags, 0, F_NFLAGS * sizeof(int), s);
    cudaMemcpyAsync(c.scal + S_TOL2, &tol2, sizeof(double), cudaMemcpyHostToDevice, s);
    k_cg_init<VT, PT><<<nblk(n), kThreads, 0, s>>>(n, r, z, p, minv, c.scal);
    cudaMemcpyAsync(c.h_scal, c.scal, S_NSCAL * sizeof(double), cudaMemcpyDeviceToHost, s);
    PG_CUDA(cudaStreamSynchronize(s));
    breakdown = false;
    rr_final = c.h_scal[S_RR0 + 1];
    if (rr_final <= tol2) return 0;

    cudaGraph_t graph;
    PG_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    for (int it = 0; it < chunk; ++it) {
        const int P = it & 1;
        k_spmv_cg<MT, VT><<<nblk(n), kThreads, 0, s>>>(n, P, c.row_ptr, c.col, K, p, c.fixed, q, c.scal, c.iflags);
        k_cg_update<VT, PT><<<nblk(n), kThreads, 0, s>>>(n, P, x, r, z, p, q, minv, c.scal, c.iflags);
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
            return cuda_fail(e, "pcg graph");
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

// ||mask(-K U)||^2 into r (FP64) and the returned value
double residual64(Ctx& c, cudaStream_t s) {
    const int n = c.n_nodes, nd = c.n_dof;
    k_spmv_plain<double, double><<<nblk(n), kThreads, 0, s>>>(n, c.row_ptr, c.col, c.K, c.U, c.fixed, c.r);
    k_neg<double><<<nblk(nd), kThreads, 0, s>>>(nd, c.r);
    cudaMemsetAsync(c.scal + S_AUX, 0, sizeof(double), s);
    k_dot_self<<<nblk(nd), kThreads, 0, s>>>(nd, c.r, c.scal + S_AUX);
    cudaMemcpyAsync(c.h_scal + S_AUX, c.scal + S_AUX, sizeof(double), cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    return c.h_scal[S_AUX];
}

}  // namespace

void set_prescribed(Ctx& c, double t_frac, cudaStream_t s) {
    k_apply_dirichlet<<<nblk(c.n_dof), kThreads, 0, s>>>(c.n_dof, c.fixed, c.ubar, t_frac, c.U);
}

int solve_linear_system(Ctx& c, const pg_solver_cfg& cfg, pg_solve_stats& st, cudaStream_t s) {
    const int n = c.n_nodes, nd = c.n_dof;
    st.iterations = 0;
    st.refinements = 0;
    st.status = PG_OK;
    st.rel_residual = 0.0;
    if (cfg.krylov != PG_KRYLOV_CG) {
        set_error("pg_solve_linear: only PG_KRYLOV_CG is available for the linear solve");
        return PG_ERR_ARG;
    }
    const int block = cfg.precond == PG_PREC_BLOCK_JACOBI ? 1 : 0;
    const int ident = cfg.precond == PG_PREC_NONE ? 1 : 0;
    const int chunk = cfg.check_every > 1 ? ((cfg.check_every + 1) & ~1) : 32;
    cudaEventRecord(c.ev0, s);
    const double rr0 = residual64(c, s);
    if (rr0 == 0.0) {
        cudaEventRecord(c.ev1, s);
        cudaEventSynchronize(c.ev1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, c.ev0, c.ev1);
        st.seconds = ms * 1e-3;
        return PG_OK;
    }
    int status = PG_OK;
    double rr = rr0;
    if (cfg.precision == PG_PRECISION_FP64) {
        k_prec_setup<double><<<nblk(n), kThreads, 0, s>>>(n, c.diag, c.K, c.fixed, block, ident, c.minv);
        k_fill<double><<<nblk(nd), kThreads, 0, s>>>(nd, c.dx, 0.0);
        bool brk = false;
        double rrf = 0.0;
        const double tol2 = cfg.rtol * cfg.rtol * rr0;
        st.iterations = pcg_run<double, double, double>(c, s, c.K, c.dx, c.r, c.z, c.p, c.q, c.minv, tol2,
                                                        cfg.max_iter, chunk, brk, rrf, status);
        k_axpy_free<double><<<nblk(nd), kThreads, 0, s>>>(nd, c.fixed, c.U, c.dx, 1.0);
        rr = residual64(c, s);
        if (status == PG_OK && rr > tol2 * 4.0) status = PG_ERR_NOT_CONVERGED;
    } else {
        // FP32 Krylov inside FP64 refinement
        k_prec_setup<float><<<nblk(n), kThreads, 0, s>>>(n, c.diag, c.K, c.fixed, block, ident, c.minvf);
        launch_to_fp32(c, s);
        const double goal = cfg.rtol * cfg.rtol * rr0;
        const double inner = cfg.inner_rtol > 0 ? cfg.inner_rtol : 1e-4;
        int total_it = 0;
        int ref = 0;
        while (rr > goal && ref < cfg.max_refine && total_it < cfg.max_iter) {
            const double sc = 1.0 / std::sqrt(rr);
            k_to_float_scaled<<<nblk(nd), kThreads, 0, s>>>(nd, c.r, c.rf, sc);
            k_fill<float><<<nblk(nd), kThreads, 0, s>>>(nd, c.xf, 0.0f);
            bool brk = false;
            double rrf = 0.0;
            int st_in = PG_OK;
            const int its = pcg_run<float, float, float>(c, s, c.Kf, c.xf, c.rf, c.zf, c.pf, c.qf, c.minvf,
                                                          inner * inner, cfg.max_iter - total_it, chunk, brk, rrf,
                                                          st_in);
            total_it += its;
            k_axpy_free_f<<<nblk(nd), kThreads, 0, s>>>(nd, c.fixed, c.U, c.xf, 1.0 / sc);
            rr = residual64(c, s);
            ++ref;
            if (brk) { status = PG_ERR_BREAKDOWN; break; }
        }
        st.iterations = total_it;
        st.refinements = ref;
        if (status == PG_OK && rr > goal) status = PG_ERR_NOT_CONVERGED;
    }
    cudaEventRecord(c.ev1, s);
    PG_CUDA(cudaEventSynchronize(c.ev1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c.ev0, c.ev1);
    st.seconds = ms * 1e-3;
    st.rel_residual = std::sqrt(rr / rr0);
    st.status = status;
    return PG_OK;
}

}  // namespace pgb
