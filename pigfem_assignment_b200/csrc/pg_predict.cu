// Learned Newton warm start: per-node features, training targets and the
// application of the MLP's output to the load extrapolation.
// The reference only has the zeroth-order predictor (U_f carried over,
// src/SolverNonlinear.cpp:254-267); this is new.
//
// From the last three converged states (U_n, U_{n-1}, U_{n-2}, reached by
// steps dt_n and dt_{n-1}) and the coming step dt, per node:
//   d_n = U_n - U_{n-1},  d_{n-1} = U_{n-1} - U_{n-2}
//   U_lin  = U_n + (dt / dt_n) d_n                      linear extrapolation
//   c      = dt (dt + dt_n) / (dt_n + dt_{n-1}) (d_n / dt_n - d_{n-1} / dt_{n-1})
//            (the quadratic extrapolation's term: U_quad = U_lin + c)
//   U_pred = U_lin + g c,   g = sum_i w_i (1 + y_i) / sum_i w_i,  w_i = |c_i|^2,
// y_i = the network's output for node i clamped to [-1, 0] (-1: the node
// follows its linear extrapolation, 0: its quadratic one).  Each node's
// network output, from its own history and damage state, votes with the
// weight its curvature term has in the prediction, and one blend g of the
// linear and quadratic extrapolations is applied to all nodes: a blend that
// varied from node to node would add a rough field, which the stiffness
// turns into a large residual (measured: ~60x the linear start's), while a
// uniform blend keeps the extrapolation smooth.
//
// Features of node i (16, scale-free, each bounded by 5): c / |d_n| (2),
// d_n / |d_n| (2), |d_{n-1}| dt_n / (|d_n| dt_{n-1}) (1), log(1 + |d_n| /
// s_inc) (1), enrichment / mirror flags (2), log(1 + the largest committed
// opening over the node's cohesive points / delta_ref) (1) and the opening's
// change over the last step / delta_ref (1), load fraction (1), dt / dt_n (1),
// Dirichlet flags (2), a constant 1 (1), 0 (1).
// Target: y* = (e . c) / (c . c) - 1 with e = U_{n+1} - U_lin over the
// node's free components, clipped to [-1, 0] (both outputs).
#include <cmath>

#include "pg_internal.cuh"
#include "pg_solve_kernels.cuh"

namespace pgb {

namespace {
inline int nblk(int n) { return (n + kThreads - 1) / kThreads; }

struct NodeHist {
    double dn[2], c[2], dnorm, dprev;
};

__device__ __forceinline__ NodeHist node_hist(const pg_pred_history& h, int i) {
    NodeHist r;
    const double q = h.dt * (h.dt + h.dt_n) / (h.dt_n + h.dt_nm1);
    double pn2 = 0.0;
    for (int d = 0; d < 2; ++d) {
        const double a = h.U_n[2 * i + d], b = h.U_nm1[2 * i + d], o = h.U_nm2[2 * i + d];
        const double dn = a - b, dp = b - o;
        r.dn[d] = dn;
        r.c[d] = q * (dn / h.dt_n - dp / h.dt_nm1);
        pn2 += dp * dp;
    }
    r.dnorm = sqrt(r.dn[0] * r.dn[0] + r.dn[1] * r.dn[1]);
    r.dprev = sqrt(pn2);
    return r;
}
}  // namespace

__global__ void k_features(int n, int n_reg, int n_enr_initial, const uint8_t* __restrict__ fixed,
                           pg_pred_history h, const double* __restrict__ isv_c, const int* __restrict__ nq_ptr,
                           const int* __restrict__ nq_list, double delta_ref, float* __restrict__ X) {
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i >= n) return;
    const NodeHist r = node_hist(h, i);
    double dmg = 0.0, dmg_prev = 0.0;
    if (nq_ptr)
        for (int k = nq_ptr[i]; k < nq_ptr[i + 1]; ++k) {
            dmg = fmax(dmg, isv_c[nq_list[k]]);
            if (h.isv_nm1) dmg_prev = fmax(dmg_prev, h.isv_nm1[nq_list[k]]);
        }
    const double eps = 1e-6 * fabs(h.s_inc);
    const double inv = 1.0 / (r.dnorm + eps);
    float f[16];
    f[0] = (float)fmax(-5.0, fmin(5.0, r.c[0] * inv));
    f[1] = (float)fmax(-5.0, fmin(5.0, r.c[1] * inv));
    f[2] = (float)(r.dn[0] * inv);
    f[3] = (float)(r.dn[1] * inv);
    f[4] = (float)fmin(5.0, r.dprev * h.dt_n / h.dt_nm1 * inv);
    f[5] = (float)fmin(5.0, log1p(r.dnorm / fabs(h.s_inc)));
    f[6] = i >= n_reg ? 1.f : 0.f;
    f[7] = i >= n_reg + n_enr_initial ? 1.f : 0.f;
    f[8] = (float)fmin(5.0, log1p(dmg / delta_ref));
    f[9] = h.isv_nm1 ? (float)fmax(-5.0, fmin(5.0, (dmg - dmg_prev) / delta_ref)) : 0.f;
    f[10] = (float)h.t_frac;
    f[11] = (float)(h.dt / h.dt_n);
    f[12] = fixed[2 * i] ? 1.f : 0.f;
    f[13] = fixed[2 * i + 1] ? 1.f : 0.f;
    f[14] = 1.f;
    f[15] = 0.f;
    float4* o = reinterpret_cast<float4*>(X + 16 * (size_t)i);
    o[0] = make_float4(f[0], f[1], f[2], f[3]);
    o[1] = make_float4(f[4], f[5], f[6], f[7]);
    o[2] = make_float4(f[8], f[9], f[10], f[11]);
    o[3] = make_float4(f[12], f[13], f[14], f[15]);
}

__global__ void k_targets(int n, const uint8_t* __restrict__ fixed, pg_pred_history h,
                          const double* __restrict__ Un1, float* __restrict__ T) {
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i >= n) return;
    const NodeHist r = node_hist(h, i);
    double ec = 0.0, cc = 0.0;
    for (int d = 0; d < 2; ++d) {
        if (fixed[2 * i + d]) continue;
        const double lin = h.U_n[2 * i + d] + (h.dt / h.dt_n) * r.dn[d];
        ec += (Un1[2 * i + d] - lin) * r.c[d];
        cc += r.c[d] * r.c[d];
    }
    const double y = cc > 0.0 ? fmax(-1.0, fmin(0.0, ec / cc - 1.0)) : -1.0;
    T[2 * i] = (float)y;
    T[2 * i + 1] = (float)y;
}

// per CTA: sum of w_i and of w_i (1 + y_i) over its nodes (free components
// of c only); the CTAs' partials are added in order on the host
constexpr int kBlendThreads = 256;
__global__ void __launch_bounds__(kBlendThreads) k_blend_partial(int n, const uint8_t* __restrict__ fixed,
                                                                 pg_pred_history h, const float* __restrict__ Y,
                                                                 double* __restrict__ part) {
    __shared__ double sw[kBlendThreads], swy[kBlendThreads];
    double w = 0.0, wy = 0.0;
    for (int i = blockIdx.x * kBlendThreads + threadIdx.x; i < n; i += kBlendThreads * gridDim.x) {
        const NodeHist r = node_hist(h, i);
        double cc = 0.0;
        for (int d = 0; d < 2; ++d)
            if (!fixed[2 * i + d]) cc += r.c[d] * r.c[d];
        const double y = fmax(-1.0, fmin(0.0, (double)Y[2 * i]));
        w += cc;
        wy += cc * (1.0 + y);
    }
    sw[threadIdx.x] = w;
    swy[threadIdx.x] = wy;
    __syncthreads();
    for (int st = kBlendThreads / 2; st > 0; st >>= 1) {
        if (threadIdx.x < st) {
            sw[threadIdx.x] += sw[threadIdx.x + st];
            swy[threadIdx.x] += swy[threadIdx.x + st];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = sw[0];
        part[2 * blockIdx.x + 1] = swy[0];
    }
}

// U = U_lin + g c on free DOFs
__global__ void k_apply(int n, const uint8_t* __restrict__ fixed, pg_pred_history h, double g,
                        double* __restrict__ U) {
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i >= n) return;
    const NodeHist r = node_hist(h, i);
    for (int d = 0; d < 2; ++d) {
        if (fixed[2 * i + d]) continue;
        U[2 * i + d] = h.U_n[2 * i + d] + (h.dt / h.dt_n) * r.dn[d] + g * r.c[d];
    }
}

// node -> cohesive quadrature points (for the damage features)
int build_node_qp_map(Ctx& c) {
    if (c.nq_ptr || c.n_coh_qp == 0) return PG_OK;
    const HostMesh& m = c.hm;
    std::vector<std::vector<int>> lists(m.n_nodes());
    for (int ci = 0; ci < m.n_cut; ++ci) {
        const CutTemplate& T = cut_template(m.cut_tmpl[ci]);
        for (int k = 0; k < T.n_coh; ++k)
            for (int v = 0; v < 4; ++v) {
                const int ln = T.coh_nodes[k][v];
                const int node = m.cut_enr[(size_t)ci * kMaxEnr + ln - 3];
                for (int q = 0; q < 2; ++q) lists[node].push_back(m.cut_coh_qp0[ci] + 2 * k + q);
            }
    }
    std::vector<int> ptr(m.n_nodes() + 1, 0), list;
    for (int i = 0; i < m.n_nodes(); ++i) {
        list.insert(list.end(), lists[i].begin(), lists[i].end());
        ptr[i + 1] = (int)list.size();
    }
    PG_CUDA(cudaMalloc((void**)&c.nq_ptr, ptr.size() * sizeof(int)));
    PG_CUDA(h2d_sync(c.nq_ptr, ptr.data(), ptr.size() * sizeof(int)));
    PG_CUDA(cudaMalloc((void**)&c.nq_list, std::max<size_t>(1, list.size()) * sizeof(int)));
    if (!list.empty()) PG_CUDA(h2d_sync(c.nq_list, list.data(), list.size() * sizeof(int)));
    return PG_OK;
}

double predictor_delta_ref(const Ctx& c) {
    if (c.coh.law == PG_COH_OP) return c.coh.p[1] > 0 ? c.coh.p[1] : 1.0;
    return c.coh.p[2] > 0 ? c.coh.p[0] / c.coh.p[2] : 1.0;
}

double predictor_app(const Ctx& c) {
    const RveSpec& s = c.hm.spec;
    const double app = (s.x1 - s.x0) * s.strain;
    return app != 0.0 ? app : 1.0;
}

bool history_ok(const pg_pred_history& h) {
    return h.U_n && h.U_nm1 && h.U_nm2 && h.dt_n > 0.0 && h.dt_nm1 > 0.0 && h.dt > 0.0 && h.s_inc != 0.0;
}

int launch_features(Ctx& c, const pg_pred_history& h, float* X, cudaStream_t s) {
    int rc = build_node_qp_map(c);
    if (rc) return rc;
    k_features<<<nblk(c.n_nodes), kThreads, 0, s>>>(c.n_nodes, c.n_reg, c.hm.n_enr_initial, c.fixed, h, c.isv_c,
                                                    c.nq_ptr, c.nq_list, predictor_delta_ref(c), X);
    PG_CUDA(cudaGetLastError());
    return PG_OK;
}

int predictor_blend(Ctx& c, const pg_pred_history& h, const float* Y, double& g, cudaStream_t s) {
    constexpr int kParts = 148 * 2;
    double* part = nullptr;
    PG_CUDA(cudaMallocAsync((void**)&part, 2 * kParts * sizeof(double), s));
    k_blend_partial<<<kParts, kBlendThreads, 0, s>>>(c.n_nodes, c.fixed, h, Y, part);
    std::vector<double> hp(2 * kParts);
    PG_CUDA(cudaMemcpyAsync(hp.data(), part, hp.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
    PG_CUDA(cudaStreamSynchronize(s));
    cudaFreeAsync(part, s);
    double w = 0.0, wy = 0.0;
    for (int b = 0; b < kParts; ++b) {
        w += hp[2 * b];
        wy += hp[2 * b + 1];
    }
    g = w > 0.0 ? std::max(0.0, std::min(1.0, wy / w)) : 0.0;
    return PG_OK;
}

int launch_apply(Ctx& c, const pg_pred_history& h, const float* Y, double scale, double* U, cudaStream_t s,
                 double* g_used) {
    double g = 0.0;
    if (Y) {
        const int rc = predictor_blend(c, h, Y, g, s);
        if (rc) return rc;
        g *= scale;
    }
    if (g_used) *g_used = g;
    k_apply<<<nblk(c.n_nodes), kThreads, 0, s>>>(c.n_nodes, c.fixed, h, g, U);
    PG_CUDA(cudaGetLastError());
    return PG_OK;
}

}  // namespace pgb

using namespace pgb;

extern "C" {

int pg_predictor_features(pg_ctx* cx, const pg_pred_history* h, float* X_dev) {
    if (!cx || !h || !X_dev || !history_ok(*h)) { set_error("pg_predictor_features: bad argument"); return PG_ERR_ARG; }
    Ctx& c = cx->c;
    cudaSetDevice(c.device);
    return launch_features(c, *h, X_dev, c.stream);
}

int pg_predictor_targets(pg_ctx* cx, const pg_pred_history* h, const double* U_np1, float* T_dev) {
    if (!cx || !h || !U_np1 || !T_dev || !history_ok(*h)) {
        set_error("pg_predictor_targets: bad argument");
        return PG_ERR_ARG;
    }
    Ctx& c = cx->c;
    cudaSetDevice(c.device);
    k_targets<<<nblk(c.n_nodes), kThreads, 0, c.stream>>>(c.n_nodes, c.fixed, *h, U_np1, T_dev);
    PG_CUDA(cudaGetLastError());
    return PG_OK;
}

int pg_predictor_apply(pg_ctx* cx, const pg_pred_history* h, const float* Y_dev, double scale, double* U_dev) {
    if (!cx || !h || !U_dev || !history_ok(*h)) { set_error("pg_predictor_apply: bad argument"); return PG_ERR_ARG; }
    Ctx& c = cx->c;
    cudaSetDevice(c.device);
    return launch_apply(c, *h, Y_dev, scale, U_dev, c.stream, nullptr);
}

int pg_ctx_attach_mlp(pg_ctx* cx, pg_mlp* m) {
    if (!cx) { set_error("pg_ctx_attach_mlp: null context"); return PG_ERR_ARG; }
    Ctx& c = cx->c;
    cudaSetDevice(c.device);
    c.mlp = m;
    if (m && !c.featX) {
        PG_CUDA(cudaMalloc((void**)&c.featX, 16 * (size_t)c.n_nodes * sizeof(float)));
        PG_CUDA(cudaMalloc((void**)&c.featY, 2 * (size_t)c.n_nodes * sizeof(float)));
    }
    return PG_OK;
}

}  // extern "C"
