// Learned Newton warm start: per-node features, training targets and the
// application of the MLP's correction to the linear load extrapolation.
// The reference only has the zeroth-order predictor (U_f carried over,
// src/SolverNonlinear.cpp:254-267); this is new.
//
// For a step from load factor t_n to t_{n+1} with ratio = dt_{n+1} / dt_n:
//   U_lin  = U_n + ratio (U_n - U_{n-1})                (free DOFs)
//   U_pred = U_lin + s * MLP(features)                  s = prescribed increment of the step
// Features of node i (16): the last increment / s (2), U_n / app (2),
// normalised position (2), enrichment / mirror flags (2), the largest
// committed opening over the node's cohesive points / delta_ref (1), load
// factor (1), ratio (1), Dirichlet flags (2), |last increment| / s (1),
// a constant 1 (1), 0 (1).  Targets: (U_{n+1} - U_lin) / s.
#include <cmath>

#include "pg_internal.cuh"
#include "pg_solve_kernels.cuh"

namespace pgb {

namespace {
inline int nblk(int n) { return (n + kThreads - 1) / kThreads; }
}

__global__ void k_features(int n, int n_reg, int n_enr_initial, const uint8_t* __restrict__ fixed,
                           const double* __restrict__ x, const double* __restrict__ y, double x0, double xs, double y0,
                           double ys, const double* __restrict__ Un, const double* __restrict__ Unm1, double s_inc,
                           double app, double t_frac, double ratio, const double* __restrict__ isv_c,
                           const int* __restrict__ nq_ptr, const int* __restrict__ nq_list, double delta_ref,
                           float* __restrict__ X) {
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i >= n) return;
    const double dux = Un[2 * i] - Unm1[2 * i], duy = Un[2 * i + 1] - Unm1[2 * i + 1];
    double dmg = 0.0;
    if (nq_ptr)
        for (int k = nq_ptr[i]; k < nq_ptr[i + 1]; ++k) dmg = fmax(dmg, isv_c[nq_list[k]]);
    float f[16];
    f[0] = (float)(dux / s_inc);
    f[1] = (float)(duy / s_inc);
    f[2] = (float)(Un[2 * i] / app);
    f[3] = (float)(Un[2 * i + 1] / app);
    f[4] = (float)((x[i] - x0) / xs);
    f[5] = (float)((y[i] - y0) / ys);
    f[6] = i >= n_reg ? 1.f : 0.f;
    f[7] = i >= n_reg + n_enr_initial ? 1.f : 0.f;
    f[8] = (float)fmin(dmg / delta_ref, 50.0);
    f[9] = (float)t_frac;
    f[10] = (float)ratio;
    f[11] = fixed[2 * i] ? 1.f : 0.f;
    f[12] = fixed[2 * i + 1] ? 1.f : 0.f;
    f[13] = (float)(sqrt(dux * dux + duy * duy) / s_inc);
    f[14] = 1.f;
    f[15] = 0.f;
    float4* o = reinterpret_cast<float4*>(X + 16 * (size_t)i);
    o[0] = make_float4(f[0], f[1], f[2], f[3]);
    o[1] = make_float4(f[4], f[5], f[6], f[7]);
    o[2] = make_float4(f[8], f[9], f[10], f[11]);
    o[3] = make_float4(f[12], f[13], f[14], f[15]);
}

__global__ void k_targets(int nd, const uint8_t* __restrict__ fixed, const double* __restrict__ Un1,
                          const double* __restrict__ Un, const double* __restrict__ Unm1, double ratio, double s_inc,
                          float* __restrict__ T) {
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i >= nd) return;
    const double lin = Un[i] + ratio * (Un[i] - Unm1[i]);
    T[i] = fixed[i] ? 0.f : (float)((Un1[i] - lin) / s_inc);
}

// gate (features, may be null): the correction is applied only at nodes that
// are enrichment nodes or carry cohesive damage (features 6 and 8); in the
// elastic bulk the linear extrapolation is already close, and any network
// output there only adds error.
__global__ void k_apply(int nd, const uint8_t* __restrict__ fixed, const double* __restrict__ Un,
                        const double* __restrict__ Unm1, double ratio, double s_inc, const float* __restrict__ Y,
                        const float* __restrict__ gate, double* __restrict__ U) {
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i >= nd || fixed[i]) return;
    bool on = Y != nullptr;
    if (on && gate) {
        const float* f = gate + 16 * (size_t)(i >> 1);
        on = f[6] > 0.5f || f[8] > 0.f;
    }
    U[i] = Un[i] + ratio * (Un[i] - Unm1[i]) + (on ? s_inc * (double)Y[i] : 0.0);
}

// node -> cohesive quadrature points (for the damage feature)
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
    PG_CUDA(cudaMemcpy(c.nq_ptr, ptr.data(), ptr.size() * sizeof(int), cudaMemcpyHostToDevice));
    PG_CUDA(cudaMalloc((void**)&c.nq_list, std::max<size_t>(1, list.size()) * sizeof(int)));
    if (!list.empty()) PG_CUDA(cudaMemcpy(c.nq_list, list.data(), list.size() * sizeof(int), cudaMemcpyHostToDevice));
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

int launch_features(Ctx& c, const double* Un, const double* Unm1, double t_frac, double ratio, double s_inc, float* X,
                    cudaStream_t s) {
    int rc = build_node_qp_map(c);
    if (rc) return rc;
    const RveSpec& sp = c.hm.spec;
    k_features<<<nblk(c.n_nodes), kThreads, 0, s>>>(
        c.n_nodes, c.n_reg, c.hm.n_enr_initial, c.fixed, c.x, c.y, sp.x0, sp.x1 - sp.x0, sp.y0, sp.y1 - sp.y0, Un,
        Unm1, s_inc, predictor_app(c), t_frac, ratio, c.isv_c, c.nq_ptr, c.nq_list, predictor_delta_ref(c), X);
    PG_CUDA(cudaGetLastError());
    return PG_OK;
}

int launch_apply(Ctx& c, const double* Un, const double* Unm1, double ratio, double s_inc, const float* Y, double* U,
                 cudaStream_t s, const float* gate) {
    k_apply<<<nblk(c.n_dof), kThreads, 0, s>>>(c.n_dof, c.fixed, Un, Unm1, ratio, s_inc, Y, gate, U);
    PG_CUDA(cudaGetLastError());
    return PG_OK;
}

}  // namespace pgb

using namespace pgb;

extern "C" {

int pg_predictor_features(pg_ctx* cx, const double* Un, const double* Unm1, double t_frac, double ratio, double s_inc,
                          float* X_dev) {
    if (!cx || !Un || !Unm1 || !X_dev || s_inc == 0.0) { set_error("pg_predictor_features: bad argument"); return PG_ERR_ARG; }
    Ctx& c = cx->c;
    cudaSetDevice(c.device);
    return launch_features(c, Un, Unm1, t_frac, ratio, s_inc, X_dev, c.stream);
}

int pg_predictor_targets(pg_ctx* cx, const double* Un1, const double* Un, const double* Unm1, double ratio,
                         double s_inc, float* T_dev) {
    if (!cx || !Un1 || !Un || !Unm1 || !T_dev || s_inc == 0.0) { set_error("pg_predictor_targets: bad argument"); return PG_ERR_ARG; }
    Ctx& c = cx->c;
    cudaSetDevice(c.device);
    k_targets<<<nblk(c.n_dof), kThreads, 0, c.stream>>>(c.n_dof, c.fixed, Un1, Un, Unm1, ratio, s_inc, T_dev);
    PG_CUDA(cudaGetLastError());
    return PG_OK;
}

int pg_predictor_apply(pg_ctx* cx, const double* Un, const double* Unm1, double ratio, double s_inc, const float* Y_dev,
                       double* U_dev) {
    if (!cx || !Un || !Unm1 || !U_dev) { set_error("pg_predictor_apply: bad argument"); return PG_ERR_ARG; }
    Ctx& c = cx->c;
    cudaSetDevice(c.device);
    return launch_apply(c, Un, Unm1, ratio, s_inc, Y_dev, U_dev, c.stream);
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
