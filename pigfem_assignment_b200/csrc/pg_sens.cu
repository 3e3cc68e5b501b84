// Adjoint shape sensitivity of the right-edge load (the homogenised stress
// sigma_11, and C_11 = sigma_11 / strain) with respect to the inclusions'
// centres and radii (sm_100a).
//
// Reference:
//   Circle_Inclusion::getIntersectionVelocity           src/InclusionCircle.cpp:176-196
//   SensitivityShapeParameter::compute_velocity         src/SensitivityShapeParameter.cpp:47-80
//   SensitivityShapeParameterStructural::Kernel*        src/SensitivityShapeParameterStructural.cpp:18-230
//   SensitivityAdjoint::solveProblem                    src/SensitivityAdjoint.cpp:23-63
//   SensitivityRightLoad::evaluate / assemble_dfdUf     src/SensitivityRightLoad.cpp:32-125
//   Problem::addShapeSensitivityParameter (X, Y, R)     src/Problem.cpp:856-861, InclusionCircle.cpp:200-227
//
// The function is f = L . P_int(U): the x reaction summed over the right
// edge and divided by the height (mean sigma_xx there).  At equilibrium
// R_f(U, d) = P_int,f = 0, so
//     df/dd = sum_e (L - lambda)_e . dP_e/dd,   K_ff lambda_f = (dF/dU_f)^T = (K L)_f,
// with lambda zero on prescribed DOFs and L zero on free ones.  Only cut
// elements depend on a shape parameter: their enrichment nodes slide along
// their parent edges with the velocity v = e s / ((x - c) . e) (e the edge
// vector, x the node, c the centre; s = r for the radius, x - c_x or
// y - c_y for the centre's coordinates), mirror nodes with their originals.
// dP_e/dd is formed analytically on the device (k_cut_sens_ad: forward-mode
// derivatives of the quadrature rows along v, at fixed U and fixed committed
// cohesive state) and dotted with (L - lambda) in place.  A central
// difference of the element force under moves of +-h v (k_cut_sens, h =
// h_rel r) remains as a cross-check of the radius derivatives.
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "pg_solve_kernels.cuh"
#include "pigfem_b200.h"

namespace pgb {
namespace {

inline int nb(int n) { return (n + kThreads - 1) / kThreads; }

// w = L on prescribed DOFs, -lambda on free ones
__global__ void k_sens_weight(int nd, const uint8_t* __restrict__ fixed, const double* __restrict__ L,
                              const double* __restrict__ lambda, double* __restrict__ w) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nd) w[i] = fixed[i] ? L[i] : -lambda[i];
}

struct SensData {
    int n_inc = 0;
    int* node_inc = nullptr;
    double* vel[3] = {nullptr, nullptr, nullptr};  // X, Y, R velocity fields (2 per node)
    double* radius = nullptr;
    double* L = nullptr;
    double* w = nullptr;
    double* sens = nullptr;
    int* param_of = nullptr;
    std::vector<double> hL;
};

int sens_setup(Ctx& c, SensData& d, int n_slots) {
    const HostMesh& m = c.hm;
    const int nn = m.n_nodes();
    d.n_inc = (int)m.spec.inclusions.size();
    std::vector<int> inc(nn, -1);
    std::vector<double> vel[3];
    for (auto& v : vel) v.assign(2 * (size_t)nn, 0.0);
    std::vector<double> rad(std::max(1, d.n_inc), 0.0);
    for (int i = 0; i < d.n_inc; ++i) rad[i] = m.spec.inclusions[i].r;
    for (int k = 0; k < m.n_enr; ++k) {
        const int node = m.n_reg + k, ic = m.enr_inc[k];
        const int na = m.enr_edge[2 * k], nbn = m.enr_edge[2 * k + 1];
        if (ic < 0 || ic >= d.n_inc) continue;
        const Inclusion& I = m.spec.inclusions[ic];
        const double dx = m.x[nbn] - m.x[na], dy = m.y[nbn] - m.y[na];
        const double px = m.x[node] - I.cx, py = m.y[node] - I.cy;
        const double den = px * dx + py * dy;
        if (den == 0.0) continue;  // tangent edge: the node does not move to first order
        inc[node] = ic;
        const double s[3] = {px, py, I.r};
        for (int kind = 0; kind < 3; ++kind) {
            vel[kind][2 * (size_t)node] = dx * s[kind] / den;
            vel[kind][2 * (size_t)node + 1] = dy * s[kind] / den;
        }
    }
    // right edge, x direction: 1 / height (SensitivityRightLoad's L / area)
    d.hL.assign(2 * (size_t)nn, 0.0);
    const int nx = m.spec.nx, ny = m.spec.ny;
    const double H = m.spec.y1 - m.spec.y0;
    for (int j = 0; j <= ny; ++j) d.hL[2 * (size_t)(nx + j * (nx + 1))] = 1.0 / H;
    PG_CUDA(cudaMalloc((void**)&d.node_inc, nn * sizeof(int)));
    for (int kind = 0; kind < 3; ++kind) {
        PG_CUDA(cudaMalloc((void**)&d.vel[kind], vel[kind].size() * sizeof(double)));
        PG_CUDA(h2d_sync(d.vel[kind], vel[kind].data(), vel[kind].size() * sizeof(double)));
    }
    PG_CUDA(cudaMalloc((void**)&d.radius, rad.size() * sizeof(double)));
    PG_CUDA(cudaMalloc((void**)&d.L, d.hL.size() * sizeof(double)));
    PG_CUDA(cudaMalloc((void**)&d.w, d.hL.size() * sizeof(double)));
    PG_CUDA(cudaMalloc((void**)&d.sens, std::max(1, n_slots) * sizeof(double)));
    PG_CUDA(cudaMalloc((void**)&d.param_of, 3 * (size_t)std::max(1, d.n_inc) * sizeof(int)));
    PG_CUDA(h2d_sync(d.node_inc, inc.data(), nn * sizeof(int)));
    PG_CUDA(h2d_sync(d.radius, rad.data(), rad.size() * sizeof(double)));
    PG_CUDA(h2d_sync(d.L, d.hL.data(), d.hL.size() * sizeof(double)));
    return PG_OK;
}

void sens_free(SensData& d) {
    for (void* p : {(void*)d.node_inc, (void*)d.vel[0], (void*)d.vel[1], (void*)d.vel[2], (void*)d.radius,
                    (void*)d.L, (void*)d.w, (void*)d.sens, (void*)d.param_of})
        if (p) cudaFree(p);
}

// f and the adjoint weights w = L - lambda at the context's U (committed
// cohesive state); leaves the tangent assembled
int sens_adjoint(Ctx& c, const pg_solver_cfg& cfg, SensData& d, double& f, pg_solve_stats& st, cudaStream_t s) {
    const int nd = c.n_dof;
    cudaMemsetAsync(c.F, 0, (size_t)nd * sizeof(double), s);
    launch_assemble(c, c.U, 1.0, true, true, s);
    c.assembled = true;
    std::vector<double> F(nd);
    PG_CUDA(cudaMemcpyAsync(F.data(), c.F, (size_t)nd * sizeof(double), cudaMemcpyDeviceToHost, s));
    PG_CUDA(cudaStreamSynchronize(s));
    f = 0.0;
    for (int i = 0; i < nd; ++i) f += d.hL[i] * F[i];
    // adjoint: mask(K) lambda = mask(K L)
    residual_into(c, s, d.L, nullptr, c.b);  // c.b = -mask(K L)
    k_scale_inplace<<<nb(nd), kThreads, 0, s>>>(nd, c.b, -1.0);
    st = pg_solve_stats{};
    int rc = krylov_solve(c, cfg, st, s);
    if (rc != PG_OK) return rc;
    if (st.status != PG_OK) {
        set_error("shape sensitivity: adjoint solve did not converge");
        return st.status;
    }
    k_sens_weight<<<nb(nd), kThreads, 0, s>>>(nd, c.fixed, d.L, c.dx, d.w);
    return PG_OK;
}

int sens_prologue(pg_ctx* cx, const pg_solver_cfg* cfg, const char* who) {
    if (!cx || !cfg) {
        set_error(std::string(who) + ": invalid argument");
        return PG_ERR_ARG;
    }
    Ctx& c = cx->c;
    cudaSetDevice(c.device);
    if (c.hm.spec.nx <= 0 || c.hm.grids.size() != 1) {
        set_error(std::string(who) + ": needs a single RVE on a structured grid");
        return PG_ERR_ARG;
    }
    return PG_OK;
}

}  // namespace
}  // namespace pgb

using namespace pgb;

extern "C" int pg_sensitivity_shape(pg_ctx* cx, const pg_solver_cfg* cfg, int32_t n_params, const int32_t* inclusion,
                                    const int32_t* kind, double* f_out, double* dfdp, pg_solve_stats* adjoint_stats) {
    int rc = sens_prologue(cx, cfg, "pg_sensitivity_shape");
    if (rc != PG_OK) return rc;
    Ctx& c = cx->c;
    const int n_inc = (int)c.hm.spec.inclusions.size();
    if (n_params < 0 || (n_params > 0 && (!inclusion || !kind))) {
        set_error("pg_sensitivity_shape: invalid parameter list");
        return PG_ERR_ARG;
    }
    // slot of each distinct (inclusion, kind); repeated parameters share one
    std::vector<int> param_of(3 * (size_t)std::max(1, n_inc), -1), slot(n_params);
    int n_slots = 0;
    for (int p = 0; p < n_params; ++p) {
        if (inclusion[p] < 0 || inclusion[p] >= n_inc || kind[p] < PG_SHAPE_X || kind[p] > PG_SHAPE_R) {
            set_error("pg_sensitivity_shape: parameter " + std::to_string(p) + " names no inclusion centre or radius");
            return PG_ERR_ARG;
        }
        int& sl = param_of[3 * (size_t)inclusion[p] + kind[p]];
        if (sl < 0) sl = n_slots++;
        slot[p] = sl;
    }
    cudaStream_t s = c.stream;
    SensData d;
    rc = sens_setup(c, d, n_slots);
    double f = 0.0;
    pg_solve_stats st{};
    if (rc == PG_OK) rc = sens_adjoint(c, *cfg, d, f, st, s);
    if (adjoint_stats) *adjoint_stats = st;
    if (rc != PG_OK) {
        sens_free(d);
        return rc;
    }
    if (f_out) *f_out = f;
    std::vector<double> hs(std::max(1, n_slots), 0.0);
    if (n_slots > 0 && c.n_cut > 0) {
        cudaMemcpyAsync(d.param_of, param_of.data(), param_of.size() * sizeof(int), cudaMemcpyHostToDevice, s);
        cudaMemsetAsync(d.sens, 0, n_slots * sizeof(double), s);
        CutArgs ca = cut_args(c, c.U, 1.0);
        ca.node_inc = d.node_inc;
        ca.wsens = d.w;
        ca.radius = d.radius;
        ca.sens = d.sens;
        ca.param_of = d.param_of;
        for (int k = 0; k < 3; ++k) {
            bool used = false;
            for (int i = 0; i < n_inc && !used; ++i) used = param_of[3 * (size_t)i + k] >= 0;
            if (!used) continue;
            ca.kind = k;
            ca.vel = d.vel[k];
            // an element touches at most three inclusions (one per cut edge)
            for (int which = 0; which < 3; ++which) {
                ca.which = which;
                launch_cut_sens_ad(c, ca, s);
            }
        }
        cudaMemcpyAsync(hs.data(), d.sens, n_slots * sizeof(double), cudaMemcpyDeviceToHost, s);
    }
    const cudaError_t e = cudaStreamSynchronize(s);
    sens_free(d);
    if (e != cudaSuccess) return cuda_fail(e, "pg_sensitivity_shape");
    PG_CUDA(cudaGetLastError());
    if (dfdp)
        for (int p = 0; p < n_params; ++p) dfdp[p] = hs[slot[p]];
    return PG_OK;
}

extern "C" int pg_sensitivity_c11(pg_ctx* cx, const pg_solver_cfg* cfg, double h_rel, double* c11, double* dc11_dr,
                                  pg_solve_stats* adjoint_stats) {
    int rc = sens_prologue(cx, cfg, "pg_sensitivity_c11");
    if (rc != PG_OK) return rc;
    if (!(h_rel >= 0.0)) {
        set_error("pg_sensitivity_c11: h_rel must be 0 (analytic) or positive (central difference)");
        return PG_ERR_ARG;
    }
    Ctx& c = cx->c;
    const double strain = c.hm.spec.strain * c.t_frac;
    if (strain == 0.0) {
        set_error("pg_sensitivity_c11: zero applied strain");
        return PG_ERR_ARG;
    }
    const int n_inc = (int)c.hm.spec.inclusions.size();
    if (h_rel == 0.0) {
        std::vector<int32_t> inc(n_inc), kind(n_inc, PG_SHAPE_R);
        for (int i = 0; i < n_inc; ++i) inc[i] = i;
        std::vector<double> g(std::max(1, n_inc));
        double f = 0.0;
        rc = pg_sensitivity_shape(cx, cfg, n_inc, inc.data(), kind.data(), &f, g.data(), adjoint_stats);
        if (rc != PG_OK) return rc;
        if (c11) *c11 = f / strain;
        if (dc11_dr)
            for (int i = 0; i < n_inc; ++i) dc11_dr[i] = g[i] / strain;
        return PG_OK;
    }
    // central difference of each cut element's internal force (cross-check)
    cudaStream_t s = c.stream;
    SensData d;
    rc = sens_setup(c, d, n_inc);
    double f = 0.0;
    pg_solve_stats st{};
    if (rc == PG_OK) rc = sens_adjoint(c, *cfg, d, f, st, s);
    if (adjoint_stats) *adjoint_stats = st;
    if (rc != PG_OK) {
        sens_free(d);
        return rc;
    }
    if (c11) *c11 = f / strain;
    cudaMemsetAsync(d.sens, 0, std::max(1, d.n_inc) * sizeof(double), s);
    CutArgs ca = cut_args(c, c.U, 1.0);
    ca.node_inc = d.node_inc;
    ca.vel = d.vel[PG_SHAPE_R];
    ca.wsens = d.w;
    ca.radius = d.radius;
    ca.sens = d.sens;
    ca.h_rel = h_rel;
    for (int which = 0; which < 3; ++which)
        for (double sgn : {1.0, -1.0}) {
            ca.which = which;
            ca.sgn = sgn;
            if (c.n_cut > 0) launch_cut_sens(c, ca, s);
        }
    PG_CUDA(cudaGetLastError());
    std::vector<double> hs(std::max(1, d.n_inc));
    cudaMemcpyAsync(hs.data(), d.sens, hs.size() * sizeof(double), cudaMemcpyDeviceToHost, s);
    const cudaError_t e = cudaStreamSynchronize(s);
    sens_free(d);
    if (e != cudaSuccess) return cuda_fail(e, "pg_sensitivity_c11");
    if (dc11_dr)
        for (int i = 0; i < d.n_inc; ++i) dc11_dr[i] = hs[i] / strain;
    return PG_OK;
}
