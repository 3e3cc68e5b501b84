// Adjoint shape sensitivity of the homogenised stiffness C_11 with respect to
// the inclusion radii (sm_100a).
//
// Reference:
//   Circle_Inclusion::getIntersectionVelocity           src/InclusionCircle.cpp:176-196
//   SensitivityShapeParameter::compute_velocity         src/SensitivityShapeParameter.cpp
//   SensitivityShapeParameterStructural::Kernel*        src/SensitivityShapeParameterStructural.cpp:18-230
//   SensitivityAdjoint::solveProblem                    src/SensitivityAdjoint.cpp:23-63
//   SensitivityRightLoad::evaluate / assemble_dfdUf     src/SensitivityRightLoad.cpp:32-125
//
// The function is f = L . P_int(U): the x reaction summed over the right
// edge and divided by the height (mean sigma_xx there), C_11 = f / strain.
// At equilibrium R_f(U, r) = P_int,f = 0, so
//     df/dr_i = sum_e (L - lambda)_e . dP_e/dr_i,   K_ff lambda_f = (dF/dU_f)^T = (K L)_f,
// with lambda zero on prescribed DOFs and L zero on free ones.  Only cut
// elements depend on a radius: their enrichment nodes slide along their
// parent edges with the velocity v = d r / ((x - c) . d) (d the edge vector,
// x the node, c the centre), mirror nodes with their originals.  dP_e/dr_i
// is the central difference of the element's internal force under a move of
// its inclusion-i enrichment nodes by +-h v (h = h_rel * r_i), at fixed U and
// fixed committed cohesive state; the cut-element kernel evaluates both
// moves and dots them with (L - lambda) in place (no dP/dr vector is stored).
// The reference differentiates B and the quadrature weights analytically; the
// element-level central difference agrees with it to O(h^2).
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
    double* vel = nullptr;
    double* radius = nullptr;
    double* L = nullptr;
    double* w = nullptr;
    double* sens = nullptr;
    std::vector<double> hL;
};

int sens_setup(Ctx& c, SensData& d) {
    const HostMesh& m = c.hm;
    const int nn = m.n_nodes();
    d.n_inc = (int)m.spec.inclusions.size();
    std::vector<int> inc(nn, -1);
    std::vector<double> vel(2 * (size_t)nn, 0.0), rad(std::max(1, d.n_inc), 0.0);
    for (int i = 0; i < d.n_inc; ++i) rad[i] = m.spec.inclusions[i].r;
    for (int k = 0; k < m.n_enr; ++k) {
        const int node = m.n_reg + k, ic = m.enr_inc[k];
        const int na = m.enr_edge[2 * k], nbn = m.enr_edge[2 * k + 1];
        if (ic < 0 || ic >= d.n_inc) continue;
        const Inclusion& I = m.spec.inclusions[ic];
        const double dx = m.x[nbn] - m.x[na], dy = m.y[nbn] - m.y[na];
        const double den = (m.x[node] - I.cx) * dx + (m.y[node] - I.cy) * dy;
        if (den == 0.0) continue;  // tangent edge: the node does not move to first order
        inc[node] = ic;
        vel[2 * (size_t)node] = dx * I.r / den;
        vel[2 * (size_t)node + 1] = dy * I.r / den;
    }
    // right edge, x direction: 1 / height
    d.hL.assign(2 * (size_t)nn, 0.0);
    const int nx = m.spec.nx, ny = m.spec.ny;
    const double H = m.spec.y1 - m.spec.y0;
    for (int j = 0; j <= ny; ++j) d.hL[2 * (size_t)(nx + j * (nx + 1))] = 1.0 / H;
    PG_CUDA(cudaMalloc((void**)&d.node_inc, nn * sizeof(int)));
    PG_CUDA(cudaMalloc((void**)&d.vel, vel.size() * sizeof(double)));
    PG_CUDA(cudaMalloc((void**)&d.radius, rad.size() * sizeof(double)));
    PG_CUDA(cudaMalloc((void**)&d.L, d.hL.size() * sizeof(double)));
    PG_CUDA(cudaMalloc((void**)&d.w, d.hL.size() * sizeof(double)));
    PG_CUDA(cudaMalloc((void**)&d.sens, rad.size() * sizeof(double)));
    PG_CUDA(cudaMemcpy(d.node_inc, inc.data(), nn * sizeof(int), cudaMemcpyHostToDevice));
    PG_CUDA(cudaMemcpy(d.vel, vel.data(), vel.size() * sizeof(double), cudaMemcpyHostToDevice));
    PG_CUDA(cudaMemcpy(d.radius, rad.data(), rad.size() * sizeof(double), cudaMemcpyHostToDevice));
    PG_CUDA(cudaMemcpy(d.L, d.hL.data(), d.hL.size() * sizeof(double), cudaMemcpyHostToDevice));
    return PG_OK;
}

void sens_free(SensData& d) {
    for (void* p : {(void*)d.node_inc, (void*)d.vel, (void*)d.radius, (void*)d.L, (void*)d.w, (void*)d.sens})
        if (p) cudaFree(p);
}

}  // namespace
}  // namespace pgb

using namespace pgb;

extern "C" int pg_sensitivity_c11(pg_ctx* cx, const pg_solver_cfg* cfg, double h_rel, double* c11, double* dc11_dr,
                                  pg_solve_stats* adjoint_stats) {
    if (!cx || !cfg || !(h_rel > 0.0)) {
        set_error("pg_sensitivity_c11: invalid argument");
        return PG_ERR_ARG;
    }
    Ctx& c = cx->c;
    cudaSetDevice(c.device);
    if (c.hm.spec.nx <= 0) {
        set_error("pg_sensitivity_c11: needs a single RVE on a structured grid");
        return PG_ERR_ARG;
    }
    cudaStream_t s = c.stream;
    const int nd = c.n_dof;
    const double strain = c.hm.spec.strain * c.t_frac;
    if (strain == 0.0) {
        set_error("pg_sensitivity_c11: zero applied strain");
        return PG_ERR_ARG;
    }
    SensData d;
    int rc = sens_setup(c, d);
    if (rc != PG_OK) {
        sens_free(d);
        return rc;
    }
    // f = L . P_int(U) and the tangent at U (committed cohesive state)
    cudaMemsetAsync(c.F, 0, (size_t)nd * sizeof(double), s);
    launch_assemble(c, c.U, 1.0, true, true, s);
    c.assembled = true;
    std::vector<double> F(nd);
    cudaMemcpyAsync(F.data(), c.F, (size_t)nd * sizeof(double), cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    double f = 0.0;
    for (int i = 0; i < nd; ++i) f += d.hL[i] * F[i];
    if (c11) *c11 = f / strain;
    // adjoint: mask(K) lambda = mask(K L)
    residual_into(c, s, d.L, nullptr, c.b);  // c.b = -mask(K L)
    k_scale_inplace<<<nb(nd), kThreads, 0, s>>>(nd, c.b, -1.0);
    pg_solve_stats st{};
    rc = krylov_solve(c, *cfg, st, s);
    if (adjoint_stats) *adjoint_stats = st;
    if (rc != PG_OK || st.status != PG_OK) {
        sens_free(d);
        if (rc != PG_OK) return rc;
        set_error("pg_sensitivity_c11: adjoint solve did not converge");
        return st.status;
    }
    k_sens_weight<<<nb(nd), kThreads, 0, s>>>(nd, c.fixed, d.L, c.dx, d.w);
    cudaMemsetAsync(d.sens, 0, std::max(1, d.n_inc) * sizeof(double), s);
    CutArgs ca = cut_args(c, c.U, 1.0);
    ca.node_inc = d.node_inc;
    ca.vel = d.vel;
    ca.wsens = d.w;
    ca.radius = d.radius;
    ca.sens = d.sens;
    ca.h_rel = h_rel;
    // an element touches at most three inclusions (one per cut edge)
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
