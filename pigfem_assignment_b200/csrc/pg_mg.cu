// Geometric multigrid preconditioner for the IGFEM system (sm_100a).
//
// The reference factors K_ff directly (MUMPS through PETSc,
// src/Solver.cpp:56-142); on the GPU the masked system is solved by CG whose
// preconditioner is one V-cycle over the structured background grid:
//   level 0     the IGFEM system itself (2x2-block CSR, regular + enrichment nodes)
//   level l>0   grid of ceil(n_{l-1}/2) cells per side, 9-point block stencil
// Prolongation interpolates the coarse correction bilinearly (in grid index
// space) onto the regular nodes of the finer grid and leaves enrichment
// DOFs to the smoother (their shape functions vanish at the regular nodes,
// so a smooth error lives in the regular DOFs).  Coarse operators are the
// Galerkin products P^T A P of the masked finer operator; a coarse DOF is
// fixed when the finer node at its position is fixed.  Smoothing is damped
// block Jacobi (2x2 node blocks), the coarsest grid (at most 4 cells per
// side) is solved by a dense LU with partial pivoting in one CTA.
//
// Precision: the outer CG always runs in FP64 (operator, vectors, dots and
// the returned residual).  PG_PRECISION_MIXED runs the whole V-cycle in FP32
// (FP32 copies of every level's operator and FP32 vectors); only the
// preconditioner changes, so the FP64 result and its residual are unchanged
// in kind.
//
// Every kernel a CG iteration launches returns at once after the device
// "done" flag is set, so captured graphs of several iterations may run past
// convergence without changing the result.
#include <cuda_runtime.h>

#include <algorithm>
#include <type_traits>
#include <cmath>
#include <vector>

#include "pg_solve_kernels.cuh"

namespace pgb {

namespace {

constexpr int kMgMaxLevels = 16;
constexpr int kMgCoarseCells = 4;        // coarsen until both sides have at most this many cells
constexpr int kMgCoarseMaxDof = 2 * (kMgCoarseCells + 1) * (kMgCoarseCells + 1);
constexpr int kMgNu1 = 2, kMgNu2 = 2;    // pre- and post-smoothing sweeps
constexpr double kMgOmega = 0.5;         // block-Jacobi damping: lambda_max(D^-1 K) reaches ~3.9 on IGFEM meshes

struct MgLevel {
    int nx = 0, ny = 0, n = 0;           // cells per side, nodes
    double* A = nullptr;                 // 36 per node: stencil block (dj+1)*3+(di+1), 2x2 row-major
    float* Af = nullptr;
    double* Dinv = nullptr;              // 4 per node
    float* Dinvf = nullptr;
    uint8_t* fixed = nullptr;            // 2 per node
    double *x = nullptr, *x2 = nullptr, *b = nullptr, *r = nullptr;
    float *xf = nullptr, *x2f = nullptr, *bf = nullptr, *rf = nullptr;
};

}  // namespace

struct MgHierarchy {
    int nlev = 0;                        // coarse levels 1..nlev (nlev is the coarsest)
    MgLevel L[kMgMaxLevels + 1];
    // level-0 V-cycle vectors
    double *x0 = nullptr, *x0b = nullptr, *r0 = nullptr;
    float *b0f = nullptr, *x0f = nullptr, *x0bf = nullptr, *r0f = nullptr;
    float* Dinv0f = nullptr;
    // coarsest dense LU (row-major, n_c x n_c) and pivots
    int nc = 0;
    double* LU = nullptr;
    int* piv = nullptr;
    // CG scalars: 0 pq, 1 rz, 2 rz_new, 3 rr, 4 tol2; flags: 0 done, 1 breakdown, 2 iterations, 3 coarse-singular
    double* sc = nullptr;
    int* fl = nullptr;
    // inclusion rigid modes (cohesive meshes): 3 per inclusion, supports disjoint
    int n_inc = 0;                       // 0: no mode space
    bool use_modes = false;
    int* z_inc = nullptr;                // per node: the inclusion whose modes touch it, -1 none
    double* zval = nullptr;              // per node: [d][k], 2 x 3
    double* E = nullptr;                 // per inclusion: Z_i^T K Z_i (3 x 3)
    double* Einv = nullptr;
    double* w = nullptr;                 // per inclusion: Z_i^T r (3)
    std::vector<void*> owned;
};

namespace {

// ---------------------------------------------------------------------------
// Grid transfer weights (grid index space).  Coarse index I sits at fine
// index pos(I) = min(2I, nf); nf is the finer grid's cell count.
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ int mg_pos(int I, int nf) { return 2 * I < nf ? 2 * I : nf; }

__host__ __device__ __forceinline__ double mg_w(int g, int nf, int I) {
    if ((g & 1) == 0) return (g >> 1) == I ? 1.0 : 0.0;
    if (g == nf) return I == ((nf + 1) >> 1) ? 1.0 : 0.0;
    return (I == ((g - 1) >> 1) || I == ((g + 1) >> 1)) ? 0.5 : 0.0;
}

// ---------------------------------------------------------------------------
// Set-up kernels
// ---------------------------------------------------------------------------
struct GalArgs {
    int nxf, nyf, nxc, nyc;
    // finer operator: BSR (level 0) or stencil
    const int* row_ptr;
    const int* col;
    const double* K;
    int n_reg;
    const double* A;
    const uint8_t* fixed_f;
    const uint8_t* fixed_c;
    double* Ac;
};

// Ac(a, a + o) = sum_{i child of a} sum_{j in row i} P_ia M_i A_ij M_j P_jb, masked by the coarse mask.
template <bool FINE_BSR>
__global__ void k_mg_galerkin(GalArgs g) {
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int ncn = (g.nxc + 1) * (g.nyc + 1);
    if (tid >= 9 * ncn) return;
    const int a = tid / 9, o = tid - 9 * a;
    const int Ia = a % (g.nxc + 1), Ja = a / (g.nxc + 1);
    const int Ib = Ia + (o % 3) - 1, Jb = Ja + (o / 3) - 1;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    if (Ib >= 0 && Ib <= g.nxc && Jb >= 0 && Jb <= g.nyc) {
        const int px = mg_pos(Ia, g.nxf), py = mg_pos(Ja, g.nyf);
        for (int cy = py - 1; cy <= py + 1; ++cy) {
            if (cy < 0 || cy > g.nyf) continue;
            const double wy = mg_w(cy, g.nyf, Ja);
            if (wy == 0.0) continue;
            for (int cx = px - 1; cx <= px + 1; ++cx) {
                if (cx < 0 || cx > g.nxf) continue;
                const double wx = mg_w(cx, g.nxf, Ia);
                if (wx == 0.0) continue;
                const int i = cx + cy * (g.nxf + 1);
                const double wi = wx * wy;
                const bool fi0 = !g.fixed_f[2 * i], fi1 = !g.fixed_f[2 * i + 1];
                if (FINE_BSR) {
                    for (int q = g.row_ptr[i]; q < g.row_ptr[i + 1]; ++q) {
                        const int j = g.col[q];
                        if (j >= g.n_reg) continue;
                        const int gx = j % (g.nxf + 1), gy = j / (g.nxf + 1);
                        const double wj = mg_w(gx, g.nxf, Ib) * mg_w(gy, g.nyf, Jb);
                        if (wj == 0.0) continue;
                        const bool fj0 = !g.fixed_f[2 * j], fj1 = !g.fixed_f[2 * j + 1];
                        const double* blk = g.K + 4 * (size_t)q;
                        const double w = wi * wj;
                        if (fi0 && fj0) acc[0] += w * blk[0];
                        if (fi0 && fj1) acc[1] += w * blk[1];
                        if (fi1 && fj0) acc[2] += w * blk[2];
                        if (fi1 && fj1) acc[3] += w * blk[3];
                    }
                } else {
                    for (int s = 0; s < 9; ++s) {
                        const int gx = cx + (s % 3) - 1, gy = cy + (s / 3) - 1;
                        if (gx < 0 || gx > g.nxf || gy < 0 || gy > g.nyf) continue;
                        const double wj = mg_w(gx, g.nxf, Ib) * mg_w(gy, g.nyf, Jb);
                        if (wj == 0.0) continue;
                        const int j = gx + gy * (g.nxf + 1);
                        const bool fj0 = !g.fixed_f[2 * j], fj1 = !g.fixed_f[2 * j + 1];
                        const double* blk = g.A + 36 * (size_t)i + 4 * s;
                        const double w = wi * wj;
                        if (fi0 && fj0) acc[0] += w * blk[0];
                        if (fi0 && fj1) acc[1] += w * blk[1];
                        if (fi1 && fj0) acc[2] += w * blk[2];
                        if (fi1 && fj1) acc[3] += w * blk[3];
                    }
                }
            }
        }
        const int b = Ib + Jb * (g.nxc + 1);
        if (g.fixed_c[2 * a]) acc[0] = acc[1] = 0.0;
        if (g.fixed_c[2 * a + 1]) acc[2] = acc[3] = 0.0;
        if (g.fixed_c[2 * b]) acc[0] = acc[2] = 0.0;
        if (g.fixed_c[2 * b + 1]) acc[1] = acc[3] = 0.0;
    }
    double* out = g.Ac + 36 * (size_t)a + 4 * o;
    for (int k = 0; k < 4; ++k) out[k] = acc[k];
}

// Coarse mask by injection: the coarse node takes the mask of the finer node at its position.
__global__ void k_mg_inject_mask(int nxf, int nxc, int nyc, int nyf, const uint8_t* fixed_f, uint8_t* fixed_c) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= (nxc + 1) * (nyc + 1)) return;
    const int I = a % (nxc + 1), J = a / (nxc + 1);
    const int i = mg_pos(I, nxf) + mg_pos(J, nyf) * (nxf + 1);
    fixed_c[2 * a] = fixed_f[2 * i];
    fixed_c[2 * a + 1] = fixed_f[2 * i + 1];
}

// Inverse of each node's masked diagonal block (stencil centre), as k_prec_setup does for level 0.
__global__ void k_mg_dinv(int n, const double* A, const uint8_t* fixed, double* Dinv, float* Dinvf) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double* b = A + 36 * (size_t)i + 16;
    const bool f0 = fixed[2 * i], f1 = fixed[2 * i + 1];
    double m[4] = {0.0, 0.0, 0.0, 0.0};
    if (!f0 && !f1) {
        const double det = b[0] * b[3] - b[1] * b[2];
        if (det != 0.0) {
            m[0] = b[3] / det;
            m[1] = -b[1] / det;
            m[2] = -b[2] / det;
            m[3] = b[0] / det;
        }
    } else {
        m[0] = (f0 || b[0] == 0.0) ? 0.0 : 1.0 / b[0];
        m[3] = (f1 || b[3] == 0.0) ? 0.0 : 1.0 / b[3];
    }
    for (int k = 0; k < 4; ++k) {
        Dinv[4 * (size_t)i + k] = m[k];
        if (Dinvf) Dinvf[4 * (size_t)i + k] = (float)m[k];
    }
}

__global__ void k_mg_to_f32(size_t n, const double* a, float* b) {
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i < n) b[i] = (float)a[i];
}

// Dense LU with partial pivoting of the coarsest operator, one CTA.
// Fixed DOFs get identity rows and columns.  fl[3] = 1 on a zero pivot.
__global__ void k_mg_coarse_factor(int nx, int ny, const double* A, const uint8_t* fixed, double* LU, int* piv,
                                   int* fl) {
    __shared__ double M[kMgCoarseMaxDof][kMgCoarseMaxDof + 1];
    __shared__ int sp[kMgCoarseMaxDof];
    __shared__ int s_pivot;
    const int nn = (nx + 1) * (ny + 1), n = 2 * nn;
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) M[e / n][e % n] = 0.0;
    __syncthreads();
    for (int t = threadIdx.x; t < 9 * nn; t += blockDim.x) {
        const int a = t / 9, o = t - 9 * a;
        const int I = a % (nx + 1) + (o % 3) - 1, J = a / (nx + 1) + (o / 3) - 1;
        if (I < 0 || I > nx || J < 0 || J > ny) continue;
        const int b = I + J * (nx + 1);
        const double* blk = A + 36 * (size_t)a + 4 * o;
        for (int d = 0; d < 2; ++d)
            for (int f = 0; f < 2; ++f)
                if (!fixed[2 * a + d] && !fixed[2 * b + f]) M[2 * a + d][2 * b + f] = blk[2 * d + f];
    }
    __syncthreads();
    for (int r = threadIdx.x; r < n; r += blockDim.x) {
        if (fixed[r]) M[r][r] = 1.0;
        sp[r] = r;
    }
    __syncthreads();
    for (int k = 0; k < n; ++k) {
        if (threadIdx.x == 0) {
            int best = k;
            for (int r = k + 1; r < n; ++r)
                if (fabs(M[r][k]) > fabs(M[best][k])) best = r;
            s_pivot = best;
            if (M[best][k] == 0.0) fl[3] = 1;
        }
        __syncthreads();
        const int pr = s_pivot;
        if (pr != k) {
            for (int c2 = threadIdx.x; c2 < n; c2 += blockDim.x) {
                const double t2 = M[k][c2];
                M[k][c2] = M[pr][c2];
                M[pr][c2] = t2;
            }
            if (threadIdx.x == 0) {
                const int t3 = sp[k];
                sp[k] = sp[pr];
                sp[pr] = t3;
            }
        }
        __syncthreads();
        const double d = M[k][k];
        for (int r = k + 1 + threadIdx.x; r < n; r += blockDim.x)
            if (d != 0.0) M[r][k] /= d;
        __syncthreads();
        for (int e = threadIdx.x; e < (n - k - 1) * (n - k - 1); e += blockDim.x) {
            const int r = k + 1 + e / (n - k - 1), c2 = k + 1 + e % (n - k - 1);
            M[r][c2] -= M[r][k] * M[k][c2];
        }
        __syncthreads();
    }
    // The coarse solve runs once per V-cycle; two substitutions of n steps,
    // each behind a barrier, cost tens of microseconds.  So the inverse is
    // formed here (column j solves L U x = P e_j, one thread per column) and
    // stored transposed in LU (LU[j n + r] = X[r][j]), with the rows and
    // columns of fixed DOFs zeroed: the solve is then one matrix-vector product.
    __shared__ double W[kMgCoarseMaxDof][kMgCoarseMaxDof + 1];
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        double* y = W[j];
        for (int r = 0; r < n; ++r) y[r] = (sp[r] == j && !fixed[j]) ? 1.0 : 0.0;
        for (int k = 0; k < n; ++k) {
            const double yk = y[k];
            for (int r = k + 1; r < n; ++r) y[r] -= M[r][k] * yk;
        }
        for (int k = n - 1; k >= 0; --k) {
            y[k] = M[k][k] != 0.0 ? y[k] / M[k][k] : 0.0;
            const double yk = y[k];
            for (int r = 0; r < k; ++r) y[r] -= M[r][k] * yk;
        }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
        const int j = e / n, r = e - j * n;
        LU[e] = fixed[r] ? 0.0 : W[j][r];
    }
    for (int r = threadIdx.x; r < n; r += blockDim.x) piv[r] = sp[r];
}

// ---------------------------------------------------------------------------
// V-cycle kernels (T = double or float; arithmetic in T)
// ---------------------------------------------------------------------------
// level 0: xout = xin + omega D^-1 mask(b - A xin) (xin null: zero)
template <typename T>
__global__ void __launch_bounds__(kThreads) k_mg_smooth_bsr(int n, const int* __restrict__ row_ptr,
                                                            const int* __restrict__ col, const T* __restrict__ K,
                                                            const T* __restrict__ Dinv, const uint8_t* __restrict__ fixed,
                                                            const T* __restrict__ b, const T* __restrict__ xin,
                                                            T* __restrict__ xout, T omega, const int* done, int resid_only) {
    if (done && done[0]) return;
    // kRowLanes lanes per block row (bsr_row_group); lane 0 of each group finishes the row
    const int t = blockIdx.x * kThreads + threadIdx.x;
    const int i = t / kRowLanes, g = t % kRowLanes;
    double y0 = 0.0, y1 = 0.0;
    if (xin) bsr_row_group<T, T>(i, i < n, g, row_ptr, col, K, xin, y0, y1);
    if (i >= n || g != 0) return;
    T r0 = b[2 * i], r1 = b[2 * i + 1];
    if (xin) {
        r0 -= (T)y0;
        r1 -= (T)y1;
    }
    if (fixed[2 * i]) r0 = 0;
    if (fixed[2 * i + 1]) r1 = 0;
    if (resid_only) {
        xout[2 * i] = r0;
        xout[2 * i + 1] = r1;
        return;
    }
    const T* m = Dinv + 4 * (size_t)i;
    const T z0 = m[0] * r0 + m[1] * r1, z1 = m[2] * r0 + m[3] * r1;
    xout[2 * i] = (xin ? xin[2 * i] : (T)0) + omega * z0;
    xout[2 * i + 1] = (xin ? xin[2 * i + 1] : (T)0) + omega * z1;
}

// GLOBAL: A and Dinv are in global memory and read as whole 2x2 blocks
// (load_block); otherwise (shared memory) element by element.
template <typename T, bool GLOBAL>
__device__ __forceinline__ void mg_smooth_node(int i, int nx, int ny, const T* __restrict__ A,
                                               const T* __restrict__ Dinv, const uint8_t* __restrict__ fixed,
                                               const T* __restrict__ b, const T* __restrict__ xin, T* __restrict__ xout,
                                               T omega, int resid_only) {
    T r0 = b[2 * i], r1 = b[2 * i + 1];
    if (xin) {
        const int I = i % (nx + 1), J = i / (nx + 1);
        T y0 = 0, y1 = 0;
        for (int s = 0; s < 9; ++s) {
            const int gx = I + (s % 3) - 1, gy = J + (s / 3) - 1;
            if (gx < 0 || gx > nx || gy < 0 || gy > ny) continue;
            const int j = gx + gy * (nx + 1);
            const T* k = A + 36 * (size_t)i + 4 * s;
            T k0, k1, k2, k3;
            if constexpr (GLOBAL) {
                double d0, d1, d2, d3;
                load_block(k, d0, d1, d2, d3);
                k0 = (T)d0; k1 = (T)d1; k2 = (T)d2; k3 = (T)d3;
            } else {
                k0 = k[0]; k1 = k[1]; k2 = k[2]; k3 = k[3];
            }
            const T x0 = xin[2 * j], x1 = xin[2 * j + 1];
            y0 += k0 * x0 + k1 * x1;
            y1 += k2 * x0 + k3 * x1;
        }
        r0 -= y0;
        r1 -= y1;
    }
    if (fixed[2 * i]) r0 = 0;
    if (fixed[2 * i + 1]) r1 = 0;
    if (resid_only) {
        xout[2 * i] = r0;
        xout[2 * i + 1] = r1;
        return;
    }
    const T* m = Dinv + 4 * (size_t)i;
    T m0, m1, m2, m3;
    if constexpr (GLOBAL) {
        double d0, d1, d2, d3;
        load_block(m, d0, d1, d2, d3);
        m0 = (T)d0; m1 = (T)d1; m2 = (T)d2; m3 = (T)d3;
    } else {
        m0 = m[0]; m1 = m[1]; m2 = m[2]; m3 = m[3];
    }
    const T z0 = m0 * r0 + m1 * r1, z1 = m2 * r0 + m3 * r1;
    xout[2 * i] = (xin ? xin[2 * i] : (T)0) + omega * z0;
    xout[2 * i + 1] = (xin ? xin[2 * i + 1] : (T)0) + omega * z1;
}

template <typename T>
__global__ void __launch_bounds__(kThreads) k_mg_smooth_st(int nx, int ny, const T* __restrict__ A,
                                                           const T* __restrict__ Dinv, const uint8_t* __restrict__ fixed,
                                                           const T* __restrict__ b, const T* __restrict__ xin,
                                                           T* __restrict__ xout, T omega, const int* done, int resid_only) {
    if (done && done[0]) return;
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i >= (nx + 1) * (ny + 1)) return;
    mg_smooth_node<T, true>(i, nx, ny, A, Dinv, fixed, b, xin, xout, omega, resid_only);
}

// bc(a) = mask_c(sum_{i child of a} P_ia rf(i))
template <typename T>
__device__ __forceinline__ void mg_restrict_node(int a, int nxf, int nyf, int nxc, const T* __restrict__ rf,
                                                 const uint8_t* fixed_c, T* __restrict__ bc) {
    const int Ia = a % (nxc + 1), Ja = a / (nxc + 1);
    const int px = mg_pos(Ia, nxf), py = mg_pos(Ja, nyf);
    T s0 = 0, s1 = 0;
    for (int cy = py - 1; cy <= py + 1; ++cy) {
        if (cy < 0 || cy > nyf) continue;
        const double wy = mg_w(cy, nyf, Ja);
        if (wy == 0.0) continue;
        for (int cx = px - 1; cx <= px + 1; ++cx) {
            if (cx < 0 || cx > nxf) continue;
            const double wx = mg_w(cx, nxf, Ia);
            if (wx == 0.0) continue;
            const int i = cx + cy * (nxf + 1);
            const T w = (T)(wx * wy);
            s0 += w * rf[2 * i];
            s1 += w * rf[2 * i + 1];
        }
    }
    bc[2 * a] = fixed_c[2 * a] ? (T)0 : s0;
    bc[2 * a + 1] = fixed_c[2 * a + 1] ? (T)0 : s1;
}

template <typename T>
__global__ void k_mg_restrict(int nxf, int nyf, int nxc, int nyc, const T* __restrict__ rf, const uint8_t* fixed_c,
                              T* __restrict__ bc, const int* done) {
    if (done && done[0]) return;
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= (nxc + 1) * (nyc + 1)) return;
    mg_restrict_node(a, nxf, nyf, nxc, rf, fixed_c, bc);
}

// xf(i) += mask_f(sum_a P_ia xc(a)) over the finer grid's nodes
template <typename T>
__device__ __forceinline__ void mg_prolong_node(int i, int nxf, int nyf, int nxc, const T* __restrict__ xc,
                                                const uint8_t* fixed_f, T* __restrict__ xf) {
    const int gx = i % (nxf + 1), gy = i / (nxf + 1);
    int Ix[2], Iy[2];
    T wxs[2], wys[2];
    int nxp, nyp;
    if ((gx & 1) == 0) { Ix[0] = gx >> 1; wxs[0] = 1; nxp = 1; }
    else if (gx == nxf) { Ix[0] = (nxf + 1) >> 1; wxs[0] = 1; nxp = 1; }
    else { Ix[0] = (gx - 1) >> 1; Ix[1] = (gx + 1) >> 1; wxs[0] = wxs[1] = (T)0.5; nxp = 2; }
    if ((gy & 1) == 0) { Iy[0] = gy >> 1; wys[0] = 1; nyp = 1; }
    else if (gy == nyf) { Iy[0] = (nyf + 1) >> 1; wys[0] = 1; nyp = 1; }
    else { Iy[0] = (gy - 1) >> 1; Iy[1] = (gy + 1) >> 1; wys[0] = wys[1] = (T)0.5; nyp = 2; }
    T s0 = 0, s1 = 0;
    for (int py = 0; py < nyp; ++py)
        for (int px = 0; px < nxp; ++px) {
            const int a = Ix[px] + Iy[py] * (nxc + 1);
            const T w = wxs[px] * wys[py];
            s0 += w * xc[2 * a];
            s1 += w * xc[2 * a + 1];
        }
    if (!fixed_f[2 * i]) xf[2 * i] += s0;
    if (!fixed_f[2 * i + 1]) xf[2 * i + 1] += s1;
}

template <typename T>
__global__ void k_mg_prolong(int nxf, int nyf, int nxc, const T* __restrict__ xc, const uint8_t* fixed_f,
                             T* __restrict__ xf, const int* done) {
    if (done && done[0]) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (nxf + 1) * (nyf + 1)) return;
    mg_prolong_node(i, nxf, nyf, nxc, xc, fixed_f, xf);
}

// The bottom of the V-cycle in one launch.  Below a few hundred nodes every
// level's kernels are latency-bound (a launch of one block costs about as
// much as one of a thousand), and the V-cycle has seven of them per level.
// So the levels from `first` down to the coarsest run in one CTA, phase after
// phase between block barriers, in the same order and with the same per-node
// arithmetic as the per-level kernels: restrict the finer residual,
// pre-smooth, residual, ..., coarse solve, then prolongate and post-smooth
// back up.  Their operators, diagonal inverses and vectors are first copied
// into shared memory (one coalesced pass), so no phase waits on L2; the
// result of level `first` goes back to its x for the caller's prolongation.
// (taking the 33x33 level as well, its operators read from L2, made the bottom
// 151 us instead of 34 us per cycle: slower than that level's seven launches)
constexpr int kMgBottomNodes = 300;        // levels at most this size may run in k_mg_bottom
constexpr int kMgBottomSmem = 220 * 1024;  // and their shared-memory copy at most this many bytes
constexpr int kMgBottomThreads = 512;
constexpr int kMgBottomLevels = 8;

template <typename T>
struct MgBottomArgs {
    int nlev;                               // levels here, the last the coarsest
    int nxf, nyf;                           // grid of the finer level restricted first
    const T* rf;                            // its residual
    int nx[kMgBottomLevels], ny[kMgBottomLevels];
    const T* A[kMgBottomLevels];
    const T* Dinv[kMgBottomLevels];
    const uint8_t* fixed[kMgBottomLevels];
    int staged[kMgBottomLevels];            // 1: A and D^-1 copied into shared memory; 0: read from global (L2)
    T* x0;                                  // level `first`'s x (global): the result
    const double* XT;                       // coarsest: transposed masked inverse
    int nc;
    T omega;
};

// shared-memory bytes of k_mg_bottom for a level of n nodes: b, x, x2, r (2 n
// each) and fixed (2 n bytes, rounded to 8), and with its operator staged A
// (36 n) and D^-1 (4 n) too
template <typename T>
size_t mg_bottom_vec_bytes(int n) {
    return (size_t)8 * n * sizeof(T) + (((size_t)2 * n + 7) & ~(size_t)7);
}
template <typename T>
size_t mg_bottom_op_bytes(int n) {
    return (size_t)(36 + 4) * n * sizeof(T);
}

template <typename T>
__global__ void __launch_bounds__(kMgBottomThreads) k_mg_bottom(MgBottomArgs<T> a, const int* done) {
    if (done && done[0]) return;
    extern __shared__ __align__(16) unsigned char g_bottom_smem[];
    __shared__ double bs[kMgCoarseMaxDof];
    const int tid = threadIdx.x;
    // carve and stage
    T* sA[kMgBottomLevels];
    T* sD[kMgBottomLevels];
    T* sb[kMgBottomLevels];
    T* sx[kMgBottomLevels];
    T* sx2[kMgBottomLevels];
    T* sr[kMgBottomLevels];
    uint8_t* sf[kMgBottomLevels];
    unsigned char* p = g_bottom_smem;
    for (int k = 0; k < a.nlev; ++k) {
        const int n = (a.nx[k] + 1) * (a.ny[k] + 1);
        T* q0 = reinterpret_cast<T*>(p);
        if (a.staged[k]) {
            sA[k] = q0;
            sD[k] = sA[k] + 36 * n;
            q0 = sD[k] + 4 * n;
        } else {
            // a larger level: its operator stays in global memory (L2), only its vectors here
            sA[k] = const_cast<T*>(a.A[k]);
            sD[k] = const_cast<T*>(a.Dinv[k]);
        }
        sb[k] = q0;
        sx[k] = sb[k] + 2 * n;
        sx2[k] = sx[k] + 2 * n;
        sr[k] = sx2[k] + 2 * n;
        sf[k] = reinterpret_cast<uint8_t*>(sr[k] + 2 * n);
        p = reinterpret_cast<unsigned char*>(sf[k]) + ((2 * n + 7) & ~7);
        if (k < a.nlev - 1 && a.staged[k]) {
            for (int q = tid; q < 36 * n; q += kMgBottomThreads) sA[k][q] = a.A[k][q];
            for (int q = tid; q < 4 * n; q += kMgBottomThreads) sD[k][q] = a.Dinv[k][q];
        }
        for (int q = tid; q < 2 * n; q += kMgBottomThreads) sf[k][q] = a.fixed[k][q];
    }
    __syncthreads();
    int nxf = a.nxf, nyf = a.nyf;
    const T* rf = a.rf;
    T* xs[kMgBottomLevels];
    for (int k = 0; k < a.nlev; ++k) {
        const int nx = a.nx[k], ny = a.ny[k], n = (nx + 1) * (ny + 1);
        for (int i = tid; i < n; i += kMgBottomThreads) mg_restrict_node(i, nxf, nyf, nx, rf, sf[k], sb[k]);
        __syncthreads();
        if (k == a.nlev - 1) {
            // coarsest: x = XT^T b (fixed DOFs 0)
            for (int q = tid; q < a.nc; q += kMgBottomThreads) bs[q] = sf[k][q] ? 0.0 : (double)sb[k][q];
            __syncthreads();
            for (int q = tid; q < a.nc; q += kMgBottomThreads) {
                double acc = 0.0;
                for (int j = 0; j < a.nc; ++j) acc += a.XT[(size_t)j * a.nc + q] * bs[j];
                sx[k][q] = sf[k][q] ? (T)0 : (T)acc;
            }
            __syncthreads();
            xs[k] = sx[k];
            break;
        }
        T* lc = sx[k];
        T* la = sx2[k];
        for (int i = tid; i < n; i += kMgBottomThreads)
            mg_smooth_node<T, false>(i, nx, ny, (const T*)sA[k], (const T*)sD[k], sf[k], (const T*)sb[k], (const T*)nullptr, lc,
                           a.omega, 0);
        __syncthreads();
        for (int it = 1; it < kMgNu1; ++it) {
            for (int i = tid; i < n; i += kMgBottomThreads)
                mg_smooth_node<T, false>(i, nx, ny, (const T*)sA[k], (const T*)sD[k], sf[k], (const T*)sb[k], (const T*)lc, la,
                               a.omega, 0);
            __syncthreads();
            T* t = lc;
            lc = la;
            la = t;
        }
        for (int i = tid; i < n; i += kMgBottomThreads)
            mg_smooth_node<T, false>(i, nx, ny, (const T*)sA[k], (const T*)sD[k], sf[k], (const T*)sb[k], (const T*)lc, sr[k],
                           a.omega, 1);
        __syncthreads();
        xs[k] = lc;
        rf = sr[k];
        nxf = nx;
        nyf = ny;
    }
    for (int k = a.nlev - 2; k >= 0; --k) {
        const int nx = a.nx[k], ny = a.ny[k], n = (nx + 1) * (ny + 1);
        T* lc = xs[k];
        T* la = lc == sx[k] ? sx2[k] : sx[k];
        for (int i = tid; i < n; i += kMgBottomThreads)
            mg_prolong_node(i, nx, ny, a.nx[k + 1], (const T*)xs[k + 1], sf[k], lc);
        __syncthreads();
        for (int it = 0; it < kMgNu2; ++it) {
            for (int i = tid; i < n; i += kMgBottomThreads)
                mg_smooth_node<T, false>(i, nx, ny, (const T*)sA[k], (const T*)sD[k], sf[k], (const T*)sb[k], (const T*)lc, la,
                               a.omega, 0);
            __syncthreads();
            T* t = lc;
            lc = la;
            la = t;
        }
        xs[k] = lc;
    }
    const int n0 = 2 * (a.nx[0] + 1) * (a.ny[0] + 1);
    for (int q = tid; q < n0; q += kMgBottomThreads) a.x0[q] = xs[0][q];
}

__global__ void k_mg_f64_to_f32(int n, const double* __restrict__ a, float* __restrict__ b, const int* done) {
    if (done && done[0]) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = (float)a[i];
}

__global__ void k_mg_f32_to_f64(int n, const float* __restrict__ a, double* __restrict__ b, const int* done) {
    if (done && done[0]) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = (double)a[i];
}

// ---------------------------------------------------------------------------
// CG kernels (FP64).  Scalars: sc[0] p.q, sc[1] r.z, sc[2] new r.z, sc[3] r.r, sc[4] tol^2.
// ---------------------------------------------------------------------------
__global__ void k_mgcg_s1(double* sc, const int* fl) {
    if (fl[0]) return;
    sc[1] = sc[2];
    sc[0] = 0.0;
    sc[3] = 0.0;
}

__global__ void __launch_bounds__(kThreads) k_mgcg_spmv(int n, const int* __restrict__ row_ptr,
                                                        const int* __restrict__ col, const double* __restrict__ K,
                                                        const double* __restrict__ p, const uint8_t* __restrict__ fixed,
                                                        double* __restrict__ q, double* sc, const int* fl,
                                                        double* ws) {
    if (fl[0]) return;
    // kRowLanes lanes per block row (bsr_row_group); lane 0 of each group finishes the row
    const int t = blockIdx.x * kThreads + threadIdx.x;
    const int i = t / kRowLanes, g = t % kRowLanes;
    double part = 0.0;
    double y0, y1;
    bsr_row_group<double, double>(i, i < n, g, row_ptr, col, K, p, y0, y1);
    if (i < n && g == 0) {
        if (fixed[2 * i]) y0 = 0.0;
        if (fixed[2 * i + 1]) y1 = 0.0;
        q[2 * i] = y0;
        q[2 * i + 1] = y1;
        part = p[2 * i] * y0 + p[2 * i + 1] * y1;
    }
    const double s = block_sum(part);
    grid_add(ws, 0, s, &sc[0]);
}

__global__ void __launch_bounds__(kThreads) k_mgcg_update(int nd, double* __restrict__ x, double* __restrict__ r,
                                                          const double* __restrict__ p, const double* __restrict__ q,
                                                          double* sc, int* fl, double* ws) {
    if (fl[0]) return;
    const double pq = sc[0];
    if (!(pq > 0.0)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            fl[1] = 1;
            fl[0] = 1;
        }
        return;
    }
    const double alpha = sc[1] / pq;
    const int i = blockIdx.x * kThreads + threadIdx.x;
    double part = 0.0;
    if (i < nd) {
        x[i] += alpha * p[i];
        const double ri = r[i] - alpha * q[i];
        r[i] = ri;
        part = ri * ri;
    }
    const double s = block_sum(part);
    grid_add(ws, 1, s, &sc[3]);
}

__global__ void k_mgcg_s2(double* sc, int* fl) {
    if (fl[0]) return;
    fl[2] += 1;
    if (sc[3] <= sc[4]) fl[0] = 1;
    sc[2] = 0.0;
}

__global__ void __launch_bounds__(kThreads) k_mgcg_dot(int nd, const double* __restrict__ a, const double* __restrict__ b,
                                                       double* out, const int* fl, double* ws) {
    if (fl[0]) return;
    const int i = blockIdx.x * kThreads + threadIdx.x;
    const double v = i < nd ? a[i] * b[i] : 0.0;
    const double s = block_sum(v);
    grid_add(ws, 2, s, out);
}

__global__ void __launch_bounds__(kThreads) k_mgcg_pupdate(int nd, const double* __restrict__ z, double* __restrict__ p,
                                                           const double* sc, const int* fl) {
    if (fl[0]) return;
    const double beta = sc[2] / sc[1];
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i < nd) p[i] = z[i] + beta * p[i];
}

__global__ void __launch_bounds__(kThreads) k_mgcg_start(int nd, const uint8_t* __restrict__ fixed,
                                                         const double* __restrict__ b, double* __restrict__ r,
                                                         double* __restrict__ x, double* sc, double* ws) {
    const int i = blockIdx.x * kThreads + threadIdx.x;
    double part = 0.0;
    if (i < nd) {
        const double v = fixed[i] ? 0.0 : b[i];
        r[i] = v;
        x[i] = 0.0;
        part = v * v;
    }
    const double s = block_sum(part);
    grid_add(ws, 1, s, &sc[3]);
}

__global__ void k_mgcg_tol(double* sc, double rtol2) { sc[4] = rtol2 * sc[3]; }

inline int nb(int n, int t = kThreads) { return (n + t - 1) / t; }


// ---------------------------------------------------------------------------
// Inclusion rigid modes.  With cohesive interfaces an inclusion whose
// interface has softened can translate and rotate against the matrix at
// little energy; the grid hierarchy cannot represent those discontinuous
// modes (its corrections are continuous), so the preconditioner adds the
// coarse correction Z (Z^T K Z)^-1 Z^T r over them (additively, so it stays
// symmetric positive definite).  Mode k of inclusion i is the rigid motion
// R_k (x translation, y translation, rotation about the centre) inside the
// inclusion and zero outside: R_k at the nodes inside, and at an enrichment
// node the value that makes the field there R_k (inclusion side) or 0
// (matrix side), i.e. minus the parent edge's interpolation of the nodal
// values.  Distinct inclusions share no element, so Z^T K Z is block
// diagonal with one 3 x 3 block per inclusion.
// ---------------------------------------------------------------------------
__global__ void k_modes_E(int n, const int* __restrict__ z_inc, const double* __restrict__ zval,
                          const int* __restrict__ row_ptr, const int* __restrict__ col, const double* __restrict__ K,
                          const uint8_t* __restrict__ fixed, double* E) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const int zi = z_inc[q];
    if (zi < 0) return;
    double y[2][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
    for (int p = row_ptr[q]; p < row_ptr[q + 1]; ++p) {
        const int cn = col[p];
        if (z_inc[cn] != zi) continue;
        const double* blk = K + 4 * (size_t)p;
        for (int d = 0; d < 2; ++d)
            for (int e = 0; e < 2; ++e) {
                if (fixed[2 * cn + e]) continue;
                const double kde = blk[2 * d + e];
                for (int l = 0; l < 3; ++l) y[d][l] += kde * zval[6 * (size_t)cn + 3 * e + l];
            }
    }
    for (int k = 0; k < 3; ++k)
        for (int l = 0; l < 3; ++l) {
            double v = 0.0;
            for (int d = 0; d < 2; ++d)
                if (!fixed[2 * q + d]) v += zval[6 * (size_t)q + 3 * d + k] * y[d][l];
            atomicAdd(&E[9 * zi + 3 * k + l], v);
        }
}

// 3 x 3 inverse per inclusion (zero when the block is numerically singular)
__global__ void k_modes_inv(int n_inc, const double* E, double* Einv) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_inc) return;
    const double* a = E + 9 * i;
    const double c00 = a[4] * a[8] - a[5] * a[7], c01 = a[5] * a[6] - a[3] * a[8], c02 = a[3] * a[7] - a[4] * a[6];
    const double det = a[0] * c00 + a[1] * c01 + a[2] * c02;
    double scale = 0.0;
    for (int k = 0; k < 9; ++k) scale = fmax(scale, fabs(a[k]));
    double* o = Einv + 9 * i;
    if (!(fabs(det) > 1e-13 * scale * scale * scale)) {
        for (int k = 0; k < 9; ++k) o[k] = 0.0;
        return;
    }
    const double r = 1.0 / det;
    o[0] = c00 * r;
    o[1] = (a[2] * a[7] - a[1] * a[8]) * r;
    o[2] = (a[1] * a[5] - a[2] * a[4]) * r;
    o[3] = c01 * r;
    o[4] = (a[0] * a[8] - a[2] * a[6]) * r;
    o[5] = (a[2] * a[3] - a[0] * a[5]) * r;
    o[6] = c02 * r;
    o[7] = (a[1] * a[6] - a[0] * a[7]) * r;
    o[8] = (a[0] * a[4] - a[1] * a[3]) * r;
}

__global__ void k_modes_zero(int n, double* w, const int* done) {
    if (done && done[0]) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) w[i] = 0.0;
}

// w_i = Z_i^T r
__global__ void k_modes_dot(int n, const int* __restrict__ z_inc, const double* __restrict__ zval,
                            const uint8_t* __restrict__ fixed, const double* __restrict__ r, double* w, const int* done) {
    if (done && done[0]) return;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const int zi = z_inc[q];
    if (zi < 0) return;
    const double r0 = fixed[2 * q] ? 0.0 : r[2 * q], r1 = fixed[2 * q + 1] ? 0.0 : r[2 * q + 1];
    for (int k = 0; k < 3; ++k)
        atomicAdd(&w[3 * zi + k], zval[6 * (size_t)q + k] * r0 + zval[6 * (size_t)q + 3 + k] * r1);
}

// z += Z_i E_i^-1 w_i
__global__ void k_modes_add(int n, const int* __restrict__ z_inc, const double* __restrict__ zval,
                            const uint8_t* __restrict__ fixed, const double* __restrict__ Einv,
                            const double* __restrict__ w, double* z, const int* done) {
    if (done && done[0]) return;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const int zi = z_inc[q];
    if (zi < 0) return;
    const double* B = Einv + 9 * zi;
    const double* wi = w + 3 * zi;
    double cc[3];
    for (int k = 0; k < 3; ++k) cc[k] = B[3 * k] * wi[0] + B[3 * k + 1] * wi[1] + B[3 * k + 2] * wi[2];
    for (int d = 0; d < 2; ++d) {
        if (fixed[2 * q + d]) continue;
        z[2 * q + d] += zval[6 * (size_t)q + 3 * d] * cc[0] + zval[6 * (size_t)q + 3 * d + 1] * cc[1] +
                        zval[6 * (size_t)q + 3 * d + 2] * cc[2];
    }
}

template <typename T>
int mg_alloc(MgHierarchy& m, T** p, size_t n) {
    *p = nullptr;
    PG_CUDA(cudaMalloc((void**)p, std::max<size_t>(n, 1) * sizeof(T)));
    PG_CUDA(fill_sync(*p, 0, std::max<size_t>(n, 1) * sizeof(T)));
    m.owned.push_back((void*)*p);
    return PG_OK;
}

// Inclusion rigid modes of a cohesive mesh (host, once per mesh).
int modes_build(Ctx& c, MgHierarchy& m) {
    const HostMesh& hm = c.hm;
    const int ni = (int)hm.spec.inclusions.size();
    if (!hm.spec.cohesive || ni == 0) return PG_OK;
    const int nn = hm.n_nodes();
    // side of every enrichment node: 1 if an inclusion-material child uses it, 0 if a matrix child does
    std::vector<int> side(hm.n_enr, -1);
    for (int ci = 0; ci < hm.n_cut; ++ci) {
        const CutTemplate& T = cut_template(hm.cut_tmpl[ci]);
        for (int ch = 0; ch < T.n_child; ++ch) {
            const int mat = hm.cut_child_mat[(size_t)ci * kMaxChildren + ch];
            for (int k = 0; k < T.child_n[ch]; ++k) {
                const int ln = T.child_nodes[ch][k];
                if (ln < 3) continue;
                const int node = hm.cut_enr[(size_t)ci * kMaxEnr + ln - 3];
                if (node >= hm.n_reg) side[node - hm.n_reg] = mat == hm.spec.matrix_mat ? 0 : 1;
            }
        }
    }
    std::vector<int> zinc(nn, -1);
    std::vector<double> zval(6 * (size_t)nn, 0.0);
    auto rigid = [&](int i, double x, double y, double out[2][3]) {
        const Inclusion& I = hm.spec.inclusions[i];
        out[0][0] = 1.0; out[0][1] = 0.0; out[0][2] = -(y - I.cy);
        out[1][0] = 0.0; out[1][1] = 1.0; out[1][2] = x - I.cx;
    };
    for (int n = 0; n < hm.n_reg; ++n) {
        const int i = hm.node_detect[n];
        if (i < 0 || i >= ni) continue;
        double R[2][3];
        rigid(i, hm.x[n], hm.y[n], R);
        zinc[n] = i;
        for (int d = 0; d < 2; ++d)
            for (int k = 0; k < 3; ++k) zval[6 * (size_t)n + 3 * d + k] = R[d][k];
    }
    for (int k = 0; k < hm.n_enr; ++k) {
        const int n = hm.n_reg + k, i = hm.enr_inc[k];
        if (i < 0 || i >= ni || side[k] < 0) continue;
        const int a = hm.enr_edge[2 * k], b = hm.enr_edge[2 * k + 1];
        const double ex = hm.x[b] - hm.x[a], ey = hm.y[b] - hm.y[a];
        const double t = ((hm.x[n] - hm.x[a]) * ex + (hm.y[n] - hm.y[a]) * ey) / (ex * ex + ey * ey);
        double Ra[2][3] = {}, Rb[2][3] = {}, Rn[2][3] = {};
        if (hm.node_detect[a] == i) rigid(i, hm.x[a], hm.y[a], Ra);
        if (hm.node_detect[b] == i) rigid(i, hm.x[b], hm.y[b], Rb);
        if (side[k] == 1) rigid(i, hm.x[n], hm.y[n], Rn);
        zinc[n] = i;
        for (int d = 0; d < 2; ++d)
            for (int q = 0; q < 3; ++q)
                zval[6 * (size_t)n + 3 * d + q] = Rn[d][q] - ((1.0 - t) * Ra[d][q] + t * Rb[d][q]);
    }
    int rc;
    if ((rc = mg_alloc(m, &m.z_inc, (size_t)nn)) || (rc = mg_alloc(m, &m.zval, 6 * (size_t)nn)) ||
        (rc = mg_alloc(m, &m.E, 9 * (size_t)ni)) || (rc = mg_alloc(m, &m.Einv, 9 * (size_t)ni)) ||
        (rc = mg_alloc(m, &m.w, 3 * (size_t)ni)))
        return rc;
    PG_CUDA(h2d_sync(m.z_inc, zinc.data(), zinc.size() * sizeof(int)));
    PG_CUDA(h2d_sync(m.zval, zval.data(), zval.size() * sizeof(double)));
    m.n_inc = ni;
    return PG_OK;
}

// Structure of the hierarchy (once per mesh).
int mg_build(Ctx& c) {
    if (c.mg) return PG_OK;
    {   // k_mg_bottom's shared-memory limit, once per device (before any graph capture)
        static bool done_dev[64] = {};
        int dev = 0;
        cudaGetDevice(&dev);
        if (dev < 0 || dev >= 64 || !done_dev[dev]) {
            PG_CUDA(cudaFuncSetAttribute(k_mg_bottom<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMgBottomSmem));
            PG_CUDA(cudaFuncSetAttribute(k_mg_bottom<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMgBottomSmem));
            if (dev >= 0 && dev < 64) done_dev[dev] = true;
        }
    }
    const int nx0 = c.hm.spec.nx, ny0 = c.hm.spec.ny;
    if (nx0 < 1 || ny0 < 1) {
        set_error("multigrid: mesh without a structured background grid");
        return PG_ERR_ARG;
    }
    MgHierarchy* m = new MgHierarchy();
    c.mg = m;
    int rc;
    const int nd0 = c.n_dof;
    if ((rc = mg_alloc(*m, &m->x0, nd0)) || (rc = mg_alloc(*m, &m->x0b, nd0)) || (rc = mg_alloc(*m, &m->r0, nd0)))
        return rc;
    if ((rc = mg_alloc(*m, &m->b0f, nd0)) || (rc = mg_alloc(*m, &m->x0f, nd0)) || (rc = mg_alloc(*m, &m->x0bf, nd0)) ||
        (rc = mg_alloc(*m, &m->r0f, nd0)) || (rc = mg_alloc(*m, &m->Dinv0f, 4 * (size_t)c.n_nodes)))
        return rc;
    int nx = nx0, ny = ny0, l = 0;
    while ((nx > kMgCoarseCells || ny > kMgCoarseCells) && l < kMgMaxLevels) {
        nx = (nx + 1) / 2;
        ny = (ny + 1) / 2;
        ++l;
        MgLevel& L = m->L[l];
        L.nx = nx;
        L.ny = ny;
        L.n = (nx + 1) * (ny + 1);
        const size_t n = L.n;
        if ((rc = mg_alloc(*m, &L.A, 36 * n)) || (rc = mg_alloc(*m, &L.Af, 36 * n)) || (rc = mg_alloc(*m, &L.Dinv, 4 * n)) ||
            (rc = mg_alloc(*m, &L.Dinvf, 4 * n)) || (rc = mg_alloc(*m, &L.fixed, 2 * n)))
            return rc;
        if ((rc = mg_alloc(*m, &L.x, 2 * n)) || (rc = mg_alloc(*m, &L.x2, 2 * n)) || (rc = mg_alloc(*m, &L.b, 2 * n)) ||
            (rc = mg_alloc(*m, &L.r, 2 * n)))
            return rc;
        if ((rc = mg_alloc(*m, &L.xf, 2 * n)) || (rc = mg_alloc(*m, &L.x2f, 2 * n)) || (rc = mg_alloc(*m, &L.bf, 2 * n)) ||
            (rc = mg_alloc(*m, &L.rf, 2 * n)))
            return rc;
    }
    if (l == 0 || (nx > kMgCoarseCells || ny > kMgCoarseCells)) {
        set_error("multigrid: grid too small or too large to coarsen");
        return PG_ERR_ARG;
    }
    m->nlev = l;
    m->nc = 2 * m->L[l].n;
    if ((rc = mg_alloc(*m, &m->LU, (size_t)m->nc * m->nc)) || (rc = mg_alloc(*m, &m->piv, m->nc)) ||
        (rc = mg_alloc(*m, &m->sc, 8)) || (rc = mg_alloc(*m, &m->fl, 8)))
        return rc;
    // coarse masks by injection
    cudaStream_t s = c.stream;
    const uint8_t* ff = c.fixed;
    int nxf = nx0, nyf = ny0;
    for (int k = 1; k <= l; ++k) {
        MgLevel& L = m->L[k];
        k_mg_inject_mask<<<nb(L.n), kThreads, 0, s>>>(nxf, L.nx, L.ny, nyf, ff, L.fixed);
        ff = L.fixed;
        nxf = L.nx;
        nyf = L.ny;
    }
    PG_CUDA(cudaGetLastError());
    PG_CUDA(cudaStreamSynchronize(s));
    return modes_build(c, *m);
}

// Numeric set-up for the current K (every solve: K changes between Newton iterations).
int mg_numeric(Ctx& c, bool f32, cudaStream_t s) {
    MgHierarchy& m = *c.mg;
    const int n0 = c.n_nodes;
    // level 0 smoother: block Jacobi of the masked K
    k_prec_setup<double><<<nb(n0), kThreads, 0, s>>>(n0, c.diag, c.K, c.fixed, 1, 0, c.minv);
    if (f32) {
        launch_to_fp32(c, s);
        k_mg_to_f32<<<nb(4 * n0), kThreads, 0, s>>>(4 * (size_t)n0, c.minv, m.Dinv0f);
    }
    int nxf = c.hm.spec.nx, nyf = c.hm.spec.ny;
    for (int k = 1; k <= m.nlev; ++k) {
        MgLevel& L = m.L[k];
        GalArgs g;
        g.nxf = nxf;
        g.nyf = nyf;
        g.nxc = L.nx;
        g.nyc = L.ny;
        g.row_ptr = c.row_ptr;
        g.col = c.col;
        g.K = c.K;
        g.n_reg = c.n_reg;
        g.A = k > 1 ? m.L[k - 1].A : nullptr;
        g.fixed_f = k > 1 ? m.L[k - 1].fixed : c.fixed;
        g.fixed_c = L.fixed;
        g.Ac = L.A;
        if (k == 1)
            k_mg_galerkin<true><<<nb(9 * L.n), kThreads, 0, s>>>(g);
        else
            k_mg_galerkin<false><<<nb(9 * L.n), kThreads, 0, s>>>(g);
        k_mg_dinv<<<nb(L.n), kThreads, 0, s>>>(L.n, L.A, L.fixed, L.Dinv, f32 ? L.Dinvf : nullptr);
        if (f32) k_mg_to_f32<<<nb(36 * L.n), kThreads, 0, s>>>(36 * (size_t)L.n, L.A, L.Af);
        nxf = L.nx;
        nyf = L.ny;
    }
    if (m.n_inc > 0 && m.use_modes) {
        cudaMemsetAsync(m.E, 0, 9 * (size_t)m.n_inc * sizeof(double), s);
        k_modes_E<<<nb(n0), kThreads, 0, s>>>(n0, m.z_inc, m.zval, c.row_ptr, c.col, c.K, c.fixed, m.E);
        k_modes_inv<<<nb(m.n_inc), kThreads, 0, s>>>(m.n_inc, m.E, m.Einv);
    }
    const MgLevel& C = m.L[m.nlev];
    cudaMemsetAsync(m.fl, 0, 8 * sizeof(int), s);
    k_mg_coarse_factor<<<1, 128, 0, s>>>(C.nx, C.ny, C.A, C.fixed, m.LU, m.piv, m.fl);
    PG_CUDA(cudaGetLastError());
    return PG_OK;
}

// One V-cycle: returns the level-0 buffer holding V(b0).  Records launches on s.
template <typename T>
const T* vcycle(Ctx& c, MgHierarchy& m, cudaStream_t s, const T* b0, const int* done);

// First level of the fused bottom (k_mg_bottom) and which of its levels have
// their operator staged in shared memory: going up from the coarsest, the
// levels of at most kMgBottomNodes nodes (at most kMgBottomLevels) whose
// vectors fit in kMgBottomSmem bytes together; then, coarsest first, each
// level's operator is staged while it still fits (the coarsest level, solved
// by its explicit inverse, needs none); the others read theirs from L2.
template <typename T>
int mg_bottom_first(const MgHierarchy& m, size_t* smem, int* staged) {
    int kb = m.nlev;
    size_t bytes = mg_bottom_vec_bytes<T>(m.L[m.nlev].n);
    for (int k = m.nlev - 1; k >= 1 && m.nlev - k + 1 <= kMgBottomLevels; --k) {
        const size_t add = mg_bottom_vec_bytes<T>(m.L[k].n);
        if (m.L[k].n > kMgBottomNodes || bytes + add > (size_t)kMgBottomSmem) break;
        bytes += add;
        kb = k;
    }
    for (int k = m.nlev; k >= kb; --k) {
        int& st = staged[k - kb];
        st = 0;
        if (k == m.nlev) continue;
        const size_t add = mg_bottom_op_bytes<T>(m.L[k].n);
        if (bytes + add <= (size_t)kMgBottomSmem) {
            bytes += add;
            st = 1;
        }
    }
    *smem = bytes;
    return kb;
}

// Levels kb .. nlev in one launch; level kb's result ends in its x (xf).
template <typename T>
void launch_bottom(MgHierarchy& m, int kb, size_t smem, const int* staged, int nxf, int nyf, const T* rf,
                   cudaStream_t s, const int* done) {
    MgBottomArgs<T> a;
    a.nlev = m.nlev - kb + 1;
    a.nxf = nxf;
    a.nyf = nyf;
    a.rf = rf;
    for (int k = kb; k <= m.nlev; ++k) {
        MgLevel& L = m.L[k];
        const int j = k - kb;
        a.nx[j] = L.nx;
        a.ny[j] = L.ny;
        a.fixed[j] = L.fixed;
        a.staged[j] = staged[j];
        if constexpr (std::is_same<T, float>::value) {
            a.A[j] = L.Af;
            a.Dinv[j] = L.Dinvf;
        } else {
            a.A[j] = L.A;
            a.Dinv[j] = L.Dinv;
        }
    }
    if constexpr (std::is_same<T, float>::value) a.x0 = m.L[kb].xf;
    else a.x0 = m.L[kb].x;
    a.XT = m.LU;
    a.nc = m.nc;
    a.omega = (T)kMgOmega;
    k_mg_bottom<T><<<1, kMgBottomThreads, smem, s>>>(a, done);
}

template <>
const double* vcycle<double>(Ctx& c, MgHierarchy& m, cudaStream_t s, const double* b0, const int* done) {
    const int n0 = c.n_nodes;
    const double om = kMgOmega;
    // level 0 pre-smoothing
    double* cur = m.x0;
    double* alt = m.x0b;
    k_mg_smooth_bsr<double><<<nb(kRowLanes * n0), kThreads, 0, s>>>(n0, c.row_ptr, c.col, c.K, c.minv, c.fixed, b0, nullptr, cur, om,
                                                          done, 0);
    for (int it = 1; it < kMgNu1; ++it) {
        k_mg_smooth_bsr<double><<<nb(kRowLanes * n0), kThreads, 0, s>>>(n0, c.row_ptr, c.col, c.K, c.minv, c.fixed, b0, cur, alt, om,
                                                              done, 0);
        std::swap(cur, alt);
    }
    k_mg_smooth_bsr<double><<<nb(kRowLanes * n0), kThreads, 0, s>>>(n0, c.row_ptr, c.col, c.K, c.minv, c.fixed, b0, cur, m.r0, om,
                                                          done, 1);
    int nxf = c.hm.spec.nx, nyf = c.hm.spec.ny;
    const double* rf = m.r0;
    double* xs[kMgMaxLevels + 1];
    xs[0] = cur;
    size_t bsm = 0;
    int staged[kMgBottomLevels];
    const int kb = mg_bottom_first<double>(m, &bsm, staged);
    for (int k = 1; k <= m.nlev; ++k) {
        MgLevel& L = m.L[k];
        if (k == kb) {  // this level and all coarser ones: one launch
            launch_bottom<double>(m, kb, bsm, staged, nxf, nyf, rf, s, done);
            xs[k] = L.x;
            break;
        }
        k_mg_restrict<double><<<nb(L.n), kThreads, 0, s>>>(nxf, nyf, L.nx, L.ny, rf, L.fixed, L.b, done);
        double* lc = L.x;
        double* la = L.x2;
        k_mg_smooth_st<double><<<nb(L.n), kThreads, 0, s>>>(L.nx, L.ny, L.A, L.Dinv, L.fixed, L.b, nullptr, lc, om, done, 0);
        for (int it = 1; it < kMgNu1; ++it) {
            k_mg_smooth_st<double><<<nb(L.n), kThreads, 0, s>>>(L.nx, L.ny, L.A, L.Dinv, L.fixed, L.b, lc, la, om, done, 0);
            std::swap(lc, la);
        }
        k_mg_smooth_st<double><<<nb(L.n), kThreads, 0, s>>>(L.nx, L.ny, L.A, L.Dinv, L.fixed, L.b, lc, L.r, om, done, 1);
        xs[k] = lc;
        rf = L.r;
        nxf = L.nx;
        nyf = L.ny;
    }
    for (int k = kb - 1; k >= 0; --k) {
        const MgLevel& Lc = m.L[k + 1];
        if (k == 0) {
            k_mg_prolong<double><<<nb(c.n_reg), kThreads, 0, s>>>(c.hm.spec.nx, c.hm.spec.ny, Lc.nx, xs[1], c.fixed, cur,
                                                                    done);
            for (int it = 0; it < kMgNu2; ++it) {
                k_mg_smooth_bsr<double><<<nb(kRowLanes * n0), kThreads, 0, s>>>(n0, c.row_ptr, c.col, c.K, c.minv, c.fixed, b0, cur,
                                                                      alt, om, done, 0);
                std::swap(cur, alt);
            }
            return cur;
        }
        MgLevel& L = m.L[k];
        double* lc = xs[k];
        double* la = lc == L.x ? L.x2 : L.x;
        k_mg_prolong<double><<<nb(L.n), kThreads, 0, s>>>(L.nx, L.ny, Lc.nx, xs[k + 1], L.fixed, lc, done);
        for (int it = 0; it < kMgNu2; ++it) {
            k_mg_smooth_st<double><<<nb(L.n), kThreads, 0, s>>>(L.nx, L.ny, L.A, L.Dinv, L.fixed, L.b, lc, la, om, done, 0);
            std::swap(lc, la);
        }
        xs[k] = lc;
    }
    return cur;
}

template <>
const float* vcycle<float>(Ctx& c, MgHierarchy& m, cudaStream_t s, const float* b0, const int* done) {
    const int n0 = c.n_nodes;
    const float om = (float)kMgOmega;
    float* cur = m.x0f;
    float* alt = m.x0bf;
    k_mg_smooth_bsr<float><<<nb(kRowLanes * n0), kThreads, 0, s>>>(n0, c.row_ptr, c.col, c.Kf, m.Dinv0f, c.fixed, b0, nullptr, cur, om,
                                                         done, 0);
    for (int it = 1; it < kMgNu1; ++it) {
        k_mg_smooth_bsr<float><<<nb(kRowLanes * n0), kThreads, 0, s>>>(n0, c.row_ptr, c.col, c.Kf, m.Dinv0f, c.fixed, b0, cur, alt, om,
                                                             done, 0);
        std::swap(cur, alt);
    }
    k_mg_smooth_bsr<float><<<nb(kRowLanes * n0), kThreads, 0, s>>>(n0, c.row_ptr, c.col, c.Kf, m.Dinv0f, c.fixed, b0, cur, m.r0f, om,
                                                         done, 1);
    int nxf = c.hm.spec.nx, nyf = c.hm.spec.ny;
    const float* rf = m.r0f;
    float* xs[kMgMaxLevels + 1];
    xs[0] = cur;
    size_t bsm = 0;
    int staged[kMgBottomLevels];
    const int kb = mg_bottom_first<float>(m, &bsm, staged);
    for (int k = 1; k <= m.nlev; ++k) {
        MgLevel& L = m.L[k];
        if (k == kb) {  // this level and all coarser ones: one launch
            launch_bottom<float>(m, kb, bsm, staged, nxf, nyf, rf, s, done);
            xs[k] = L.xf;
            break;
        }
        k_mg_restrict<float><<<nb(L.n), kThreads, 0, s>>>(nxf, nyf, L.nx, L.ny, rf, L.fixed, L.bf, done);
        float* lc = L.xf;
        float* la = L.x2f;
        k_mg_smooth_st<float><<<nb(L.n), kThreads, 0, s>>>(L.nx, L.ny, L.Af, L.Dinvf, L.fixed, L.bf, nullptr, lc, om, done, 0);
        for (int it = 1; it < kMgNu1; ++it) {
            k_mg_smooth_st<float><<<nb(L.n), kThreads, 0, s>>>(L.nx, L.ny, L.Af, L.Dinvf, L.fixed, L.bf, lc, la, om, done, 0);
            std::swap(lc, la);
        }
        k_mg_smooth_st<float><<<nb(L.n), kThreads, 0, s>>>(L.nx, L.ny, L.Af, L.Dinvf, L.fixed, L.bf, lc, L.rf, om, done, 1);
        xs[k] = lc;
        rf = L.rf;
        nxf = L.nx;
        nyf = L.ny;
    }
    for (int k = kb - 1; k >= 0; --k) {
        const MgLevel& Lc = m.L[k + 1];
        if (k == 0) {
            k_mg_prolong<float><<<nb(c.n_reg), kThreads, 0, s>>>(c.hm.spec.nx, c.hm.spec.ny, Lc.nx, xs[1], c.fixed, cur, done);
            for (int it = 0; it < kMgNu2; ++it) {
                k_mg_smooth_bsr<float><<<nb(kRowLanes * n0), kThreads, 0, s>>>(n0, c.row_ptr, c.col, c.Kf, m.Dinv0f, c.fixed, b0, cur,
                                                                     alt, om, done, 0);
                std::swap(cur, alt);
            }
            return cur;
        }
        MgLevel& L = m.L[k];
        float* lc = xs[k];
        float* la = lc == L.xf ? L.x2f : L.xf;
        k_mg_prolong<float><<<nb(L.n), kThreads, 0, s>>>(L.nx, L.ny, Lc.nx, xs[k + 1], L.fixed, lc, done);
        for (int it = 0; it < kMgNu2; ++it) {
            k_mg_smooth_st<float><<<nb(L.n), kThreads, 0, s>>>(L.nx, L.ny, L.Af, L.Dinvf, L.fixed, L.bf, lc, la, om, done, 0);
            std::swap(lc, la);
        }
        xs[k] = lc;
    }
    return cur;
}

// z = M^-1 r through one V-cycle (FP64 in, FP64 out).
void mg_apply(Ctx& c, MgHierarchy& m, bool f32, cudaStream_t s, const double* r, double* z, const int* done) {
    const int nd = c.n_dof;
    if (f32) {
        k_mg_f64_to_f32<<<nb(nd), kThreads, 0, s>>>(nd, r, m.b0f, done);
        const float* x = vcycle<float>(c, m, s, m.b0f, done);
        k_mg_f32_to_f64<<<nb(nd), kThreads, 0, s>>>(nd, x, z, done);
    } else {
        const double* x = vcycle<double>(c, m, s, r, done);
        k_copy<double><<<nb(nd), kThreads, 0, s>>>(nd, x, z);
    }
    if (m.n_inc > 0 && m.use_modes) {
        const int n = c.n_nodes;
        k_modes_zero<<<nb(3 * m.n_inc), kThreads, 0, s>>>(3 * m.n_inc, m.w, done);
        k_modes_dot<<<nb(n), kThreads, 0, s>>>(n, m.z_inc, m.zval, c.fixed, r, m.w, done);
        k_modes_add<<<nb(n), kThreads, 0, s>>>(n, m.z_inc, m.zval, c.fixed, m.Einv, m.w, z, done);
    }
}

}  // namespace

int mg_prepare(Ctx& c, bool f32, bool modes, cudaStream_t s) {
    int rc = mg_build(c);
    if (rc != PG_OK) return rc;
    c.mg->use_modes = modes;
    if ((rc = mg_numeric(c, f32, s))) return rc;
    int fl[8] = {};
    cudaMemcpyAsync(fl, c.mg->fl, sizeof fl, cudaMemcpyDeviceToHost, s);
    PG_CUDA(cudaStreamSynchronize(s));
    if (fl[3]) {
        set_error("multigrid: singular coarsest operator");
        return PG_ERR_BREAKDOWN;
    }
    return PG_OK;
}

void mg_precondition(Ctx& c, bool f32, cudaStream_t s, const double* r, double* z) {
    mg_apply(c, *c.mg, f32, s, r, z, nullptr);
}

void mg_free(Ctx& c) {
    if (!c.mg) return;
    for (void* p : c.mg->owned) cudaFree(p);
    delete c.mg;
    c.mg = nullptr;
}

// CG on mask(K) dx = mask(b) (b = c.b, dx = c.dx) preconditioned by one
// V-cycle per iteration.  Fills st.iterations, st.rel_residual (true FP64
// residual) and st.status.
int mg_pcg_solve(Ctx& c, const pg_solver_cfg& cfg, pg_solve_stats& st, cudaStream_t s) {
    int rc = mg_build(c);
    if (rc != PG_OK) return rc;
    MgHierarchy& m = *c.mg;
    const bool f32 = cfg.precision == PG_PRECISION_MIXED;
    m.use_modes = cfg.inclusion_modes != 0;
    if ((rc = mg_numeric(c, f32, s))) return rc;
    const int n = c.n_nodes, nd = c.n_dof;
    cudaMemsetAsync(m.sc, 0, 8 * sizeof(double), s);
    k_mgcg_start<<<nb(nd), kThreads, 0, s>>>(nd, c.fixed, c.b, c.r, c.dx, m.sc, c.red_active);
    k_mgcg_tol<<<1, 1, 0, s>>>(m.sc, cfg.rtol * cfg.rtol);
    // z = V(r), p = z, sc[2] = r.z
    mg_apply(c, m, f32, s, c.r, c.z, nullptr);
    k_copy<double><<<nb(nd), kThreads, 0, s>>>(nd, c.z, c.p);
    k_mgcg_dot<<<nb(nd), kThreads, 0, s>>>(nd, c.r, c.z, m.sc + 2, m.fl, c.red_active);
    int hf[8] = {};
    double hs[8] = {};
    cudaMemcpyAsync(hs, m.sc, sizeof hs, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(hf, m.fl, sizeof hf, cudaMemcpyDeviceToHost, s);
    PG_CUDA(cudaStreamSynchronize(s));
    if (hf[3]) {
        set_error("multigrid: singular coarsest operator");
        st.status = PG_ERR_BREAKDOWN;
        return PG_OK;
    }
    const double bb = hs[3];
    int iters = 0;
    bool breakdown = false;
    if (bb > 0.0 && cfg.max_iter > 0) {
        constexpr int kChunk = 2;
        cudaGraph_t graph;
        PG_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        for (int it = 0; it < kChunk; ++it) {
            k_mgcg_s1<<<1, 1, 0, s>>>(m.sc, m.fl);
            k_mgcg_spmv<<<nb(kRowLanes * n), kThreads, 0, s>>>(n, c.row_ptr, c.col, c.K, c.p, c.fixed, c.q, m.sc, m.fl,
                                                                 c.red_active);
            k_mgcg_update<<<nb(nd), kThreads, 0, s>>>(nd, c.dx, c.r, c.p, c.q, m.sc, m.fl, c.red_active);
            k_mgcg_s2<<<1, 1, 0, s>>>(m.sc, m.fl);
            mg_apply(c, m, f32, s, c.r, c.z, m.fl);
            k_mgcg_dot<<<nb(nd), kThreads, 0, s>>>(nd, c.r, c.z, m.sc + 2, m.fl, c.red_active);
            k_mgcg_pupdate<<<nb(nd), kThreads, 0, s>>>(nd, c.z, c.p, m.sc, m.fl);
        }
        PG_CUDA(cudaStreamEndCapture(s, &graph));
        cudaGraphExec_t exec = nullptr;
        const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        if (ie != cudaSuccess) return cuda_fail(ie, "multigrid CG graph");
        while (true) {
            cudaGraphLaunch(exec, s);
            cudaMemcpyAsync(hf, m.fl, sizeof hf, cudaMemcpyDeviceToHost, s);
            const cudaError_t e = cudaStreamSynchronize(s);
            if (e != cudaSuccess) {
                cudaGraphExecDestroy(exec);
                return cuda_fail(e, "multigrid CG");
            }
            iters = hf[2];
            if (hf[0] || iters >= cfg.max_iter) break;
        }
        cudaGraphExecDestroy(exec);
        breakdown = hf[1] != 0;
    }
    const double rr = residual_into(c, s, c.dx, c.b, c.r);
    st.iterations = iters;
    st.refinements = 0;
    st.rel_residual = bb > 0.0 ? std::sqrt(rr / bb) : 0.0;
    if (breakdown)
        st.status = PG_ERR_BREAKDOWN;
    else
        st.status = rr <= 4.0 * cfg.rtol * cfg.rtol * bb ? PG_OK : PG_ERR_NOT_CONVERGED;
    return PG_OK;
}

}  // namespace pgb
