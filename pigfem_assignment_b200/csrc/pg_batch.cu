// Many independent linear-elastic RVEs of uneven size assembled and solved
// together (sm_100a).
//
// The reference solves one RVE per run (Problem::solve_problem,
// src/Problem.cpp:400-418); a batch here is the block-diagonal union of the
// RVEs' IGFEM systems.  The meshes are concatenated node by node (each RVE's
// regular then enrichment nodes), so one launch of each assembly kernel
// covers every RVE, and the solve is CG with per-RVE scalars: every RVE has
// its own step lengths, its own residual target (rtol times its own right-
// hand side) and stops on its own, while the kernels keep running over the
// whole batch until the last RVE converges.  The preconditioner is either
// block Jacobi or one multigrid V-cycle whose levels are the union of every
// RVE's own grid hierarchy (RVEs of different sizes have different depths:
// an RVE's coarsest grid is solved by its own dense LU, one CTA per RVE, while
// larger RVEs keep coarsening).  The CG iterations of a whole batch run as
// CUDA graphs.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <sys/mman.h>
#include <vector>

#include "pg_solve_kernels.cuh"
#include "pigfem_b200.h"

namespace pgb {

namespace {

constexpr int kBMaxDepth = 16;
constexpr int kBCoarseCells = 4;
constexpr int kBCoarseMaxDof = 2 * (kBCoarseCells + 1) * (kBCoarseCells + 1);
constexpr int kBCoarseStride = kBCoarseMaxDof * kBCoarseMaxDof;
constexpr double kBOmega = 0.5;  // block-Jacobi damping (lambda_max(D^-1 K) reaches ~3.9)

// One RVE's grid at one depth of the hierarchy.
struct BDesc {
    int off;            // first node of this grid in the depth's arrays
    int nx, ny;         // cells per side
    int foff;           // first node of the finer grid (depth 0: the RVE's first node in the batch mesh)
    int fnx, fny;       // finer grid cells
    int coarsest;       // 1: the RVE's deepest grid (solved by its dense LU)
    int present;        // 0: the RVE has no grid at this depth
};

struct BDepth {
    int n = 0;                         // nodes of all RVEs present at this depth
    int* node_rve = nullptr;           // n
    BDesc* desc = nullptr;             // one per RVE (unused for RVEs absent at this depth)
    double *A = nullptr, *Dinv = nullptr;
    float *Af = nullptr, *Dinvf = nullptr;
    uint8_t* fixed = nullptr;
    double *x = nullptr, *x2 = nullptr, *b = nullptr, *r = nullptr;
    float *xf = nullptr, *x2f = nullptr, *bf = nullptr, *rf = nullptr;
};

__host__ __device__ __forceinline__ int b_pos(int I, int nf) { return 2 * I < nf ? 2 * I : nf; }

__host__ __device__ __forceinline__ double b_w(int g, int nf, int I) {
    if ((g & 1) == 0) return (g >> 1) == I ? 1.0 : 0.0;
    if (g == nf) return I == ((nf + 1) >> 1) ? 1.0 : 0.0;
    return (I == ((g - 1) >> 1) || I == ((g + 1) >> 1)) ? 0.5 : 0.0;
}

inline int nb(long long n, int t = kThreads) { return (int)((n + t - 1) / t); }

// ---------------------------------------------------------------------------
// Multigrid set-up kernels over one depth of the union hierarchy
// ---------------------------------------------------------------------------
__global__ void k_b_inject_mask(int n, const int* node_rve, const BDesc* D, const uint8_t* fixed_f, uint8_t* fixed_c) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= n) return;
    const BDesc L = D[node_rve[a]];
    const int la = a - L.off;
    const int I = la % (L.nx + 1), J = la / (L.nx + 1);
    const int i = L.foff + b_pos(I, L.fnx) + b_pos(J, L.fny) * (L.fnx + 1);
    fixed_c[2 * a] = fixed_f[2 * i];
    fixed_c[2 * a + 1] = fixed_f[2 * i + 1];
}

// Galerkin product P^T M A M P of one depth from the finer one (BSR at depth 1).
template <bool FINE_BSR>
__global__ void k_b_galerkin(int n, const int* node_rve, const BDesc* D, const int* row_ptr, const int* col,
                             const double* K, const double* A, const uint8_t* fixed_f, const uint8_t* fixed_c,
                             double* Ac) {
    const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (tid >= 9LL * n) return;
    const int a = (int)(tid / 9), o = (int)(tid - 9LL * a);
    const BDesc L = D[node_rve[a]];
    const int la = a - L.off;
    const int Ia = la % (L.nx + 1), Ja = la / (L.nx + 1);
    const int Ib = Ia + (o % 3) - 1, Jb = Ja + (o / 3) - 1;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    if (Ib >= 0 && Ib <= L.nx && Jb >= 0 && Jb <= L.ny) {
        const int nreg_f = (L.fnx + 1) * (L.fny + 1);
        const int px = b_pos(Ia, L.fnx), py = b_pos(Ja, L.fny);
        for (int cy = py - 1; cy <= py + 1; ++cy) {
            if (cy < 0 || cy > L.fny) continue;
            const double wy = b_w(cy, L.fny, Ja);
            if (wy == 0.0) continue;
            for (int cx = px - 1; cx <= px + 1; ++cx) {
                if (cx < 0 || cx > L.fnx) continue;
                const double wx = b_w(cx, L.fnx, Ia);
                if (wx == 0.0) continue;
                const int i = L.foff + cx + cy * (L.fnx + 1);
                const double wi = wx * wy;
                const bool fi0 = !fixed_f[2 * i], fi1 = !fixed_f[2 * i + 1];
                if (FINE_BSR) {
                    for (int q = row_ptr[i]; q < row_ptr[i + 1]; ++q) {
                        const int jl = col[q] - L.foff;
                        if (jl < 0 || jl >= nreg_f) continue;  // enrichment columns: no coarse part
                        const int gx = jl % (L.fnx + 1), gy = jl / (L.fnx + 1);
                        const double wj = b_w(gx, L.fnx, Ib) * b_w(gy, L.fny, Jb);
                        if (wj == 0.0) continue;
                        const int j = L.foff + jl;
                        const bool fj0 = !fixed_f[2 * j], fj1 = !fixed_f[2 * j + 1];
                        const double* blk = K + 4 * (size_t)q;
                        const double w = wi * wj;
                        if (fi0 && fj0) acc[0] += w * blk[0];
                        if (fi0 && fj1) acc[1] += w * blk[1];
                        if (fi1 && fj0) acc[2] += w * blk[2];
                        if (fi1 && fj1) acc[3] += w * blk[3];
                    }
                } else {
                    for (int s = 0; s < 9; ++s) {
                        const int gx = cx + (s % 3) - 1, gy = cy + (s / 3) - 1;
                        if (gx < 0 || gx > L.fnx || gy < 0 || gy > L.fny) continue;
                        const double wj = b_w(gx, L.fnx, Ib) * b_w(gy, L.fny, Jb);
                        if (wj == 0.0) continue;
                        const int j = L.foff + gx + gy * (L.fnx + 1);
                        const bool fj0 = !fixed_f[2 * j], fj1 = !fixed_f[2 * j + 1];
                        const double* blk = A + 36 * (size_t)i + 4 * s;
                        const double w = wi * wj;
                        if (fi0 && fj0) acc[0] += w * blk[0];
                        if (fi0 && fj1) acc[1] += w * blk[1];
                        if (fi1 && fj0) acc[2] += w * blk[2];
                        if (fi1 && fj1) acc[3] += w * blk[3];
                    }
                }
            }
        }
        const int b = L.off + Ib + Jb * (L.nx + 1);
        if (fixed_c[2 * a]) acc[0] = acc[1] = 0.0;
        if (fixed_c[2 * a + 1]) acc[2] = acc[3] = 0.0;
        if (fixed_c[2 * b]) acc[0] = acc[2] = 0.0;
        if (fixed_c[2 * b + 1]) acc[1] = acc[3] = 0.0;
    }
    double* out = Ac + 36 * (size_t)a + 4 * o;
    for (int k = 0; k < 4; ++k) out[k] = acc[k];
}

__global__ void k_b_dinv(int n, const double* A, const uint8_t* fixed, double* Dinv, float* Dinvf, float* Af) {
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
        Dinvf[4 * (size_t)i + k] = (float)m[k];
    }
    for (int k = 0; k < 36; ++k) Af[36 * (size_t)i + k] = (float)A[36 * (size_t)i + k];
}

// Coarsest grid of every RVE: dense LU with partial pivoting, one CTA per RVE.
struct BCoarse {
    int depth, off, nx, ny;
};

__global__ void k_b_coarse_factor(const BCoarse* cd, double* const* Adepth, uint8_t* const* Fdepth, double* LU, int* piv,
                                  int* bad) {
    __shared__ double M[kBCoarseMaxDof][kBCoarseMaxDof + 1];
    __shared__ int sp[kBCoarseMaxDof];
    __shared__ int s_pivot;
    const int r = blockIdx.x;
    const BCoarse C = cd[r];
    const double* A = Adepth[C.depth];
    const uint8_t* fixed = Fdepth[C.depth];
    const int nn = (C.nx + 1) * (C.ny + 1), n = 2 * nn;
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) M[e / n][e % n] = 0.0;
    __syncthreads();
    for (int t = threadIdx.x; t < 9 * nn; t += blockDim.x) {
        const int a = t / 9, o = t - 9 * a;
        const int I = a % (C.nx + 1) + (o % 3) - 1, J = a / (C.nx + 1) + (o / 3) - 1;
        if (I < 0 || I > C.nx || J < 0 || J > C.ny) continue;
        const int b = I + J * (C.nx + 1);
        const double* blk = A + 36 * (size_t)(C.off + a) + 4 * o;
        for (int d = 0; d < 2; ++d)
            for (int f = 0; f < 2; ++f)
                if (!fixed[2 * (C.off + a) + d] && !fixed[2 * (C.off + b) + f]) M[2 * a + d][2 * b + f] = blk[2 * d + f];
    }
    __syncthreads();
    for (int q = threadIdx.x; q < n; q += blockDim.x) {
        if (fixed[2 * C.off + q]) M[q][q] = 1.0;
        sp[q] = q;
    }
    __syncthreads();
    for (int k = 0; k < n; ++k) {
        if (threadIdx.x == 0) {
            int best = k;
            for (int q = k + 1; q < n; ++q)
                if (fabs(M[q][k]) > fabs(M[best][k])) best = q;
            s_pivot = best;
            if (M[best][k] == 0.0) bad[r] = 1;
        }
        __syncthreads();
        const int pr = s_pivot;
        if (pr != k) {
            for (int c = threadIdx.x; c < n; c += blockDim.x) {
                const double t2 = M[k][c];
                M[k][c] = M[pr][c];
                M[pr][c] = t2;
            }
            if (threadIdx.x == 0) {
                const int t3 = sp[k];
                sp[k] = sp[pr];
                sp[pr] = t3;
            }
        }
        __syncthreads();
        const double d = M[k][k];
        for (int q = k + 1 + threadIdx.x; q < n; q += blockDim.x)
            if (d != 0.0) M[q][k] /= d;
        __syncthreads();
        for (int e = threadIdx.x; e < (n - k - 1) * (n - k - 1); e += blockDim.x) {
            const int q = k + 1 + e / (n - k - 1), c = k + 1 + e % (n - k - 1);
            M[q][c] -= M[q][k] * M[k][c];
        }
        __syncthreads();
    }
    double* LUr = LU + (size_t)r * kBCoarseStride;
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) LUr[e] = M[e / n][e % n];
    for (int q = threadIdx.x; q < n; q += blockDim.x) piv[r * kBCoarseMaxDof + q] = sp[q];
}

// ---------------------------------------------------------------------------
// V-cycle kernels (arithmetic in T)
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(kThreads) k_b_smooth_st(int n, const int* __restrict__ node_rve, const BDesc* D,
                                                          const T* __restrict__ A, const T* __restrict__ Dinv,
                                                          const uint8_t* __restrict__ fixed, const T* __restrict__ b,
                                                          const T* __restrict__ xin, T* __restrict__ xout, T omega,
                                                          const int* done, int resid_only) {
    if (done && done[0]) return;
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i >= n) return;
    const BDesc L = D[node_rve[i]];
    if (L.coarsest) return;  // that RVE's grid is solved by its dense LU
    T r0 = b[2 * i], r1 = b[2 * i + 1];
    if (xin) {
        const int li = i - L.off;
        const int I = li % (L.nx + 1), J = li / (L.nx + 1);
        T y0 = 0, y1 = 0;
        for (int s = 0; s < 9; ++s) {
            const int gx = I + (s % 3) - 1, gy = J + (s / 3) - 1;
            if (gx < 0 || gx > L.nx || gy < 0 || gy > L.ny) continue;
            const int j = L.off + gx + gy * (L.nx + 1);
            const T* k = A + 36 * (size_t)i + 4 * s;
            const T x0 = xin[2 * j], x1 = xin[2 * j + 1];
            y0 += k[0] * x0 + k[1] * x1;
            y1 += k[2] * x0 + k[3] * x1;
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
    const T z0 = m[0] * r0 + m[1] * r1, z1 = m[2] * r0 + m[3] * r1;
    xout[2 * i] = (xin ? xin[2 * i] : (T)0) + omega * z0;
    xout[2 * i + 1] = (xin ? xin[2 * i + 1] : (T)0) + omega * z1;
}

// level-0 block-Jacobi sweep over the batch's block-CSR rows
template <typename T>
__global__ void __launch_bounds__(kThreads) k_b_smooth_bsr(int n, const int* __restrict__ row_ptr,
                                                           const int* __restrict__ col, const T* __restrict__ K,
                                                           const T* __restrict__ Dinv, const uint8_t* __restrict__ fixed,
                                                           const T* __restrict__ b, const T* __restrict__ xin,
                                                           T* __restrict__ xout, T omega, const int* done, int resid_only) {
    if (done && done[0]) return;
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i >= n) return;
    T r0 = b[2 * i], r1 = b[2 * i + 1];
    if (xin) {
        T y0 = 0, y1 = 0;
        for (int q = row_ptr[i]; q < row_ptr[i + 1]; ++q) {
            const int j = col[q];
            const T* k = K + 4 * (size_t)q;
            const T x0 = xin[2 * j], x1 = xin[2 * j + 1];
            y0 += k[0] * x0 + k[1] * x1;
            y1 += k[2] * x0 + k[3] * x1;
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
    const T z0 = m[0] * r0 + m[1] * r1, z1 = m[2] * r0 + m[3] * r1;
    xout[2 * i] = (xin ? xin[2 * i] : (T)0) + omega * z0;
    xout[2 * i + 1] = (xin ? xin[2 * i + 1] : (T)0) + omega * z1;
}

// b_c(a) = mask_c(sum_{i child of a} P_ia r_f(i)) over the nodes of one depth
template <typename T>
__global__ void k_b_restrict(int n, const int* __restrict__ node_rve, const BDesc* D, const T* __restrict__ rf,
                             const uint8_t* fixed_c, T* __restrict__ bc, const int* done) {
    if (done && done[0]) return;
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= n) return;
    const BDesc L = D[node_rve[a]];
    const int la = a - L.off;
    const int Ia = la % (L.nx + 1), Ja = la / (L.nx + 1);
    const int px = b_pos(Ia, L.fnx), py = b_pos(Ja, L.fny);
    T s0 = 0, s1 = 0;
    for (int cy = py - 1; cy <= py + 1; ++cy) {
        if (cy < 0 || cy > L.fny) continue;
        const double wy = b_w(cy, L.fny, Ja);
        if (wy == 0.0) continue;
        for (int cx = px - 1; cx <= px + 1; ++cx) {
            if (cx < 0 || cx > L.fnx) continue;
            const double wx = b_w(cx, L.fnx, Ia);
            if (wx == 0.0) continue;
            const int i = L.foff + cx + cy * (L.fnx + 1);
            const T w = (T)(wx * wy);
            s0 += w * rf[2 * i];
            s1 += w * rf[2 * i + 1];
        }
    }
    bc[2 * a] = fixed_c[2 * a] ? (T)0 : s0;
    bc[2 * a + 1] = fixed_c[2 * a + 1] ? (T)0 : s1;
}

// x_f(i) += mask_f(sum_a P_ia x_c(a)) over the regular nodes of the finer grids.
// nf nodes of the finer depth; for depth 0 node_rve_f is the batch's node map
// and the descriptor of depth 1 gives each RVE's fine grid (foff, fnx, fny).
template <typename T>
__global__ void k_b_prolong(int nf, const int* __restrict__ node_rve_f, const BDesc* Dc, const T* __restrict__ xc,
                            const uint8_t* fixed_f, T* __restrict__ xf, const int* done) {
    if (done && done[0]) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nf) return;
    const BDesc L = Dc[node_rve_f[i]];
    if (!L.present) return;  // that RVE's grid at the finer depth is its coarsest
    const int li = i - L.foff;
    if (li < 0 || li >= (L.fnx + 1) * (L.fny + 1)) return;  // enrichment nodes: no coarse part
    const int gx = li % (L.fnx + 1), gy = li / (L.fnx + 1);
    int Ix[2], Iy[2];
    T wxs[2], wys[2];
    int nxp, nyp;
    if ((gx & 1) == 0) { Ix[0] = gx >> 1; wxs[0] = 1; nxp = 1; }
    else if (gx == L.fnx) { Ix[0] = (L.fnx + 1) >> 1; wxs[0] = 1; nxp = 1; }
    else { Ix[0] = (gx - 1) >> 1; Ix[1] = (gx + 1) >> 1; wxs[0] = wxs[1] = (T)0.5; nxp = 2; }
    if ((gy & 1) == 0) { Iy[0] = gy >> 1; wys[0] = 1; nyp = 1; }
    else if (gy == L.fny) { Iy[0] = (L.fny + 1) >> 1; wys[0] = 1; nyp = 1; }
    else { Iy[0] = (gy - 1) >> 1; Iy[1] = (gy + 1) >> 1; wys[0] = wys[1] = (T)0.5; nyp = 2; }
    T s0 = 0, s1 = 0;
    for (int py = 0; py < nyp; ++py)
        for (int px = 0; px < nxp; ++px) {
            const int a = L.off + Ix[px] + Iy[py] * (L.nx + 1);
            const T w = wxs[px] * wys[py];
            s0 += w * xc[2 * a];
            s1 += w * xc[2 * a + 1];
        }
    if (!fixed_f[2 * i]) xf[2 * i] += s0;
    if (!fixed_f[2 * i + 1]) xf[2 * i + 1] += s1;
}

// Every RVE's coarsest grid: x = U^-1 L^-1 P b, one CTA per RVE.
template <typename T>
__global__ void k_b_coarse_solve(const BCoarse* cd, const double* __restrict__ LU, const int* __restrict__ piv,
                                 uint8_t* const* Fdepth, T* const* Bdepth, T* const* Xdepth, const int* done) {
    if (done && done[0]) return;
    __shared__ double y[kBCoarseMaxDof];
    const int r = blockIdx.x;
    const BCoarse C = cd[r];
    const int n = 2 * (C.nx + 1) * (C.ny + 1);
    const uint8_t* fixed = Fdepth[C.depth] + 2 * C.off;
    const T* b = Bdepth[C.depth] + 2 * C.off;
    T* x = Xdepth[C.depth] + 2 * C.off;
    const double* LUr = LU + (size_t)r * kBCoarseStride;
    const int* pv = piv + r * kBCoarseMaxDof;
    for (int q = threadIdx.x; q < n; q += blockDim.x) y[q] = fixed[pv[q]] ? 0.0 : (double)b[pv[q]];
    __syncthreads();
    for (int k = 0; k < n; ++k) {
        const double yk = y[k];
        for (int q = k + 1 + threadIdx.x; q < n; q += blockDim.x) y[q] -= LUr[q * n + k] * yk;
        __syncthreads();
    }
    for (int k = n - 1; k >= 0; --k) {
        if (threadIdx.x == 0) y[k] = LUr[k * n + k] != 0.0 ? y[k] / LUr[k * n + k] : 0.0;
        __syncthreads();
        const double yk = y[k];
        for (int q = threadIdx.x; q < k; q += blockDim.x) y[q] -= LUr[q * n + k] * yk;
        __syncthreads();
    }
    for (int q = threadIdx.x; q < n; q += blockDim.x) x[q] = fixed[q] ? (T)0 : (T)y[q];
}

__global__ void k_b_f64_to_f32(int n, const double* __restrict__ a, float* __restrict__ b, const int* done) {
    if (done && done[0]) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = (float)a[i];
}

__global__ void k_b_f32_to_f64(int n, const float* __restrict__ a, double* __restrict__ b, const int* done) {
    if (done && done[0]) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = (double)a[i];
}

// z = M^-1 r (block Jacobi), whole batch
__global__ void k_b_jacobi(int n, const double* __restrict__ minv, const double* __restrict__ r, double* __restrict__ z,
                           const int* done) {
    if (done && done[0]) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double* m = minv + 4 * (size_t)i;
    const double r0 = r[2 * i], r1 = r[2 * i + 1];
    z[2 * i] = m[0] * r0 + m[1] * r1;
    z[2 * i + 1] = m[2] * r0 + m[3] * r1;
}

// ---------------------------------------------------------------------------
// Per-RVE CG.  Scalars per RVE (8 doubles): 0 p.q, 1 r.z, 2 new r.z, 3 r.r,
// 4 tol^2, 5 b.b, 6 true r.r; flags per RVE (4 ints): 0 done, 1 breakdown,
// 2 iterations.  g[0]: RVEs done, g[1]: all done.
// ---------------------------------------------------------------------------
// Segmented sum: lanes of a warp that share one RVE reduce by shuffles; a
// warp that straddles two RVEs adds lane by lane.
__device__ __forceinline__ void seg_add(double v, int rve, double* acc, int stride, int slot) {
    const unsigned full = 0xffffffffu;
    const int r0 = __shfl_sync(full, rve, 0);
    if (__all_sync(full, rve == r0)) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(full, v, o);
        if ((threadIdx.x & 31) == 0 && rve >= 0) atomicAdd(&acc[(size_t)rve * stride + slot], v);
    } else if (rve >= 0 && v != 0.0) {
        atomicAdd(&acc[(size_t)rve * stride + slot], v);
    }
}

__global__ void __launch_bounds__(kThreads) k_bcg_start(int nd, const int* __restrict__ node_rve,
                                                        const uint8_t* __restrict__ fixed, const double* __restrict__ b,
                                                        double* __restrict__ r, double* __restrict__ x, double* sc) {
    const int i = blockIdx.x * kThreads + threadIdx.x;
    double v = 0.0;
    int rve = -1;
    if (i < nd) {
        v = fixed[i] ? 0.0 : b[i];
        r[i] = v;
        x[i] = 0.0;
        rve = node_rve[i >> 1];
    }
    seg_add(v * v, rve, sc, 8, 3);
}

__global__ void k_bcg_tol(int nr, double* sc, int* fl, int* g, double rtol2) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nr) return;
    double* s = sc + 8 * r;
    s[5] = s[3];
    s[4] = rtol2 * s[3];
    if (s[3] == 0.0) {
        fl[4 * r] = 1;
        atomicAdd(&g[0], 1);
    }
}

__global__ void k_bcg_alldone(int nr, int* g) {
    if (g[0] >= nr) g[1] = 1;
}

__global__ void k_bcg_s1(int nr, double* sc, const int* fl, const int* g) {
    if (g[1]) return;
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nr || fl[4 * r]) return;
    double* s = sc + 8 * r;
    s[1] = s[2];
    s[0] = 0.0;
    s[3] = 0.0;
}

__global__ void __launch_bounds__(kThreads) k_bcg_spmv(int n, const int* __restrict__ node_rve,
                                                       const int* __restrict__ row_ptr, const int* __restrict__ col,
                                                       const double* __restrict__ K, const double* __restrict__ p,
                                                       const uint8_t* __restrict__ fixed, double* __restrict__ q,
                                                       double* sc, const int* g) {
    if (g[1]) return;
    const int i = blockIdx.x * kThreads + threadIdx.x;
    double part = 0.0;
    int rve = -1;
    if (i < n) {
        double y0, y1;
        bsr_row<double, double>(i, row_ptr, col, K, p, y0, y1);
        if (fixed[2 * i]) y0 = 0.0;
        if (fixed[2 * i + 1]) y1 = 0.0;
        q[2 * i] = y0;
        q[2 * i + 1] = y1;
        part = p[2 * i] * y0 + p[2 * i + 1] * y1;
        rve = node_rve[i];
    }
    seg_add(part, rve, sc, 8, 0);
}

__global__ void __launch_bounds__(kThreads) k_bcg_update(int nd, const int* __restrict__ node_rve,
                                                         double* __restrict__ x, double* __restrict__ r,
                                                         const double* __restrict__ p, const double* __restrict__ q,
                                                         double* sc, int* fl, const int* g) {
    if (g[1]) return;
    const int i = blockIdx.x * kThreads + threadIdx.x;
    double part = 0.0;
    int rve = -1;
    if (i < nd) {
        rve = node_rve[i >> 1];
        const double* s = sc + 8 * rve;
        if (!fl[4 * rve]) {
            const double pq = s[0];
            if (pq > 0.0) {
                const double alpha = s[1] / pq;
                x[i] += alpha * p[i];
                const double ri = r[i] - alpha * q[i];
                r[i] = ri;
                part = ri * ri;
            } else {
                fl[4 * rve + 1] = 1;
            }
        }
    }
    seg_add(part, rve, sc, 8, 3);
}

__global__ void k_bcg_s2(int nr, double* sc, int* fl, int* g) {
    if (g[1]) return;
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nr || fl[4 * r]) return;
    double* s = sc + 8 * r;
    fl[4 * r + 2] += 1;
    if (fl[4 * r + 1] || s[3] <= s[4]) {
        fl[4 * r] = 1;
        atomicAdd(&g[0], 1);
    }
    s[2] = 0.0;
}

__global__ void __launch_bounds__(kThreads) k_bcg_dot(int nd, const int* __restrict__ node_rve, const double* __restrict__ a,
                                                      const double* __restrict__ b, double* sc, int slot, const int* g) {
    if (g && g[1]) return;
    const int i = blockIdx.x * kThreads + threadIdx.x;
    double v = 0.0;
    int rve = -1;
    if (i < nd) {
        v = a[i] * b[i];
        rve = node_rve[i >> 1];
    }
    seg_add(v, rve, sc, 8, slot);
}

__global__ void __launch_bounds__(kThreads) k_bcg_pupdate(int nd, const int* __restrict__ node_rve,
                                                          const double* __restrict__ z, double* __restrict__ p,
                                                          const double* sc, const int* fl, const int* g) {
    if (g[1]) return;
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i >= nd) return;
    const int rve = node_rve[i >> 1];
    if (fl[4 * rve]) return;
    const double* s = sc + 8 * rve;
    p[i] = z[i] + (s[2] / s[1]) * p[i];
}

template <typename T>
int b_alloc(std::vector<void*>& owned, T** p, size_t n) {
    *p = nullptr;
    PG_CUDA(cudaMalloc((void**)p, std::max<size_t>(n, 1) * sizeof(T)));
    PG_CUDA(fill_sync(*p, 0, std::max<size_t>(n, 1) * sizeof(T)));
    owned.push_back((void*)*p);
    return PG_OK;
}

template <typename T>
int b_upload(std::vector<void*>& owned, T** p, const std::vector<T>& v) {
    int rc = b_alloc(owned, p, v.size());
    if (rc) return rc;
    if (!v.empty()) PG_CUDA(h2d_sync(*p, v.data(), v.size() * sizeof(T)));
    return PG_OK;
}

}  // namespace
}  // namespace pgb

struct pg_batch {
    int n_rve = 0;
    // host seconds of the set-up: mesh copies, merge, context (uploads, grid
    // tiles, cut tables, fold order), multigrid hierarchy
    double setup_s[7] = {0, 0, 0, 0, 0, 0, 0};
    std::vector<std::pair<int, int>> grid;  // background grid (nx, ny) of each RVE
    std::vector<int> noff;              // first node of each RVE (+ total)
    std::vector<int> eoff;              // first element of each RVE (+ total)
    pg_ctx ctx;                         // the merged system
    // union multigrid hierarchy
    int dmax = 0;
    std::vector<int> depth;             // per RVE
    pgb::BDepth lv[pgb::kBMaxDepth + 1];
    int* node_rve0 = nullptr;           // batch nodes -> RVE
    pgb::BDesc* desc1 = nullptr;        // alias of lv[1].desc (fine grids of depth 0)
    pgb::BCoarse* coarse = nullptr;     // per RVE
    double** Aptr = nullptr;            // per depth (device arrays of device pointers)
    uint8_t** Fptr = nullptr;
    double** Bptr = nullptr;
    double** Xptr = nullptr;
    float** Bfptr = nullptr;
    float** Xfptr = nullptr;
    double* LU = nullptr;
    int* piv = nullptr;
    int* bad = nullptr;
    double *x0 = nullptr, *x0b = nullptr, *r0 = nullptr;
    float *b0f = nullptr, *x0f = nullptr, *x0bf = nullptr, *r0f = nullptr, *Dinv0f = nullptr;
    // per-RVE CG
    double* sc = nullptr;
    int* fl = nullptr;
    int* g = nullptr;
    std::vector<void*> owned;
};

namespace pgb {
namespace {

// Concatenates the RVE meshes into one block-diagonal mesh: every array's
// place per RVE first (prefix sums of the sizes), then the RVEs copied and
// renumbered in parallel, each into its own range.
void merge_meshes(const pg_mesh* const* ms, int R, HostMesh& out, std::vector<int>& noff, std::vector<int>& eoff) {
    out = HostMesh();
    auto M = [&](int r) -> const HostMesh& { return ms[r]->m; };
    noff.assign(R + 1, 0);
    eoff.assign(R + 1, 0);
    std::vector<int> moff(R + 1, 0), coff(R + 1, 0), boff(R + 1, 0), qoff(R + 1, 0), koff(R + 1, 0);
    for (int r = 0; r < R; ++r) {
        noff[r + 1] = noff[r] + M(r).n_nodes();
        eoff[r + 1] = eoff[r] + M(r).n_elem;
        moff[r + 1] = moff[r] + (int)M(r).spec.materials.size();
        coff[r + 1] = coff[r] + M(r).n_cut;
        boff[r + 1] = boff[r] + M(r).n_blocks();
        qoff[r + 1] = qoff[r] + M(r).n_coh_qp;
        koff[r + 1] = koff[r] + (int)M(r).ne_list.size();
    }
    // the place of each RVE's part of one array, and the array sized to all
    // (its pages backed by huge pages where the host allows it: sizing a
    // multi-GB array otherwise costs a page fault per 4 KB)
    auto place = [&](auto field, auto& dst) {
        std::vector<size_t> o(R + 1, 0);
        for (int r = 0; r < R; ++r) o[r + 1] = o[r] + (M(r).*field).size();
        dst.reserve(o[R]);
        const size_t bytes = o[R] * sizeof(dst[0]);
        if (bytes >= (8u << 20)) {
            const uintptr_t a = (reinterpret_cast<uintptr_t>(dst.data()) + 4095) & ~uintptr_t(4095);
            const uintptr_t e = reinterpret_cast<uintptr_t>(dst.data()) + bytes;
            if (e > a) madvise(reinterpret_cast<void*>(a), e - a, MADV_HUGEPAGE);
        }
        dst.resize(o[R]);
        return o;
    };
    const auto o_x = place(&HostMesh::x, out.x);
    place(&HostMesh::y, out.y);
    const auto o_conn = place(&HostMesh::conn, out.conn);
    const auto o_emat = place(&HostMesh::elem_mat, out.elem_mat);
    place(&HostMesh::elem_cut, out.elem_cut);
    const auto o_cut = place(&HostMesh::cut_elem, out.cut_elem);
    place(&HostMesh::cut_tmpl, out.cut_tmpl);
    const auto o_cenr = place(&HostMesh::cut_enr, out.cut_enr);
    const auto o_cchm = place(&HostMesh::cut_child_mat, out.cut_child_mat);
    const auto o_ccoh = place(&HostMesh::cut_coh_mat, out.cut_coh_mat);
    place(&HostMesh::cut_coh_qp0, out.cut_coh_qp0);
    const auto o_fix = place(&HostMesh::fixed, out.fixed);
    place(&HostMesh::ubar, out.ubar);
    const auto o_col = place(&HostMesh::col, out.col);
    const auto o_diag = place(&HostMesh::diag_slot, out.diag_slot);
    const auto o_nel = place(&HostMesh::ne_list, out.ne_list);
    const auto o_slot = place(&HostMesh::cut_slot, out.cut_slot);
    out.row_ptr.assign((size_t)noff[R] + 1, 0);
    out.ne_ptr.assign((size_t)noff[R] + 1, 0);
    parallel_for(R, 1, [&](long long rr) {
        const int r = (int)rr;
        const HostMesh& m = M(r);
        const int no = noff[r], eo = eoff[r], mo = moff[r], co = coff[r], bo = boff[r], qo = qoff[r], ko = koff[r];
        std::copy(m.x.begin(), m.x.end(), out.x.begin() + o_x[r]);
        std::copy(m.y.begin(), m.y.end(), out.y.begin() + o_x[r]);
        for (size_t i = 0; i < m.conn.size(); ++i) out.conn[o_conn[r] + i] = m.conn[i] + no;
        for (size_t i = 0; i < m.elem_mat.size(); ++i) {
            out.elem_mat[o_emat[r] + i] = m.elem_mat[i] + mo;
            out.elem_cut[o_emat[r] + i] = m.elem_cut[i] >= 0 ? m.elem_cut[i] + co : -1;
        }
        for (size_t i = 0; i < m.cut_elem.size(); ++i) {
            out.cut_elem[o_cut[r] + i] = m.cut_elem[i] + eo;
            out.cut_tmpl[o_cut[r] + i] = m.cut_tmpl[i];
            out.cut_coh_qp0[o_cut[r] + i] = m.cut_coh_qp0[i] + qo;
        }
        for (size_t i = 0; i < m.cut_enr.size(); ++i) out.cut_enr[o_cenr[r] + i] = m.cut_enr[i] >= 0 ? m.cut_enr[i] + no : -1;
        for (size_t i = 0; i < m.cut_child_mat.size(); ++i)
            out.cut_child_mat[o_cchm[r] + i] = m.cut_child_mat[i] >= 0 ? m.cut_child_mat[i] + mo : -1;
        std::copy(m.cut_coh_mat.begin(), m.cut_coh_mat.end(), out.cut_coh_mat.begin() + o_ccoh[r]);
        std::copy(m.fixed.begin(), m.fixed.end(), out.fixed.begin() + o_fix[r]);
        std::copy(m.ubar.begin(), m.ubar.end(), out.ubar.begin() + o_fix[r]);
        for (size_t i = 1; i < m.row_ptr.size(); ++i) out.row_ptr[no + i] = m.row_ptr[i] + bo;
        for (size_t i = 0; i < m.col.size(); ++i) out.col[o_col[r] + i] = m.col[i] + no;
        for (size_t i = 0; i < m.diag_slot.size(); ++i) out.diag_slot[o_diag[r] + i] = m.diag_slot[i] + bo;
        for (size_t i = 1; i < m.ne_ptr.size(); ++i) out.ne_ptr[no + i] = m.ne_ptr[i] + ko;
        for (size_t i = 0; i < m.ne_list.size(); ++i) {
            const int v = m.ne_list[i];
            out.ne_list[o_nel[r] + i] = (((v >> 2) + eo) << 2) | (v & 3);
        }
        for (size_t i = 0; i < m.cut_slot.size(); ++i) out.cut_slot[o_slot[r] + i] = m.cut_slot[i] >= 0 ? m.cut_slot[i] + bo : -1;
    });
    out.spec = M(0).spec;
    out.spec.materials.clear();
    out.spec.inclusions.clear();
    out.spec.nx = out.spec.ny = 0;
    out.n_reg = noff[R];  // every node counts as "regular" for the batch-level views
    out.n_enr = 0;
    out.n_elem = eoff[R];
    out.n_cut = coff[R];
    out.n_coh_qp = qoff[R];
    for (int r = 0; r < R; ++r) {
        const HostMesh& m = M(r);
        out.spec.materials.insert(out.spec.materials.end(), m.spec.materials.begin(), m.spec.materials.end());
        out.n_free += m.n_free;
        for (const auto& gb : m.grids)
            out.grids.push_back({gb.nx, gb.ny, gb.node_off + noff[r], gb.elem_off + eoff[r], gb.n_reg});
    }
}

// Builds the union hierarchy (structure once per batch).
int batch_mg_build(pg_batch& B) {
    Ctx& c = B.ctx.c;
    const int R = B.n_rve;
    auto& own = B.owned;
    int rc;
    B.depth.assign(R, 0);
    // per-RVE grid sizes per depth
    std::vector<std::vector<std::pair<int, int>>> dims(R);
    for (int r = 0; r < R; ++r) {
        int nx = B.grid[r].first, ny = B.grid[r].second;
        dims[r].push_back({nx, ny});
        while ((nx > kBCoarseCells || ny > kBCoarseCells) && (int)dims[r].size() <= kBMaxDepth) {
            nx = (nx + 1) / 2;
            ny = (ny + 1) / 2;
            dims[r].push_back({nx, ny});
        }
        if (dims[r].size() < 2 || nx > kBCoarseCells || ny > kBCoarseCells) {
            set_error("pg_batch: an RVE grid cannot be coarsened to at most 4 cells per side");
            return PG_ERR_ARG;
        }
        B.depth[r] = (int)dims[r].size() - 1;
        B.dmax = std::max(B.dmax, B.depth[r]);
    }
    // depth-0 node map
    std::vector<int> nr0(B.noff[R]);
    for (int r = 0; r < R; ++r)
        for (int i = B.noff[r]; i < B.noff[r + 1]; ++i) nr0[i] = r;
    if ((rc = b_upload(own, &B.node_rve0, nr0))) return rc;
    std::vector<int> prev_off(R);
    for (int r = 0; r < R; ++r) prev_off[r] = B.noff[r];
    std::vector<double*> Ap(B.dmax + 1, nullptr), Bp(B.dmax + 1, nullptr), Xp(B.dmax + 1, nullptr);
    std::vector<uint8_t*> Fp(B.dmax + 1, nullptr);
    std::vector<float*> Bfp(B.dmax + 1, nullptr), Xfp(B.dmax + 1, nullptr);
    std::vector<BCoarse> cd(R);
    for (int d = 1; d <= B.dmax; ++d) {
        BDepth& L = B.lv[d];
        std::vector<BDesc> desc(R, BDesc{0, 0, 0, 0, 0, 0, 0, 0});
        std::vector<int> nr;
        int off = 0;
        for (int r = 0; r < R; ++r) {
            if (B.depth[r] < d) continue;
            BDesc D;
            D.off = off;
            D.nx = dims[r][d].first;
            D.ny = dims[r][d].second;
            D.foff = prev_off[r];
            D.fnx = dims[r][d - 1].first;
            D.fny = dims[r][d - 1].second;
            D.coarsest = B.depth[r] == d ? 1 : 0;
            D.present = 1;
            desc[r] = D;
            const int n = (D.nx + 1) * (D.ny + 1);
            for (int k = 0; k < n; ++k) nr.push_back(r);
            if (D.coarsest) cd[r] = BCoarse{d, off, D.nx, D.ny};
            prev_off[r] = off;
            off += n;
        }
        L.n = off;
        const size_t n = (size_t)std::max(off, 1);
        if ((rc = b_upload(own, &L.node_rve, nr)) || (rc = b_upload(own, &L.desc, desc))) return rc;
        if ((rc = b_alloc(own, &L.A, 36 * n)) || (rc = b_alloc(own, &L.Af, 36 * n)) || (rc = b_alloc(own, &L.Dinv, 4 * n)) ||
            (rc = b_alloc(own, &L.Dinvf, 4 * n)) || (rc = b_alloc(own, &L.fixed, 2 * n)))
            return rc;
        if ((rc = b_alloc(own, &L.x, 2 * n)) || (rc = b_alloc(own, &L.x2, 2 * n)) || (rc = b_alloc(own, &L.b, 2 * n)) ||
            (rc = b_alloc(own, &L.r, 2 * n)) || (rc = b_alloc(own, &L.xf, 2 * n)) || (rc = b_alloc(own, &L.x2f, 2 * n)) ||
            (rc = b_alloc(own, &L.bf, 2 * n)) || (rc = b_alloc(own, &L.rf, 2 * n)))
            return rc;
        Ap[d] = L.A;
        Fp[d] = L.fixed;
        Bp[d] = L.b;
        Xp[d] = L.x2;  // the V-cycle's final buffer at every depth (even sweep counts)
        Bfp[d] = L.bf;
        Xfp[d] = L.x2f;
        const uint8_t* ff = d == 1 ? c.fixed : B.lv[d - 1].fixed;
        k_b_inject_mask<<<nb(L.n), kThreads, 0, c.stream>>>(L.n, L.node_rve, L.desc, ff, L.fixed);
    }
    B.desc1 = B.lv[1].desc;
    if ((rc = b_upload(own, &B.coarse, cd)) || (rc = b_upload(own, &B.Aptr, Ap)) || (rc = b_upload(own, &B.Fptr, Fp)) ||
        (rc = b_upload(own, &B.Bptr, Bp)) || (rc = b_upload(own, &B.Xptr, Xp)) || (rc = b_upload(own, &B.Bfptr, Bfp)) ||
        (rc = b_upload(own, &B.Xfptr, Xfp)))
        return rc;
    if ((rc = b_alloc(own, &B.LU, (size_t)R * kBCoarseStride)) || (rc = b_alloc(own, &B.piv, (size_t)R * kBCoarseMaxDof)) ||
        (rc = b_alloc(own, &B.bad, (size_t)R)))
        return rc;
    const size_t nd = (size_t)c.n_dof;
    if ((rc = b_alloc(own, &B.x0, nd)) || (rc = b_alloc(own, &B.x0b, nd)) || (rc = b_alloc(own, &B.r0, nd)) ||
        (rc = b_alloc(own, &B.b0f, nd)) || (rc = b_alloc(own, &B.x0f, nd)) || (rc = b_alloc(own, &B.x0bf, nd)) ||
        (rc = b_alloc(own, &B.r0f, nd)) || (rc = b_alloc(own, &B.Dinv0f, 4 * (size_t)c.n_nodes)))
        return rc;
    if ((rc = b_alloc(own, &B.sc, 8 * (size_t)R)) || (rc = b_alloc(own, &B.fl, 4 * (size_t)R)) || (rc = b_alloc(own, &B.g, 8)))
        return rc;
    PG_CUDA(cudaGetLastError());
    PG_CUDA(cudaStreamSynchronize(c.stream));
    return PG_OK;
}

// Numeric set-up for the current K.
int batch_mg_numeric(pg_batch& B, bool f32, cudaStream_t s) {
    Ctx& c = B.ctx.c;
    const int n0 = c.n_nodes;
    k_prec_setup<double><<<nb(n0), kThreads, 0, s>>>(n0, c.diag, c.K, c.fixed, 1, 0, c.minv);
    if (f32) {
        launch_to_fp32(c, s);
        k_b_f64_to_f32<<<nb(4LL * n0), kThreads, 0, s>>>(4 * n0, c.minv, B.Dinv0f, nullptr);
    }
    for (int d = 1; d <= B.dmax; ++d) {
        BDepth& L = B.lv[d];
        if (d == 1)
            k_b_galerkin<true><<<nb(9LL * L.n), kThreads, 0, s>>>(L.n, L.node_rve, L.desc, c.row_ptr, c.col, c.K, nullptr,
                                                                  c.fixed, L.fixed, L.A);
        else
            k_b_galerkin<false><<<nb(9LL * L.n), kThreads, 0, s>>>(L.n, L.node_rve, L.desc, nullptr, nullptr, nullptr,
                                                                   B.lv[d - 1].A, B.lv[d - 1].fixed, L.fixed, L.A);
        k_b_dinv<<<nb(L.n), kThreads, 0, s>>>(L.n, L.A, L.fixed, L.Dinv, L.Dinvf, L.Af);
    }
    cudaMemsetAsync(B.bad, 0, (size_t)B.n_rve * sizeof(int), s);
    k_b_coarse_factor<<<B.n_rve, 128, 0, s>>>(B.coarse, B.Aptr, B.Fptr, B.LU, B.piv, B.bad);
    PG_CUDA(cudaGetLastError());
    return PG_OK;
}

// One union V-cycle: returns the level-0 buffer holding V(b0).
template <typename T>
struct BV;

template <>
struct BV<double> {
    static const double* run(pg_batch& B, cudaStream_t s, const double* b0, const int* done) {
        Ctx& c = B.ctx.c;
        const int n0 = c.n_nodes;
        const double om = kBOmega;
        double* cur = B.x0;
        double* alt = B.x0b;
        k_b_smooth_bsr<double><<<nb(n0), kThreads, 0, s>>>(n0, c.row_ptr, c.col, c.K, c.minv, c.fixed, b0, nullptr, cur,
                                                             om, done, 0);
        k_b_smooth_bsr<double><<<nb(n0), kThreads, 0, s>>>(n0, c.row_ptr, c.col, c.K, c.minv, c.fixed, b0, cur, alt, om,
                                                             done, 0);
        std::swap(cur, alt);
        k_b_smooth_bsr<double><<<nb(n0), kThreads, 0, s>>>(n0, c.row_ptr, c.col, c.K, c.minv, c.fixed, b0, cur, B.r0, om,
                                                             done, 1);
        const double* rf = B.r0;
        for (int d = 1; d <= B.dmax; ++d) {
            BDepth& L = B.lv[d];
            k_b_restrict<double><<<nb(L.n), kThreads, 0, s>>>(L.n, L.node_rve, L.desc, rf, L.fixed, L.b, done);
            if (d == B.dmax) break;
            // RVEs that continue: two sweeps (x, then x2), residual into r
            k_b_smooth_st<double><<<nb(L.n), kThreads, 0, s>>>(L.n, L.node_rve, L.desc, L.A, L.Dinv, L.fixed, L.b, nullptr,
                                                                 L.x, om, done, 0);
            k_b_smooth_st<double><<<nb(L.n), kThreads, 0, s>>>(L.n, L.node_rve, L.desc, L.A, L.Dinv, L.fixed, L.b, L.x, L.x2,
                                                                 om, done, 0);
            k_b_smooth_st<double><<<nb(L.n), kThreads, 0, s>>>(L.n, L.node_rve, L.desc, L.A, L.Dinv, L.fixed, L.b, L.x2, L.r,
                                                                 om, done, 1);
            rf = L.r;
        }
        k_b_coarse_solve<double><<<B.n_rve, 128, 0, s>>>(B.coarse, B.LU, B.piv, B.Fptr, B.Bptr, B.Xptr, done);
        for (int d = B.dmax - 1; d >= 1; --d) {
            BDepth& L = B.lv[d];
            const BDepth& C = B.lv[d + 1];
            k_b_prolong<double><<<nb(L.n), kThreads, 0, s>>>(L.n, L.node_rve, C.desc, C.x2, L.fixed, L.x2, done);
            k_b_smooth_st<double><<<nb(L.n), kThreads, 0, s>>>(L.n, L.node_rve, L.desc, L.A, L.Dinv, L.fixed, L.b, L.x2, L.x,
                                                                 om, done, 0);
            k_b_smooth_st<double><<<nb(L.n), kThreads, 0, s>>>(L.n, L.node_rve, L.desc, L.A, L.Dinv, L.fixed, L.b, L.x, L.x2,
                                                                 om, done, 0);
        }
        k_b_prolong<double><<<nb(n0), kThreads, 0, s>>>(n0, B.node_rve0, B.desc1, B.lv[1].x2, c.fixed, cur, done);
        for (int it = 0; it < 2; ++it) {
            k_b_smooth_bsr<double><<<nb(n0), kThreads, 0, s>>>(n0, c.row_ptr, c.col, c.K, c.minv, c.fixed, b0, cur, alt, om,
                                                                 done, 0);
            std::swap(cur, alt);
        }
        return cur;
    }
};

template <>
struct BV<float> {
    static const float* run(pg_batch& B, cudaStream_t s, const float* b0, const int* done) {
        Ctx& c = B.ctx.c;
        const int n0 = c.n_nodes;
        const float om = (float)kBOmega;
        float* cur = B.x0f;
        float* alt = B.x0bf;
        k_b_smooth_bsr<float><<<nb(n0), kThreads, 0, s>>>(n0, c.row_ptr, c.col, c.Kf, B.Dinv0f, c.fixed, b0, nullptr, cur,
                                                            om, done, 0);
        k_b_smooth_bsr<float><<<nb(n0), kThreads, 0, s>>>(n0, c.row_ptr, c.col, c.Kf, B.Dinv0f, c.fixed, b0, cur, alt, om,
                                                            done, 0);
        std::swap(cur, alt);
        k_b_smooth_bsr<float><<<nb(n0), kThreads, 0, s>>>(n0, c.row_ptr, c.col, c.Kf, B.Dinv0f, c.fixed, b0, cur, B.r0f,
                                                            om, done, 1);
        const float* rf = B.r0f;
        for (int d = 1; d <= B.dmax; ++d) {
            BDepth& L = B.lv[d];
            k_b_restrict<float><<<nb(L.n), kThreads, 0, s>>>(L.n, L.node_rve, L.desc, rf, L.fixed, L.bf, done);
            if (d == B.dmax) break;
            k_b_smooth_st<float><<<nb(L.n), kThreads, 0, s>>>(L.n, L.node_rve, L.desc, L.Af, L.Dinvf, L.fixed, L.bf, nullptr,
                                                                L.xf, om, done, 0);
            k_b_smooth_st<float><<<nb(L.n), kThreads, 0, s>>>(L.n, L.node_rve, L.desc, L.Af, L.Dinvf, L.fixed, L.bf, L.xf,
                                                                L.x2f, om, done, 0);
            k_b_smooth_st<float><<<nb(L.n), kThreads, 0, s>>>(L.n, L.node_rve, L.desc, L.Af, L.Dinvf, L.fixed, L.bf, L.x2f,
                                                                L.rf, om, done, 1);
            rf = L.rf;
        }
        k_b_coarse_solve<float><<<B.n_rve, 128, 0, s>>>(B.coarse, B.LU, B.piv, B.Fptr, B.Bfptr, B.Xfptr, done);
        for (int d = B.dmax - 1; d >= 1; --d) {
            BDepth& L = B.lv[d];
            const BDepth& C = B.lv[d + 1];
            k_b_prolong<float><<<nb(L.n), kThreads, 0, s>>>(L.n, L.node_rve, C.desc, C.x2f, L.fixed, L.x2f, done);
            k_b_smooth_st<float><<<nb(L.n), kThreads, 0, s>>>(L.n, L.node_rve, L.desc, L.Af, L.Dinvf, L.fixed, L.bf, L.x2f,
                                                                L.xf, om, done, 0);
            k_b_smooth_st<float><<<nb(L.n), kThreads, 0, s>>>(L.n, L.node_rve, L.desc, L.Af, L.Dinvf, L.fixed, L.bf, L.xf,
                                                                L.x2f, om, done, 0);
        }
        k_b_prolong<float><<<nb(n0), kThreads, 0, s>>>(n0, B.node_rve0, B.desc1, B.lv[1].x2f, c.fixed, cur, done);
        for (int it = 0; it < 2; ++it) {
            k_b_smooth_bsr<float><<<nb(n0), kThreads, 0, s>>>(n0, c.row_ptr, c.col, c.Kf, B.Dinv0f, c.fixed, b0, cur, alt,
                                                                om, done, 0);
            std::swap(cur, alt);
        }
        return cur;
    }
};

void batch_precondition(pg_batch& B, int precond, bool f32, cudaStream_t s, const double* r, double* z, const int* done) {
    Ctx& c = B.ctx.c;
    const int nd = c.n_dof;
    if (precond != PG_PREC_MG) {
        k_b_jacobi<<<nb(c.n_nodes), kThreads, 0, s>>>(c.n_nodes, c.minv, r, z, done);
        return;
    }
    if (f32) {
        k_b_f64_to_f32<<<nb(nd), kThreads, 0, s>>>(nd, r, B.b0f, done);
        const float* x = BV<float>::run(B, s, B.b0f, done);
        k_b_f32_to_f64<<<nb(nd), kThreads, 0, s>>>(nd, x, z, done);
    } else {
        const double* x = BV<double>::run(B, s, r, done);
        cudaMemcpyAsync(z, x, (size_t)nd * sizeof(double), cudaMemcpyDeviceToDevice, s);
    }
}

}  // namespace
}  // namespace pgb

using namespace pgb;

extern "C" {

int pg_batch_create(const pg_mesh* const* meshes, int32_t n_rve, int32_t device, pg_batch** out) {
    if (!meshes || !out || n_rve <= 0) { set_error("pg_batch_create: invalid argument"); return PG_ERR_ARG; }
    *out = nullptr;
    for (int r = 0; r < n_rve; ++r) {
        if (!meshes[r]) { set_error("pg_batch_create: null mesh"); return PG_ERR_ARG; }
        if (meshes[r]->m.spec.cohesive) {
            set_error("pg_batch_create: batches hold linear-elastic RVEs (no cohesive interfaces)");
            return PG_ERR_ARG;
        }
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        set_error("pg_batch_create: no CUDA device (this library has no CPU fallback)");
        return PG_ERR_CUDA;
    }
    if (device < 0 || device >= ndev) { set_error("pg_batch_create: invalid device"); return PG_ERR_ARG; }
    pg_batch* B = new (std::nothrow) pg_batch;
    if (!B) { set_error("pg_batch_create: out of host memory"); return PG_ERR_ARG; }
    B->n_rve = n_rve;
    auto now = [] { return std::chrono::steady_clock::now(); };
    auto secs = [](auto a, auto b) { return std::chrono::duration<double>(b - a).count(); };
    auto t0 = now();
    for (int r = 0; r < n_rve; ++r) B->grid.push_back({meshes[r]->m.spec.nx, meshes[r]->m.spec.ny});
    auto t1 = now();
    HostMesh merged;
    merge_meshes(meshes, n_rve, merged, B->noff, B->eoff);
    auto t2 = now();
    int rc = ctx_create(std::move(merged), device, B->ctx.c);
    auto t3 = now();
    if (rc == PG_OK) rc = batch_mg_build(*B);
    B->setup_s[0] = secs(t0, t1);
    B->setup_s[1] = secs(t1, t2);
    for (int k = 0; k < 4; ++k) B->setup_s[2 + k] = B->ctx.c.setup_s[k];
    B->setup_s[6] = secs(t3, now());
    if (rc != PG_OK) {
        pg_batch_destroy(B);
        return rc;
    }
    *out = B;
    return PG_OK;
}

void pg_batch_destroy(pg_batch* B) {
    if (!B) return;
    cudaSetDevice(B->ctx.c.device);
    for (void* p : B->owned) cudaFree(p);
    free_ctx(B->ctx.c);
    delete B;
}

pg_ctx* pg_batch_context(pg_batch* B) { return B ? &B->ctx : nullptr; }

int pg_batch_setup_times(const pg_batch* B, double* seconds) {
    if (!B || !seconds) { set_error("pg_batch_setup_times: null argument"); return PG_ERR_ARG; }
    for (int k = 0; k < 7; ++k) seconds[k] = B->setup_s[k];
    return PG_OK;
}

int pg_batch_info(const pg_batch* B, int32_t* node_offset, int32_t* element_offset, int32_t* depth) {
    if (!B) { set_error("pg_batch_info: null batch"); return PG_ERR_ARG; }
    for (int r = 0; r <= B->n_rve; ++r) {
        if (node_offset) node_offset[r] = B->noff[r];
        if (element_offset) element_offset[r] = B->eoff[r];
    }
    if (depth)
        for (int r = 0; r < B->n_rve; ++r) depth[r] = B->depth[r];
    return PG_OK;
}

int pg_batch_solve(pg_batch* B, const pg_solver_cfg* cfg, pg_solve_stats* per_rve, pg_solve_stats* total) {
    if (!B || !cfg) { set_error("pg_batch_solve: invalid argument"); return PG_ERR_ARG; }
    Ctx& c = B->ctx.c;
    cudaSetDevice(c.device);
    if (cfg->krylov != PG_KRYLOV_CG) { set_error("pg_batch_solve: batches are solved by CG"); return PG_ERR_ARG; }
    cudaStream_t s = c.stream;
    const int R = B->n_rve, n = c.n_nodes, nd = c.n_dof;
    const bool f32 = cfg->precision == PG_PRECISION_MIXED;
    const int pc = cfg->precond;
    cudaEventRecord(c.ev0, s);
    if (!c.assembled) {
        int rc = launch_assemble(c, c.U, 0.0, false, true, s);
        if (rc) return rc;
        c.assembled = true;
    }
    // b = mask(-K U_p) with every RVE's prescribed values at load factor 1
    set_prescribed(c, 1.0, s);
    residual_into(c, s, c.U, nullptr, c.b);
    if (pc == PG_PREC_MG) {
        int rc = batch_mg_numeric(*B, f32, s);
        if (rc) return rc;
    } else {
        k_prec_setup<double><<<nb(n), kThreads, 0, s>>>(n, c.diag, c.K, c.fixed, pc == PG_PREC_BLOCK_JACOBI, pc == PG_PREC_NONE,
                                                        c.minv);
    }
    cudaMemsetAsync(B->sc, 0, 8 * (size_t)R * sizeof(double), s);
    cudaMemsetAsync(B->fl, 0, 4 * (size_t)R * sizeof(int), s);
    cudaMemsetAsync(B->g, 0, 8 * sizeof(int), s);
    k_bcg_start<<<nb(nd), kThreads, 0, s>>>(nd, B->node_rve0, c.fixed, c.b, c.r, c.dx, B->sc);
    k_bcg_tol<<<nb(R, 128), 128, 0, s>>>(R, B->sc, B->fl, B->g, cfg->rtol * cfg->rtol);
    k_bcg_alldone<<<1, 1, 0, s>>>(R, B->g);
    batch_precondition(*B, pc, f32, s, c.r, c.z, nullptr);
    cudaMemcpyAsync(c.p, c.z, (size_t)nd * sizeof(double), cudaMemcpyDeviceToDevice, s);
    k_bcg_dot<<<nb(nd), kThreads, 0, s>>>(nd, B->node_rve0, c.r, c.z, B->sc, 2, nullptr);
    std::vector<int> hbad(R, 0);
    if (pc == PG_PREC_MG) {
        cudaMemcpyAsync(hbad.data(), B->bad, R * sizeof(int), cudaMemcpyDeviceToHost, s);
    }
    PG_CUDA(cudaStreamSynchronize(s));
    for (int r = 0; r < R; ++r)
        if (hbad[r]) {
            set_error("pg_batch_solve: singular coarsest operator in one RVE");
            return PG_ERR_BREAKDOWN;
        }
    const int chunk = pc == PG_PREC_MG ? 2 : (cfg->check_every > 1 ? cfg->check_every : 32);
    cudaGraph_t graph;
    PG_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    for (int it = 0; it < chunk; ++it) {
        k_bcg_s1<<<nb(R, 128), 128, 0, s>>>(R, B->sc, B->fl, B->g);
        k_bcg_spmv<<<nb(n), kThreads, 0, s>>>(n, B->node_rve0, c.row_ptr, c.col, c.K, c.p, c.fixed, c.q, B->sc, B->g);
        k_bcg_update<<<nb(nd), kThreads, 0, s>>>(nd, B->node_rve0, c.dx, c.r, c.p, c.q, B->sc, B->fl, B->g);
        k_bcg_s2<<<nb(R, 128), 128, 0, s>>>(R, B->sc, B->fl, B->g);
        k_bcg_alldone<<<1, 1, 0, s>>>(R, B->g);
        batch_precondition(*B, pc, f32, s, c.r, c.z, B->g + 1);
        k_bcg_dot<<<nb(nd), kThreads, 0, s>>>(nd, B->node_rve0, c.r, c.z, B->sc, 2, B->g);
        k_bcg_pupdate<<<nb(nd), kThreads, 0, s>>>(nd, B->node_rve0, c.z, c.p, B->sc, B->fl, B->g);
    }
    PG_CUDA(cudaStreamEndCapture(s, &graph));
    cudaGraphExec_t exec = nullptr;
    const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ie != cudaSuccess) return cuda_fail(ie, "pg_batch_solve graph");
    int hg[8] = {};
    int launched = 0;
    while (true) {
        cudaGraphLaunch(exec, s);
        launched += chunk;
        cudaMemcpyAsync(hg, B->g, sizeof hg, cudaMemcpyDeviceToHost, s);
        const cudaError_t e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) {
            cudaGraphExecDestroy(exec);
            return cuda_fail(e, "pg_batch_solve");
        }
        if (hg[1] || launched >= cfg->max_iter) break;
    }
    cudaGraphExecDestroy(exec);
    // true residual per RVE
    residual_into(c, s, c.dx, c.b, c.r);
    k_bcg_dot<<<nb(nd), kThreads, 0, s>>>(nd, B->node_rve0, c.r, c.r, B->sc, 6, nullptr);
    k_axpy_free<double><<<nb(nd), kThreads, 0, s>>>(nd, c.fixed, c.U, c.dx, 1.0);
    cudaEventRecord(c.ev1, s);
    std::vector<double> hs(8 * (size_t)R);
    std::vector<int> hf(4 * (size_t)R);
    cudaMemcpyAsync(hs.data(), B->sc, hs.size() * sizeof(double), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(hf.data(), B->fl, hf.size() * sizeof(int), cudaMemcpyDeviceToHost, s);
    PG_CUDA(cudaStreamSynchronize(s));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c.ev0, c.ev1);
    int worst = PG_OK, max_it = 0, n_bad = 0;
    double worst_rel = 0.0;
    for (int r = 0; r < R; ++r) {
        pg_solve_stats st{};
        st.iterations = hf[4 * r + 2];
        const double bb = hs[8 * r + 5];
        st.rel_residual = bb > 0.0 ? std::sqrt(hs[8 * r + 6] / bb) : 0.0;
        st.seconds = ms * 1e-3;
        if (hf[4 * r + 1]) st.status = PG_ERR_BREAKDOWN;
        else if (!(hs[8 * r + 6] <= 4.0 * cfg->rtol * cfg->rtol * bb)) st.status = PG_ERR_NOT_CONVERGED;
        else st.status = PG_OK;
        if (st.status != PG_OK) {
            ++n_bad;
            worst = st.status;
        }
        max_it = std::max(max_it, st.iterations);
        worst_rel = std::max(worst_rel, st.rel_residual);
        if (per_rve) per_rve[r] = st;
    }
    if (total) {
        total->iterations = max_it;
        total->refinements = 0;
        total->rel_residual = worst_rel;
        total->seconds = ms * 1e-3;
        total->newton_iterations = 0;
        total->status = worst;
    }
    if (n_bad) {
        set_error("pg_batch_solve: " + std::to_string(n_bad) + " RVE(s) did not reach the tolerance");
        return worst;
    }
    return PG_OK;
}

int pg_batch_get_solution(pg_batch* B, int32_t rve, double* U_host) {
    if (!B || !U_host || rve < 0 || rve >= B->n_rve) { set_error("pg_batch_get_solution: invalid argument"); return PG_ERR_ARG; }
    Ctx& c = B->ctx.c;
    cudaSetDevice(c.device);
    const size_t n = 2 * (size_t)(B->noff[rve + 1] - B->noff[rve]);
    PG_CUDA(cudaMemcpyAsync(U_host, c.U + 2 * (size_t)B->noff[rve], n * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    PG_CUDA(cudaStreamSynchronize(c.stream));
    return PG_OK;
}

}  // extern "C"
