// Vector/SpMV kernels of the Krylov solves (see pg_solve.cu for the scalar
// bookkeeping they implement).
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "pg_internal.cuh"

namespace pgb {

constexpr int kThreads = 256;

enum : int {
    S_PQ0 = 0, S_RZ0 = 2, S_RR0 = 4, S_TOL2 = 6, S_AUX = 8, S_NSCAL = 16
};
enum : int { F_DONE = 0, F_BREAKDOWN = 1, F_ITERS = 2, F_NFLAGS = 8 };

// Deterministic grid sums.  A reduction workspace holds its slot capacity
// (ws[0], in blocks), kRedSlots arrival tickets (from ws[1], two per double)
// and kRedSlots x capacity block partials (from ws[kRedHeader]).  Slots:
// 0-3 for the scalar sums of one kernel, 4 + j for the j-th product of the
// GMRES multi-dot.  Sequential kernels on one stream may reuse a slot.
constexpr int kRedSlots = 72;
constexpr int kRedHeader = 40;
inline size_t red_ws_doubles(int cap) { return (size_t)kRedHeader + (size_t)kRedSlots * (size_t)cap; }

__device__ __forceinline__ double block_sum(double d) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) d += __shfl_down_sync(0xffffffffu, d, o);
    __shared__ double sh[32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[wid] = d;
    __syncthreads();
    d = 0.0;
    if (wid == 0) {
        d = (lane < (int)(blockDim.x >> 5)) ? sh[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) d += __shfl_down_sync(0xffffffffu, d, o);
    }
    return d;  // valid in thread 0
}

// Adds the sum over the grid's blocks of s (each block's s valid in its
// thread 0) to *out in a fixed order: every block stores its s in the slot's
// partials, and the last block to take a ticket adds them in block order
// (a fixed tree over fixed strided sums) -- the same bits on every run,
// where atomically added block sums vary with the blocks' arrival.  Every
// thread of the block must call it.  A null workspace (a solve that asked
// for no fixed order) or a grid larger than the workspace's capacity falls
// back to the atomic sum.
__device__ __forceinline__ void grid_add(double* ws, int slot, double s, double* out) {
    __shared__ int s_last;
    if (ws == nullptr || (int)gridDim.x > (int)ws[0]) {
        if (threadIdx.x == 0) atomicAdd(out, s);
        return;
    }
    const int cap = (int)ws[0];
    unsigned* tickets = reinterpret_cast<unsigned*>(ws + 1);
    double* part = ws + kRedHeader + (size_t)slot * cap;
    if (threadIdx.x == 0) {
        part[blockIdx.x] = s;
        __threadfence();
        const unsigned t = atomicAdd(&tickets[slot], 1u);
        s_last = (t == gridDim.x - 1) ? 1 : 0;
    }
    __syncthreads();
    if (s_last) {
        __threadfence();
        double acc = 0.0;
        for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) acc += __ldcg(&part[b]);
        acc = block_sum(acc);
        if (threadIdx.x == 0) {
            *out += acc;
            tickets[slot] = 0u;
        }
    }
}

// y_i = sum_j K_ij x_j over 2x2 blocks (FP64 accumulation), masked rows zeroed
template <typename MT, typename VT>
__device__ __forceinline__ void bsr_row(int i, const int* __restrict__ row_ptr, const int* __restrict__ col,
                                        const MT* __restrict__ K, const VT* __restrict__ x, double& y0, double& y1) {
    const int r0 = row_ptr[i], r1 = row_ptr[i + 1];
    y0 = 0.0;
    y1 = 0.0;
    for (int k = r0; k < r1; ++k) {
        const int j = col[k];
        const MT* b = K + 4 * (size_t)k;
        const double x0 = (double)x[2 * j], x1 = (double)x[2 * j + 1];
        y0 += (double)b[0] * x0 + (double)b[1] * x1;
        y1 += (double)b[2] * x0 + (double)b[3] * x1;
    }
}

// One 2x2 block of K (row-major), read-only: one 256-bit load for FP64 blocks
// (K is a cudaMalloc allocation, so every block is 32-byte aligned), one
// 128-bit load for FP32 ones.
__device__ __forceinline__ void load_block(const double* p, double& a, double& b, double& c, double& d) {
    asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];" : "=d"(a), "=d"(b), "=d"(c), "=d"(d) : "l"(p));
}
__device__ __forceinline__ void load_block(const float* p, double& a, double& b, double& c, double& d) {
    const float4 v = __ldg(reinterpret_cast<const float4*>(p));
    a = v.x;
    b = v.y;
    c = v.z;
    d = v.w;
}

// Block row i of K times x with kRowLanes lanes per row: lane g of the row's
// group takes blocks r0 + g, r0 + g + kRowLanes, ..., so a group's loads of K
// are contiguous; two shuffles give every lane of the group the row's sum.
// A lane issues the column and block loads of kRowUnroll of its blocks at
// once, then their x gathers (a row of up to 12 blocks: one round of each).
// Every lane of the warp must call it (valid = false for padding rows).
constexpr int kRowLanes = 4;
constexpr int kRowUnroll = 3;
template <typename MT, typename VT>
__device__ __forceinline__ void bsr_row_group(int i, bool valid, int g, const int* __restrict__ row_ptr,
                                              const int* __restrict__ col, const MT* __restrict__ K,
                                              const VT* __restrict__ x, double& y0, double& y1) {
    double a0 = 0.0, a1 = 0.0;
    if (valid) {
        const int r1 = __ldg(&row_ptr[i + 1]);
        for (int base = __ldg(&row_ptr[i]) + g; base < r1; base += kRowLanes * kRowUnroll) {
            int j[kRowUnroll];
            double b[kRowUnroll][4];
#pragma unroll
            for (int u = 0; u < kRowUnroll; ++u) {
                const int k = base + u * kRowLanes;
                j[u] = -1;
                b[u][0] = b[u][1] = b[u][2] = b[u][3] = 0.0;
                if (k < r1) {
                    j[u] = __ldg(&col[k]);
                    load_block(K + 4 * (size_t)k, b[u][0], b[u][1], b[u][2], b[u][3]);
                }
            }
#pragma unroll
            for (int u = 0; u < kRowUnroll; ++u) {
                if (j[u] >= 0) {
                    const double x0 = (double)x[2 * j[u]], x1 = (double)x[2 * j[u] + 1];
                    a0 += b[u][0] * x0 + b[u][1] * x1;
                    a1 += b[u][2] * x0 + b[u][3] * x1;
                }
            }
        }
    }
    a0 += __shfl_xor_sync(0xffffffffu, a0, 1);
    a1 += __shfl_xor_sync(0xffffffffu, a1, 1);
    a0 += __shfl_xor_sync(0xffffffffu, a0, 2);
    a1 += __shfl_xor_sync(0xffffffffu, a1, 2);
    y0 = a0;
    y1 = a1;
}

template <typename MT, typename VT>
__global__ void __launch_bounds__(kThreads) k_spmv_plain(int n, const int* __restrict__ row_ptr, const int* __restrict__ col,
                                                          const MT* __restrict__ K, const VT* __restrict__ x,
                                                          const uint8_t* __restrict__ fixed, VT* __restrict__ y) {
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i >= n) return;
    double y0, y1;
    bsr_row<MT, VT>(i, row_ptr, col, K, x, y0, y1);
    y[2 * i] = fixed[2 * i] ? (VT)0 : (VT)y0;
    y[2 * i + 1] = fixed[2 * i + 1] ? (VT)0 : (VT)y1;
}

template <typename MT, typename VT>
__global__ void __launch_bounds__(kThreads) k_spmv_cg(int n, int P, const int* __restrict__ row_ptr, const int* __restrict__ col,
                                                       const MT* __restrict__ K, const VT* __restrict__ p,
                                                       const uint8_t* __restrict__ fixed, VT* __restrict__ q, double* scal,
                                                       const int* flags, double* ws) {
    if (flags[F_DONE]) return;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        scal[S_RZ0 + P] = 0.0;
        scal[S_RR0 + P] = 0.0;
    }
    const int i = blockIdx.x * kThreads + threadIdx.x;
    double part = 0.0;
    if (i < n) {
        double y0, y1;
        bsr_row<MT, VT>(i, row_ptr, col, K, p, y0, y1);
        const VT q0 = fixed[2 * i] ? (VT)0 : (VT)y0;
        const VT q1 = fixed[2 * i + 1] ? (VT)0 : (VT)y1;
        q[2 * i] = q0;
        q[2 * i + 1] = q1;
        part = (double)p[2 * i] * (double)q0 + (double)p[2 * i + 1] * (double)q1;
    }
    const double s = block_sum(part);
    grid_add(ws, 0, s, &scal[S_PQ0 + P]);
}

template <typename VT>
__global__ void k_neg(int nd, VT* r) {
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i < nd) r[i] = -r[i];
}

template <typename VT, typename PT>
__device__ __forceinline__ void apply_prec(const PT* __restrict__ minv, int node, double r0, double r1, double& z0, double& z1) {
    const PT* m = minv + 4 * (size_t)node;
    z0 = (double)m[0] * r0 + (double)m[1] * r1;
    z1 = (double)m[2] * r0 + (double)m[3] * r1;
}

template <typename VT, typename PT>
__global__ void __launch_bounds__(kThreads) k_cg_init(int n, const VT* __restrict__ r, VT* __restrict__ z, VT* __restrict__ p,
                                                       const PT* __restrict__ minv, double* scal, double* ws) {
    const int i = blockIdx.x * kThreads + threadIdx.x;
    double prz = 0.0, prr = 0.0;
    if (i < n) {
        const double r0 = (double)r[2 * i], r1 = (double)r[2 * i + 1];
        double z0, z1;
        apply_prec<VT, PT>(minv, i, r0, r1, z0, z1);
        z[2 * i] = (VT)z0;
        z[2 * i + 1] = (VT)z1;
        p[2 * i] = (VT)z0;
        p[2 * i + 1] = (VT)z1;
        prz = r0 * z0 + r1 * z1;
        prr = r0 * r0 + r1 * r1;
    }
    const double a = block_sum(prz);
    const double b = block_sum(prr);
    grid_add(ws, 1, a, &scal[S_RZ0 + 1]);
    grid_add(ws, 2, b, &scal[S_RR0 + 1]);
}

template <typename VT, typename PT>
__global__ void __launch_bounds__(kThreads) k_cg_update(int n, int P, VT* __restrict__ x, VT* __restrict__ r, VT* __restrict__ z,
                                                         const VT* __restrict__ p, const VT* __restrict__ q,
                                                         const PT* __restrict__ minv, double* scal, int* flags,
                                                         double* ws) {
    if (flags[F_DONE]) return;
    const int Q = 1 - P;
    const double pq = scal[S_PQ0 + P];
    if (!(pq > 0.0)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            flags[F_BREAKDOWN] = 1;
            flags[F_DONE] = 1;
        }
        return;
    }
    const double alpha = scal[S_RZ0 + Q] / pq;
    const int i = blockIdx.x * kThreads + threadIdx.x;
    double prz = 0.0, prr = 0.0;
    if (i < n) {
        const double r0 = (double)r[2 * i] - alpha * (double)q[2 * i];
        const double r1 = (double)r[2 * i + 1] - alpha * (double)q[2 * i + 1];
        x[2 * i] = (VT)((double)x[2 * i] + alpha * (double)p[2 * i]);
        x[2 * i + 1] = (VT)((double)x[2 * i + 1] + alpha * (double)p[2 * i + 1]);
        r[2 * i] = (VT)r0;
        r[2 * i + 1] = (VT)r1;
        double z0, z1;
        apply_prec<VT, PT>(minv, i, r0, r1, z0, z1);
        z[2 * i] = (VT)z0;
        z[2 * i + 1] = (VT)z1;
        prz = r0 * z0 + r1 * z1;
        prr = r0 * r0 + r1 * r1;
    }
    const double a = block_sum(prz);
    const double b = block_sum(prr);
    grid_add(ws, 1, a, &scal[S_RZ0 + P]);
    grid_add(ws, 2, b, &scal[S_RR0 + P]);
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        scal[S_PQ0 + Q] = 0.0;
        flags[F_ITERS] += 1;
    }
}

template <typename VT>
__global__ void __launch_bounds__(kThreads) k_cg_pupdate(int n, int P, const VT* __restrict__ z, VT* __restrict__ p,
                                                          double* scal, int* flags) {
    if (flags[F_DONE]) return;
    const int Q = 1 - P;
    const double rz = scal[S_RZ0 + P];
    const double rz_old = scal[S_RZ0 + Q];
    if (blockIdx.x == 0 && threadIdx.x == 0 && scal[S_RR0 + P] <= scal[S_TOL2]) flags[F_DONE] = 1;
    const double beta = rz / rz_old;
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i < n) {
        p[2 * i] = (VT)((double)z[2 * i] + beta * (double)p[2 * i]);
        p[2 * i + 1] = (VT)((double)z[2 * i + 1] + beta * (double)p[2 * i + 1]);
    }
}

// Per-node preconditioner: inverse of the masked 2x2 diagonal block (block
// Jacobi), inverse diagonal (Jacobi) or the free-DOF identity.
template <typename PT>
__global__ void k_prec_setup(int n, const int* __restrict__ diag, const double* __restrict__ K,
                             const uint8_t* __restrict__ fixed, int block, int ident, PT* minv) {
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i >= n) return;
    const double* b = K + 4 * (size_t)diag[i];
    const bool f0 = fixed[2 * i], f1 = fixed[2 * i + 1];
    double m[4] = {0.0, 0.0, 0.0, 0.0};
    if (ident) {
        m[0] = f0 ? 0.0 : 1.0;
        m[3] = f1 ? 0.0 : 1.0;
    } else if (block && !f0 && !f1) {
        const double det = b[0] * b[3] - b[1] * b[2];
        m[0] = b[3] / det;
        m[1] = -b[1] / det;
        m[2] = -b[2] / det;
        m[3] = b[0] / det;
    } else {
        m[0] = f0 ? 0.0 : 1.0 / b[0];
        m[3] = f1 ? 0.0 : 1.0 / b[3];
    }
    for (int k = 0; k < 4; ++k) minv[4 * (size_t)i + k] = (PT)m[k];
}

template <typename VT>
__global__ void k_fill(int n, VT* v, VT a) {
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i < n) v[i] = a;
}

template <typename VT>
__global__ void k_axpy_free(int nd, const uint8_t* __restrict__ fixed, double* U, const VT* __restrict__ e, double s) {
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i < nd && !fixed[i]) U[i] += s * (double)e[i];
}

__global__ inline void k_axpy_free_f(int nd, const uint8_t* __restrict__ fixed, double* U, const float* __restrict__ e,
                                     double s) {
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i < nd && !fixed[i]) U[i] += s * (double)e[i];
}

__global__ inline void k_to_float_scaled(int nd, const double* __restrict__ a, float* b, double s) {
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i < nd) b[i] = (float)(a[i] * s);
}

__global__ inline void k_dot_self(int nd, const double* __restrict__ a, double* out, double* ws) {
    const int i = blockIdx.x * kThreads + threadIdx.x;
    const double v = (i < nd) ? a[i] * a[i] : 0.0;
    const double s = block_sum(v);
    grid_add(ws, 3, s, out);
}

__global__ inline void k_apply_dirichlet(int nd, const uint8_t* __restrict__ fixed, const double* __restrict__ ubar,
                                         double tf, double* U) {
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i < nd && fixed[i]) U[i] = tf * ubar[i];
}

// out = mask(b) - out  (b may be null: zero)
__global__ inline void k_rhs_minus(int nd, const uint8_t* __restrict__ fixed, const double* __restrict__ b, double* out) {
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i < nd) out[i] = fixed[i] ? 0.0 : ((b ? b[i] : 0.0) - out[i]);
}

template <typename VT>
__global__ void k_copy(int n, const VT* __restrict__ a, VT* __restrict__ b) {
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i < n) b[i] = a[i];
}

__global__ inline void k_scale_copy(int n, const double* __restrict__ a, double* __restrict__ b, double s) {
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i < n) b[i] = s * a[i];
}

__global__ inline void k_scale_inplace(int n, double* a, double s) {
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i < n) a[i] *= s;
}

// z = M^-1 v per node (2x2 blocks)
__global__ inline void k_apply_prec_vec(int n, const double* __restrict__ minv, const double* __restrict__ v,
                                        double* __restrict__ z) {
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i >= n) return;
    const double* m = minv + 4 * (size_t)i;
    const double v0 = v[2 * i], v1 = v[2 * i + 1];
    z[2 * i] = m[0] * v0 + m[1] * v1;
    z[2 * i + 1] = m[2] * v0 + m[3] * v1;
}

// out[j] += V_j . w for j < k (V: k vectors of length nd, contiguous)
__global__ inline void k_multidot(int nd, int k, const double* __restrict__ V, const double* __restrict__ w,
                                  double* out, double* ws) {
    for (int j = 0; j < k; ++j) {
        const double* vj = V + (size_t)j * nd;
        double part = 0.0;
        for (int i = blockIdx.x * kThreads + threadIdx.x; i < nd; i += gridDim.x * kThreads) part += vj[i] * w[i];
        const double s = block_sum(part);
        grid_add(ws, 4 + j, s, &out[j]);
    }
}

// w -= sum_j h_j V_j
__global__ inline void k_multi_axpy(int nd, int k, const double* __restrict__ V, const double* __restrict__ h,
                                    double* w) {
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i >= nd) return;
    double acc = w[i];
    for (int j = 0; j < k; ++j) acc -= h[j] * V[(size_t)j * nd + i];
    w[i] = acc;
}

// q += sum_j y_j V_j
__global__ inline void k_multi_axpy_add(int nd, int k, const double* __restrict__ V, const double* __restrict__ y,
                                        double* q) {
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i >= nd) return;
    double acc = q[i];
    for (int j = 0; j < k; ++j) acc += y[j] * V[(size_t)j * nd + i];
    q[i] = acc;
}

// ---------------- MINRES (symmetric indefinite, SPD preconditioner) ----------------
// Scalar slots (device), updated by one thread per iteration.
enum : int {
    M_BETA = 16, M_OLDB, M_ALFA, M_BB, M_DBAR, M_EPSLN, M_PHIBAR, M_CS, M_SN, M_PHI, M_DELTA, M_OLDEPS, M_DENOM,
    M_BETA1, M_TOL, M_ITER, M_NSCAL
};

// v = y / beta
__global__ inline void k_mr_v(int nd, const double* __restrict__ y, double* __restrict__ v, const double* scal,
                              const int* flags) {
    if (flags[F_DONE]) return;
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i < nd) v[i] = y[i] / scal[M_BETA];
}

// y = mask(K v) - (beta/oldb) r1 ; alfa += v.y
template <typename MT>
__global__ void __launch_bounds__(kThreads) k_mr_av(int n, const int* __restrict__ row_ptr, const int* __restrict__ col,
                                                    const MT* __restrict__ K, const double* __restrict__ v,
                                                    const uint8_t* __restrict__ fixed, const double* __restrict__ r1,
                                                    double* __restrict__ y, double* scal, const int* flags,
                                                    double* ws) {
    if (flags[F_DONE]) return;
    const double c = scal[M_OLDB] > 0.0 ? scal[M_BETA] / scal[M_OLDB] : 0.0;
    const int i = blockIdx.x * kThreads + threadIdx.x;
    double part = 0.0;
    if (i < n) {
        double y0, y1;
        bsr_row<MT, double>(i, row_ptr, col, K, v, y0, y1);
        y0 = fixed[2 * i] ? 0.0 : y0 - c * r1[2 * i];
        y1 = fixed[2 * i + 1] ? 0.0 : y1 - c * r1[2 * i + 1];
        y[2 * i] = y0;
        y[2 * i + 1] = y1;
        part = v[2 * i] * y0 + v[2 * i + 1] * y1;
    }
    const double s = block_sum(part);
    grid_add(ws, 0, s, &scal[M_ALFA]);
}

// y -= (alfa/beta) r2; r2new = y (written over r1); z = M^-1 r2new (into y); bb += r2new.z
__global__ inline void __launch_bounds__(kThreads) k_mr_2(int n, double* __restrict__ y, const double* __restrict__ r2,
                                                           double* __restrict__ r1_to_r2new,
                                                           const double* __restrict__ minv, double* scal, const int* flags,
                                                           double* ws) {
    if (flags[F_DONE]) return;
    const double c = scal[M_ALFA] / scal[M_BETA];
    const int i = blockIdx.x * kThreads + threadIdx.x;
    double part = 0.0;
    if (i < n) {
        const double a0 = y[2 * i] - c * r2[2 * i], a1 = y[2 * i + 1] - c * r2[2 * i + 1];
        r1_to_r2new[2 * i] = a0;
        r1_to_r2new[2 * i + 1] = a1;
        const double* m = minv + 4 * (size_t)i;
        const double z0 = m[0] * a0 + m[1] * a1, z1 = m[2] * a0 + m[3] * a1;
        y[2 * i] = z0;
        y[2 * i + 1] = z1;
        part = a0 * z0 + a1 * z1;
    }
    const double s = block_sum(part);
    grid_add(ws, 1, s, &scal[M_BB]);
}

// Lanczos / Givens scalar recurrences of MINRES (Paige & Saunders 1975)
__global__ inline void k_mr_scalars(double* sc, int* flags) {
    if (flags[F_DONE]) return;
    const double alfa = sc[M_ALFA];
    const double beta_new = sqrt(fmax(sc[M_BB], 0.0));
    sc[M_OLDB] = sc[M_BETA];
    const double oldeps = sc[M_EPSLN];
    const double delta = sc[M_CS] * sc[M_DBAR] + sc[M_SN] * alfa;
    const double gbar = sc[M_SN] * sc[M_DBAR] - sc[M_CS] * alfa;
    sc[M_EPSLN] = sc[M_SN] * beta_new;
    sc[M_DBAR] = -sc[M_CS] * beta_new;
    const double gamma = fmax(sqrt(gbar * gbar + beta_new * beta_new), 1e-300);
    sc[M_CS] = gbar / gamma;
    sc[M_SN] = beta_new / gamma;
    sc[M_PHI] = sc[M_CS] * sc[M_PHIBAR];
    sc[M_PHIBAR] = sc[M_SN] * sc[M_PHIBAR];
    sc[M_DELTA] = delta;
    sc[M_OLDEPS] = oldeps;
    sc[M_DENOM] = 1.0 / gamma;
    sc[M_BETA] = beta_new;
    sc[M_ALFA] = 0.0;
    sc[M_BB] = 0.0;
    flags[F_ITERS] += 1;
    if (sc[M_PHIBAR] <= sc[M_TOL] * sc[M_BETA1] || beta_new == 0.0) flags[F_DONE] = 1;
}

// w_new = (v - oldeps w_{k-2} - delta w_{k-1}) / gamma, written over w_{k-2}; x += phi w_new
__global__ inline void k_mr_w(int nd, const double* __restrict__ v, double* __restrict__ wkm2,
                              const double* __restrict__ wkm1, double* __restrict__ x, const double* scal,
                              const int* flags) {
    // runs after k_mr_scalars of the same iteration: F_DONE may already be set by it,
    // the update of this iteration still has to be applied
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i >= nd) return;
    if (flags[F_DONE] > 1) return;
    const double w = (v[i] - scal[M_OLDEPS] * wkm2[i] - scal[M_DELTA] * wkm1[i]) * scal[M_DENOM];
    wkm2[i] = w;
    x[i] += scal[M_PHI] * w;
}

// after an iteration's w-update, a DONE flag raised by this iteration's scalars becomes final
__global__ inline void k_mr_seal(int* flags) {
    if (flags[F_DONE] == 1) flags[F_DONE] = 2;
}

// z = M^-1 r with |diag| Jacobi (SPD preconditioner for MINRES)
__global__ inline void k_prec_absjacobi(int n, const int* __restrict__ diag, const double* __restrict__ K,
                                        const uint8_t* __restrict__ fixed, double* minv) {
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i >= n) return;
    const double* b = K + 4 * (size_t)diag[i];
    double* m = minv + 4 * (size_t)i;
    m[0] = fixed[2 * i] ? 0.0 : 1.0 / fabs(b[0]);
    m[1] = 0.0;
    m[2] = 0.0;
    m[3] = fixed[2 * i + 1] ? 0.0 : 1.0 / fabs(b[3]);
}

__global__ inline void k_dot2(int nd, const double* __restrict__ a, const double* __restrict__ b, double* out,
                              double* ws) {
    const int i = blockIdx.x * kThreads + threadIdx.x;
    const double v = (i < nd) ? a[i] * b[i] : 0.0;
    const double s = block_sum(v);
    grid_add(ws, 3, s, out);
}

// out = mask(a)
__global__ inline void k_mask_copy(int nd, const uint8_t* __restrict__ fixed, const double* __restrict__ a, double* out) {
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i < nd) out[i] = fixed[i] ? 0.0 : a[i];
}

// out = U + s d on free DOFs, U on prescribed DOFs
__global__ inline void k_axpy_to(int nd, const uint8_t* __restrict__ fixed, const double* __restrict__ U,
                                 const double* __restrict__ d, double s, double* out) {
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i < nd) out[i] = fixed[i] ? U[i] : U[i] + s * d[i];
}

// U += ratio (U - Uold) on free DOFs (linear extrapolation in load)
__global__ inline void k_extrapolate(int nd, const uint8_t* __restrict__ fixed, double* U, const double* __restrict__ Uold,
                                     double ratio) {
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i < nd && !fixed[i]) U[i] += ratio * (U[i] - Uold[i]);
}

}  // namespace pgb
