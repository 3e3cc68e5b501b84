// Block-Jacobi PCG on a caller-owned system, with no device allocation.
//
// Some callers cannot let this library call cudaMalloc: a host framework
// that owns all device memory through its own allocator or a fixed budget,
// code that runs where allocating would synchronise the device or is not
// permitted (inside another library's stream-ordered callbacks, a memory
// pool that must not grow), and foreign-language bindings that only hold
// pointers to buffers they manage themselves.  pg_pcg_solve_static serves
// them: the caller passes the matrix, mask, right-hand side and solution
// buffers, and the Krylov work vectors live in one fixed array in the
// library's own device image, sized for kStaticMaxNodes nodes and held on
// every GPU that loads the library until the process exits.
//
// Set-up: the first call on a device, with that device current, looks the
// array's device address up with cudaGetSymbolAddress and keeps it; make
// that first call before any stream capture.  Every call on a device shares
// the one array and finds the previous call's contents there; everything
// the solve reads before writing is cleared by the call itself.  Calls that
// overlap on the GPU (several streams or host threads at once) race on the
// array and must be serialised by the caller.  The looked-up address belongs
// to the device's current CUDA context: after cudaDeviceReset on that device
// it is stale, so a process that resets a device must not call this entry
// point on it again.
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <mutex>

#include "pg_solve_kernels.cuh"
#include "pigfem_b200.h"

namespace pgb {

namespace {

constexpr int kStaticMaxNodes = PG_STATIC_MAX_NODES;
constexpr int kStaticChunk = 32;   // iterations launched between two host reads of the status flags
// set-up outcomes in the breakdown flag (CG itself writes 1 there)
constexpr int kStaticNoDiag = 2;    // a free DOF whose row has no diagonal block
constexpr int kStaticSingular = 3;  // a free DOF's diagonal block (or pivot) is zero or not finite

// Layout (doubles): r, z, p, q (2 * kStaticMaxNodes each), minv (4 per
// node), the CG scalars (S_NSCAL), the CG flags (F_NFLAGS ints, 8 bytes
// per slot so the offsets stay 8-byte aligned).
constexpr size_t kOffR = 0;
constexpr size_t kOffZ = kOffR + 2 * (size_t)kStaticMaxNodes;
constexpr size_t kOffP = kOffZ + 2 * (size_t)kStaticMaxNodes;
constexpr size_t kOffQ = kOffP + 2 * (size_t)kStaticMaxNodes;
constexpr size_t kOffMinv = kOffQ + 2 * (size_t)kStaticMaxNodes;
constexpr size_t kOffScal = kOffMinv + 4 * (size_t)kStaticMaxNodes;
constexpr size_t kOffFlags = kOffScal + S_NSCAL;
// the deterministic grid sums' workspace (grid_add): one partial per block of the largest grid
constexpr int kStaticRedCap = (kStaticMaxNodes + kThreads - 1) / kThreads + 1;
constexpr size_t kOffRed = kOffFlags + F_NFLAGS;
constexpr size_t kScratchDoubles = kOffRed + (size_t)kRedHeader + (size_t)kRedSlots * kStaticRedCap;

// In host code this name is only a handle for cudaGetSymbolAddress, not a
// device address.
static __device__ __align__(256) double g_pcg_scratch[kScratchDoubles];

std::mutex g_setup_mutex;
double* g_scratch_dev[64] = {};

// the workspace's capacity and cleared tickets
__global__ void k_static_red_init(double* ws) {
    if (threadIdx.x == 0) ws[0] = (double)kStaticRedCap;
    if (threadIdx.x > 0 && threadIdx.x < kRedHeader) ws[threadIdx.x] = 0.0;
}

// Block-Jacobi inverse of each node's masked 2x2 diagonal block, found by
// scanning the row for the diagonal column (the caller's pattern carries
// no diagonal index).  Fixed DOFs get 0; a free DOF whose partner is fixed
// gets the scalar inverse.
__global__ void k_static_prec(int n, const int* __restrict__ row_ptr, const int* __restrict__ col,
                              const double* __restrict__ K, const uint8_t* __restrict__ fixed, double* minv,
                              int* flags) {
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i >= n) return;
    const double* b = nullptr;
    for (int q = row_ptr[i]; q < row_ptr[i + 1]; ++q)
        if (col[q] == i) {
            b = K + 4 * (size_t)q;
            break;
        }
    double m[4] = {0.0, 0.0, 0.0, 0.0};
    const bool f0 = fixed[2 * i], f1 = fixed[2 * i + 1];
    if (b == nullptr) {
        if (!f0 || !f1) flags[F_BREAKDOWN] = kStaticNoDiag;  // a free DOF without a diagonal block
    } else if (!f0 && !f1) {
        const double det = b[0] * b[3] - b[1] * b[2];
        if (det == 0.0 || !isfinite(det)) flags[F_BREAKDOWN] = kStaticSingular;
        m[0] = b[3] / det;
        m[1] = -b[1] / det;
        m[2] = -b[2] / det;
        m[3] = b[0] / det;
    } else {
        const double piv = f0 ? b[3] : b[0];
        if (!(f0 && f1) && (piv == 0.0 || !isfinite(piv))) flags[F_BREAKDOWN] = kStaticSingular;
        m[0] = f0 ? 0.0 : 1.0 / b[0];
        m[3] = f1 ? 0.0 : 1.0 / b[3];
    }
    for (int k = 0; k < 4; ++k) minv[4 * (size_t)i + k] = m[k];
}

// r = mask(b), x = 0
__global__ void k_static_start(int nd, const uint8_t* __restrict__ fixed, const double* __restrict__ b, double* r,
                               double* x) {
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i >= nd) return;
    r[i] = fixed[i] ? 0.0 : b[i];
    x[i] = 0.0;
}

// scal[S_TOL2] = rtol^2 * ||mask(b)||^2 (from the initial r.r of k_cg_init)
__global__ void k_static_tol(double* scal, double rtol2) { scal[S_TOL2] = rtol2 * scal[S_RR0 + 1]; }

// out = ||mask(b) - mask(K) x||^2 and ||mask(b)||^2, accumulated into out[0..1]
__global__ void __launch_bounds__(kThreads) k_static_resid(int n, const int* __restrict__ row_ptr,
                                                           const int* __restrict__ col, const double* __restrict__ K,
                                                           const double* __restrict__ x,
                                                           const uint8_t* __restrict__ fixed,
                                                           const double* __restrict__ b, double* out, double* ws) {
    const int i = blockIdx.x * kThreads + threadIdx.x;
    double rr = 0.0, bb = 0.0;
    if (i < n) {
        double y0, y1;
        bsr_row<double, double>(i, row_ptr, col, K, x, y0, y1);
        const double b0 = fixed[2 * i] ? 0.0 : b[2 * i], b1 = fixed[2 * i + 1] ? 0.0 : b[2 * i + 1];
        const double r0 = fixed[2 * i] ? 0.0 : b0 - y0, r1 = fixed[2 * i + 1] ? 0.0 : b1 - y1;
        rr = r0 * r0 + r1 * r1;
        bb = b0 * b0 + b1 * b1;
    }
    const double a = block_sum(rr);
    const double c = block_sum(bb);
    grid_add(ws, 1, a, &out[0]);
    grid_add(ws, 2, c, &out[1]);
}

// Device address of the scratch array on the current device (looked up once).
int scratch_on_current_device(double** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "pg_pcg_solve_static: cudaGetDevice");
    if (dev < 0 || dev >= 64) {
        set_error("pg_pcg_solve_static: device ordinal beyond 63");
        return PG_ERR_ARG;
    }
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_dev[dev]) {
        double* p = nullptr;
        e = cudaGetSymbolAddress((void**)&p, g_pcg_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "pg_pcg_solve_static: cudaGetSymbolAddress");
        g_scratch_dev[dev] = p;
    }
    *out = g_scratch_dev[dev];
    return PG_OK;
}

}  // namespace

}  // namespace pgb

using namespace pgb;

namespace {

int pcg_static(int32_t n_nodes, const int32_t* row_ptr, const int32_t* col, const double* K, const uint8_t* fixed,
               const double* b, double* x, double rtol, int32_t max_iter, void* stream, pg_solve_stats* stats) {
    if (n_nodes > kStaticMaxNodes) {
        char msg[160];
        std::snprintf(msg, sizeof msg, "pg_pcg_solve_static: %d nodes exceed the fixed scratch capacity of %d nodes",
                      (int)n_nodes, kStaticMaxNodes);
        set_error(msg);
        return PG_ERR_LIMIT;
    }
    if (n_nodes <= 0 || !row_ptr || !col || !K || !fixed || !b || !x || !stats || !(rtol > 0.0) || max_iter < 0) {
        set_error("pg_pcg_solve_static: invalid argument");
        return PG_ERR_ARG;
    }
    const auto t0 = std::chrono::steady_clock::now();
    double* base = nullptr;
    int rc = scratch_on_current_device(&base);
    if (rc != PG_OK) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    const int n = n_nodes, nd = 2 * n_nodes;
    double* r = base + kOffR;
    double* z = base + kOffZ;
    double* p = base + kOffP;
    double* q = base + kOffQ;
    double* minv = base + kOffMinv;
    double* scal = base + kOffScal;
    int* flags = reinterpret_cast<int*>(base + kOffFlags);
    double* ws = base + kOffRed;
    const int gb = (n + kThreads - 1) / kThreads, gd = (nd + kThreads - 1) / kThreads;

    cudaError_t e = cudaMemsetAsync(scal, 0, (S_NSCAL + F_NFLAGS) * sizeof(double), s);
    if (e != cudaSuccess) return cuda_fail(e, "pg_pcg_solve_static: clearing the scalars and flags");
    k_static_red_init<<<1, kRedHeader, 0, s>>>(ws);
    k_static_start<<<gd, kThreads, 0, s>>>(nd, fixed, b, r, x);
    k_static_prec<<<gb, kThreads, 0, s>>>(n, row_ptr, col, K, fixed, minv, flags);
    k_cg_init<double, double><<<gb, kThreads, 0, s>>>(n, r, z, p, minv, scal, ws);
    k_static_tol<<<1, 1, 0, s>>>(scal, rtol * rtol);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "pg_pcg_solve_static: launch");

    int hf[F_NFLAGS] = {};
    double hs[S_NSCAL] = {};
    e = cudaMemcpyAsync(hs, scal, sizeof hs, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(hf, flags, sizeof hf, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(e, "pg_pcg_solve_static: set-up");
    if (hf[F_BREAKDOWN] == kStaticNoDiag) {
        set_error("pg_pcg_solve_static: a free DOF has no diagonal block in the pattern");
        return PG_ERR_ARG;
    }
    if (hf[F_BREAKDOWN] == kStaticSingular) {
        set_error("pg_pcg_solve_static: singular diagonal block (zero or non-finite determinant or pivot)");
        return PG_ERR_BREAKDOWN;
    }
    int iters = 0, launched = 0;
    bool done = hs[S_RR0 + 1] <= hs[S_TOL2] || hs[S_RR0 + 1] == 0.0;
    while (!done && launched < max_iter) {
        // iteration k uses the scalar slots of parity k & 1
        const int m = max_iter - launched < kStaticChunk ? max_iter - launched : kStaticChunk;
        for (int it = 0; it < m; ++it) {
            const int P = (launched + it) & 1;
            k_spmv_cg<double, double><<<gb, kThreads, 0, s>>>(n, P, row_ptr, col, K, p, fixed, q, scal, flags, ws);
            k_cg_update<double, double><<<gb, kThreads, 0, s>>>(n, P, x, r, z, p, q, minv, scal, flags, ws);
            k_cg_pupdate<double><<<gb, kThreads, 0, s>>>(n, P, z, p, scal, flags);
        }
        launched += m;
        e = cudaMemcpyAsync(hf, flags, sizeof hf, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return cuda_fail(e, "pg_pcg_solve_static: iterations");
        iters = hf[F_ITERS];
        done = hf[F_DONE] != 0;
    }
    // true residual of the returned x (the q slot of the scratch is free now)
    e = cudaMemsetAsync(q, 0, 2 * sizeof(double), s);
    if (e != cudaSuccess) return cuda_fail(e, "pg_pcg_solve_static: clearing the residual accumulator");
    k_static_resid<<<gb, kThreads, 0, s>>>(n, row_ptr, col, K, x, fixed, b, q, ws);
    double res[2] = {0.0, 0.0};
    e = cudaMemcpyAsync(res, q, sizeof res, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(e, "pg_pcg_solve_static: residual");

    stats->iterations = iters;
    stats->refinements = 0;
    stats->newton_iterations = 0;
    stats->rel_residual = res[1] > 0.0 ? std::sqrt(res[0] / res[1]) : 0.0;
    stats->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (hf[F_BREAKDOWN]) {
        stats->status = PG_ERR_BREAKDOWN;
        set_error("pg_pcg_solve_static: CG breakdown (operator not positive definite on the free DOFs)");
        return PG_ERR_BREAKDOWN;
    }
    // the recursive residual met rtol; accept the true one within a small factor
    if (!(res[0] <= 4.0 * rtol * rtol * res[1])) {
        stats->status = PG_ERR_NOT_CONVERGED;
        set_error("pg_pcg_solve_static: iteration budget exhausted before the tolerance");
        return PG_ERR_NOT_CONVERGED;
    }
    stats->status = PG_OK;
    return PG_OK;
}

}  // namespace

extern "C" int pg_pcg_solve_static(int32_t n_nodes, const int32_t* row_ptr, const int32_t* col, const double* K,
                                   const uint8_t* fixed, const double* b, double* x, double rtol, int32_t max_iter,
                                   void* stream, pg_solve_stats* stats) {
    // stats describes this call on every return, the early ones included
    constexpr int kUnset = -1;
    if (stats) {
        *stats = pg_solve_stats{};
        stats->status = kUnset;
    }
    const int rc = pcg_static(n_nodes, row_ptr, col, K, fixed, b, x, rtol, max_iter, stream, stats);
    if (stats && stats->status == kUnset) stats->status = rc;
    return rc;
}
