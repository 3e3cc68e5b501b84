// Per-node MLP of the learned Newton warm start: BF16 tensor-core (tcgen05)
// forward, backward and weight-gradient kernels with FP32 accumulation in
// tensor memory, plus an FP32 Adam step.  The reference has no learned
// component; the network is a 16 -> 64 -> 64 -> 16 ReLU MLP (two outputs used)
// over per-node features of a load step.
//
// One CTA (4 warps, 128 threads) owns a 128-row tile of nodes: thread t holds
// row t.  Every GEMM is D[128 x N] (+)= A[128 x K] * B[N x K]^T issued by one
// thread as tcgen05.mma.cta_group::1.kind::f16 (BF16 x BF16 -> FP32) with both
// operands in shared memory in the canonical K-major layout without swizzle:
// 8-row x 16-byte core matrices, K-adjacent core matrices 128 B apart (LBO),
// 8-row groups SBO = (K/8)*128 B apart.  D lives in tensor memory (lane = row,
// one 32-bit column per output) and is read back with tcgen05.ld 32x32b.
// Completion is signalled by tcgen05.commit to an mbarrier whose wait is
// bounded; on timeout the kernel records an error, frees its tensor memory
// and returns.
//
// Weight gradients: dW2 and dW1 come out of one M=128 GEMM whose A stacks
// dZ2^T over dZ1^T and whose B stacks H1^T over X^T (the off-diagonal blocks
// are not read); dW3 uses A = [dY^T; 0].  They accumulate in tensor memory
// over all tiles a CTA processes; each CTA then writes its part of the
// gradient to its own slot and k_grad_sum adds the parts in CTA order.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <new>
#include <random>
#include <vector>

#include "pg_internal.cuh"

namespace pgb {
namespace mlp {

constexpr int IN = 16, HID = 64, OUT = 16, USED = 2, TILE = 128, NT = 128;
constexpr uint32_t TMEM_COLS = 512;
// tensor-memory columns
constexpr uint32_t C_Z1 = 0, C_Z2 = 64, C_Y = 128, C_DW12 = 256, C_DW3 = 384;

// shared-memory map (bytes from the 1024-aligned dynamic base)
constexpr uint32_t O_X = 0;                       // A 128 x 16        4 KB
constexpr uint32_t O_W1 = O_X + 4096;             // B  64 x 16        2 KB
constexpr uint32_t O_H1 = O_W1 + 2048;            // A 128 x 64       16 KB
constexpr uint32_t O_W2 = O_H1 + 16384;           // B  64 x 64        8 KB
constexpr uint32_t O_H2 = O_W2 + 8192;            // A 128 x 64       16 KB
constexpr uint32_t O_W3 = O_H2 + 16384;           // B  16 x 64        2 KB
constexpr uint32_t O_DY = O_W3 + 2048;            // A 128 x 16        4 KB
constexpr uint32_t O_W3T = O_DY + 4096;           // B  64 x 16        2 KB
constexpr uint32_t O_DZ2 = O_W3T + 2048;          // A 128 x 64       16 KB
constexpr uint32_t O_W2T = O_DZ2 + 16384;         // B  64 x 64        8 KB
constexpr uint32_t O_AT = O_W2T + 8192;           // A 128 x 128 (dZ2^T ; dZ1^T)   32 KB
constexpr uint32_t O_BT = O_AT + 32768;           // B  80 x 128 (H1^T ; X^T)      20 KB
constexpr uint32_t O_A3 = O_BT + 20480;           // A 128 x 128 (dY^T ; 0)        32 KB
constexpr uint32_t O_B3 = O_A3 + 32768;           // B  64 x 128 (H2^T)            16 KB
constexpr uint32_t SMEM_BYTES = O_B3 + 16384;     // 182 KB
// The allocation also covers O_B3 + 32 KB: every operand's core-matrix grid
// (rows/8 x K/8 groups of 128 B) read with either stride interpretation stays
// inside the allocation.
constexpr uint32_t SMEM_ALLOC = O_B3 + 32768 + 1024;

struct Params {
    float* W1; float* b1; float* W2; float* b2; float* W3; float* b3;
};

constexpr int kW1 = HID * IN, kB1 = HID, kW2 = HID * HID, kB2 = HID, kW3 = OUT * HID, kB3 = OUT;
constexpr int kNParams = kW1 + kB1 + kW2 + kB2 + kW3 + kB3;

__host__ __device__ inline Params carve(float* base) {
    Params q;
    q.W1 = base;
    q.b1 = q.W1 + kW1;
    q.W2 = q.b1 + kB1;
    q.b2 = q.W2 + kW2;
    q.W3 = q.b2 + kB2;
    q.b3 = q.W3 + kW3;
    return q;
}

// Sum over a warp's lanes by a fixed butterfly: every lane gets the same
// value, in the same order on every run.
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// byte offset of element (row, k) in a canonical K-major tile with K columns
__device__ __forceinline__ uint32_t kmaj(int row, int k, int K) {
    return (uint32_t)((row >> 3) * (K * 16) + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, int K) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((128u >> 4) & 0x3FFFu) << 16;                 // LBO: K-adjacent core matrices
    d |= (uint64_t)(((uint32_t)(K * 16) >> 4) & 0x3FFFu) << 32;   // SBO: 8-row groups
    d |= (uint64_t)1 << 46;                                       // descriptor version (sm_100)
    return d;                                                     // base offset 0, no swizzle
}

__device__ __forceinline__ uint32_t idesc_bf16(int M, int N) {
    return (1u << 4)                       // D: FP32
           | (1u << 7)                     // A: BF16
           | (1u << 10)                    // B: BF16
           | ((uint32_t)(N >> 3) << 17)    // N
           | ((uint32_t)(M >> 4) << 24);   // M (A, B K-major; no negation)
}

__device__ __forceinline__ void umma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void umma_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}

constexpr int kPollLimit = 1 << 22;  // polls of a completion wait before it gives up

__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t phase, int polls) {
    for (int it = 0; it < polls; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(mbar), "r"(phase)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void st_bf16(uint8_t* base, uint32_t off, float v) {
    *reinterpret_cast<__nv_bfloat16*>(base + off) = __float2bfloat16_rn(v);
}

// thread's row of a K-major A tile: K/8 16-byte stores
__device__ __forceinline__ void st_row(uint8_t* base, int row, const float* v, int K) {
    for (int c = 0; c < K / 8; ++c) {
        __align__(16) __nv_bfloat16 h[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) h[i] = __float2bfloat16_rn(v[8 * c + i]);
        *reinterpret_cast<uint4*>(base + kmaj(row, 8 * c, K)) = *reinterpret_cast<const uint4*>(h);
    }
}

// How the completion waits of one launch behave: polls before a wait gives
// up, and (self-test only) a GEMM whose MMAs are not issued, so that nothing
// ever arrives on its mbarrier and its wait must run out.
struct WaitCfg {
    int polls;
    int skip_gemm;  // index of the GEMM not issued, -1: none
};

// Issues the K/16 MMAs of one GEMM (thread 0) and waits for them (all threads).
// Returns false on a timed-out wait; `inflight` then says whether MMAs of this
// CTA are still pending on the phase `phase` (left unflipped).
__device__ __forceinline__ bool gemm(uint32_t sbase, uint32_t a_off, uint32_t b_off, int K, int N, uint32_t d_tmem,
                                     bool accumulate, uint32_t mbar, uint32_t& phase, const WaitCfg& wc, int& index,
                                     bool& inflight) {
    const bool issue = index++ != wc.skip_gemm;
    fence_async_smem();
    fence_before();
    __syncthreads();
    if (threadIdx.x == 0 && issue) {
        fence_after();
        const uint32_t id = idesc_bf16(128, N);
        for (int ks = 0; ks < K / 16; ++ks) {
            const uint64_t a = sdesc(sbase + a_off + 256u * ks, K);
            const uint64_t b = sdesc(sbase + b_off + 256u * ks, K);
            umma(d_tmem, a, b, id, (accumulate || ks > 0) ? 1u : 0u);
        }
        umma_commit(mbar);
    }
    bool ok = mbar_wait(mbar, phase, wc.polls);
    ok = __syncthreads_and(ok) != 0;  // every thread takes the same branch afterwards
    if (!ok) {
        inflight = issue;
        return false;
    }
    phase ^= 1u;
    fence_after();
    return ok;
}

// Training (kTrain) or inference pass over n rows.  Training writes this
// CTA's gradient (kNParams floats, summed over its tiles) to gpart + CTA *
// kNParams and its share of the loss to lpart[CTA]; k_grad_sum adds the CTAs'
// parts in CTA order.  Every sum inside a CTA has a fixed order too (warp
// butterflies, then the four warps in order, then the tiles in order), so a
// gradient is the same bits on every run.
template <bool kTrain>
__global__ void __launch_bounds__(NT, 1) k_mlp(const float* __restrict__ X, const float* __restrict__ T, int n,
                                               Params p, float* gpart, float* Y_out, double* lpart, int* err,
                                               WaitCfg wc) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(sm);
    __shared__ __align__(8) uint64_t mbar_storage;
    __shared__ uint32_t tmem_slot;
    constexpr int NB = HID + HID + OUT;  // bias gradients: b1, b2, b3
    __shared__ float sgb[NB];
    __shared__ float sloss;
    __shared__ float swarp[NT / 32][NB + 1];  // per warp: this tile's bias-gradient and loss sums
    const int tid = threadIdx.x, warp = tid >> 5;
    const uint32_t mbar = (uint32_t)__cvta_generic_to_shared(&mbar_storage);

    // stage the weights as BF16 B operands (and transposes for the backward)
    for (int i = tid; i < HID * IN; i += NT) {
        const int o = i / IN, k = i % IN;
        st_bf16(sm, O_W1 + kmaj(o, k, IN), p.W1[i]);
    }
    for (int i = tid; i < HID * HID; i += NT) {
        const int o = i / HID, k = i % HID;
        st_bf16(sm, O_W2 + kmaj(o, k, HID), p.W2[i]);
        if (kTrain) st_bf16(sm, O_W2T + kmaj(k, o, HID), p.W2[i]);
    }
    for (int i = tid; i < OUT * HID; i += NT) {
        const int o = i / HID, k = i % HID;
        st_bf16(sm, O_W3 + kmaj(o, k, HID), p.W3[i]);
        if (kTrain) st_bf16(sm, O_W3T + kmaj(k, o, OUT), p.W3[i]);
    }
    if (kTrain) {
        for (int i = tid; i < 32768 / 16; i += NT) reinterpret_cast<uint4*>(sm + O_A3)[i] = make_uint4(0, 0, 0, 0);
        for (int i = tid; i < NB; i += NT) sgb[i] = 0.f;
        for (int i = tid; i < (NT / 32) * (NB + 1); i += NT) (&swarp[0][0])[i] = 0.f;
        if (tid == 0) sloss = 0.f;
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         (uint32_t)__cvta_generic_to_shared(&tmem_slot)),
                     "r"(TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = tmem_slot;
    const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
    uint32_t phase = 0;
    bool ok = true;
    bool first = true;
    int gi = 0;             // GEMMs issued so far (WaitCfg::skip_gemm)
    bool inflight = false;  // a timed-out wait left MMAs of this CTA pending
    const int ntiles = (n + TILE - 1) / TILE;
    for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        const int row = tile * TILE + tid;
        const bool valid = row < n;
        float x[IN];
#pragma unroll
        for (int i = 0; i < IN; ++i) x[i] = valid ? X[(size_t)row * IN + i] : 0.f;
        st_row(sm + O_X, tid, x, IN);
        if (kTrain)
            for (int i = 0; i < IN; ++i) st_bf16(sm, O_BT + kmaj(HID + i, tid, TILE), x[i]);
        // ---- layer 1
        ok = gemm(sbase, O_X, O_W1, IN, HID, tmem + C_Z1, false, mbar, phase, wc, gi, inflight);
        if (!ok) break;
        float h1[HID];
        uint64_t m1 = 0;
        for (int c = 0; c < HID; c += 16) tmem_ld16(tmem + lane_base + C_Z1 + c, h1 + c);
        for (int j = 0; j < HID; ++j) {
            const float z = h1[j] + p.b1[j];
            h1[j] = z > 0.f ? z : 0.f;
            if (z > 0.f) m1 |= (1ull << j);
        }
        st_row(sm + O_H1, tid, h1, HID);
        if (kTrain)
            for (int j = 0; j < HID; ++j) st_bf16(sm, O_BT + kmaj(j, tid, TILE), h1[j]);
        // ---- layer 2
        ok = gemm(sbase, O_H1, O_W2, HID, HID, tmem + C_Z2, false, mbar, phase, wc, gi, inflight);
        if (!ok) break;
        float h2[HID];
        uint64_t m2 = 0;
        for (int c = 0; c < HID; c += 16) tmem_ld16(tmem + lane_base + C_Z2 + c, h2 + c);
        for (int j = 0; j < HID; ++j) {
            const float z = h2[j] + p.b2[j];
            h2[j] = z > 0.f ? z : 0.f;
            if (z > 0.f) m2 |= (1ull << j);
        }
        st_row(sm + O_H2, tid, h2, HID);
        if (kTrain)
            for (int j = 0; j < HID; ++j) st_bf16(sm, O_B3 + kmaj(j, tid, TILE), h2[j]);
        // ---- layer 3
        ok = gemm(sbase, O_H2, O_W3, HID, OUT, tmem + C_Y, false, mbar, phase, wc, gi, inflight);
        if (!ok) break;
        float y[OUT];
        tmem_ld16(tmem + lane_base + C_Y, y);
        for (int o = 0; o < OUT; ++o) y[o] += p.b3[o];
        if (!kTrain) {
            if (valid) {
                Y_out[2 * (size_t)row] = y[0];
                Y_out[2 * (size_t)row + 1] = y[1];
            }
            continue;
        }
        // ---- backward
        float dy[OUT];
        float lrow = 0.f;
        for (int o = 0; o < OUT; ++o) dy[o] = 0.f;
        if (valid)
            for (int o = 0; o < USED; ++o) {
                const float e = y[o] - T[2 * (size_t)row + o];
                dy[o] = 2.f * e / (float)n;
                lrow += e * e;
            }
        const int lane = tid & 31;
        {
            const float ls = warp_sum(lrow);
            if (lane == 0) swarp[warp][NB] = ls;
        }
        for (int o = 0; o < USED; ++o) {
            const float v = warp_sum(dy[o]);
            if (lane == 0) swarp[warp][2 * HID + o] = v;
        }
        st_row(sm + O_DY, tid, dy, OUT);
        for (int o = 0; o < USED; ++o) st_bf16(sm, O_A3 + kmaj(o, tid, TILE), dy[o]);
        ok = gemm(sbase, O_DY, O_W3T, OUT, HID, tmem + C_Z1, false, mbar, phase, wc, gi, inflight);  // dH2
        if (!ok) break;
        float d2[HID];
        for (int c = 0; c < HID; c += 16) tmem_ld16(tmem + lane_base + C_Z1 + c, d2 + c);
#pragma unroll
        for (int j = 0; j < HID; ++j) {
            d2[j] = ((m2 >> j) & 1ull) ? d2[j] : 0.f;
            const float v = warp_sum(d2[j]);
            if (lane == 0) swarp[warp][HID + j] = v;
        }
        st_row(sm + O_DZ2, tid, d2, HID);
        for (int j = 0; j < HID; ++j) st_bf16(sm, O_AT + kmaj(j, tid, TILE), d2[j]);
        ok = gemm(sbase, O_DZ2, O_W2T, HID, HID, tmem + C_Z2, false, mbar, phase, wc, gi, inflight);  // dH1
        if (!ok) break;
        float d1[HID];
        for (int c = 0; c < HID; c += 16) tmem_ld16(tmem + lane_base + C_Z2 + c, d1 + c);
#pragma unroll
        for (int j = 0; j < HID; ++j) {
            d1[j] = ((m1 >> j) & 1ull) ? d1[j] : 0.f;
            const float v = warp_sum(d1[j]);
            if (lane == 0) swarp[warp][j] = v;
            st_bf16(sm, O_AT + kmaj(HID + j, tid, TILE), d1[j]);
        }
        // this tile's sums, the warps added in order (the tile's other smem
        // writes are fenced by the barrier inside the next GEMM)
        __syncthreads();
        for (int i = tid; i <= NB; i += NT) {
            const float v = ((swarp[0][i] + swarp[1][i]) + swarp[2][i]) + swarp[3][i];
            if (i < NB) sgb[i] += v;
            else sloss += v;
        }
        // weight gradients, accumulated in tensor memory over this CTA's tiles
        ok = gemm(sbase, O_AT, O_BT, TILE, HID + IN, tmem + C_DW12, !first, mbar, phase, wc, gi, inflight);
        if (!ok) break;
        ok = gemm(sbase, O_A3, O_B3, TILE, HID, tmem + C_DW3, !first, mbar, phase, wc, gi, inflight);
        if (!ok) break;
        first = false;
    }
    if (!ok && threadIdx.x == 0) atomicExch(err, 1);
    // MMAs still pending after a timed-out wait write tensor memory: wait for
    // them (bounded again) before that memory is freed below
    if (!ok && inflight) mbar_wait(mbar, phase, kPollLimit);
    if (kTrain) {
        // this CTA's part: D12 rows 0..63: dW2 (cols 0..63); rows 64..127:
        // dW1 (cols 64..79); D3 rows 0..15: dW3 (the rows of unused outputs
        // zero); every entry written, zero when the CTA stopped early
        Params g = carve(gpart + (size_t)blockIdx.x * kNParams);
        const bool have = ok && !first;
        const int m = tid;
        float v[16];
        if (m < HID) {
            for (int c = 0; c < HID; c += 16) {
                if (have) tmem_ld16(tmem + lane_base + C_DW12 + c, v);
                for (int i = 0; i < 16; ++i) g.W2[m * HID + c + i] = have ? v[i] : 0.f;
            }
        } else {
            if (have) tmem_ld16(tmem + lane_base + C_DW12 + HID, v);
            for (int i = 0; i < IN; ++i) g.W1[(m - HID) * IN + i] = have ? v[i] : 0.f;
        }
        for (int c = 0; c < HID; c += 16) {
            if (have) tmem_ld16(tmem + lane_base + C_DW3 + c, v);
            if (m < OUT)
                for (int i = 0; i < 16; ++i) g.W3[m * HID + c + i] = (have && m < USED) ? v[i] : 0.f;
        }
        __syncthreads();
        for (int i = tid; i < HID; i += NT) {
            g.b1[i] = have ? sgb[i] : 0.f;
            g.b2[i] = have ? sgb[HID + i] : 0.f;
        }
        if (tid < OUT) g.b3[tid] = have ? sgb[2 * HID + tid] : 0.f;
        if (tid == 0) lpart[blockIdx.x] = have ? (double)sloss / (double)n : 0.0;
    }
    fence_before();
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
}

// g[i] = the CTAs' parts of parameter i added in CTA order; *loss likewise
__global__ void k_grad_sum(const float* __restrict__ part, int nparts, float* g, const double* __restrict__ lpart,
                           double* loss) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < kNParams) {
        float acc = 0.f;
        for (int b = 0; b < nparts; ++b) acc += part[(size_t)b * kNParams + i];
        g[i] = acc;
    }
    if (i == 0) {
        double l = 0.0;
        for (int b = 0; b < nparts; ++b) l += lpart[b];
        *loss = l;
    }
}

__global__ void k_adam(float* p, const float* g, float* m, float* v, int n, float lr, float b1, float b2, float eps,
                       float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}


}  // namespace mlp
}  // namespace pgb

struct pg_mlp {
    int device = 0;
    cudaStream_t stream = nullptr;
    float* params = nullptr;   // kNParams
    float* grads = nullptr;
    float* m = nullptr;
    float* v = nullptr;
    double* loss = nullptr;
    float* gpart = nullptr;    // per CTA of a gradient launch: its part of the gradient (kNParams)
    double* lpart = nullptr;   // and of the loss
    int* err = nullptr;
    float* probe = nullptr;    // one tile of inputs and outputs for pg_mlp_wait_selftest
    int step = 0;
    int n_sms = 148;
};

using namespace pgb;
using namespace pgb::mlp;

extern "C" {

int pg_mlp_create(int32_t device, uint64_t seed, pg_mlp** out) {
    if (!out) { set_error("pg_mlp_create: null output"); return PG_ERR_ARG; }
    *out = nullptr;
    pg_mlp* m = new (std::nothrow) pg_mlp;
    if (!m) { set_error("pg_mlp_create: out of host memory"); return PG_ERR_ARG; }
    m->device = device;
    PG_CUDA(cudaSetDevice(device));
    PG_CUDA(cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking));
    PG_CUDA(cudaMalloc((void**)&m->params, 4 * kNParams * sizeof(float)));
    m->grads = m->params + kNParams;
    m->m = m->grads + kNParams;
    m->v = m->m + kNParams;
    PG_CUDA(fill_sync(m->params, 0, 4 * kNParams * sizeof(float)));
    PG_CUDA(cudaMalloc((void**)&m->loss, sizeof(double)));
    PG_CUDA(cudaMalloc((void**)&m->err, sizeof(int)));
    PG_CUDA(fill_sync(m->err, 0, sizeof(int)));
    PG_CUDA(cudaMalloc((void**)&m->probe, TILE * (IN + 2) * sizeof(float)));
    PG_CUDA(fill_sync(m->probe, 0, TILE * (IN + 2) * sizeof(float)));
    cudaDeviceGetAttribute(&m->n_sms, cudaDevAttrMultiProcessorCount, device);
    PG_CUDA(cudaMalloc((void**)&m->gpart, (size_t)m->n_sms * kNParams * sizeof(float)));
    PG_CUDA(cudaMalloc((void**)&m->lpart, (size_t)m->n_sms * sizeof(double)));
    PG_CUDA(cudaFuncSetAttribute(k_mlp<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_ALLOC));
    PG_CUDA(cudaFuncSetAttribute(k_mlp<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_ALLOC));
    // He initialisation (host, seeded), last layer scaled to start near zero output
    std::mt19937_64 rng(seed);
    std::normal_distribution<float> nd(0.f, 1.f);
    std::vector<float> h(kNParams, 0.f);
    Params hp = carve(h.data());
    for (int i = 0; i < kW1; ++i) hp.W1[i] = nd(rng) * std::sqrt(2.f / IN);
    for (int i = 0; i < kW2; ++i) hp.W2[i] = nd(rng) * std::sqrt(2.f / HID);
    for (int o = 0; o < USED; ++o)
        for (int j = 0; j < HID; ++j) hp.W3[o * HID + j] = 0.1f * nd(rng) * std::sqrt(1.f / HID);
    PG_CUDA(h2d_sync(m->params, h.data(), kNParams * sizeof(float)));
    *out = m;
    return PG_OK;
}

void pg_mlp_destroy(pg_mlp* m) {
    if (!m) return;
    cudaSetDevice(m->device);
    if (m->params) cudaFree(m->params);
    if (m->loss) cudaFree(m->loss);
    if (m->gpart) cudaFree(m->gpart);
    if (m->lpart) cudaFree(m->lpart);
    if (m->err) cudaFree(m->err);
    if (m->probe) cudaFree(m->probe);
    if (m->stream) cudaStreamDestroy(m->stream);
    delete m;
}

int32_t pg_mlp_param_count(void) { return kNParams; }

int pg_mlp_params(pg_mlp* m, float* host, int32_t set) {
    if (!m || !host) { set_error("pg_mlp_params: null argument"); return PG_ERR_ARG; }
    cudaSetDevice(m->device);
    PG_CUDA(cudaStreamSynchronize(m->stream));
    if (set) {
        PG_CUDA(h2d_sync(m->params, host, kNParams * sizeof(float)));
        PG_CUDA(fill_sync(m->m, 0, 2 * kNParams * sizeof(float)));
        m->step = 0;
    } else {
        PG_CUDA(cudaMemcpy(host, m->params, kNParams * sizeof(float), cudaMemcpyDeviceToHost));
    }
    return PG_OK;
}

int pg_mlp_grads(pg_mlp* m, float* host) {
    if (!m || !host) { set_error("pg_mlp_grads: null argument"); return PG_ERR_ARG; }
    cudaSetDevice(m->device);
    PG_CUDA(cudaStreamSynchronize(m->stream));
    PG_CUDA(cudaMemcpy(host, m->grads, kNParams * sizeof(float), cudaMemcpyDeviceToHost));
    return PG_OK;
}

static int mlp_check_err(pg_mlp* m) {
    int e = 0;
    PG_CUDA(cudaMemcpyAsync(&e, m->err, sizeof(int), cudaMemcpyDeviceToHost, m->stream));
    PG_CUDA(cudaStreamSynchronize(m->stream));
    if (e) {
        cudaMemsetAsync(m->err, 0, sizeof(int), m->stream);
        set_error("pg_mlp: tensor-core completion wait timed out");
        return PG_ERR_STATE;
    }
    return PG_OK;
}

// Y_dev[2n] = MLP(X_dev[16n]) (device pointers)
int pg_mlp_forward(pg_mlp* m, const float* X_dev, int32_t n, float* Y_dev, void* stream) {
    if (!m || (n > 0 && (!X_dev || !Y_dev))) { set_error("pg_mlp_forward: null argument"); return PG_ERR_ARG; }
    if (n <= 0) return PG_OK;
    cudaSetDevice(m->device);
    cudaStream_t s = stream ? (cudaStream_t)stream : m->stream;
    const int tiles = (n + TILE - 1) / TILE;
    const int grid = tiles < m->n_sms ? tiles : m->n_sms;
    Params p = carve(m->params);
    k_mlp<false><<<grid, NT, SMEM_ALLOC, s>>>(X_dev, nullptr, n, p, nullptr, Y_dev, nullptr, m->err,
                                              WaitCfg{kPollLimit, -1});
    PG_CUDA(cudaGetLastError());
    if (s == m->stream) return mlp_check_err(m);
    return PG_OK;
}

// Self-test of the bounded completion wait: one forward tile whose first GEMM
// is not issued, so nothing arrives on its mbarrier and the wait must give up
// after `polls` polls.  Nothing is in flight when it does, so the kernel
// records its error word, frees its tensor memory and returns; the call
// returns the timeout status and the network stays usable.
int pg_mlp_wait_selftest(pg_mlp* m, int32_t polls) {
    if (!m || polls < 1) { set_error("pg_mlp_wait_selftest: bad argument"); return PG_ERR_ARG; }
    cudaSetDevice(m->device);
    Params p = carve(m->params);
    k_mlp<false><<<1, NT, SMEM_ALLOC, m->stream>>>(m->probe, nullptr, TILE, p, nullptr, m->probe + TILE * IN, nullptr, m->err,
                                                   WaitCfg{polls, 0});
    PG_CUDA(cudaGetLastError());
    return mlp_check_err(m);
}

// gradients of the mean-squared loss over all n rows into the internal buffer; loss to *loss_host
int pg_mlp_gradient(pg_mlp* m, const float* X_dev, const float* T_dev, int32_t n, double* loss_host) {
    if (!m || !X_dev || !T_dev || n <= 0) { set_error("pg_mlp_gradient: bad argument"); return PG_ERR_ARG; }
    cudaSetDevice(m->device);
    cudaStream_t s = m->stream;
    const int tiles = (n + TILE - 1) / TILE;
    const int grid = tiles < m->n_sms ? tiles : m->n_sms;
    Params p = carve(m->params);
    k_mlp<true><<<grid, NT, SMEM_ALLOC, s>>>(X_dev, T_dev, n, p, m->gpart, nullptr, m->lpart, m->err,
                                             WaitCfg{kPollLimit, -1});
    PG_CUDA(cudaGetLastError());
    k_grad_sum<<<(kNParams + 255) / 256, 256, 0, s>>>(m->gpart, grid, m->grads, m->lpart, m->loss);
    PG_CUDA(cudaGetLastError());
    int rc = mlp_check_err(m);
    if (rc) return rc;
    if (loss_host) PG_CUDA(cudaMemcpy(loss_host, m->loss, sizeof(double), cudaMemcpyDeviceToHost));
    return PG_OK;
}

int pg_mlp_adam(pg_mlp* m, float lr) {
    if (!m) { set_error("pg_mlp_adam: null"); return PG_ERR_ARG; }
    cudaSetDevice(m->device);
    m->step += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, (float)m->step), c2 = 1.f - std::pow(b2, (float)m->step);
    k_adam<<<(kNParams + 255) / 256, 256, 0, m->stream>>>(m->params, m->grads, m->m, m->v, kNParams, lr, b1, b2, 1e-8f,
                                                        c1, c2);
    PG_CUDA(cudaGetLastError());
    return PG_OK;
}

// Minibatch training: `epochs` passes over n rows in batches of `batch` rows
// (the caller shuffles).  Writes the mean loss of every epoch to loss_hist.
int pg_mlp_train(pg_mlp* m, const float* X_dev, const float* T_dev, int32_t n, int32_t epochs, int32_t batch, float lr,
                 double* loss_hist) {
    if (!m || !X_dev || !T_dev || n <= 0 || batch <= 0) { set_error("pg_mlp_train: bad argument"); return PG_ERR_ARG; }
    for (int ep = 0; ep < epochs; ++ep) {
        double acc = 0.0;
        int nb = 0;
        for (int s0 = 0; s0 < n; s0 += batch) {
            const int nn = (n - s0) < batch ? (n - s0) : batch;
            double l = 0.0;
            int rc = pg_mlp_gradient(m, X_dev + (size_t)s0 * IN, T_dev + (size_t)s0 * 2, nn, &l);
            if (rc) return rc;
            rc = pg_mlp_adam(m, lr);
            if (rc) return rc;
            acc += l;
            ++nb;
        }
        if (loss_hist) loss_hist[ep] = acc / (nb ? nb : 1);
    }
    return PG_OK;
}

}  // extern "C"
