// BF16 tensor-core GEMM for the learned closure on sm_100a (tcgen05 + TMEM).
//
//   C[M x N] = A[M x K] * B[N x K]^T     A, B: bf16, row-major, K contiguous
//                                        accumulation: fp32 in tensor memory
//
// One CTA computes a 128 x NT tile (NT = 64, 128 or 256) with 128 threads,
// over all of K or over one of `ksplit` K ranges (blockIdx.z; fp32 partial
// tiles, summed by a second kernel):
//   - all threads stage 128 x 64 (A) and NT x 64 (B) bf16 blocks into shared
//     memory with 16-byte cp.async copies, three stages deep (two blocks in
//     flight while the tensor cores work on a third), in the canonical
//     no-swizzle K-major layout of the tensor cores: 8 x 16-byte core
//     matrices, the two K halves of an MMA 128 B apart (LBO), 8-row groups
//     1024 B apart (SBO);
//   - thread 0 issues tcgen05.mma (kind::f16, M = 128, N = NT, K = 16) four
//     times per 64-wide block into the TMEM accumulator and commits them to
//     the stage's mbarrier, so the copies of blocks k+1 and k+2 overlap the
//     MMAs of k;
//   - the epilogue reads the accumulator with tcgen05.ld (warp w owns rows
//     32w..32w+31, one row per thread) and applies one of the closure's
//     fused epilogues (bias, GELU, GELU', transposed copies, fp32 store).
// Every mbarrier wait is bounded: past the limit the CTA records an error
// and skips the rest, then frees its tensor memory.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace od {
namespace mlp {

constexpr int BM = 128;        // rows per CTA tile
constexpr int BK = 64;         // K per pipeline stage
constexpr int STAGES = 3;
constexpr long long kWaitLimit = 1LL << 26;

enum Epi : int {
    kStoreF32 = 0,     // C (+ bias) -> fp32 [M x N] (ldc = N)
    kBiasGelu = 1,     // z = C + bias -> z fp32, gelu(z) -> bf16 [M x N] and bf16 transpose [N x M]
    kGeluGrad = 2,     // dz = C * gelu'(z_in) -> bf16 [M x N] and bf16 transpose [N x M]
    kApplyRhs = 3,     // rhs[v][row*64 + p] += rhs_scale[v] * (C + bias) for column v*64 + p < 320, row < rows
};

struct GemmArgs {
    const __nv_bfloat16* A;   // [M x K]
    const __nv_bfloat16* B;   // [N x K]
    int M, N, K;
    const float* bias;        // [N] or null
    float* out_f32;           // kStoreF32: C; kBiasGelu: z
    __nv_bfloat16* out_bf;    // kBiasGelu: gelu(z); kGeluGrad: dz
    __nv_bfloat16* out_bfT;   // transposed copy ([N x M]) or null
    const float* z_in;        // kGeluGrad: the layer's pre-activation [M x N]
    int* err;                 // set to 1 when a bounded wait gives up
    int ksplit;               // > 1 (kStoreF32 only): partial sums into ws[split][M][N]
    float* ws;
    float* rhs;               // kApplyRhs: the solver's RHS (5 planes of rhs_npts values)
    long long rhs_npts;
    int rhs_rows;             // elements (rows beyond are padding)
    float rhs_scale[5];
};

// Arguments of the fused inference kernel (od_mlp_fused.cuh): the whole
// network on 128-row tiles, output added into the solver's RHS.
struct FusedArgs {
    const __nv_bfloat16* X;      // [M x 896] standardised features
    const __nv_bfloat16* Wt;     // the weights in step order and shared-memory layout (tile_fused_weights)
    const float* bias[4];
    float* rhs;                  // the solver's RHS: 5 planes of rhs_npts values
    long long rhs_npts;
    int rhs_rows;                // elements (rows beyond are padding)
    float rhs_scale[5];
    int* err;
};

// launches the fused inference kernel on M rows (a multiple of 128)
cudaError_t launch_fused(const FusedArgs& a, int M, cudaStream_t s);

// bytes of the fused kernel's weight image
constexpr size_t kFusedWeightBytes = 884736;

// writes the weight image the fused kernel streams: for each of its 30 K
// steps the B tile (256 or 160 rows x 64 columns of one layer) in the
// shared-memory core-matrix layout, so that one bulk copy fills a stage.
// W: [256 x 896], [256 x 256], [256 x 256], [>= 320 x 256] bf16.
cudaError_t tile_fused_weights(const __nv_bfloat16* const W[4], __nv_bfloat16* Wt, cudaStream_t s);

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= 1ull << 46;  // descriptor version of sm_100
    // base offset 0, leading-byte-offset mode 0, layout type 0 (no swizzle)
    return d;
}

// kind::f16 instruction descriptor: bf16 x bf16 -> f32, both K-major
__host__ __device__ constexpr uint32_t instr_desc(int m, int n) {
    return (1u << 4)                       // D format f32
           | (1u << 7)                     // A format bf16
           | (1u << 10)                    // B format bf16
           | ((uint32_t)(n >> 3) << 17)    // N / 8
           | ((uint32_t)(m >> 4) << 24);   // M / 16
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

// Bounded wait for the given phase parity: false after `limit` polls (the
// caller then sets its error flag, waits for its own copies with the same
// bound, frees its tensor memory and returns).
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, long long limit = kWaitLimit) {
    for (long long it = 0; it < limit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}

// GELU in its tanh form (Hendrycks & Gimpel, "Gaussian Error Linear Units",
// 2016): gelu(z) = z/2 (1 + tanh(k (z + 0.044715 z^3))), k = sqrt(2/pi), with
// tanh from the single-instruction tanh.approx.f32 (relative error about
// 2^-11, below the bf16 rounding the activations get next).
__device__ __forceinline__ float tanh_fast(float x) {
    float r;
    asm("tanh.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

constexpr float kGeluK = 0.7978845608028654f;   // sqrt(2 / pi)

__device__ __forceinline__ float gelu(float z) {
    const float t = tanh_fast(kGeluK * fmaf(0.044715f * z, z * z, z));
    return 0.5f * z * (1.0f + t);
}

// d gelu / dz = (1 + t)/2 + z/2 (1 - t^2) k (1 + 3 * 0.044715 z^2)
__device__ __forceinline__ float gelu_grad(float z) {
    const float z2 = z * z;
    const float t = tanh_fast(kGeluK * fmaf(0.044715f * z, z2, z));
    return 0.5f * (1.0f + t) + 0.5f * z * (1.0f - t * t) * kGeluK * fmaf(0.134145f, z2, 1.0f);
}

// smem offset of (row r, 16-byte K chunk kc) inside a tile
__device__ __forceinline__ uint32_t tile_off(int r, int kc) {
    return (uint32_t)((r >> 3) * 1024 + kc * 128 + (r & 7) * 16);
}

template <int NT>
struct Smem {
    alignas(1024) unsigned char a[STAGES][BM * BK * 2];
    alignas(1024) unsigned char b[STAGES][NT * BK * 2];
    alignas(8) unsigned long long bar[STAGES];
    alignas(8) unsigned long long done_bar;
    uint32_t tmem_base;
    int failed;
};

template <int NT>
__device__ __forceinline__ void load_stage(const GemmArgs& g, Smem<NT>& s, int st, int m0, int n0, int kb) {
    const int t = threadIdx.x;
    const int k0 = kb * BK;
    // A: 128 rows x 8 chunks; 8 consecutive threads cover rows r..r+7 of one chunk
#pragma unroll
    for (int i = 0; i < (BM * 8) / 128; ++i) {
        const int c = t + 128 * i;
        const int r = (c & 7) + 8 * (c >> 6);
        const int kc = (c >> 3) & 7;
        cp_async16(smem_addr(s.a[st]) + tile_off(r, kc), g.A + (size_t)(m0 + r) * g.K + k0 + kc * 8);
    }
#pragma unroll
    for (int i = 0; i < (NT * 8) / 128; ++i) {
        const int c = t + 128 * i;
        const int r = (c & 7) + 8 * (c >> 6);
        const int kc = (c >> 3) & 7;
        cp_async16(smem_addr(s.b[st]) + tile_off(r, kc), g.B + (size_t)(n0 + r) * g.K + k0 + kc * 8);
    }
}

template <int NT, int EPI>
__global__ void __launch_bounds__(128, 1) gemm_kernel(const GemmArgs g) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    // 1024-byte aligned view of the dynamic shared memory
    Smem<NT>& s = *reinterpret_cast<Smem<NT>*>(
        smem_raw + ((1024 - (smem_addr(smem_raw) & 1023)) & 1023));
    const int t = threadIdx.x;
    const int warp = t >> 5;
    const int m0 = blockIdx.x * BM;
    const int n0 = blockIdx.y * NT;
    const int ks = g.ksplit > 1 ? g.ksplit : 1;
    const int KB = g.K / BK / ks;             // K blocks of this CTA's range
    const int kb0 = (int)blockIdx.z * KB;
    constexpr uint32_t kCols = NT;  // fp32 accumulator: one column per N

    if (t == 0) {
        for (int i = 0; i < STAGES; ++i) mbar_init(smem_addr(&s.bar[i]), 1);
        mbar_init(smem_addr(&s.done_bar), 1);
        s.failed = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&s.tmem_base)),
                     "r"(kCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s.tmem_base;
    const uint32_t idesc = instr_desc(BM, NT);

    // prologue: blocks 0 .. STAGES-2, one cp.async group each (empty groups
    // past the end keep the group count equal to the block count)
#pragma unroll
    for (int i = 0; i < STAGES - 1; ++i) {
        if (i < KB) load_stage<NT>(g, s, i, m0, n0, kb0 + i);
        asm volatile("cp.async.commit_group;" ::: "memory");
    }
    for (int kb = 0; kb < KB; ++kb) {
        const int st = kb % STAGES;
        // block kb has landed in stage st (at most STAGES-2 newer groups pending)
        asm volatile("cp.async.wait_group %0;" ::"n"(STAGES - 2) : "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (t == 0 && !s.failed) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t a0 = smem_addr(s.a[st]), b0 = smem_addr(s.b[st]);
#pragma unroll
            for (int k = 0; k < BK / 16; ++k) {
                const uint64_t ad = smem_desc(a0 + k * 256, 128, 1024);
                const uint64_t bd = smem_desc(b0 + k * 256, 128, 1024);
                const uint32_t acc = (kb > 0 || k > 0) ? 1u : 0u;
                asm volatile(
                    "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                    " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}" ::"r"(tmem),
                    "l"(ad), "l"(bd), "r"(idesc), "r"(acc)
                    : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_addr(&s.bar[st]))
                         : "memory");
        }
        // prefetch block kb+STAGES-1 into the stage of block kb-1 once its MMAs are done
        const int nb = kb + STAGES - 1;
        if (nb < KB) {
            const int nst = nb % STAGES;
            if (kb >= 1) {
                // completion number (kb-1)/STAGES of bar[nst]
                const uint32_t parity = (uint32_t)(((kb - 1) / STAGES) & 1);
                if (!mbar_wait(smem_addr(&s.bar[nst]), parity)) {
                    s.failed = 1;
                    if (g.err) atomicExch(g.err, 1);
                }
            }
            __syncthreads();
            if (!s.failed) load_stage<NT>(g, s, nst, m0, n0, kb0 + nb);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    }
    // all MMAs done: commit once more on the final barrier
    if (t == 0 && !s.failed) {
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         smem_addr(&s.done_bar))
                     : "memory");
    }
    __syncthreads();
    bool ok = !s.failed;
    if (ok && !mbar_wait(smem_addr(&s.done_bar), 0)) {
        ok = false;
        if (g.err) atomicExch(g.err, 1);
    }
    ok = __all_sync(0xffffffffu, ok);  // tcgen05.ld is warp-collective
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (ok) {
        // Epilogue per 32-column chunk: the accumulator rows come out of TMEM
        // one row per thread; row-major outputs go through a 32 x 32 shared
        // staging tile (XOR-swizzled, in the now idle operand buffer) so that
        // each store instruction writes one contiguous row segment.
        const int lane = t & 31;
        const int row0 = m0 + warp * 32;
        float* stg = reinterpret_cast<float*>(s.a[0]) + warp * 1024;
        const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll 1
        for (int c0 = 0; c0 < NT; c0 += 32) {
            uint32_t r[32];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
                "[%16];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                  "=r"(r[15])
                : "r"(lane_base + (uint32_t)c0));
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
                "[%16];"
                : "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]),
                  "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]),
                  "=r"(r[30]), "=r"(r[31])
                : "r"(lane_base + (uint32_t)(c0 + 16)));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            const int n = n0 + c0;
            float v[32];
#pragma unroll
            for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
            if constexpr (EPI == kGeluGrad) {
                // z_in of this row chunk, read row by row (coalesced) through the staging tile
#pragma unroll
                for (int rr = 0; rr < 32; ++rr) stg[rr * 32 + (lane ^ rr)] = g.z_in[(size_t)(row0 + rr) * g.N + n + lane];
                __syncwarp();
#pragma unroll
                for (int j = 0; j < 32; ++j) v[j] *= gelu_grad(stg[lane * 32 + (j ^ lane)]);
                __syncwarp();
            } else {
                if (g.bias && !(EPI == kStoreF32 && ks > 1)) {
#pragma unroll
                    for (int j = 0; j < 32; ++j) v[j] += g.bias[n + j];
                }
            }
            // row-major fp32 output: C, the split-K partial, or z
            if constexpr (EPI == kApplyRhs) {
                // columns n..n+31 lie in one variable's 64-point block
                const int var = n >> 6;
                if (var < 5) {
                    const float sc = g.rhs_scale[var];
#pragma unroll
                    for (int j = 0; j < 32; ++j) stg[lane * 32 + (j ^ lane)] = v[j];
                    __syncwarp();
                    float* base = g.rhs + (size_t)var * g.rhs_npts + (n & 63) + lane;
                    // all 32 row segments loaded first (one memory round trip), then updated
                    float cur[32];
#pragma unroll
                    for (int rr = 0; rr < 32; ++rr)
                        cur[rr] = row0 + rr < g.rhs_rows ? base[(size_t)(row0 + rr) * 64] : 0.f;
#pragma unroll
                    for (int rr = 0; rr < 32; ++rr)
                        if (row0 + rr < g.rhs_rows) base[(size_t)(row0 + rr) * 64] = cur[rr] + sc * stg[rr * 32 + (lane ^ rr)];
                    __syncwarp();
                }
            }
            if constexpr (EPI == kStoreF32 || EPI == kBiasGelu) {
                // (z of a hidden layer is kept only for training: null at inference)
                float* dst = EPI == kStoreF32 && ks > 1 ? g.ws + (size_t)blockIdx.z * g.M * g.N : g.out_f32;
                if (dst) {
#pragma unroll
                    for (int j = 0; j < 32; ++j) stg[lane * 32 + (j ^ lane)] = v[j];
                    __syncwarp();
#pragma unroll 4
                    for (int rr = 0; rr < 32; ++rr)
                        dst[(size_t)(row0 + rr) * g.N + n + lane] = stg[rr * 32 + (lane ^ rr)];
                    __syncwarp();
                }
            }
            // bf16 outputs: gelu(z) or dz, row-major and (optionally) transposed
            if constexpr (EPI == kBiasGelu || EPI == kGeluGrad) {
                if constexpr (EPI == kBiasGelu) {
#pragma unroll
                    for (int j = 0; j < 32; ++j) v[j] = gelu(v[j]);
                }
#pragma unroll
                for (int j = 0; j < 32; ++j) v[j] = __bfloat162float(__float2bfloat16_rn(v[j]));
                if (g.out_bfT) {
#pragma unroll
                    for (int j = 0; j < 32; ++j) g.out_bfT[(size_t)(n + j) * g.M + row0 + lane] = __float2bfloat16_rn(v[j]);
                }
#pragma unroll
                for (int j = 0; j < 32; ++j) stg[lane * 32 + (j ^ lane)] = v[j];
                __syncwarp();
#pragma unroll 4
                for (int rr = 0; rr < 32; ++rr)
                    g.out_bf[(size_t)(row0 + rr) * g.N + n + lane] = __float2bfloat16_rn(stg[rr * 32 + (lane ^ rr)]);
                __syncwarp();
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols) : "memory");
    }
}

template <int NT>
constexpr size_t gemm_smem_bytes() {
    return sizeof(Smem<NT>) + 1024;
}


}  // namespace mlp
}  // namespace od
