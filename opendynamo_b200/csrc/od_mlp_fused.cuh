// Fused closure inference on sm_100a (tcgen05 + TMEM): the whole per-element
// network 896 -> 256 -> 256 -> 256 -> 320 for a tile of 128 elements in one
// CTA, its output added straight into the solver's RHS.
//
// The hidden activations never leave the SM: each layer's epilogue reads the
// accumulator from tensor memory (tcgen05.ld), adds the bias, applies GELU,
// rounds to bf16 and writes the result into shared memory in the canonical
// K-major core-matrix layout the next layer's MMAs read as their A operand.
// Only the features (layer 1's A, written in this kernel's tile layout by
// the features kernel or by phase A) and the weights (every layer's B, from a
// step-ordered image in the shared-memory layout, tile_fused_weights) are
// streamed, in 64-wide K blocks, four stages deep, as bulk copies that
// complete on the stage's `full` mbarrier.
//
// Warp roles: a load warp (lane 0 issues the bulk copies, refilling each
// stage as soon as its MMAs are complete, up to four steps ahead of the
// MMAs), an MMA warp (lane 0
// issues tcgen05.mma, kind::f16, M = 128, K = 16, and commits each stage's
// MMAs to its `bar` mbarrier and each layer's last MMAs to a `done`
// mbarrier) and 16 epilogue warps (warp w: TMEM lanes 32 (w % 4) .. +31). The
// layers alternate between two accumulators of 256 TMEM columns, so a
// layer's MMAs never wait for the epilogue of the layer before to finish
// reading its accumulator. A hidden layer's epilogue runs k-block by k-block
// (64 columns; each warp 16 of them) and releases each k-block of the next
// layer's input on a `kready` mbarrier, so the next layer's MMAs start on the
// first k-block while the epilogue works on the rest. The output layer runs
// as two passes of N = 160 (columns 0-159 and 160-319: variables 0-2.5 and
// 2.5-5), the first pass's epilogue beside the second pass's MMAs.
//
// Shared memory (197 KiB, 198 KiB with the alignment slack the launch adds):
// one 64 KiB activation buffer of four 128 x 64 k-blocks, four 32 KiB weight
// stages and the biases (the RHS update reduces straight from registers). A
// layer's epilogue overwrites its own input in place: it starts only after
// all of the layer's MMAs have completed. During layer 1 the activation
// buffer holds the feature stages instead (layer 1's output is written after
// its last MMA). Tensor memory: 512 fp32 columns, two accumulators.
// Every mbarrier wait is bounded: past the limit the CTA records an error,
// skips the remaining work, waits for its own copies and MMAs and frees its
// tensor memory.
#pragma once

#include "od_mlp.cuh"

namespace od {
namespace mlp {

constexpr int kFIn = 896, kFHid = 256, kFOut = 320, kFPass = 160;
constexpr int kFStages = 4;
constexpr int kFEpiThreads = 512;   // 16 epilogue warps: warp w reads TMEM lanes 32 (w % 4) .. +31
constexpr int kFThreads = kFEpiThreads + 64;   // + the MMA warp and the load warp
constexpr int kFGroups = kFEpiThreads / 128;   // column groups of the output epilogue
constexpr int kFUnits = 5;   // hidden layers 1-3, output passes 0 and 1
constexpr int kFSteps = kFIn / BK + 2 * (kFHid / BK) + 2 * (kFHid / BK);   // 14 + 4 + 4 + 2 x 4 = 30
constexpr uint32_t kFStageBytes = kFHid * BK * 2;      // weight tile of a hidden-layer step
constexpr uint32_t kFOutStageBytes = kFPass * BK * 2;  // weight tile of an output step
static_assert(22 * kFStageBytes + 8 * kFOutStageBytes == kFusedWeightBytes, "weight image size");

struct FusedSmem {
    alignas(1024) unsigned char h[4][BM * BK * 2];   // activations [k-block]; layer 1: feature stages
    alignas(1024) unsigned char b[kFStages][kFHid * BK * 2];   // weight stages
    alignas(16) float bias[3 * kFHid + kFOut];   // the four layers' biases, read by every epilogue
    alignas(8) unsigned long long bar[kFStages];    // the stage's MMAs are complete (stage free)
    alignas(8) unsigned long long full[kFStages];   // the stage's weight tile has landed
    alignas(8) unsigned long long done[2];          // unit u's MMAs are complete: done[u & 1], completion u >> 1
    alignas(8) unsigned long long kready[kFHid / BK];   // k-block kb of hidden layer u's output written: completion u
    uint32_t tmem_base;
    int failed;
};

constexpr size_t fused_smem_bytes() { return sizeof(FusedSmem) + 1024; }

// step -> (layer 0..3, pass of the output layer, K block)
struct FStep {
    int layer, pass, kb;
};

__device__ __forceinline__ FStep fused_step(int s) {
    if (s < 14) return {0, 0, s};
    if (s < 18) return {1, 0, s - 14};
    if (s < 22) return {2, 0, s - 18};
    return {3, (s - 22) >> 2, (s - 22) & 3};
}

// unit of a step: hidden layers 0-2, output passes 3 and 4; its accumulator is u & 1
__device__ __forceinline__ int fused_unit(const FStep& f) { return f.layer < 3 ? f.layer : 3 + f.pass; }

// byte offset of step s's weight tile in the image, and its size
__device__ __forceinline__ uint32_t fused_w_off(int s) {
    return s < 22 ? (uint32_t)s * kFStageBytes : 22u * kFStageBytes + (uint32_t)(s - 22) * kFOutStageBytes;
}
__device__ __forceinline__ uint32_t fused_w_bytes(int s) { return s < 22 ? kFStageBytes : kFOutStageBytes; }

constexpr uint32_t kFXBytes = BM * BK * 2;   // feature block of a layer-1 step

// The load warp's lane 0: the weight tile of step s (and for layer 1 the tile's feature
// block) into its stage, bulk copies that complete on the stage's `full`
// barrier. with_x = false posts the barrier's byte count for both but copies
// only the weights; fused_load_x then adds the features.
__device__ __forceinline__ void fused_load_x(const FusedArgs& g, FusedSmem& sm, int s, int tile) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(sm.h[s % kFStages])),
                 "l"(reinterpret_cast<const char*>(g.X) + ((size_t)tile * (kFIn / BK) + s) * kFXBytes), "r"(kFXBytes),
                 "r"(smem_addr(&sm.full[s % kFStages]))
                 : "memory");
}

__device__ __forceinline__ void fused_load(const FusedArgs& g, FusedSmem& sm, int s, int tile, bool with_x = true) {
    const int st = s % kFStages;
    const uint32_t bar = smem_addr(&sm.full[st]);
    const uint32_t wbytes = fused_w_bytes(s);
    const bool feat = s < kFIn / BK;
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar),
                 "r"(wbytes + (feat ? kFXBytes : 0u))
                 : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(sm.b[st])),
                 "l"(reinterpret_cast<const char*>(g.Wt) + fused_w_off(s)), "r"(wbytes), "r"(bar)
                 : "memory");
    if (feat && with_x) fused_load_x(g, sm, s, tile);
}

// 32 accumulator columns of this thread's row (TMEM lane) starting at column c
__device__ __forceinline__ void fused_tmem_ld32(uint32_t lane_base, int c, float* v) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(lane_base + (uint32_t)c));
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(lane_base + (uint32_t)(c + 16)));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
}

// 16 accumulator columns of this thread's row (TMEM lane) starting at column c
__device__ __forceinline__ void fused_tmem_ld16(uint32_t lane_base, int c, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(lane_base + (uint32_t)c));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
}

// Epilogue of hidden layer l from accumulator acc: bias + GELU -> bf16 rows
// into the activation buffer (K-major tiles of 64 columns), k-block by
// k-block. Each thread takes one row (its TMEM lane) and 16 columns of every
// k-block (warp w / 4 picks which), then releases the k-block to the next
// layer's MMAs on kready[kb] (also when `ok` is false and nothing was
// written: the arrivals keep the barrier's count).
__device__ __forceinline__ void fused_hidden_epilogue(const FusedArgs& g, FusedSmem& sm, int l, uint32_t acc,
                                                      bool ok) {
    const int t = threadIdx.x, warp = t >> 5, quarter = warp & 3, sub = warp >> 2;
    const int row = quarter * 32 + (t & 31);
    const uint32_t lane_base = acc + ((uint32_t)(quarter * 32) << 16);
    const float* bias = sm.bias + l * kFHid;
#pragma unroll 1
    for (int kb = 0; kb < kFHid / BK; ++kb) {
        if (ok) {
            const int c0 = kb * BK + sub * 16;
            float v[16];
            fused_tmem_ld16(lane_base, c0, v);   // warp-collective: every lane takes part
            uint32_t pk[8];
#pragma unroll
            for (int h = 0; h < 8; ++h) {
                const __nv_bfloat162 p2 = __floats2bfloat162_rn(gelu(v[2 * h] + bias[c0 + 2 * h]),
                                                                gelu(v[2 * h + 1] + bias[c0 + 2 * h + 1]));
                pk[h] = *reinterpret_cast<const uint32_t*>(&p2);
            }
            const uint32_t dst = smem_addr(sm.h[kb]) + tile_off(row, sub * 2);
            asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(dst), "r"(pk[0]), "r"(pk[1]), "r"(pk[2]),
                         "r"(pk[3])
                         : "memory");
            asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(dst + 128u), "r"(pk[4]), "r"(pk[5]),
                         "r"(pk[6]), "r"(pk[7])
                         : "memory");
            // generic-proxy writes of the activations -> visible to the MMAs
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        }
        // this thread's accumulator reads are complete before the k-block's release
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(&sm.kready[kb])) : "memory");
    }
}

// Epilogue of output pass p: rhs[var][row*64 + point] += scale[var] * (C + bias)
// for the columns var*64 + point of this pass. Each thread owns one row (its
// TMEM lane) and 32 consecutive columns, 32 consecutive RHS values: eight
// 16-byte vector reductions, one contribution per RHS value (the same
// rounding as load + add + store, without the load's round trip), and no
// staging tile, so that the shared memory holds four weight stages.
__device__ __forceinline__ void fused_out_epilogue(const FusedArgs& g, FusedSmem& sm, int pass, uint32_t tmem,
                                                   int m0) {
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31, quarter = warp & 3, grp = warp >> 2;
    const uint32_t lane_base = tmem + ((uint32_t)(quarter * 32) << 16);
    const int row = m0 + quarter * 32 + lane;
#pragma unroll 1
    for (int c0 = grp * 32; c0 < kFPass; c0 += 32 * kFGroups) {   // 32-column chunks, round robin over the groups
        float v[32];
        fused_tmem_ld32(lane_base, c0, v);   // warp-collective: every lane takes part
        const int n = pass * kFPass + c0;    // 32 columns inside one variable's 64-point block
        const int var = n >> 6;
        const float sc = var == 0 ? g.rhs_scale[0] : var == 1 ? g.rhs_scale[1] : var == 2 ? g.rhs_scale[2]
                       : var == 3 ? g.rhs_scale[3] : g.rhs_scale[4];
        if (row >= g.rhs_rows) continue;
        float* base = g.rhs + (size_t)var * g.rhs_npts + (size_t)row * 64 + (n & 63);
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const float a0 = sc * (v[4 * q] + sm.bias[3 * kFHid + n + 4 * q]);
            const float a1 = sc * (v[4 * q + 1] + sm.bias[3 * kFHid + n + 4 * q + 1]);
            const float a2 = sc * (v[4 * q + 2] + sm.bias[3 * kFHid + n + 4 * q + 2]);
            const float a3 = sc * (v[4 * q + 3] + sm.bias[3 * kFHid + n + 4 * q + 3]);
            asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(base + 4 * q), "f"(a0), "f"(a1),
                         "f"(a2), "f"(a3)
                         : "memory");
        }
    }
}

// Records a failed wait: the CTA's flag and the caller's error word.
__device__ __forceinline__ void fused_fail(const FusedArgs& g, FusedSmem& sm) {
    *(volatile int*)&sm.failed = 1;
    if (g.err) atomicExch(g.err, 1);
}

__device__ __forceinline__ bool fused_failed(FusedSmem& sm) { return *(volatile int*)&sm.failed != 0; }

// Load warp (its lane 0): the bulk copies of every step, kFStages steps ahead
// of the MMAs. Step s reuses the stage of step s - kFStages once that step's
// MMAs are complete (its `bar` commit).
__device__ __forceinline__ void fused_loader(const FusedArgs& g, FusedSmem& sm) {
    int issued = 0;
    // The weights and biases do not depend on the kernel launched before this
    // one (phase A or the features kernel, which may let this kernel start
    // early): the first weight tiles are requested before waiting for it, the
    // features after.
    for (int i = 0; i < kFStages; ++i) {
        fused_load(g, sm, i, blockIdx.x, false);
        ++issued;
    }
    asm volatile("griddepcontrol.wait;" ::: "memory");
    for (int i = 0; i < kFStages; ++i) fused_load_x(g, sm, i, blockIdx.x);
    for (int s = kFStages; s < kFSteps && !fused_failed(sm); ++s) {
        if (!mbar_wait(smem_addr(&sm.bar[s % kFStages]), (uint32_t)((s / kFStages - 1) & 1))) {
            fused_fail(g, sm);
            break;
        }
        fused_load(g, sm, s, blockIdx.x);
        ++issued;
    }
    // before the CTA frees its memory no copy may still be writing it: wait
    // for the last fill of every stage (they have landed already unless a
    // wait failed)
    for (int s = issued - kFStages; s < issued; ++s)
        if (s >= 0 && !mbar_wait(smem_addr(&sm.full[s % kFStages]), (uint32_t)((s / kFStages) & 1)))
            fused_fail(g, sm);
}

// MMA warp (its lane 0): the tcgen05.mma of every step in step order. A
// hidden layer's or output pass's step kb waits for k-block kb of the layer
// before (kready); every step waits for its stage (full). Each step's MMAs
// are committed to the stage's `bar` (stage free) and a layer's last ones
// also to `done` (accumulator complete).
__device__ __forceinline__ void fused_mma(const FusedArgs& g, FusedSmem& sm, uint32_t tmem) {
    int last_mma = -1;   // last step whose MMAs were issued
    for (int s = 0; s < kFSteps && !fused_failed(sm); ++s) {
        const FStep f = fused_step(s);
        const int u = fused_unit(f);
        const int st = s % kFStages;
        if (u >= 1 && u <= 3) {
            // k-block f.kb of hidden layer u - 1's output (its completion u - 1)
            if (!mbar_wait(smem_addr(&sm.kready[f.kb]), (uint32_t)((u - 1) & 1))) {
                fused_fail(g, sm);
                break;
            }
        }
        if (!mbar_wait(smem_addr(&sm.full[st]), (uint32_t)((s / kFStages) & 1))) {
            fused_fail(g, sm);
            break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const int n = f.layer == 3 ? kFPass : kFHid;
        const uint32_t idesc = instr_desc(BM, n);
        const uint32_t acc = tmem + (uint32_t)((u & 1) * kFHid);
        const uint32_t a0 = smem_addr(sm.h[f.layer == 0 ? st : f.kb]);
        const uint32_t b0 = smem_addr(sm.b[st]);
#pragma unroll
        for (int k = 0; k < BK / 16; ++k) {
            const uint64_t ad = smem_desc(a0 + k * 256, 128, 1024);
            const uint64_t bd = smem_desc(b0 + k * 256, 128, 1024);
            const uint32_t accumulate = (f.kb > 0 || k > 0) ? 1u : 0u;
            asm volatile(
                "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}" ::"r"(acc),
                "l"(ad), "l"(bd), "r"(idesc), "r"(accumulate)
                : "memory");
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         smem_addr(&sm.bar[st]))
                     : "memory");
        last_mma = s;
        if (s + 1 == kFSteps || fused_step(s + 1).kb == 0)
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_addr(&sm.done[u & 1]))
                         : "memory");
    }
    // no MMA may still be running when the CTA frees its tensor memory (only
    // after a failed wait has no epilogue waited for the last ones)
    if (last_mma >= 0 &&
        !mbar_wait(smem_addr(&sm.bar[last_mma % kFStages]), (uint32_t)((last_mma / kFStages) & 1)))
        fused_fail(g, sm);
}

__global__ void __launch_bounds__(kFThreads, 1) mlp_fused_kernel(const FusedArgs g) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    FusedSmem& sm = *reinterpret_cast<FusedSmem*>(smem_raw + ((1024 - (smem_addr(smem_raw) & 1023)) & 1023));
    const int t = threadIdx.x, warp = t >> 5;
    const int m0 = blockIdx.x * BM;
    constexpr uint32_t kCols = 2 * kFHid;   // two accumulators

    if (t == 0) {
        for (int i = 0; i < kFStages; ++i) {
            mbar_init(smem_addr(&sm.bar[i]), 1);
            mbar_init(smem_addr(&sm.full[i]), 1);
        }
        for (int i = 0; i < 2; ++i) mbar_init(smem_addr(&sm.done[i]), 1);
        for (int i = 0; i < kFHid / BK; ++i) mbar_init(smem_addr(&sm.kready[i]), kFEpiThreads);
        sm.failed = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&sm.tmem_base)),
                     "r"(kCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    for (int i = t; i < 3 * kFHid + kFOut; i += kFThreads)
        sm.bias[i] = i < kFHid ? g.bias[0][i] : i < 2 * kFHid ? g.bias[1][i - kFHid]
                   : i < 3 * kFHid ? g.bias[2][i - 2 * kFHid] : g.bias[3][i - 3 * kFHid];
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = sm.tmem_base;

    if (warp == kFEpiThreads / 32) {
        if ((t & 31) == 0) fused_mma(g, sm, tmem);
        __syncwarp();
    } else if (warp == kFEpiThreads / 32 + 1) {
        if ((t & 31) == 0) fused_loader(g, sm);
        __syncwarp();
    } else {
        // the RHS the output epilogues add to is written by the kernel before
        asm volatile("griddepcontrol.wait;" ::: "memory");
        for (int u = 0; u < kFUnits; ++u) {
            bool ok = !fused_failed(sm);
            if (ok && !mbar_wait(smem_addr(&sm.done[u & 1]), (uint32_t)((u >> 1) & 1))) {
                fused_fail(g, sm);
                ok = false;
            }
            ok = __all_sync(0xffffffffu, ok);   // tcgen05.ld is warp-collective
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t acc = tmem + (uint32_t)((u & 1) * kFHid);
            if (u < 3)
                fused_hidden_epilogue(g, sm, u, acc, ok);
            else if (ok)
                fused_out_epilogue(g, sm, u - 3, acc, m0);
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols) : "memory");
    }
}

}  // namespace mlp
}  // namespace od
