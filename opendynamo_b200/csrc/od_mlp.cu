// Closure network kernels: the tcgen05 GEMM launcher and the small
// element-wise kernels of MLP training (bf16 conversion, transposes, the
// loss gradient, bias gradients, Adam).

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "../../include/opendynamo.h"
#include "od_mlp.cuh"
#include "od_mlp_fused.cuh"

namespace od {
namespace mlp {

constexpr long long kSMs = 148;  // B200

// out = sum of the ksplit partial tiles (+ bias)
__global__ void splitk_reduce_kernel(const float* __restrict__ ws, int ks, long long mn, int N,
                                     const float* __restrict__ bias, float* __restrict__ out) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= mn) return;
    float v = 0.f;
    for (int z = 0; z < ks; ++z) v += ws[z * mn + i];
    if (bias) v += bias[i % N];
    out[i] = v;
}

template <int NT, int EPI>
cudaError_t launch_gemm_t(const GemmArgs& g, cudaStream_t s) {
    const size_t smem = gemm_smem_bytes<NT>();
    // the shared-memory limit is set once per device (a host call per launch
    // cost more than the small GEMMs themselves)
    static bool prepared[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!prepared[dev]) {
        e = cudaFuncSetAttribute(gemm_kernel<NT, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        prepared[dev] = true;
    }
    const int ks = g.ksplit > 1 ? g.ksplit : 1;
    dim3 grid((unsigned)(g.M / BM), (unsigned)(g.N / NT), (unsigned)ks);
    gemm_kernel<NT, EPI><<<grid, 128, smem, s>>>(g);
    e = cudaGetLastError();
    if (e == cudaSuccess && ks > 1) {
        const long long mn = (long long)g.M * g.N;
        splitk_reduce_kernel<<<(unsigned)((mn + 255) / 256), 256, 0, s>>>(g.ws, ks, mn, g.N, g.bias, g.out_f32);
        e = cudaGetLastError();
    }
    return e;
}

template <int EPI>
cudaError_t launch_nt(const GemmArgs& g, int nt, cudaStream_t s) {
    if (nt == 256) return launch_gemm_t<256, EPI>(g, s);
    if (nt == 128) return launch_gemm_t<128, EPI>(g, s);
    return launch_gemm_t<64, EPI>(g, s);
}

// C = A B^T with the epilogue `epi`; M % 128 == 0, N % 64 == 0, K % 64 == 0.
// Tile width: the widest of 256 / 128 / 64 dividing N that still gives two
// CTAs per SM (the epilogue has four warps per CTA and wants company),
// else 64. kStoreF32 products with few tiles and a long K (weight gradients)
// split K when the caller passes a workspace of ksplit * M * N floats.
cudaError_t launch_gemm(const GemmArgs& g0, int epi, cudaStream_t s, size_t ws_floats) {
    if (g0.M <= 0 || g0.N <= 0 || g0.K <= 0 || g0.M % BM || g0.N % 64 || g0.K % BK) return cudaErrorInvalidValue;
    GemmArgs g = g0;
    const long long rows = g.M / BM;
    int nt = 64;
    for (int c : {256, 128}) {
        if (g.N % c == 0 && rows * (g.N / c) >= 2 * kSMs) {
            nt = c;
            break;
        }
    }
    g.ksplit = 1;
    if (epi == kStoreF32 && g.ws) {
        const long long tiles = rows * (g.N / nt);
        const int kblocks = g.K / BK;
        int ks = 1;
        while (tiles * ks < 2 * kSMs && kblocks % (2 * ks) == 0 && kblocks / (2 * ks) >= 2 &&
               (size_t)(2 * ks) * g.M * g.N <= ws_floats)
            ks *= 2;
        g.ksplit = ks;
    }
    switch (epi) {
        case kStoreF32: return launch_nt<kStoreF32>(g, nt, s);
        case kBiasGelu: return launch_nt<kBiasGelu>(g, nt, s);
        case kGeluGrad: return launch_nt<kGeluGrad>(g, nt, s);
        case kApplyRhs: return launch_nt<kApplyRhs>(g, nt, s);
        default: return cudaErrorInvalidValue;
    }
}

__global__ void tile_fused_weights_kernel(const __nv_bfloat16* __restrict__ W0, const __nv_bfloat16* __restrict__ W1,
                                          const __nv_bfloat16* __restrict__ W2, const __nv_bfloat16* __restrict__ W3,
                                          __nv_bfloat16* __restrict__ Wt) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;   // 16-byte chunk of the image
    if (q >= kFusedWeightBytes / 16) return;
    const uint32_t byte = q * 16;
    int s;
    uint32_t within;
    if (byte < 22u * kFStageBytes) {
        s = (int)(byte / kFStageBytes);
        within = byte % kFStageBytes;
    } else {
        s = 22 + (int)((byte - 22u * kFStageBytes) / kFOutStageBytes);
        within = (byte - 22u * kFStageBytes) % kFOutStageBytes;
    }
    const FStep f = fused_step(s);
    const int r = (int)(within / 1024) * 8 + (int)(within % 128) / 16;   // inverse of tile_off
    const int kc = (int)(within % 1024) / 128;
    const int K = f.layer == 0 ? kFIn : kFHid;
    const int n0 = f.layer == 3 ? f.pass * kFPass : 0;
    const __nv_bfloat16* W = f.layer == 0 ? W0 : f.layer == 1 ? W1 : f.layer == 2 ? W2 : W3;
    *reinterpret_cast<uint4*>(reinterpret_cast<char*>(Wt) + byte) =
        *reinterpret_cast<const uint4*>(W + (size_t)(n0 + r) * K + f.kb * BK + kc * 8);
}

cudaError_t tile_fused_weights(const __nv_bfloat16* const W[4], __nv_bfloat16* Wt, cudaStream_t s) {
    constexpr unsigned n = (unsigned)(kFusedWeightBytes / 16);
    tile_fused_weights_kernel<<<(n + 255) / 256, 256, 0, s>>>(W[0], W[1], W[2], W[3], Wt);
    return cudaGetLastError();
}

cudaError_t launch_fused(const FusedArgs& a, int M, cudaStream_t s) {
    if (M <= 0 || M % BM) return cudaErrorInvalidValue;
    static bool prepared[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!prepared[dev]) {
        e = cudaFuncSetAttribute(mlp_fused_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fused_smem_bytes());
        if (e != cudaSuccess) return e;
        prepared[dev] = true;
    }
    // programmatic dependent launch: the prologue and the first weight copies
    // overlap the tail of the kernel before (griddepcontrol.wait in the kernel
    // orders everything that reads its results)
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)(M / BM));
    cfg.blockDim = dim3(kFThreads);
    cfg.dynamicSmemBytes = fused_smem_bytes();
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, mlp_fused_kernel, a);
}

// Self-test of the bounded mbarrier wait of the tcgen05 kernels: a barrier
// nothing arrives on must give up after `limit` polls; after one arrival the
// same wait completes. out[0] = first wait completed, out[1] = second.
__global__ void mbar_wait_selftest_kernel(long long limit, int* out) {
    __shared__ __align__(8) unsigned long long bar;
    if (threadIdx.x != 0) return;
    const uint32_t b = smem_addr(&bar);
    mbar_init(b, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    const bool first = mbar_wait(b, 0, limit);
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(b) : "memory");
    const bool second = mbar_wait(b, 0, limit);
    out[0] = first ? 1 : 0;
    out[1] = second ? 1 : 0;
}

}  // namespace mlp
}  // namespace od

extern "C" int od_mlp_wait_selftest(long long limit, int device, int* first_completed, int* second_completed) {
    if (limit <= 0 || !first_completed || !second_completed) return OD_ERR_ARG;
    int prev = 0;
    if (cudaGetDevice(&prev) != cudaSuccess || cudaSetDevice(device) != cudaSuccess) return OD_ERR_CUDA;
    int* d = nullptr;
    int h[2] = {-1, -1};
    cudaError_t e = cudaMalloc((void**)&d, 2 * sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(d, 0xff, 2 * sizeof(int));
    if (e == cudaSuccess) {
        od::mlp::mbar_wait_selftest_kernel<<<1, 32>>>(limit, d);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(h, d, sizeof h, cudaMemcpyDeviceToHost);
    if (d) cudaFree(d);
    cudaSetDevice(prev);
    if (e != cudaSuccess) return OD_ERR_CUDA;
    *first_completed = h[0];
    *second_completed = h[1];
    return OD_OK;
}

extern "C" int od_gemm_bf16(int M, int N, int K, const void* dA, const void* dB, float* dC, const float* dbias,
                            void* stream) {
    if (!dA || !dB || !dC) return OD_ERR_ARG;
    if (M <= 0 || N <= 0 || K <= 0 || M % 128 || N % 64 || K % 64) return OD_ERR_ARG;
    int* err = nullptr;
    float* ws = nullptr;
    cudaStream_t s = (cudaStream_t)stream;
    const size_t ws_floats = (size_t)16 * M * N;
    cudaError_t e = cudaMallocAsync((void**)&err, sizeof(int), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(err, 0, sizeof(int), s);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&ws, ws_floats * sizeof(float), s);
    od::mlp::GemmArgs g{};
    g.A = (const __nv_bfloat16*)dA;
    g.B = (const __nv_bfloat16*)dB;
    g.M = M;
    g.N = N;
    g.K = K;
    g.bias = dbias;
    g.out_f32 = dC;
    g.err = err;
    g.ws = ws;
    if (e == cudaSuccess) e = od::mlp::launch_gemm(g, od::mlp::kStoreF32, s, ws_floats);
    int herr = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (err) cudaFreeAsync(err, s);
    if (ws) cudaFreeAsync(ws, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return OD_ERR_CUDA;
    return herr ? OD_ERR_CUDA : OD_OK;
}
