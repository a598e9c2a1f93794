// Closure network kernels: the tcgen05 GEMM launcher and the small
// element-wise kernels of MLP training (bf16 conversion, transposes, the
// loss gradient, bias gradients, Adam).

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "../../include/opendynamo.h"
#include "od_mlp.cuh"

namespace od {
namespace mlp {

template <int NT, int EPI>
cudaError_t launch_gemm_t(const GemmArgs& g, cudaStream_t s) {
    const size_t smem = gemm_smem_bytes<NT>();
    cudaError_t e = cudaFuncSetAttribute(gemm_kernel<NT, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    dim3 grid((unsigned)(g.M / BM), (unsigned)(g.N / NT));
    gemm_kernel<NT, EPI><<<grid, 128, smem, s>>>(g);
    return cudaGetLastError();
}

// C = A B^T with the epilogue `epi`; M % 128 == 0, N % 128 == 0, K % 64 == 0.
cudaError_t launch_gemm(const GemmArgs& g, int epi, cudaStream_t s) {
    if (g.M <= 0 || g.N <= 0 || g.K <= 0 || g.M % BM || g.N % 128 || g.K % BK) return cudaErrorInvalidValue;
    const bool wide = g.N % 256 == 0;
    switch (epi) {
        case kStoreF32: return wide ? launch_gemm_t<256, kStoreF32>(g, s) : launch_gemm_t<128, kStoreF32>(g, s);
        case kBiasGelu: return wide ? launch_gemm_t<256, kBiasGelu>(g, s) : launch_gemm_t<128, kBiasGelu>(g, s);
        case kGeluGrad: return wide ? launch_gemm_t<256, kGeluGrad>(g, s) : launch_gemm_t<128, kGeluGrad>(g, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace mlp
}  // namespace od

extern "C" int od_gemm_bf16(int M, int N, int K, const void* dA, const void* dB, float* dC, const float* dbias,
                            void* stream) {
    if (!dA || !dB || !dC) return OD_ERR_ARG;
    if (M <= 0 || N <= 0 || K <= 0 || M % 128 || N % 128 || K % 64) return OD_ERR_ARG;
    int* err = nullptr;
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = cudaMallocAsync((void**)&err, sizeof(int), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(err, 0, sizeof(int), s);
    od::mlp::GemmArgs g{};
    g.A = (const __nv_bfloat16*)dA;
    g.B = (const __nv_bfloat16*)dB;
    g.M = M;
    g.N = N;
    g.K = K;
    g.bias = dbias;
    g.out_f32 = dC;
    g.err = err;
    if (e == cudaSuccess) e = od::mlp::launch_gemm(g, od::mlp::kStoreF32, s);
    int herr = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (err) cudaFreeAsync(err, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return OD_ERR_CUDA;
    return herr ? OD_ERR_CUDA : OD_OK;
}
