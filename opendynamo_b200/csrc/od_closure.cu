// Learned closure: a per-element MLP (896 -> 256 -> 256 -> 256 -> 320,
// GELU) that corrects the RHS of an under-resolved coarse run.
//
// Kernels here:
//   project   L2 projection of a fine FR P=3 state (or RHS) onto the coarse
//             P=3 basis of elements `factor` times larger per axis (exact for
//             the piecewise cubic fine field: Gauss-Legendre quadrature of the
//             fine elements, the coarse mass matrix is diagonal at the GL
//             points)
//   features  64 points x (5 conserved + 9 velocity gradients) per element,
//             standardised with per-channel constants and clipped to +-8,
//             bf16 rows
//   apply     rhs += out_scale[v] * network output (between the two phases
//             of an RK stage)
//   training  loss gradient, bias gradients, gathers and Adam
// The network's matrix products run on the tcgen05 GEMM of od_mlp.cuh.

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/opendynamo.h"
#include "od_launch.h"
#include "od_mlp.cuh"

namespace od {
TablesD host_fr_tables();
namespace mlp {
cudaError_t launch_gemm(const GemmArgs& g, int epi, cudaStream_t s, size_t ws_floats);
}
}  // namespace od

namespace {

using bf16 = __nv_bfloat16;
constexpr int kIn = 896, kHid = 256, kOut = 320, kOutPad = 384, kChan = 14;
constexpr float kClip = 8.0f;  // standardised inputs are clipped to +-kClip (states outside the training range)

// ---------------------------------------------------------------- projection
struct ProjParams {
    int nxc, nyc, nzc, f;
    float P[4][32];  // P[i][a]: coarse node i from fine sample a (a < 4 f)
};

template <class TS, class TD>
__global__ void __launch_bounds__(256) project_kernel(const TS* __restrict__ src, TD* __restrict__ dst,
                                                      ProjParams pp) {
    extern __shared__ float sh[];  // (4f)^3 fine samples, then 4 x (4f)^2, then 16 x 4f
    const int F = 4 * pp.f;
    float* u = sh;
    float* t1 = u + F * F * F;
    float* t2 = t1 + 4 * F * F;
    const long long ec = blockIdx.x;
    const int cx = (int)(ec % pp.nxc), cy = (int)((ec / pp.nxc) % pp.nyc), cz = (int)(ec / ((long long)pp.nxc * pp.nyc));
    const long long nxf = (long long)pp.nxc * pp.f, nyf = (long long)pp.nyc * pp.f, nzf = (long long)pp.nzc * pp.f;
    const long long npf = nxf * nyf * nzf * 64, npc = (long long)pp.nxc * pp.nyc * pp.nzc * 64;
    for (int v = 0; v < 5; ++v) {
        __syncthreads();
        for (int s = threadIdx.x; s < F * F * F; s += blockDim.x) {
            const int a = s % F, b = (s / F) % F, c = s / (F * F);
            const long long fe = (cx * pp.f + a / 4) + nxf * ((cy * pp.f + b / 4) + nyf * (long long)(cz * pp.f + c / 4));
            u[s] = (float)src[v * npf + fe * 64 + (a & 3) + 4 * (b & 3) + 16 * (c & 3)];
        }
        __syncthreads();
        // x: t1[i][b][c]
        for (int s = threadIdx.x; s < 4 * F * F; s += blockDim.x) {
            const int i = s & 3, bc = s >> 2;
            float acc = 0.f;
            for (int a = 0; a < F; ++a) acc += pp.P[i][a] * u[a + F * bc];
            t1[s] = acc;  // index i + 4 (b + F c)
        }
        __syncthreads();
        // y: t2[i][j][c]
        for (int s = threadIdx.x; s < 16 * F; s += blockDim.x) {
            const int i = s & 3, j = (s >> 2) & 3, c = s >> 4;
            float acc = 0.f;
            for (int b = 0; b < F; ++b) acc += pp.P[j][b] * t1[i + 4 * (b + F * c)];
            t2[s] = acc;  // index i + 4 j + 16 c
        }
        __syncthreads();
        if (threadIdx.x < 64) {
            const int i = threadIdx.x & 3, j = (threadIdx.x >> 2) & 3, k = threadIdx.x >> 4;
            float acc = 0.f;
            for (int c = 0; c < F; ++c) acc += pp.P[k][c] * t2[i + 4 * j + 16 * c];
            dst[v * npc + ec * 64 + threadIdx.x] = (TD)acc;
        }
    }
}

ProjParams proj_params(int nxc, int nyc, int nzc, int f) {
    ProjParams pp{};
    pp.nxc = nxc;
    pp.nyc = nyc;
    pp.nzc = nzc;
    pp.f = f;
    const od::TablesD t = od::host_fr_tables();
    double w[4];
    for (int a = 0; a < 4; ++a) {
        const double x = t.pts[a];
        const double p4 = (35 * x * x * x * x - 30 * x * x + 3) / 8.0, p3 = (5 * x * x * x - 3 * x) / 2.0;
        const double dp4 = 4.0 * (x * p4 - p3) / (x * x - 1.0);
        w[a] = 2.0 / ((1.0 - x * x) * dp4 * dp4);
    }
    auto lag = [&](int i, double xi) {
        double r = 1.0;
        for (int m = 0; m < 4; ++m)
            if (m != i) r *= (xi - t.pts[m]) / (t.pts[i] - t.pts[m]);
        return r;
    };
    for (int i = 0; i < 4; ++i)
        for (int a = 0; a < 4 * f; ++a) {
            const int q = a / 4, jf = a % 4;
            const double xc = -1.0 + (2.0 * q + 1.0 + t.pts[jf]) / f;
            pp.P[i][a] = (float)(w[jf] * lag(i, xc) / (f * w[i]));
        }
    return pp;
}

// ---------------------------------------------------------------- features
struct FeatParams {
    int nx, ny, nz;
    float jac[3];
    float D[16];
    float mean[kChan], inv_scale[kChan];
};

// X: row-major [element][channel * 64 + point]; a thread per point.
template <class T>
__global__ void __launch_bounds__(64) features_kernel(const T* __restrict__ u, FeatParams fp, bf16* __restrict__ X) {
    __shared__ float q[4][64];
    const long long e = blockIdx.x;
    const long long npts = (long long)fp.nx * fp.ny * fp.nz * 64;
    const int p = threadIdx.x, i = p & 3, j = (p >> 2) & 3, k = p >> 4;
    float c[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) c[v] = (float)u[v * npts + e * 64 + p];
#pragma unroll
    for (int v = 0; v < 4; ++v) q[v][p] = c[v];
    __syncthreads();
    float d[4][3];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        float sx = 0.f, sy = 0.f, sz = 0.f;
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            sx += fp.D[i * 4 + m] * q[v][m + 4 * j + 16 * k];
            sy += fp.D[j * 4 + m] * q[v][i + 4 * m + 16 * k];
            sz += fp.D[k * 4 + m] * q[v][i + 4 * j + 16 * m];
        }
        d[v][0] = sx * fp.jac[0];
        d[v][1] = sy * fp.jac[1];
        d[v][2] = sz * fp.jac[2];
    }
    const float ir = 1.0f / c[0];
    float ch[kChan];
#pragma unroll
    for (int v = 0; v < 5; ++v) ch[v] = c[v];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) ch[5 + 3 * a + b] = (d[1 + a][b] - c[1 + a] * ir * d[0][b]) * ir;
    bf16* row = X + e * kIn + p;
#pragma unroll
    for (int ch_i = 0; ch_i < kChan; ++ch_i)
        row[ch_i * 64] = __float2bfloat16_rn(fminf(fmaxf((ch[ch_i] - fp.mean[ch_i]) * fp.inv_scale[ch_i], -kClip),
                                                   kClip));
}

// The same features for the fused inference kernel, written in its layout:
// per 128-element tile, per channel (one 64-wide K block) the 128 x 64 block
// in the shared-memory core-matrix layout, so that one bulk copy fills a
// feature stage. f32 state. 16 threads per element, 4 elements per block:
// thread l owns the x-line (j, k) = (l & 3, l >> 2) of its element, takes the
// x derivatives of its four points in registers and the y / z derivatives
// from the four x-lines of its k-plane / j-column in shared memory (128-bit
// loads), in the same operation order as features_kernel. The channels are
// staged in shared memory and stored as 16-byte chunks.
constexpr int kFeatEpb = 4;

__global__ void __launch_bounds__(16 * kFeatEpb) features_tiled_kernel(const float* __restrict__ u, FeatParams fp,
                                                                        bf16* __restrict__ X, long long nelem) {
    __shared__ __align__(16) float q[kFeatEpb][4][64];
    __shared__ __align__(16) bf16 st[kFeatEpb][kChan][64];
    // the fused inference kernel that follows may start its prologue now
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    const int es = threadIdx.x >> 4, l = threadIdx.x & 15, j = l & 3, k = l >> 2;
    const long long e = (long long)blockIdx.x * kFeatEpb + es;
    const bool live = e < nelem;
    const long long ec = live ? e : 0;
    const long long npts = (long long)fp.nx * fp.ny * fp.nz * 64;
    float c[5][4];
#pragma unroll
    for (int v = 0; v < 5; ++v) {
        const float4 w = __ldg(reinterpret_cast<const float4*>(u + v * npts + ec * 64 + 4 * l));
        c[v][0] = w.x;
        c[v][1] = w.y;
        c[v][2] = w.z;
        c[v][3] = w.w;
        if (v < 4) *reinterpret_cast<float4*>(&q[es][v][4 * l]) = w;
    }
    __syncthreads();
    float d[4][3][4];   // [var][direction][point of the line]
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        float ly[4][4], lz[4][4];   // the x-lines (m, k) and (j, m), m = 0..3
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            const float4 a = *reinterpret_cast<const float4*>(&q[es][v][4 * (m + 4 * k)]);
            const float4 b = *reinterpret_cast<const float4*>(&q[es][v][4 * (j + 4 * m)]);
            ly[m][0] = a.x; ly[m][1] = a.y; ly[m][2] = a.z; ly[m][3] = a.w;
            lz[m][0] = b.x; lz[m][1] = b.y; lz[m][2] = b.z; lz[m][3] = b.w;
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            float sx = 0.f, sy = 0.f, sz = 0.f;
#pragma unroll
            for (int m = 0; m < 4; ++m) {
                sx += fp.D[i * 4 + m] * c[v][m];
                sy += fp.D[j * 4 + m] * ly[m][i];
                sz += fp.D[k * 4 + m] * lz[m][i];
            }
            d[v][0][i] = sx * fp.jac[0];
            d[v][1][i] = sy * fp.jac[1];
            d[v][2][i] = sz * fp.jac[2];
        }
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int p = i + 4 * l;
        const float ir = 1.0f / c[0][i];
        float ch[kChan];
#pragma unroll
        for (int v = 0; v < 5; ++v) ch[v] = c[v][i];
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) ch[5 + 3 * a + b] = (d[1 + a][b][i] - c[1 + a][i] * ir * d[0][b][i]) * ir;
#pragma unroll
        for (int ch_i = 0; ch_i < kChan; ++ch_i)
            st[es][ch_i][p] = __float2bfloat16_rn(fminf(fmaxf((ch[ch_i] - fp.mean[ch_i]) * fp.inv_scale[ch_i], -kClip),
                                                        kClip));
    }
    __syncthreads();
    if (!live) return;
    bf16* tile = X + (e >> 7) * (128 * kIn);
    for (int q8 = l; q8 < kChan * 8; q8 += 16) {
        const int ch_i = q8 >> 3, kc = q8 & 7;
        *reinterpret_cast<uint4*>(tile + ch_i * (128 * 64) + od::mlp::tile_off((int)(e & 127), kc) / 2) =
            *reinterpret_cast<const uint4*>(&st[es][ch_i][8 * kc]);
    }
}

FeatParams feat_params(int nx, int ny, int nz, double lx, double ly, double lz, const float* mean,
                       const float* scale) {
    FeatParams fp{};
    fp.nx = nx;
    fp.ny = ny;
    fp.nz = nz;
    fp.jac[0] = (float)(2.0 * nx / lx);
    fp.jac[1] = (float)(2.0 * ny / ly);
    fp.jac[2] = (float)(2.0 * nz / lz);
    const od::TablesD t = od::host_fr_tables();
    for (int a = 0; a < 16; ++a) fp.D[a] = (float)t.D[a];
    for (int c = 0; c < kChan; ++c) {
        fp.mean[c] = mean ? mean[c] : 0.f;
        fp.inv_scale[c] = scale ? 1.0f / scale[c] : 1.f;
    }
    return fp;
}

// rhs[v][e*64+p] += scale[v] * Y[e][v*64+p]
template <class T>
__global__ void apply_kernel(T* __restrict__ rhs, const float* __restrict__ Y, long long nelem, float s0, float s1,
                             float s2, float s3, float s4) {
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long npts = nelem * 64;
    if (idx >= npts * 5) return;
    const int v = (int)(idx / npts);
    const long long r = idx - v * npts;
    const long long e = r >> 6;
    const int p = (int)(r & 63);
    const float sc = v == 0 ? s0 : v == 1 ? s1 : v == 2 ? s2 : v == 3 ? s3 : s4;
    rhs[idx] = (T)((float)rhs[idx] + sc * Y[e * kOutPad + v * 64 + p]);
}

// ---------------------------------------------------------------- training kernels
// dY = g (Y - T) on the valid block (rows < mv, columns < kOut), 0 elsewhere;
// bf16 [M x 384] and its transpose; loss += sum (Y - T)^2
__global__ void loss_grad_kernel(const float* __restrict__ Y, const float* __restrict__ T, int M, int mv, float g,
                                 bf16* __restrict__ dY, bf16* __restrict__ dYT, double* loss) {
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    float sq = 0.f;
    if (idx < (long long)M * kOutPad) {
        const int m = (int)(idx / kOutPad), n = (int)(idx % kOutPad);
        float d = 0.f;
        if (m < mv && n < kOut) {
            const float r = Y[idx] - T[idx];
            d = g * r;
            sq = r * r;
        }
        const bf16 b = __float2bfloat16_rn(d);
        dY[idx] = b;
        dYT[(long long)n * M + m] = b;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sq += __shfl_down_sync(0xffffffffu, sq, o);
    if ((threadIdx.x & 31) == 0 && sq != 0.f) atomicAdd(loss, (double)sq);
}

// out[n] = sum_m AT[n][m] (bf16 -> fp32): bias gradients from the transposed
// copies, one block per row, coalesced
__global__ void __launch_bounds__(256) rowsum_kernel(const bf16* __restrict__ AT, int M, float* __restrict__ out) {
    __shared__ float red[8];
    const bf16* row = AT + (long long)blockIdx.x * M;
    float s = 0.f;
    for (int m = threadIdx.x; m < M; m += blockDim.x) s += __bfloat162float(row[m]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.f;
        for (int w = 0; w < 8; ++w) t += red[w];
        out[blockIdx.x] = t;
    }
}

// rows of a bf16 pool (and a bf16 target pool) into a batch: X [M x 896], X^T, T [M x 384] fp32
__global__ void gather_kernel(const bf16* __restrict__ Xp, const bf16* __restrict__ Tp, const long long* __restrict__ rows,
                              int mv, int M, bf16* __restrict__ X, bf16* __restrict__ XT, float* __restrict__ T) {
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx < (long long)M * kIn) {
        const int m = (int)(idx / kIn), c = (int)(idx % kIn);
        const bf16 v = m < mv ? Xp[rows[m] * kIn + c] : __float2bfloat16_rn(0.f);
        X[idx] = v;
        XT[(long long)c * M + m] = v;
    }
    if (idx < (long long)M * kOutPad) {
        const int m = (int)(idx / kOutPad), c = (int)(idx % kOutPad);
        T[idx] = (m < mv && c < kOut) ? __bfloat162float(Tp[rows[m] * kOut + c]) : 0.f;
    }
}

// Adam on fp32 master weights, then the bf16 copies (W and W^T) of the layer
__global__ void adam_kernel(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m1,
                            float* __restrict__ m2, long long n, float lr, float b1, float b2, float eps, float c1,
                            float c2, int rows, int cols, bf16* __restrict__ wb, bf16* __restrict__ wbT) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float a = b1 * m1[i] + (1.f - b1) * gi;
    const float b = b2 * m2[i] + (1.f - b2) * gi * gi;
    m1[i] = a;
    m2[i] = b;
    const float wn = w[i] - lr * (a / c1) / (sqrtf(b / c2) + eps);
    w[i] = wn;
    if (wb) {
        const bf16 h = __float2bfloat16_rn(wn);
        wb[i] = h;
        const int r = (int)(i / cols), c = (int)(i % cols);
        wbT[(long long)c * rows + r] = h;
    }
}

// bf16 copies of all layers from the fp32 master weights
__global__ void cast_weights_kernel(const float* __restrict__ w, long long n, int rows, int cols,
                                    bf16* __restrict__ wb, bf16* __restrict__ wbT) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const bf16 h = __float2bfloat16_rn(w[i]);
    wb[i] = h;
    const int r = (int)(i / cols), c = (int)(i % cols);
    wbT[(long long)c * rows + r] = h;
}

__global__ void f32_to_bf16_kernel(const float* __restrict__ a, bf16* __restrict__ b, long long n) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = __float2bfloat16_rn(a[i]);
}

unsigned blocks(long long n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

// ------------------------------------------------------------------ network
struct od_mlp {
    int device = 0;
    int mmax = 0;                    // batch capacity (rows, multiple of 128)
    cudaStream_t stream = nullptr;
    // parameters: fp32 master, Adam moments, gradients (same flat layout)
    float *w = nullptr, *m1 = nullptr, *m2 = nullptr, *g = nullptr;
    long long nparam = 0;
    long long off_w[4], off_b[4];
    int rows[4], cols[4];
    bf16 *wb[4] = {}, *wbT[4] = {};
    bf16* wt = nullptr;   // the fused inference kernel's weight image (refreshed with wb)
    // activations
    float* Z[3] = {};
    bf16 *A[3] = {}, *AT[3] = {};
    float* Y = nullptr;
    bf16 *dY = nullptr, *dYT = nullptr;
    bf16 *dZa = nullptr, *dZaT = nullptr, *dZb = nullptr, *dZbT = nullptr;
    bf16 *X = nullptr, *XT = nullptr;   // gathered batch (training)
    float* T = nullptr;
    long long* rows_d = nullptr;
    double* loss = nullptr;
    int* err = nullptr;
    float* ws = nullptr;            // split-K partial sums of the weight gradients
    size_t ws_floats = 0;
    long long step = 0;
    std::string msg;
    // closure attachment (features of the coarse state + output scaling)
    float mean[kChan], scale[kChan], out_scale[5];
    bool fused = true;       // inference as one kernel (mlp_fused_kernel) on an f32 state
    bf16* Xc = nullptr;      // features of the attached solver's elements
    float* Yc = nullptr;
    long long nelem_c = 0, mpad_c = 0;
    FeatParams fp{};
    bool attached_f64 = false;
};

namespace {

int mfail(od_mlp* m, int code, const std::string& s) {
    if (m) m->msg = s;
    return code;
}

cudaError_t gemm(od_mlp* m, const bf16* A, const bf16* B, int M, int N, int K, int epi, const float* bias,
                 float* of32, bf16* obf, bf16* obfT, const float* zin) {
    od::mlp::GemmArgs a{};
    a.A = A;
    a.B = B;
    a.M = M;
    a.N = N;
    a.K = K;
    a.bias = bias;
    a.out_f32 = of32;
    a.out_bf = obf;
    a.out_bfT = obfT;
    a.z_in = zin;
    a.err = m->err;
    a.ws = m->ws;
    return od::mlp::launch_gemm(a, epi, m->stream, m->ws_floats);
}

// hidden layers of M rows of X (bf16 [M x 896]); training keeps the
// pre-activations and the transposed activations
cudaError_t hidden(od_mlp* m, const bf16* X, int M, bool train) {
    cudaError_t e = cudaSuccess;
    const bf16* in = X;
    int kin = kIn;
    for (int l = 0; l < 3 && e == cudaSuccess; ++l) {
        e = gemm(m, in, m->wb[l], M, kHid, kin, od::mlp::kBiasGelu, m->w + m->off_b[l], train ? m->Z[l] : nullptr,
                 m->A[l], train ? m->AT[l] : nullptr, nullptr);
        in = m->A[l];
        kin = kHid;
    }
    return e;
}

// forward of M rows of X into Y [M x 384]
cudaError_t forward(od_mlp* m, const bf16* X, int M, float* Y, bool keep_t) {
    cudaError_t e = hidden(m, X, M, keep_t);
    if (e == cudaSuccess)
        e = gemm(m, m->A[2], m->wb[3], M, kOutPad, kHid, od::mlp::kStoreF32, m->w + m->off_b[3], Y, nullptr, nullptr,
                 nullptr);
    return e;
}

// gradients of 1/(mv*320) sum (Y - T)^2 w.r.t. all parameters into m->g
cudaError_t backward(od_mlp* m, const bf16* XT, int M, int mv) {
    cudaError_t e = cudaMemsetAsync(m->loss, 0, sizeof(double), m->stream);
    const float gs = 2.0f / ((float)mv * (float)kOut);
    loss_grad_kernel<<<blocks((long long)M * kOutPad, 256), 256, 0, m->stream>>>(m->Y, m->T, M, mv, gs, m->dY,
                                                                                    m->dYT, m->loss);
    if (e == cudaSuccess) e = cudaGetLastError();
    // layer 4
    if (e == cudaSuccess)
        e = gemm(m, m->dYT, m->AT[2], kOutPad, kHid, M, od::mlp::kStoreF32, nullptr, m->g + m->off_w[3], nullptr,
                 nullptr, nullptr);
    rowsum_kernel<<<kOutPad, 256, 0, m->stream>>>(m->dYT, M, m->g + m->off_b[3]);
    if (e == cudaSuccess)
        e = gemm(m, m->dY, m->wbT[3], M, kHid, kOutPad, od::mlp::kGeluGrad, nullptr, nullptr, m->dZa, m->dZaT,
                 m->Z[2]);
    bf16 *dz = m->dZa, *dzT = m->dZaT, *nz = m->dZb, *nzT = m->dZbT;
    for (int l = 2; l >= 0 && e == cudaSuccess; --l) {
        // weights of layer l: input is A[l-1] (or X for l = 0)
        const bf16* inT = l == 0 ? XT : m->AT[l - 1];
        const int kin = l == 0 ? kIn : kHid;
        e = gemm(m, dzT, inT, kHid, kin, M, od::mlp::kStoreF32, nullptr, m->g + m->off_w[l], nullptr, nullptr,
                 nullptr);
        rowsum_kernel<<<kHid, 256, 0, m->stream>>>(dzT, M, m->g + m->off_b[l]);
        if (e == cudaSuccess && l > 0) {
            e = gemm(m, dz, m->wbT[l], M, kHid, kHid, od::mlp::kGeluGrad, nullptr, nullptr, nz, nzT, m->Z[l - 1]);
            std::swap(dz, nz);
            std::swap(dzT, nzT);
        }
    }
    if (e == cudaSuccess) e = cudaGetLastError();
    return e;
}

int check_err(od_mlp* m) {
    int h = 0;
    cudaError_t e = cudaMemcpyAsync(&h, m->err, sizeof(int), cudaMemcpyDeviceToHost, m->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(m->stream);
    if (e != cudaSuccess) return mfail(m, OD_ERR_CUDA, cudaGetErrorString(e));
    if (h) return mfail(m, OD_ERR_CUDA, "tensor-core GEMM wait timed out");
    return OD_OK;
}

}  // namespace

extern "C" {

int od_mlp_create(int max_rows, int device, od_mlp** out) {
    if (!out || max_rows <= 0) return OD_ERR_ARG;
    *out = nullptr;
    od_mlp* m = new od_mlp();
    m->device = device;
    m->mmax = (max_rows + 127) / 128 * 128;
    const int R[4] = {kHid, kHid, kHid, kOutPad}, C[4] = {kIn, kHid, kHid, kHid};
    long long off = 0;
    for (int l = 0; l < 4; ++l) {
        m->rows[l] = R[l];
        m->cols[l] = C[l];
        m->off_w[l] = off;
        off += (long long)R[l] * C[l];
        m->off_b[l] = off;
        off += R[l];
    }
    m->nparam = off;
    for (int c = 0; c < kChan; ++c) {
        m->mean[c] = 0.f;
        m->scale[c] = 1.f;
    }
    for (int v = 0; v < 5; ++v) m->out_scale[v] = 1.f;
    *out = m;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking);
    const size_t P = sizeof(float) * (size_t)m->nparam;
    const size_t M = (size_t)m->mmax;
    auto mal = [&](void** p, size_t n) {
        if (e == cudaSuccess) e = cudaMalloc(p, n);
        if (e == cudaSuccess) e = cudaMemset(*p, 0, n);
    };
    mal((void**)&m->w, P);
    mal((void**)&m->m1, P);
    mal((void**)&m->m2, P);
    mal((void**)&m->g, P);
    for (int l = 0; l < 4; ++l) {
        mal((void**)&m->wb[l], sizeof(bf16) * R[l] * C[l]);
        mal((void**)&m->wbT[l], sizeof(bf16) * R[l] * C[l]);
    }
    mal((void**)&m->wt, od::mlp::kFusedWeightBytes);
    for (int l = 0; l < 3; ++l) {
        mal((void**)&m->Z[l], sizeof(float) * M * kHid);
        mal((void**)&m->A[l], sizeof(bf16) * M * kHid);
        mal((void**)&m->AT[l], sizeof(bf16) * M * kHid);
    }
    mal((void**)&m->Y, sizeof(float) * M * kOutPad);
    mal((void**)&m->dY, sizeof(bf16) * M * kOutPad);
    mal((void**)&m->dYT, sizeof(bf16) * M * kOutPad);
    mal((void**)&m->dZa, sizeof(bf16) * M * kHid);
    mal((void**)&m->dZaT, sizeof(bf16) * M * kHid);
    mal((void**)&m->dZb, sizeof(bf16) * M * kHid);
    mal((void**)&m->dZbT, sizeof(bf16) * M * kHid);
    mal((void**)&m->X, sizeof(bf16) * M * kIn);
    mal((void**)&m->XT, sizeof(bf16) * M * kIn);
    mal((void**)&m->T, sizeof(float) * M * kOutPad);
    mal((void**)&m->rows_d, sizeof(long long) * M);
    mal((void**)&m->loss, sizeof(double));
    mal((void**)&m->err, sizeof(int));
    m->ws_floats = (size_t)32 * kOutPad * kIn;
    mal((void**)&m->ws, sizeof(float) * m->ws_floats);
    if (e != cudaSuccess) return mfail(m, OD_ERR_CUDA, std::string("od_mlp_create: ") + cudaGetErrorString(e));
    return OD_OK;
}

void od_mlp_destroy(od_mlp* m) {
    if (!m) return;
    cudaSetDevice(m->device);
    if (m->stream) cudaStreamSynchronize(m->stream);
    void* ps[] = {m->w, m->m1, m->m2, m->g, m->wb[0], m->wb[1], m->wb[2], m->wb[3], m->wbT[0], m->wbT[1], m->wbT[2],
                  m->wbT[3], m->Z[0], m->Z[1], m->Z[2], m->A[0], m->A[1], m->A[2], m->AT[0], m->AT[1], m->AT[2],
                  m->Y, m->dY, m->dYT, m->dZa, m->dZaT, m->dZb, m->dZbT, m->X, m->XT, m->T, m->rows_d, m->loss,
                  m->err, m->Xc, m->Yc, m->ws, m->wt};
    for (void* p : ps)
        if (p) cudaFree(p);
    if (m->stream) cudaStreamDestroy(m->stream);
    delete m;
}

const char* od_mlp_last_error(const od_mlp* m) { return m ? m->msg.c_str() : ""; }

long long od_mlp_param_count(const od_mlp* m) { return m ? m->nparam : 0; }

// host fp32 parameters (flat: W1 [256x896], b1, W2, b2, W3, b3, W4 [384x256], b4 [384];
// rows 320..383 of W4 and b4 must be zero) -> device, bf16 copies, Adam reset
int od_mlp_set_params(od_mlp* m, const float* host) {
    if (!m || !host) return OD_ERR_ARG;
    cudaSetDevice(m->device);
    const size_t P = sizeof(float) * (size_t)m->nparam;
    cudaError_t e = cudaMemcpyAsync(m->w, host, P, cudaMemcpyHostToDevice, m->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(m->m1, 0, P, m->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(m->m2, 0, P, m->stream);
    for (int l = 0; l < 4 && e == cudaSuccess; ++l) {
        const long long n = (long long)m->rows[l] * m->cols[l];
        cast_weights_kernel<<<blocks(n, 256), 256, 0, m->stream>>>(m->w + m->off_w[l], n, m->rows[l], m->cols[l],
                                                                    m->wb[l], m->wbT[l]);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = od::mlp::tile_fused_weights(m->wb, m->wt, m->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(m->stream);
    m->step = 0;
    if (e != cudaSuccess) return mfail(m, OD_ERR_CUDA, cudaGetErrorString(e));
    return OD_OK;
}

int od_mlp_get_params(od_mlp* m, float* host) {
    if (!m || !host) return OD_ERR_ARG;
    cudaSetDevice(m->device);
    cudaError_t e = cudaMemcpyAsync(host, m->w, sizeof(float) * (size_t)m->nparam, cudaMemcpyDeviceToHost, m->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(m->stream);
    return e == cudaSuccess ? OD_OK : mfail(m, OD_ERR_CUDA, cudaGetErrorString(e));
}

// Y [rows x 384] fp32 (device) of X [rows x 896] bf16 (device); rows % 128 == 0
int od_mlp_forward(od_mlp* m, const void* X, int rows, float* Y) {
    if (!m || !X || !Y || rows <= 0 || rows % 128 || rows > m->mmax) return OD_ERR_ARG;
    cudaSetDevice(m->device);
    cudaError_t e = cudaMemsetAsync(m->err, 0, sizeof(int), m->stream);
    if (e == cudaSuccess) e = forward(m, (const bf16*)X, rows, Y, false);
    if (e != cudaSuccess) return mfail(m, OD_ERR_CUDA, cudaGetErrorString(e));
    return check_err(m);
}

// Gradients (host fp32, flat layout) and loss of a batch given as device rows:
// X [rows x 896] bf16, XT its transpose [896 x rows], T [rows x 384] fp32;
// only the first `valid` rows and 320 columns count.
int od_mlp_gradients(od_mlp* m, const void* X, const void* XT, const float* T, int rows, int valid, float* grads,
                     double* loss) {
    if (!m || !X || !XT || !T || rows <= 0 || rows % 128 || rows > m->mmax || valid <= 0 || valid > rows)
        return OD_ERR_ARG;
    cudaSetDevice(m->device);
    cudaError_t e = cudaMemsetAsync(m->err, 0, sizeof(int), m->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(m->T, T, sizeof(float) * (size_t)rows * kOutPad, cudaMemcpyDeviceToDevice, m->stream);
    if (e == cudaSuccess) e = forward(m, (const bf16*)X, rows, m->Y, true);
    if (e == cudaSuccess) e = backward(m, (const bf16*)XT, rows, valid);
    double l = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&l, m->loss, sizeof(double), cudaMemcpyDeviceToHost, m->stream);
    if (e == cudaSuccess && grads)
        e = cudaMemcpyAsync(grads, m->g, sizeof(float) * (size_t)m->nparam, cudaMemcpyDeviceToHost, m->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(m->stream);
    if (e != cudaSuccess) return mfail(m, OD_ERR_CUDA, cudaGetErrorString(e));
    if (loss) *loss = l / ((double)valid * kOut);
    return check_err(m);
}

// One Adam step on a batch gathered from device pools: features Xpool
// [n x 896] bf16, targets Tpool [n x 320] bf16, row indices `rows_host`
// (count = batch). Returns the batch's mean squared error (before the step).
int od_mlp_train_step(od_mlp* m, const void* Xpool, const void* Tpool, const long long* rows_host, int batch,
                      float lr, double* loss) {
    if (!m || !Xpool || !Tpool || !rows_host || batch <= 0 || batch > m->mmax) return OD_ERR_ARG;
    cudaSetDevice(m->device);
    const int M = (batch + 127) / 128 * 128;
    cudaError_t e = cudaMemsetAsync(m->err, 0, sizeof(int), m->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(m->rows_d, rows_host, sizeof(long long) * batch, cudaMemcpyHostToDevice, m->stream);
    gather_kernel<<<blocks((long long)M * kIn, 256), 256, 0, m->stream>>>(
        (const bf16*)Xpool, (const bf16*)Tpool, m->rows_d, batch, M, m->X, m->XT, m->T);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e == cudaSuccess) e = forward(m, m->X, M, m->Y, true);
    if (e == cudaSuccess) e = backward(m, m->XT, M, batch);
    m->step++;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float c1 = 1.f - std::pow(b1, (float)m->step), c2 = 1.f - std::pow(b2, (float)m->step);
    for (int l = 0; l < 4 && e == cudaSuccess; ++l) {
        const long long nw = (long long)m->rows[l] * m->cols[l];
        adam_kernel<<<blocks(nw, 256), 256, 0, m->stream>>>(m->w + m->off_w[l], m->g + m->off_w[l], m->m1 + m->off_w[l],
                                                              m->m2 + m->off_w[l], nw, lr, b1, b2, eps, c1, c2,
                                                              m->rows[l], m->cols[l], m->wb[l], m->wbT[l]);
        adam_kernel<<<blocks(m->rows[l], 256), 256, 0, m->stream>>>(m->w + m->off_b[l], m->g + m->off_b[l],
                                                                     m->m1 + m->off_b[l], m->m2 + m->off_b[l],
                                                                     m->rows[l], lr, b1, b2, eps, c1, c2, 1,
                                                                     m->rows[l], nullptr, nullptr);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = od::mlp::tile_fused_weights(m->wb, m->wt, m->stream);
    double l = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&l, m->loss, sizeof(double), cudaMemcpyDeviceToHost, m->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(m->stream);
    if (e != cudaSuccess) return mfail(m, OD_ERR_CUDA, cudaGetErrorString(e));
    if (loss) *loss = l / ((double)batch * kOut);
    return check_err(m);
}

// Normalisation of the closure's inputs and outputs.
int od_mlp_set_fused(od_mlp* m, int on) {
    if (!m) return OD_ERR_ARG;
    m->fused = on != 0;
    return OD_OK;
}

int od_mlp_set_scaling(od_mlp* m, const float* mean14, const float* scale14, const float* out_scale5) {
    if (!m || !mean14 || !scale14 || !out_scale5) return OD_ERR_ARG;
    std::memcpy(m->mean, mean14, sizeof m->mean);
    std::memcpy(m->scale, scale14, sizeof m->scale);
    std::memcpy(m->out_scale, out_scale5, sizeof m->out_scale);
    return OD_OK;
}

// ---- data kernels on caller-owned device memory (stream-ordered) ----

int od_project(const void* src, int src_f64, int nxc, int nyc, int nzc, int factor, void* dst, int dst_f64,
               void* stream) {
    if (!src || !dst || nxc <= 0 || nyc <= 0 || nzc <= 0 || factor < 1 || factor > 8) return OD_ERR_ARG;
    const ProjParams pp = proj_params(nxc, nyc, nzc, factor);
    const int F = 4 * factor;
    const size_t sm = sizeof(float) * ((size_t)F * F * F + 4 * F * F + 16 * F);
    const long long ne = (long long)nxc * nyc * nzc;
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = cudaSuccess;
#define OD_PROJ(TS, TD)                                                                                   \
    do {                                                                                                  \
        e = cudaFuncSetAttribute(project_kernel<TS, TD>, cudaFuncAttributeMaxDynamicSharedMemorySize,     \
                                 (int)sm);                                                                \
        if (e == cudaSuccess) project_kernel<TS, TD><<<(unsigned)ne, 256, sm, s>>>((const TS*)src, (TD*)dst, pp); \
    } while (0)
    if (src_f64 && dst_f64)
        OD_PROJ(double, double);
    else if (src_f64)
        OD_PROJ(double, float);
    else if (dst_f64)
        OD_PROJ(float, double);
    else
        OD_PROJ(float, float);
#undef OD_PROJ
    if (e == cudaSuccess) e = cudaGetLastError();
    return e == cudaSuccess ? OD_OK : OD_ERR_CUDA;
}

int od_closure_features(const void* state, int u_f64, int nx, int ny, int nz, double lx, double ly, double lz,
                        const float* mean14, const float* scale14, void* X, void* stream) {
    if (!state || !X || nx <= 0 || ny <= 0 || nz <= 0) return OD_ERR_ARG;
    const FeatParams fp = feat_params(nx, ny, nz, lx, ly, lz, mean14, scale14);
    const long long ne = (long long)nx * ny * nz;
    cudaStream_t s = (cudaStream_t)stream;
    if (u_f64)
        features_kernel<double><<<(unsigned)ne, 64, 0, s>>>((const double*)state, fp, (bf16*)X);
    else
        features_kernel<float><<<(unsigned)ne, 64, 0, s>>>((const float*)state, fp, (bf16*)X);
    return cudaGetLastError() == cudaSuccess ? OD_OK : OD_ERR_CUDA;
}

int od_f32_to_bf16(const float* a, void* b, long long n, void* stream) {
    if (!a || !b || n < 0) return OD_ERR_ARG;
    f32_to_bf16_kernel<<<blocks(n, 256), 256, 0, (cudaStream_t)stream>>>(a, (bf16*)b, n);
    return cudaGetLastError() == cudaSuccess ? OD_OK : OD_ERR_CUDA;
}

}  // extern "C"

// ------------------------------------------------------------------ solver hook
// Between phase A (which leaves the RHS in the solver's RHS buffer) and
// phase B of every RK stage: features of the stage's input state, network
// forward, rhs += out_scale * output. With the fused network on an f32
// state, phase A writes the features itself (closure_stage_features) and
// closure_network_hook runs the network alone.
namespace od {
static_assert(kChan == kFeatChan && kClip == kFeatClip, "phase A writes the same features");

bool closure_stage_features(void* user, StageFeatures* out) {
    od_mlp* m = (od_mlp*)user;
    if (!m || !m->fused || m->attached_f64 || !m->Xc) return false;
    out->X = m->Xc;
    for (int d = 0; d < 3; ++d) out->jac[d] = m->fp.jac[d];
    for (int a = 0; a < 16; ++a) out->D[a] = m->fp.D[a];
    for (int c = 0; c < kChan; ++c) {
        out->mean[c] = m->fp.mean[c];
        out->inv_scale[c] = m->fp.inv_scale[c];
    }
    return true;
}

cudaError_t closure_network_hook(void* user, const void* u_in, void* rhs, cudaStream_t s) {
    (void)u_in;
    od_mlp* m = (od_mlp*)user;
    od::mlp::FusedArgs a{};
    a.X = m->Xc;
    a.Wt = m->wt;
    for (int l = 0; l < 4; ++l) a.bias[l] = m->w + m->off_b[l];
    a.rhs = (float*)rhs;
    a.rhs_npts = m->nelem_c * 64;
    a.rhs_rows = (int)m->nelem_c;
    for (int v = 0; v < 5; ++v) a.rhs_scale[v] = m->out_scale[v];
    a.err = m->err;
    return od::mlp::launch_fused(a, (int)m->mpad_c, s);
}

cudaError_t closure_stage_hook(void* user, const void* u_in, void* rhs, cudaStream_t s) {
    od_mlp* m = (od_mlp*)user;
    cudaError_t e = cudaSuccess;
    if (m->attached_f64)
        features_kernel<double><<<(unsigned)m->nelem_c, 64, 0, s>>>((const double*)u_in, m->fp, m->Xc);
    else if (m->fused)
        features_tiled_kernel<<<(unsigned)((m->nelem_c + kFeatEpb - 1) / kFeatEpb), 16 * kFeatEpb, 0, s>>>(
            (const float*)u_in, m->fp, m->Xc, (long long)m->nelem_c);
    else
        features_kernel<float><<<(unsigned)m->nelem_c, 64, 0, s>>>((const float*)u_in, m->fp, m->Xc);
    e = cudaGetLastError();
    // the network runs on the solver's stream; the last layer's epilogue adds
    // out_scale * (output) into the RHS directly (f32 state)
    cudaStream_t keep = m->stream;
    m->stream = s;
    if (e == cudaSuccess && m->fused && !m->attached_f64) {
        // the whole network per 128-element tile in one kernel, output into the RHS
        od::mlp::FusedArgs a{};
        a.X = m->Xc;
        a.Wt = m->wt;
        for (int l = 0; l < 4; ++l) {
            a.bias[l] = m->w + m->off_b[l];
        }
        a.rhs = (float*)rhs;
        a.rhs_npts = m->nelem_c * 64;
        a.rhs_rows = (int)m->nelem_c;
        for (int v = 0; v < 5; ++v) a.rhs_scale[v] = m->out_scale[v];
        a.err = m->err;
        e = od::mlp::launch_fused(a, (int)m->mpad_c, s);
        m->stream = keep;
        return e;
    }
    if (e == cudaSuccess) e = hidden(m, m->Xc, (int)m->mpad_c, false);
    if (e == cudaSuccess) {
        if (m->attached_f64) {
            e = gemm(m, m->A[2], m->wb[3], (int)m->mpad_c, kOutPad, kHid, od::mlp::kStoreF32, m->w + m->off_b[3],
                     m->Yc, nullptr, nullptr, nullptr);
            const long long n = m->nelem_c * 64 * 5;
            const float* o = m->out_scale;
            if (e == cudaSuccess)
                apply_kernel<double><<<blocks(n, 256), 256, 0, s>>>((double*)rhs, m->Yc, m->nelem_c, o[0], o[1], o[2],
                                                                    o[3], o[4]);
        } else {
            od::mlp::GemmArgs a{};
            a.A = m->A[2];
            a.B = m->wb[3];
            a.M = (int)m->mpad_c;
            a.N = kOutPad;
            a.K = kHid;
            a.bias = m->w + m->off_b[3];
            a.err = m->err;
            a.rhs = (float*)rhs;
            a.rhs_npts = m->nelem_c * 64;
            a.rhs_rows = (int)m->nelem_c;
            for (int v = 0; v < 5; ++v) a.rhs_scale[v] = m->out_scale[v];
            e = od::mlp::launch_gemm(a, od::mlp::kApplyRhs, s, 0);
        }
        if (e == cudaSuccess) e = cudaGetLastError();
    }
    m->stream = keep;
    return e;
}

// prepares the network for a solver's mesh; returns 0 or an OD_ERR code
int closure_prepare(od_mlp* m, int nx, int ny, int nz, double lx, double ly, double lz, bool f64) {
    const long long ne = (long long)nx * ny * nz;
    const long long mp = (ne + 127) / 128 * 128;
    if (mp > m->mmax) return mfail(m, OD_ERR_SIZE, "mesh has more elements than the network's batch capacity");
    cudaSetDevice(m->device);
    if (m->Xc) cudaFree(m->Xc);
    if (m->Yc) cudaFree(m->Yc);
    m->Xc = nullptr;
    m->Yc = nullptr;
    cudaError_t e = cudaMalloc(&m->Xc, sizeof(bf16) * mp * kIn);
    if (e == cudaSuccess) e = cudaMemset(m->Xc, 0, sizeof(bf16) * mp * kIn);
    if (e == cudaSuccess) e = cudaMalloc(&m->Yc, sizeof(float) * mp * kOutPad);
    if (e != cudaSuccess) return mfail(m, OD_ERR_CUDA, cudaGetErrorString(e));
    m->nelem_c = ne;
    m->mpad_c = mp;
    m->fp = feat_params(nx, ny, nz, lx, ly, lz, m->mean, m->scale);
    m->attached_f64 = f64;
    return OD_OK;
}
}  // namespace od
