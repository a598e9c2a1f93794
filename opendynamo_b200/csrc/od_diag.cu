// Flow diagnostics of a state on the device: volume integrals (mass,
// x-momentum, total energy, kinetic energy, enstrophy) and x-z plane
// averages at every y row of solution points (the mean profile and the
// second moments a Reynolds-stress comparison needs).
//
// Quadrature: Gauss-Legendre weights of the solution points times the
// element Jacobian (h/2 per axis). Gradients for the vorticity are the
// element-local FR derivative D (no interface correction).
//
// One block of 64 threads per element, one thread per solution point; the
// element's state goes through shared memory for the derivatives. Sums are
// formed in double: a block reduction per element, then one global double
// atomicAdd per element and quantity (a diagnostic, not a hot path).

#include <cuda_runtime.h>

#include "od_launch.h"

namespace od {
namespace {

struct DiagParams {
    int nx, ny, nz;
    double hx, hy, hz;   // element sizes
    double w[4];         // GL weights on [-1, 1]
    double D[16];        // D[a*4+m] = l'_m(x_a)
};

__device__ __forceinline__ void block_add(double v, double* red, double* out, int tid) {
    // 64 threads: two warps
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((tid & 31) == 0) red[tid >> 5] = v;
    __syncthreads();
    if (tid == 0) atomicAdd(out, red[0] + red[1]);
    __syncthreads();
}

template <class S>
__global__ void __launch_bounds__(64) diag_kernel(const S* __restrict__ u, DiagParams P, double* vol,
                                                  double* prof) {
    __shared__ double q[4][64];   // rho, rho u, rho v, rho w
    __shared__ double red[2];
    __shared__ double lev[4][8];  // plane sums of this element's four y rows
    const long long nelem = (long long)P.nx * P.ny * P.nz;
    const long long npts = nelem * 64;
    const int tid = threadIdx.x;
    const long long e = blockIdx.x;
    const int ey = (int)((e / P.nx) % P.ny);
    const int i = tid & 3, j = (tid >> 2) & 3, k = tid >> 4;
    double qv[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) qv[v] = (double)u[v * npts + e * 64 + tid];
#pragma unroll
    for (int v = 0; v < 4; ++v) q[v][tid] = qv[v];
    if (tid < 32) lev[tid >> 3][tid & 7] = 0.0;
    __syncthreads();
    // derivatives of rho and momentum along x, y, z (reference space, then jac)
    const double jac[3] = {2.0 / P.hx, 2.0 / P.hy, 2.0 / P.hz};
    double dq[4][3];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        double sx = 0, sy = 0, sz = 0;
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            sx += P.D[i * 4 + m] * q[v][m + 4 * j + 16 * k];
            sy += P.D[j * 4 + m] * q[v][i + 4 * m + 16 * k];
            sz += P.D[k * 4 + m] * q[v][i + 4 * j + 16 * m];
        }
        dq[v][0] = sx * jac[0];
        dq[v][1] = sy * jac[1];
        dq[v][2] = sz * jac[2];
    }
    const double rho = qv[0], ir = 1.0 / rho;
    const double vel[3] = {qv[1] * ir, qv[2] * ir, qv[3] * ir};
    double dv[3][3];  // dv[a][b] = d vel_a / d x_b
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) dv[a][b] = (dq[1 + a][b] - vel[a] * dq[0][b]) * ir;
    const double wx = dv[2][1] - dv[1][2], wy = dv[0][2] - dv[2][0], wz = dv[1][0] - dv[0][1];
    const double ke = 0.5 * rho * (vel[0] * vel[0] + vel[1] * vel[1] + vel[2] * vel[2]);
    const double ens = 0.5 * rho * (wx * wx + wy * wy + wz * wz);
    const double wvol = P.w[i] * P.w[j] * P.w[k] * (0.125 * P.hx * P.hy * P.hz);
    block_add(wvol * rho, red, vol + 0, tid);
    block_add(wvol * qv[1], red, vol + 1, tid);
    block_add(wvol * qv[4], red, vol + 2, tid);
    block_add(wvol * ke, red, vol + 3, tid);
    block_add(wvol * ens, red, vol + 4, tid);
    block_add(wvol, red, vol + 5, tid);
    if (prof) {
        const double wpl = P.w[i] * P.w[k] * (0.25 * P.hx * P.hz);
        const double m[8] = {rho, vel[0], vel[1], vel[2], vel[0] * vel[0], vel[1] * vel[1], vel[2] * vel[2],
                             vel[0] * vel[1]};
#pragma unroll
        for (int c = 0; c < 8; ++c) atomicAdd(&lev[j][c], wpl * m[c]);
        __syncthreads();
        if (tid < 32) atomicAdd(&prof[(ey * 4 + (tid >> 3)) * 8 + (tid & 7)], lev[tid >> 3][tid & 7]);
    }
}

}  // namespace

cudaError_t launch_diag(const void* u, bool u_f64, int nx, int ny, int nz, double lx, double ly, double lz,
                        const TablesD& tab, double* d_vol6, double* d_prof, cudaStream_t s) {
    DiagParams P;
    P.nx = nx;
    P.ny = ny;
    P.nz = nz;
    P.hx = lx / nx;
    P.hy = ly / ny;
    P.hz = lz / nz;
    // GL weights from the points: w_i = 2 / ((1 - x^2) P'_4(x)^2)
    for (int a = 0; a < 4; ++a) {
        const double x = tab.pts[a];
        const double dp4 = (4.0 * (x * (35 * x * x * x * x - 30 * x * x + 3) / 8.0) -
                            4.0 * ((5 * x * x * x - 3 * x) / 2.0)) / (x * x - 1.0);
        P.w[a] = 2.0 / ((1.0 - x * x) * dp4 * dp4);
    }
    for (int a = 0; a < 16; ++a) P.D[a] = tab.D[a];
    const long long nelem = (long long)nx * ny * nz;
    if (nelem > 0x7fffffffLL) return cudaErrorInvalidValue;
    if (u_f64)
        diag_kernel<double><<<(unsigned)nelem, 64, 0, s>>>((const double*)u, P, d_vol6, d_prof);
    else
        diag_kernel<float><<<(unsigned)nelem, 64, 0, s>>>((const float*)u, P, d_vol6, d_prof);
    return cudaGetLastError();
}

}  // namespace od
