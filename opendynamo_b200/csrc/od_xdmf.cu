// ParaView conversion of state files (the reference's scripts/h5_to_xdmf.py):
// the element-major planes are reordered into the global solution-point
// tensor with the derived velocity magnitude and pressure on the GPU, then
// written as a chunked point-field file and an XDMF description.

#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/opendynamo.h"

namespace od {
namespace {

constexpr int kEZ = 8;            // elements along z per block
constexpr int kRow = 68;          // shared-memory floats per element (64 + 4 pad)
constexpr int kFields = 7;

// shared-memory slot of point p = i + 4j + 16k of local element el: rows of
// 17 per k so that the z-runs of the write phase hit distinct banks
__device__ __forceinline__ int slot(int el, int p) { return el * kRow + (p >> 4) * 17 + (p & 15); }

// numpy.maximum: NaN if either operand is NaN
__device__ __forceinline__ float nan_max(float a, float b) { return (a != a || b != b) ? __int_as_float(0x7fc00000) : (a > b ? a : b); }

// One block: the kEZ elements (ex, ey, ez0 .. ez0 + kEZ - 1). Loads their
// 64-point blocks (contiguous), derives vel and p per point, and writes,
// per field and per (i, j), the run of 4 * kEZ consecutive z points.
template <class S>
__global__ void __launch_bounds__(256) point_fields_kernel(const S* __restrict__ u, int nx, int ny, int nz,
                                                           long long npts, float* __restrict__ out) {
    __shared__ float f[kFields][kEZ * kRow];
    const int ex = blockIdx.x, ey = blockIdx.y, ez0 = blockIdx.z * kEZ;
    const int nez = min(kEZ, nz - ez0);
    for (int idx = threadIdx.x; idx < nez * 64; idx += blockDim.x) {
        const int el = idx >> 6, p = idx & 63;
        const long long src = (ex + (long long)nx * (ey + (long long)ny * (ez0 + el))) * 64 + p;
        float q[5];
#pragma unroll
        for (int v = 0; v < 5; ++v) q[v] = (float)u[v * npts + src];
        // operation order of h5_to_xdmf.py:76-79, f32, no contraction
        const float r = nan_max(q[0], 1e-30f);
        const float k2 = __fadd_rn(__fadd_rn(__fmul_rn(q[1], q[1]), __fmul_rn(q[2], q[2])), __fmul_rn(q[3], q[3]));
        const float vel = __fdiv_rn(__fsqrt_rn(k2), r);
        const float pr = nan_max(1e-7f, __fmul_rn(0.4f, __fsub_rn(q[4], __fdiv_rn(__fmul_rn(0.5f, k2), r))));
        const int s = slot(el, p);
#pragma unroll
        for (int v = 0; v < 5; ++v) f[v][s] = q[v];
        f[5][s] = vel;
        f[6][s] = pr;
    }
    __syncthreads();
    const int run = nez * 4;
    const long long npy = 4LL * ny, npz = 4LL * nz, ntot = 64LL * nx * ny * nz;
    for (int idx = threadIdx.x; idx < 16 * run; idx += blockDim.x) {
        const int ij = idx / run, zz = idx - ij * run;
        const int i = ij & 3, j = ij >> 2, el = zz >> 2, k = zz & 3;
        const long long o = ((4LL * ex + i) * npy + 4LL * ey + j) * npz + 4LL * ez0 + zz;
        const int s = slot(el, i + 4 * j + 16 * k);
#pragma unroll
        for (int c = 0; c < kFields; ++c) out[c * ntot + o] = f[c][s];
    }
}

const char* const kNames[kFields] = {"rho", "rhou", "rhov", "rhow", "E", "vel", "p"};

void put(char* err, int len, const std::string& s) {
    if (err && len > 0) std::snprintf(err, (size_t)len, "%s", s.c_str());
}

void copy_out(char* dst, size_t len, const std::string& s) {
    if (dst && len > 0) std::snprintf(dst, len, "%s", s.c_str());
}

// Path.with_suffix(suffix) of the script (h5_to_xdmf.py:81, 142)
std::string with_suffix(const std::string& path, const char* suffix) {
    const size_t slash = path.find_last_of('/');
    const size_t name0 = slash == std::string::npos ? 0 : slash + 1;
    const size_t dot = path.find_last_of('.');
    if (dot != std::string::npos && dot > name0 && dot + 1 < path.size()) return path.substr(0, dot) + suffix;
    return path + suffix;
}

std::string base_name(const std::string& path) {
    const size_t slash = path.find_last_of('/');
    return slash == std::string::npos ? path : path.substr(slash + 1);
}

std::string fmt_g(const char* f, double x) {
    char b[64];
    std::snprintf(b, sizeof b, f, x);
    return b;
}

}  // namespace
}  // namespace od

extern "C" int od_point_fields(const void* planes, int u_f64, int nx, int ny, int nz, float* out, void* stream) {
    if (!planes || !out || nx <= 0 || ny <= 0 || nz <= 0) return OD_ERR_ARG;
    const long long npts = 64LL * nx * ny * nz;
    dim3 grid((unsigned)nx, (unsigned)ny, (unsigned)((nz + od::kEZ - 1) / od::kEZ));
    if (ny > 65535 || grid.z > 65535) return OD_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    if (u_f64)
        od::point_fields_kernel<double><<<grid, 256, 0, s>>>((const double*)planes, nx, ny, nz, npts, out);
    else
        od::point_fields_kernel<float><<<grid, 256, 0, s>>>((const float*)planes, nx, ny, nz, npts, out);
    return cudaGetLastError() == cudaSuccess ? OD_OK : OD_ERR_CUDA;
}

extern "C" long long od_xdmf_text(char* buf, size_t len, const char* h5_name, int npx, int npy, int npz, double lx,
                                  double ly, double lz, unsigned long long step, double t) {
    if (!h5_name || npx <= 0 || npy <= 0 || npz <= 0) return -1;
    std::string x;
    x += "<?xml version=\"1.0\" ?>\n<!DOCTYPE Xdmf SYSTEM \"Xdmf.dtd\" []>\n<Xdmf Version=\"2.0\">\n  <Domain>\n";
    x += "    <Grid Name=\"FR_Grid\" GridType=\"Uniform\" t_step=\"" + std::to_string(step) + "\" t_time=\"" +
         od::fmt_g("%.6g", t) + "\">\n";
    x += "      <Topology TopologyType=\"3DRectMesh\" Dimensions=\"" + std::to_string(npz + 1) + " " +
         std::to_string(npy + 1) + " " + std::to_string(npx + 1) + "\"/>\n";
    x += "      <Geometry GeometryType=\"VXVYVZ\">\n";
    const int n[3] = {npx, npy, npz};
    const double L[3] = {lx, ly, lz};
    for (int d = 0; d < 3; ++d) {
        x += "        <DataItem Dimensions=\"" + std::to_string(n[d] + 1) +
             "\" NumberType=\"Float\" Precision=\"8\" Format=\"XML\">\n          ";
        // numpy.linspace(0, L, n + 1): i * (L / n) + 0, the last point exactly L
        const double step_d = L[d] / n[d];
        for (int i = 0; i <= n[d]; ++i) {
            const double v = i == n[d] ? L[d] : (double)i * step_d + 0.0;
            if (i) x += " ";
            x += od::fmt_g("%.10g", v);
        }
        x += "\n        </DataItem>\n";
    }
    x += "      </Geometry>\n";
    for (int c = 0; c < od::kFields; ++c) {
        if (c) x += "\n";
        x += std::string("      <Attribute Name=\"") + od::kNames[c] + "\" AttributeType=\"Scalar\" Center=\"Cell\">\n";
        x += "        <DataItem Dimensions=\"" + std::to_string(npz) + " " + std::to_string(npy) + " " +
             std::to_string(npx) + "\" NumberType=\"Float\" Precision=\"4\" Format=\"HDF\">\n";
        x += std::string("          ") + h5_name + ":/data/" + od::kNames[c] + "\n";
        x += "        </DataItem>\n      </Attribute>";
    }
    x += "\n    </Grid>\n  </Domain>\n</Xdmf>\n";
    if (buf && len > 0) std::snprintf(buf, len, "%s", x.c_str());
    return (long long)x.size();
}

extern "C" int od_xdmf_convert(const char* src, char* out_h5, size_t out_h5_len, char* out_xmf, size_t out_xmf_len,
                               char* err, int err_len) {
    using namespace od;
    if (!src) {
        put(err, err_len, "no source file");
        return OD_ERR_ARG;
    }
    int nx = 0, ny = 0, nz = 0, fr = 0;
    unsigned long long step = 0;
    double t = 0, lx = 0, ly = 0, lz = 0;
    char ureal[4] = {0};
    if (od_state_info(src, &nx, &ny, &nz, &fr, &step, &t, &lx, &ly, &lz, ureal) != 0) {
        put(err, err_len, base_name(src) + ": " + od_state_error());
        return OD_ERR_IO;
    }
    const int f64 = std::strcmp(ureal, "f64") == 0;
    const size_t npts = (size_t)nx * ny * nz * 64;
    const size_t es = f64 ? 8 : 4;
    std::vector<unsigned char> host(5 * npts * es);
    if (od_state_load(src, host.data(), host.size(), f64, nx, ny, nz, &step, &t) != 0) {
        put(err, err_len, base_name(src) + ": " + od_state_error());
        return OD_ERR_IO;
    }
    void* d_in = nullptr;
    float* d_out = nullptr;
    std::vector<float> fields(kFields * npts);
    cudaError_t e = cudaMalloc(&d_in, host.size());
    if (e == cudaSuccess) e = cudaMalloc((void**)&d_out, fields.size() * sizeof(float));
    if (e == cudaSuccess) e = cudaMemcpy(d_in, host.data(), host.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && od_point_fields(d_in, f64, nx, ny, nz, d_out, nullptr) != OD_OK) e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(fields.data(), d_out, fields.size() * sizeof(float), cudaMemcpyDeviceToHost);
    if (d_in) cudaFree(d_in);
    if (d_out) cudaFree(d_out);
    if (e != cudaSuccess) {
        put(err, err_len, std::string("CUDA: ") + cudaGetErrorString(e));
        return OD_ERR_CUDA;
    }
    const std::string h5 = with_suffix(src, ".pv.h5"), xmf = with_suffix(src, ".xmf");
    if (od_fields_save(h5.c_str(), fields.data(), kFields, kNames, 4LL * nx, 4LL * ny, 4LL * nz, 48, "gzip4") != 0) {
        put(err, err_len, od_state_error());
        return OD_ERR_IO;
    }
    const long long n = od_xdmf_text(nullptr, 0, base_name(h5).c_str(), 4 * nx, 4 * ny, 4 * nz, lx, ly, lz, step, t);
    std::vector<char> text((size_t)n + 1);
    od_xdmf_text(text.data(), text.size(), base_name(h5).c_str(), 4 * nx, 4 * ny, 4 * nz, lx, ly, lz, step, t);
    FILE* fp = std::fopen(xmf.c_str(), "wb");
    const bool ok = fp && std::fwrite(text.data(), 1, (size_t)n, fp) == (size_t)n;
    if (fp && std::fclose(fp) != 0) {
        put(err, err_len, "cannot write " + xmf);
        return OD_ERR_IO;
    }
    if (!ok) {
        put(err, err_len, "cannot write " + xmf);
        return OD_ERR_IO;
    }
    copy_out(out_h5, out_h5_len, h5);
    copy_out(out_xmf, out_xmf_len, xmf);
    return OD_OK;
}
