// TEST INFRASTRUCTURE ONLY — runner for the reference's own kernels.
//
// Loads one PTX module built by oracle/build_ref.py from the reference's CUDA
// sources and replays the reference host's device work with the CUDA driver
// API, as src/solver.rs does through cudarc:
//   setup_fr_operators   solver.rs:464-510   tables cast to COMPUTE_REAL, uploaded to the
//                                              six __constant__ symbols
//   allocate_buffers     solver.rs:574-601   u, u_prev (U), rhs (RHS), 6 j + 6 slice arrays
//                                              (COMPUTE_REAL), all zeroed
//   launch_configs       solver.rs:532-572   volume nelem x 64, faces 64-thread blocks of 4
//                                              faces, wall 2*nx*nz x 16, RK for_num_elems(size/4)
//   launch_rhs_stage     solver.rs:610-694   volume, face x, face y, [wall], face z
//   launch_rk_stage      solver.rs:699-738
//   the step loop        solver.rs:262-317   stage 1 into u_prev + swap, stages 2 and 3 in place
// The driver library is opened at run time; the primary context is used so the
// runtime API (torch, libopendynamo) shares it.

#include <dlfcn.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

namespace {

typedef int CUresult;
typedef int CUdevice;
typedef void* CUcontext;
typedef void* CUmodule;
typedef void* CUfunction;
typedef void* CUstream;
typedef void* CUevent;
typedef unsigned long long CUdeviceptr;

struct Driver {
    void* h = nullptr;
    CUresult (*cuInit)(unsigned);
    CUresult (*cuDeviceGet)(CUdevice*, int);
    CUresult (*cuDevicePrimaryCtxRetain)(CUcontext*, CUdevice);
    CUresult (*cuDevicePrimaryCtxRelease)(CUdevice);
    CUresult (*cuCtxSetCurrent)(CUcontext);
    CUresult (*cuModuleLoadData)(CUmodule*, const void*);
    CUresult (*cuModuleUnload)(CUmodule);
    CUresult (*cuModuleGetFunction)(CUfunction*, CUmodule, const char*);
    CUresult (*cuModuleGetGlobal)(CUdeviceptr*, size_t*, CUmodule, const char*);
    CUresult (*cuMemAlloc)(CUdeviceptr*, size_t);
    CUresult (*cuMemFree)(CUdeviceptr);
    CUresult (*cuMemsetD8)(CUdeviceptr, unsigned char, size_t);
    CUresult (*cuMemcpyHtoD)(CUdeviceptr, const void*, size_t);
    CUresult (*cuMemcpyDtoH)(void*, CUdeviceptr, size_t);
    CUresult (*cuMemcpyHtoDAsync)(CUdeviceptr, const void*, size_t, CUstream);
    CUresult (*cuMemcpyDtoHAsync)(void*, CUdeviceptr, size_t, CUstream);
    CUresult (*cuMemcpyDtoDAsync)(CUdeviceptr, CUdeviceptr, size_t, CUstream);
    CUresult (*cuStreamWaitEvent)(CUstream, CUevent, unsigned);
    CUresult (*cuEventSynchronize)(CUevent);
    CUresult (*cuLaunchKernel)(CUfunction, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned,
                               CUstream, void**, void**);
    CUresult (*cuStreamCreate)(CUstream*, unsigned);
    CUresult (*cuStreamDestroy)(CUstream);
    CUresult (*cuStreamSynchronize)(CUstream);
    CUresult (*cuEventCreate)(CUevent*, unsigned);
    CUresult (*cuEventDestroy)(CUevent);
    CUresult (*cuEventRecord)(CUevent, CUstream);
    CUresult (*cuEventElapsedTime)(float*, CUevent, CUevent);
    CUresult (*cuGetErrorString)(CUresult, const char**);
    CUresult (*cuFuncGetAttribute)(int*, int, CUfunction);

    bool load(std::string& err) {
        if (h) return true;
        h = dlopen("libcuda.so.1", RTLD_NOW | RTLD_GLOBAL);
        if (!h) {
            err = "libcuda.so.1 not available";
            return false;
        }
#define SYM(name, str)                                            \
    name = reinterpret_cast<decltype(name)>(dlsym(h, str));      \
    if (!name) {                                                  \
        err = std::string("missing driver symbol ") + str;        \
        return false;                                             \
    }
        SYM(cuInit, "cuInit");
        SYM(cuDeviceGet, "cuDeviceGet");
        SYM(cuDevicePrimaryCtxRetain, "cuDevicePrimaryCtxRetain");
        SYM(cuDevicePrimaryCtxRelease, "cuDevicePrimaryCtxRelease_v2");
        SYM(cuCtxSetCurrent, "cuCtxSetCurrent");
        SYM(cuModuleLoadData, "cuModuleLoadData");
        SYM(cuModuleUnload, "cuModuleUnload");
        SYM(cuModuleGetFunction, "cuModuleGetFunction");
        SYM(cuModuleGetGlobal, "cuModuleGetGlobal_v2");
        SYM(cuMemAlloc, "cuMemAlloc_v2");
        SYM(cuMemFree, "cuMemFree_v2");
        SYM(cuMemsetD8, "cuMemsetD8_v2");
        SYM(cuMemcpyHtoD, "cuMemcpyHtoD_v2");
        SYM(cuMemcpyDtoH, "cuMemcpyDtoH_v2");
        SYM(cuMemcpyHtoDAsync, "cuMemcpyHtoDAsync_v2");
        SYM(cuMemcpyDtoHAsync, "cuMemcpyDtoHAsync_v2");
        SYM(cuMemcpyDtoDAsync, "cuMemcpyDtoDAsync_v2");
        SYM(cuStreamWaitEvent, "cuStreamWaitEvent");
        SYM(cuEventSynchronize, "cuEventSynchronize");
        SYM(cuLaunchKernel, "cuLaunchKernel");
        SYM(cuStreamCreate, "cuStreamCreate");
        SYM(cuStreamDestroy, "cuStreamDestroy_v2");
        SYM(cuStreamSynchronize, "cuStreamSynchronize");
        SYM(cuEventCreate, "cuEventCreate");
        SYM(cuEventDestroy, "cuEventDestroy_v2");
        SYM(cuEventRecord, "cuEventRecord");
        SYM(cuEventElapsedTime, "cuEventElapsedTime");
        SYM(cuGetErrorString, "cuGetErrorString");
        SYM(cuFuncGetAttribute, "cuFuncGetAttribute");
#undef SYM
        return true;
    }
};

Driver drv;

// FR tables (fr_math.rs:107-142) in double, computed independently of the product.
void fr_tables(double pts[4], double D[16], double eL[4], double eR[4], double gL[4], double gR[4]) {
    auto leg = [](int p, double x) {
        if (p == 0) return 1.0;
        if (p == 1) return x;
        double a = 1.0, b = x, v = 0.0;
        for (int k = 2; k <= p; ++k) {
            v = ((2.0 * k - 1.0) * x * b - (k - 1.0) * a) / k;
            a = b;
            b = v;
        }
        return v;
    };
    auto dleg = [&](int p, double x) { return p == 0 ? 0.0 : p / (x * x - 1.0) * (x * leg(p, x) - leg(p - 1, x)); };
    for (int i = 0; i < 4; ++i) {
        double x = std::cos(M_PI * (i + 0.75) / 4.5);
        for (;;) {
            double s = leg(4, x) / dleg(4, x);
            x -= s;
            if (std::fabs(s) < 1e-14) break;
        }
        pts[i] = x;
    }
    for (int a = 0; a < 4; ++a)
        for (int b = a + 1; b < 4; ++b)
            if (pts[b] < pts[a]) std::swap(pts[a], pts[b]);
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
            if (i != j) {
                double num = 1, den = 1;
                for (int k = 0; k < 4; ++k) {
                    if (k != i && k != j) num *= pts[i] - pts[k];
                    if (k != j) den *= pts[j] - pts[k];
                }
                D[i * 4 + j] = num / den;
            } else {
                double s = 0;
                for (int k = 0; k < 4; ++k)
                    if (k != i) s += 1.0 / (pts[i] - pts[k]);
                D[i * 4 + i] = s;
            }
        }
    for (int i = 0; i < 4; ++i) {
        double l = 1, r = 1;
        for (int j = 0; j < 4; ++j)
            if (j != i) {
                l *= (-1.0 - pts[j]) / (pts[i] - pts[j]);
                r *= (1.0 - pts[j]) / (pts[i] - pts[j]);
            }
        eL[i] = l;
        eR[i] = r;
        double d3 = dleg(3, pts[i]), d4 = dleg(4, pts[i]);
        gR[i] = 0.5 * (d3 + d4);
        gL[i] = 0.5 * -1.0 * (d3 - d4);
    }
}

}  // namespace

extern "C" {

typedef struct {
    int nx, ny, nz;
    float lx, ly, lz;  // config values (f32), cast to COMPUTE_REAL as solver.rs:516-530
    int y_wall;
    int u_f64, rhs_f64, c_f64;
    int device;
} refh_params;

}  // extern "C"

struct refh {
    refh_params p;
    CUcontext ctx = nullptr;
    CUdevice dev = 0;
    CUmodule mod = nullptr;
    CUstream stream = nullptr;
    CUfunction k_vol, k_fx, k_fy, k_fw, k_fz, k_rk, k_rk1;
    CUdeviceptr u = 0, u_prev = 0, rhs = 0, j[6] = {}, sl[6] = {};
    size_t nelem, npts, state_size, us, rs, cs;
    std::string err;
    std::vector<CUevent> ev;
    unsigned rk_block = 1024;  // cudarc for_num_elems; clamped to what the RK kernels can launch
    // asynchronous host copies (refh_set_state_async / refh_get_state_async):
    // staging and snapshot buffers with their hand-over events
    CUdeviceptr stage = 0, snap = 0;
    CUevent ev_staged = nullptr, ev_taken = nullptr, ev_snap = nullptr, ev_copied = nullptr;
};

namespace {

int fail(refh* h, CUresult r, const char* what) {
    const char* s = nullptr;
    if (drv.cuGetErrorString) drv.cuGetErrorString(r, &s);
    if (h) h->err = std::string(what) + ": " + (s ? s : "?");
    return -2;
}

#define CK(h, call, what)                     \
    do {                                      \
        CUresult _r = (call);                 \
        if (_r != 0) return fail(h, _r, what); \
    } while (0)

int upload_constants(refh* h) {
    double pts[4], D[16], eL[4], eR[4], gL[4], gR[4];
    fr_tables(pts, D, eL, eR, gL, gR);
    struct Sym {
        const char* name;
        const double* v;
        int n;
    } syms[] = {{"c_points", pts, 4},       {"c_extrap_left", eL, 4},  {"c_extrap_right", eR, 4},
                {"c_g_left_prime", gL, 4},  {"c_g_right_prime", gR, 4}, {"c_d_matrix", D, 16}};
    for (auto& s : syms) {
        CUdeviceptr ptr;
        size_t bytes;
        CK(h, drv.cuModuleGetGlobal(&ptr, &bytes, h->mod, s.name), s.name);
        if (h->p.c_f64) {
            CK(h, drv.cuMemcpyHtoD(ptr, s.v, sizeof(double) * s.n), "constant upload");
        } else {
            float f[16];
            for (int i = 0; i < s.n; ++i) f[i] = (float)s.v[i];
            CK(h, drv.cuMemcpyHtoD(ptr, f, sizeof(float) * s.n), "constant upload");
        }
    }
    return 0;
}

// COMPUTE_REAL scalar argument storage
struct Scalar {
    double d;
    float f;
    void set(double v) {
        d = v;
        f = (float)v;
    }
    void* ptr(bool c64) { return c64 ? (void*)&d : (void*)&f; }
};

int launch(refh* h, CUfunction f, unsigned grid, unsigned block, void** args, const char* what) {
    CK(h, drv.cuLaunchKernel(f, grid, 1, 1, block, 1, 1, 0, h->stream, args, nullptr), what);
    return 0;
}

int rhs_stage(refh* h) {
    const bool c64 = h->p.c_f64;
    int nx = h->p.nx, ny = h->p.ny, nz = h->p.nz;
    Scalar lx, ly, lz;
    lx.set(c64 ? (double)h->p.lx : (double)(float)h->p.lx);
    ly.set(c64 ? (double)h->p.ly : (double)(float)h->p.ly);
    lz.set(c64 ? (double)h->p.lz : (double)(float)h->p.lz);
    void* av[] = {&h->u, &h->rhs, &h->sl[0], &h->sl[1], &h->sl[2], &h->sl[3], &h->sl[4], &h->sl[5],
                  &nx, &ny, &nz, lx.ptr(c64), ly.ptr(c64), lz.ptr(c64)};
    if (int r = launch(h, h->k_vol, (unsigned)h->nelem, 64, av, "volume")) return r;
    void* ax[] = {&h->u, &h->j[0], &h->j[1], &h->sl[0], &h->sl[1], &nx, &ny, &nz, lx.ptr(c64)};
    if (int r = launch(h, h->k_fx, (unsigned)((h->nelem + 3) / 4), 64, ax, "face x")) return r;
    void* ay[] = {&h->u, &h->j[2], &h->j[3], &h->sl[2], &h->sl[3], &nx, &ny, &nz, ly.ptr(c64)};
    if (int r = launch(h, h->k_fy, (unsigned)(nx * ((ny + 3) / 4) * nz), 64, ay, "face y")) return r;
    if (h->p.y_wall) {
        if (int r = launch(h, h->k_fw, (unsigned)(2 * nx * nz), 16, ay, "face y wall")) return r;
    }
    void* az[] = {&h->u, &h->j[4], &h->j[5], &h->sl[4], &h->sl[5], &nx, &ny, &nz, lz.ptr(c64)};
    return launch(h, h->k_fz, (unsigned)(nx * ny * ((nz + 3) / 4)), 64, az, "face z");
}

int rk_stage(refh* h, bool stage1, CUdeviceptr dst, CUdeviceptr src, double a, double b, double c) {
    const bool c64 = h->p.c_f64;
    int nx = h->p.nx, ny = h->p.ny, nz = h->p.nz;
    int size = (int)h->state_size;
    Scalar lx, ly, lz, sa, sb, sc;
    lx.set(h->p.lx);
    ly.set(h->p.ly);
    lz.set(h->p.lz);
    sa.set(a);
    sb.set(b);
    sc.set(c);
    // cudarc LaunchConfig::for_num_elems: 1024 threads per block (h->rk_block,
    // lower only where the kernel cannot launch 1024 threads on this GPU)
    unsigned n4 = (unsigned)(h->state_size / 4);
    unsigned blk = h->rk_block;
    unsigned grid = (n4 + blk - 1) / blk;
    if (stage1) {
        void* args[] = {&dst, &src, &h->rhs, &h->j[0], &h->j[1], &h->j[2], &h->j[3], &h->j[4], &h->j[5],
                        &nx, &ny, &nz, lx.ptr(c64), ly.ptr(c64), lz.ptr(c64), sa.ptr(c64), sc.ptr(c64), &size};
        return launch(h, h->k_rk1, grid, blk, args, "rk stage 1");
    }
    void* args[] = {&dst, &src, &h->rhs, &h->j[0], &h->j[1], &h->j[2], &h->j[3], &h->j[4], &h->j[5],
                    &nx, &ny, &nz, lx.ptr(c64), ly.ptr(c64), lz.ptr(c64), sa.ptr(c64), sb.ptr(c64), sc.ptr(c64),
                    &size};
    return launch(h, h->k_rk, grid, blk, args, "rk stage");
}

// COMPUTE_REAL evaluation of a host constant
double in_c(bool c64, double x) { return c64 ? x : (double)(float)x; }

}  // namespace

extern "C" {

const char* refh_last_error(refh* h) { return h ? h->err.c_str() : "null"; }

int refh_create(const char* ptx_path, const refh_params* p, refh** out) {
    std::string err;
    *out = nullptr;
    if (!drv.load(err)) return -1;
    refh* h = new refh();
    *out = h;
    h->p = *p;
    CK(h, drv.cuInit(0), "cuInit");
    CK(h, drv.cuDeviceGet(&h->dev, p->device), "cuDeviceGet");
    CK(h, drv.cuDevicePrimaryCtxRetain(&h->ctx, h->dev), "cuDevicePrimaryCtxRetain");
    CK(h, drv.cuCtxSetCurrent(h->ctx), "cuCtxSetCurrent");
    std::ifstream f(ptx_path, std::ios::binary);
    if (!f) {
        h->err = std::string("cannot open ") + ptx_path;
        return -1;
    }
    std::stringstream ss;
    ss << f.rdbuf();
    std::string ptx = ss.str();
    CK(h, drv.cuModuleLoadData(&h->mod, ptx.c_str()), "cuModuleLoadData");
    CK(h, drv.cuModuleGetFunction(&h->k_vol, h->mod, "compute_rhs_volume_kernel"), "volume kernel");
    CK(h, drv.cuModuleGetFunction(&h->k_fx, h->mod, "compute_face_flux_x_kernel"), "face x kernel");
    CK(h, drv.cuModuleGetFunction(&h->k_fy, h->mod, "compute_face_flux_y_kernel"), "face y kernel");
    CK(h, drv.cuModuleGetFunction(&h->k_fw, h->mod, "compute_face_flux_y_wall_kernel"), "wall kernel");
    CK(h, drv.cuModuleGetFunction(&h->k_fz, h->mod, "compute_face_flux_z_kernel"), "face z kernel");
    CK(h, drv.cuModuleGetFunction(&h->k_rk, h->mod, "rk_stage_kernel"), "rk kernel");
    CK(h, drv.cuModuleGetFunction(&h->k_rk1, h->mod, "rk_stage1_kernel"), "rk1 kernel");
    if (int r = upload_constants(h)) return r;
    // The f64 RK kernels need more than 64 registers per thread, so the
    // 1024-thread blocks of cudarc's for_num_elems exceed the register file
    // (CUDA_ERROR_LAUNCH_OUT_OF_RESOURCES). Element-wise kernels: a smaller
    // block changes no arithmetic.
    for (CUfunction f : {h->k_rk, h->k_rk1}) {
        int maxt = 1024;
        CK(h, drv.cuFuncGetAttribute(&maxt, 0 /* CU_FUNC_ATTRIBUTE_MAX_THREADS_PER_BLOCK */, f), "rk attribute");
        unsigned b = (unsigned)(maxt / 32 * 32);
        if (b < h->rk_block) h->rk_block = b;
    }
    CK(h, drv.cuStreamCreate(&h->stream, 1), "cuStreamCreate");
    h->nelem = (size_t)p->nx * p->ny * p->nz;
    h->npts = h->nelem * 64;
    h->state_size = h->npts * 5;
    h->us = p->u_f64 ? 8 : 4;
    h->rs = p->rhs_f64 ? 8 : 4;
    h->cs = p->c_f64 ? 8 : 4;
    CK(h, drv.cuMemAlloc(&h->u, h->state_size * h->us), "alloc u");
    CK(h, drv.cuMemAlloc(&h->u_prev, h->state_size * h->us), "alloc u_prev");
    CK(h, drv.cuMemAlloc(&h->rhs, h->state_size * h->rs), "alloc rhs");
    CK(h, drv.cuMemsetD8(h->u, 0, h->state_size * h->us), "zero");
    CK(h, drv.cuMemsetD8(h->u_prev, 0, h->state_size * h->us), "zero");
    CK(h, drv.cuMemsetD8(h->rhs, 0, h->state_size * h->rs), "zero");
    for (int q = 0; q < 6; ++q) {
        CK(h, drv.cuMemAlloc(&h->j[q], h->nelem * 16 * 5 * h->cs), "alloc j");
        CK(h, drv.cuMemAlloc(&h->sl[q], h->nelem * 16 * 12 * h->cs), "alloc slices");
        CK(h, drv.cuMemsetD8(h->j[q], 0, h->nelem * 16 * 5 * h->cs), "zero");
        CK(h, drv.cuMemsetD8(h->sl[q], 0, h->nelem * 16 * 12 * h->cs), "zero");
    }
    return 0;
}

void refh_destroy(refh* h) {
    if (!h) return;
    if (h->ctx) {
        drv.cuCtxSetCurrent(h->ctx);
        if (h->stream) drv.cuStreamSynchronize(h->stream);
        for (auto e : h->ev) drv.cuEventDestroy(e);
        CUevent aev[] = {h->ev_staged, h->ev_taken, h->ev_snap, h->ev_copied};
        if (h->ev_staged) drv.cuEventSynchronize(h->ev_staged);
        if (h->ev_copied) drv.cuEventSynchronize(h->ev_copied);
        for (auto e : aev)
            if (e) drv.cuEventDestroy(e);
        CUdeviceptr bufs[] = {h->u, h->u_prev, h->rhs, h->stage, h->snap};
        for (auto b : bufs)
            if (b) drv.cuMemFree(b);
        for (int q = 0; q < 6; ++q) {
            if (h->j[q]) drv.cuMemFree(h->j[q]);
            if (h->sl[q]) drv.cuMemFree(h->sl[q]);
        }
        if (h->stream) drv.cuStreamDestroy(h->stream);
        if (h->mod) drv.cuModuleUnload(h->mod);
        drv.cuDevicePrimaryCtxRelease(h->dev);
    }
    delete h;
}

size_t refh_state_bytes(refh* h) { return h->state_size * h->us; }

int refh_set_state(refh* h, const void* host, size_t bytes) {
    if (bytes != h->state_size * h->us) return -3;
    CK(h, drv.cuCtxSetCurrent(h->ctx), "ctx");
    CK(h, drv.cuMemcpyHtoDAsync(h->u, host, bytes, h->stream), "upload");
    CK(h, drv.cuStreamSynchronize(h->stream), "sync");
    return 0;
}

int refh_get_state(refh* h, void* host, size_t bytes) {
    if (bytes != h->state_size * h->us) return -3;
    CK(h, drv.cuCtxSetCurrent(h->ctx), "ctx");
    CK(h, drv.cuMemcpyDtoHAsync(host, h->u, bytes, h->stream), "download");
    CK(h, drv.cuStreamSynchronize(h->stream), "sync");
    return 0;
}

// Asynchronous upload on `stream`: host -> staging buffer, then the compute
// stream takes it over as u at this point of its order (a device copy). The
// same hand-over as od_set_state_async, so both bench arms pipeline their
// host copies alike.
int refh_set_state_async(refh* h, const void* host, size_t bytes, void* stream) {
    if (!stream) return refh_set_state(h, host, bytes);
    if (bytes != h->state_size * h->us) return -3;
    CK(h, drv.cuCtxSetCurrent(h->ctx), "ctx");
    if (!h->stage) {
        CK(h, drv.cuMemAlloc(&h->stage, bytes), "alloc staging buffer");
        CK(h, drv.cuEventCreate(&h->ev_staged, 2 /* CU_EVENT_DISABLE_TIMING */), "event");
        CK(h, drv.cuEventCreate(&h->ev_taken, 2), "event");
        CK(h, drv.cuEventRecord(h->ev_taken, h->stream), "event record");
    }
    CUstream s = (CUstream)stream;
    CK(h, drv.cuStreamWaitEvent(s, h->ev_taken, 0), "wait");
    CK(h, drv.cuMemcpyHtoDAsync(h->stage, host, bytes, s), "upload");
    CK(h, drv.cuEventRecord(h->ev_staged, s), "event record");
    CK(h, drv.cuStreamWaitEvent(h->stream, h->ev_staged, 0), "wait");
    CK(h, drv.cuMemcpyDtoDAsync(h->u, h->stage, bytes, h->stream), "take over");
    CK(h, drv.cuEventRecord(h->ev_taken, h->stream), "event record");
    return 0;
}

// Asynchronous download on `stream` of u as of this point of the compute
// stream, through a device snapshot (as od_get_state_async).
int refh_get_state_async(refh* h, void* host, size_t bytes, void* stream) {
    if (!stream) return refh_get_state(h, host, bytes);
    if (bytes != h->state_size * h->us) return -3;
    CK(h, drv.cuCtxSetCurrent(h->ctx), "ctx");
    if (!h->snap) {
        CK(h, drv.cuMemAlloc(&h->snap, bytes), "alloc snapshot buffer");
        CK(h, drv.cuEventCreate(&h->ev_snap, 2), "event");
        CK(h, drv.cuEventCreate(&h->ev_copied, 2), "event");
        CK(h, drv.cuEventRecord(h->ev_copied, h->stream), "event record");
    }
    CUstream s = (CUstream)stream;
    CK(h, drv.cuStreamWaitEvent(h->stream, h->ev_copied, 0), "wait");
    CK(h, drv.cuMemcpyDtoDAsync(h->snap, h->u, bytes, h->stream), "snapshot");
    CK(h, drv.cuEventRecord(h->ev_snap, h->stream), "event record");
    CK(h, drv.cuStreamWaitEvent(s, h->ev_snap, 0), "wait");
    CK(h, drv.cuMemcpyDtoHAsync(host, h->snap, bytes, s), "download");
    CK(h, drv.cuEventRecord(h->ev_copied, s), "event record");
    return 0;
}

// which: 0 u, 1 u_prev, 2 rhs, 3..8 slices (xl xr yl yr zl zr), 9..14 j (xl xr yl yr zl zr)
int refh_read(refh* h, int which, void* host, size_t bytes) {
    CK(h, drv.cuCtxSetCurrent(h->ctx), "ctx");
    CK(h, drv.cuStreamSynchronize(h->stream), "sync");
    CUdeviceptr src;
    size_t need;
    if (which == 0) { src = h->u; need = h->state_size * h->us; }
    else if (which == 1) { src = h->u_prev; need = h->state_size * h->us; }
    else if (which == 2) { src = h->rhs; need = h->state_size * h->rs; }
    else if (which >= 3 && which < 9) { src = h->sl[which - 3]; need = h->nelem * 16 * 12 * h->cs; }
    else if (which >= 9 && which < 15) { src = h->j[which - 9]; need = h->nelem * 16 * 5 * h->cs; }
    else return -1;
    if (bytes != need) return -3;
    CK(h, drv.cuMemcpyDtoH(host, src, bytes), "read");
    return 0;
}

// launch_rhs_stage on the current u
int refh_rhs_stage(refh* h) {
    CK(h, drv.cuCtxSetCurrent(h->ctx), "ctx");
    return rhs_stage(h);
}

// launch_rk_stage: stage1 -> dst u_prev, src u; else dst u, src u_prev
int refh_rk(refh* h, int stage1, double a, double b, double c) {
    CK(h, drv.cuCtxSetCurrent(h->ctx), "ctx");
    if (stage1) return rk_stage(h, true, h->u_prev, h->u, a, b, c);
    return rk_stage(h, false, h->u, h->u_prev, a, b, c);
}

int refh_swap(refh* h) {
    std::swap(h->u, h->u_prev);
    return 0;
}

// n SSP-RK3 steps exactly as solver.rs:262-317; dt is the config's f32 value.
int refh_step(refh* h, int n, float dt_cfg) {
    CK(h, drv.cuCtxSetCurrent(h->ctx), "ctx");
    const bool c64 = h->p.c_f64;
    const double dt = in_c(c64, (double)dt_cfg);
    const double c2 = in_c(c64, in_c(c64, 0.25) * dt);
    const double c3 = in_c(c64, in_c(c64, 2.0 / 3.0) * dt);
    for (int s = 0; s < n; ++s) {
        if (int r = rhs_stage(h)) return r;
        if (int r = rk_stage(h, true, h->u_prev, h->u, 1.0, 0.0, dt)) return r;
        std::swap(h->u, h->u_prev);
        if (int r = rhs_stage(h)) return r;
        if (int r = rk_stage(h, false, h->u, h->u_prev, 0.75, 0.25, c2)) return r;
        if (int r = rhs_stage(h)) return r;
        if (int r = rk_stage(h, false, h->u, h->u_prev, in_c(c64, 1.0 / 3.0), in_c(c64, 2.0 / 3.0), c3)) return r;
    }
    return 0;
}

int refh_sync(refh* h) {
    CK(h, drv.cuCtxSetCurrent(h->ctx), "ctx");
    CK(h, drv.cuStreamSynchronize(h->stream), "sync");
    return 0;
}

// Device time of n steps (CUDA events on the harness stream).
int refh_time_steps(refh* h, int n, float dt_cfg, float* ms) {
    CK(h, drv.cuCtxSetCurrent(h->ctx), "ctx");
    if (h->ev.empty()) {
        CUevent a, b;
        CK(h, drv.cuEventCreate(&a, 0), "event");
        CK(h, drv.cuEventCreate(&b, 0), "event");
        h->ev = {a, b};
    }
    CK(h, drv.cuEventRecord(h->ev[0], h->stream), "record");
    if (int r = refh_step(h, n, dt_cfg)) return r;
    CK(h, drv.cuEventRecord(h->ev[1], h->stream), "record");
    CK(h, drv.cuStreamSynchronize(h->stream), "sync");
    CK(h, drv.cuEventElapsedTime(ms, h->ev[0], h->ev[1]), "elapsed");
    return 0;
}

int refh_rk_block(refh* h) { return (int)h->rk_block; }

int refh_launches_per_step(refh* h) { return 3 * (h->p.y_wall ? 6 : 5); }

}  // extern "C"
