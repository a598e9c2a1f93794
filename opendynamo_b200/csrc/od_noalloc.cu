// od_rhs_noalloc: the full right-hand side of a device-resident state,
// without allocating anything (declared in include/opendynamo.h).
//
// Some callers of this library cannot allocate device memory at the moment
// they need a right-hand side: code running inside another framework's step
// or plugin callback, where that framework owns the device memory and
// forbids (or would deadlock on) allocations made behind its back, and
// fixed-footprint loops that must not grow their memory after start-up. For
// them this entry point needs no context and calls no cudaMalloc, cudaFree or
// allocating library routine: the caller passes the state and the output,
// and the only scratch the kernels need — the per-face viscous and interface
// fluxes phase B reads from the neighbours — lives in the static device
// array below.
//
// The array is OD_NOALLOC_SCRATCH_BYTES (16 MiB) in every GPU that loads the
// library, held until the process exits. All calls share it and it keeps the
// last call's contents; every entry a call reads is first written by that
// same call, so nothing has to start at zero. Calls whose kernels overlap on
// the GPU (different streams, or different host threads) race on the array:
// order them on one stream or serialize them.
//
// Host code cannot pass the array's name to a kernel (in host code it is a
// host-side stand-in, not a device address). The first call on each device
// looks up the device address with cudaGetSymbolAddress, with that device
// current, and caches it; make that first call before any stream capture.
// With CUDA's lazy module loading (the default since CUDA 12.2) that first
// call is also where the driver loads this library's kernels and
// materialises the array on the device, which does take device memory: make
// the first call for each device and precision combination during
// initialisation, outside any window in which allocation is forbidden.
// Every later call allocates nothing.

#include <mutex>

#include "../../include/opendynamo.h"
#include "od_launch.h"

namespace {

static __device__ __align__(256) unsigned char g_noalloc_scratch[OD_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
void* g_scratch_ptr[kMaxDevices] = {};
bool g_prepared[kMaxDevices][5] = {};

}  // namespace

namespace od {
TablesD host_fr_tables();
}

extern "C" int od_rhs_noalloc(const od_params* p, const void* d_state, void* d_rhs, size_t bytes, void* stream) {
    if (!p || !d_state || !d_rhs) return OD_ERR_ARG;
    if (p->nx <= 0 || p->ny <= 0 || p->nz <= 0 || p->flux < 0 || p->flux > 2 || !(p->lx > 0) || !(p->ly > 0) ||
        !(p->lz > 0) || p->device < 0 || p->device >= kMaxDevices)
        return OD_ERR_ARG;
    if (p->viscosity_model != OD_VISC_CONSTANT &&
        (p->viscosity_model != OD_VISC_SUTHERLAND || !(p->t_ref > 0) || !(p->s_suth >= 0)))
        return OD_ERR_ARG;
    od::Combo combo;
    if (p->mixed) {
        if (p->u_real != OD_F64 || p->compute_real != OD_F32) return OD_ERR_ARG;
        combo = od::kMixed;
    } else if (p->u_real == OD_F32) {
        combo = p->compute_real == OD_F32 ? od::kF32 : od::kU32C64;
    } else {
        combo = p->compute_real == OD_F64 ? od::kF64 : od::kU64C32;
    }
    const bool s_double = p->u_real == OD_F64;
    const bool c_double = p->compute_real == OD_F64 && !p->mixed;
    const long long nelem = (long long)p->nx * p->ny * p->nz;
    if ((size_t)nelem * 64 * 5 * (s_double ? 8 : 4) != bytes) return OD_ERR_SIZE;
    if (d_state == d_rhs) return OD_ERR_ARG;
    // plus-face viscous fluxes (3 faces x 4 components) and minus-face
    // records F_I - 1/2 Fv (3 faces x 5 components), 16 points each, per element
    const size_t scratch = (size_t)nelem * od::kFaceWords * (c_double ? 8 : 4);
    if (scratch > (size_t)OD_NOALLOC_SCRATCH_BYTES) return OD_ERR_SCRATCH;

    int prev = 0;
    if (cudaGetDevice(&prev) != cudaSuccess) return OD_ERR_CUDA;
    if (cudaSetDevice(p->device) != cudaSuccess) return OD_ERR_CUDA;
    cudaError_t (*launch)(const od::StageLaunch&, cudaStream_t) = nullptr;
    cudaError_t (*prepare)() = nullptr;
    switch (combo) {
        case od::kF32: launch = od::launch_stage_f32; prepare = od::prepare_kernels_f32; break;
        case od::kF64: launch = od::launch_stage_f64; prepare = od::prepare_kernels_f64; break;
        case od::kU64C32: launch = od::launch_stage_u64c32; prepare = od::prepare_kernels_u64c32; break;
        case od::kU32C64: launch = od::launch_stage_u32c64; prepare = od::prepare_kernels_u32c64; break;
        default: launch = od::launch_stage_mixed; prepare = od::prepare_kernels_mixed; break;
    }
    {
        // once per device: the scratch array's device address; once per
        // device and precision: the kernels' shared-memory limits
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        if (!g_scratch_ptr[p->device]) {
            void* ptr = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
            if (e != cudaSuccess || !ptr) {
                cudaSetDevice(prev);
                return OD_ERR_CUDA;
            }
            g_scratch_ptr[p->device] = ptr;
        }
        if (!g_prepared[p->device][combo]) {
            if (prepare() != cudaSuccess) {
                cudaSetDevice(prev);
                return OD_ERR_CUDA;
            }
            g_prepared[p->device][combo] = true;
        }
    }

    od::StageLaunch L{};
    L.u_in = d_state;
    L.u0 = nullptr;
    L.u_out = d_rhs;
    L.fv = g_scratch_ptr[p->device];
    L.rhs = nullptr;  // RHS evaluation: phase B adds its terms to d_rhs in place
    L.nx = p->nx;
    L.ny = p->ny;
    L.nz = p->nz;
    L.y_wall = p->y_wall;
    L.nelem = nelem;
    L.tab = od::host_fr_tables();
    const double Ls[3] = {p->lx, p->ly, p->lz};
    const int ns[3] = {p->nx, p->ny, p->nz};
    for (int d = 0; d < 3; ++d)
        L.jac[d] = c_double ? 2.0 / (Ls[d] / (double)ns[d]) : (double)(2.0f / ((float)Ls[d] / (float)ns[d]));
    L.ra = 0.0;
    L.rb = 0.0;
    L.rc = 1.0;
    L.mu = p->mu;
    L.forcing = p->forcing;
    L.suth = p->viscosity_model == OD_VISC_SUTHERLAND ? p->s_suth / p->t_ref : -1.0;
    int flags = 0;
    if (c_double) {
        if (p->q_real == OD_F32) flags |= od::kRoundQ;
        if (p->rhs_real == OD_F32) flags |= od::kRoundRhs;
        if (p->ref_compat & OD_COMPAT_Y_SLICE_F32) flags |= od::kRefYSlice;
    }
    L.flags = flags;
    L.flux = p->flux;
    L.epb_a = 4;
    L.epb_b = 2;   // the phase-B kernel od_rhs runs (a thread per element, variable and x-line)
    L.phases = 3;
    L.e0 = 0;
    L.e1 = nelem;
    L.fast_math = p->fast_math != 0;
    cudaError_t e = launch(L, (cudaStream_t)stream);
    cudaSetDevice(prev);
    return e == cudaSuccess ? OD_OK : OD_ERR_CUDA;
}
