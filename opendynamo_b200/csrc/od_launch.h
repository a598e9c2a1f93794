// Host-side launch interface between the C-ABI layer and the templated
// stage kernels. Each precision combination is compiled in its own
// translation unit (od_inst_*.cu) so the kernel variants build in parallel.
#pragma once

#include <cuda_runtime.h>

namespace od {

enum StageFlags : int {
    kHasU0 = 1,      // out = ra*u0 + rb*u_in + rc*R (else rb*u_in + rc*R)
    kRoundQ = 2,     // round the gradient through f32 (q_real = f32 with f64 compute)
    kRoundRhs = 4,   // round the volume RHS through f32 (rhs_real = f32 with f64 compute)
    kDeferRK = 8,    // phase A stores the RHS, phase B performs the RK combination
    kRefYSlice = 16, // f64 compute: round the y-face gradient traces as the reference's __fmul_rn does
};

// Face-flux scratch per element, in compute-type words: the viscous fluxes
// of the three plus faces ([dir 3][var 1..4][face pt 16]) followed by the
// minus-face records ([dir 3][var 5][face pt 16]) F_I - 1/2 Fv_own.
constexpr int kFvWords = 3 * 4 * 16;
constexpr int kFaceWords = kFvWords + 3 * 5 * 16;

// FR operator tables in double (the host computes them once, as
// src/fr_math.rs:107-142 does, then each launch casts to its own types).
struct TablesD {
    double pts[4], D[16], eL[4], eR[4], gL[4], gR[4];
};

// The learned closure's input, written by phase A when the closure is
// attached (f32 state, constant viscosity): each element's 14 channels x 64
// points as bf16 in the fused inference kernel's tile layout, with the
// features kernel's parameters and operation order. Channels: rho, rho*u,
// rho*v, rho*w, E and d(u_a)/d(x_b); standardised inputs are clipped to
// +-kFeatClip.
constexpr int kFeatChan = 14;
constexpr float kFeatClip = 8.0f;

struct StageFeatures {
    void* X;              // bf16 tiles: [element / 128][channel][128 x 64 core-matrix layout]
    float jac[3];
    float D[16];
    float mean[kFeatChan], inv_scale[kFeatChan];
};

struct StageLaunch {
    const void* u_in;
    const void* u0;      // null on stage 1 / single RHS evaluations
    void* u_out;
    void* fv;            // face-flux scratch (kFaceWords per element)
    void* rhs;           // RHS buffer of the deferred RK combination (null otherwise)
    const StageFeatures* feat;   // phase A also writes the closure's features (null otherwise)
    int nx, ny, nz, y_wall;
    long long nelem;
    TablesD tab;
    double jac[3];       // already evaluated in the compute type
    double ra, rb, rc;   // already evaluated in the state-arithmetic type
    double mu, forcing;
    double suth;            // Sutherland S = s_suth / t_ref; < 0: constant mu
    int flags;           // kHasU0 | kRoundQ | kRoundRhs
    int flux;            // 0 slau2, 1 ausm+, 2 rusanov
    int epb_a, epb_b;    // elements per block of phase A / phase B
    bool fast_math;      // approximate f32 division / square root (the reference's default build)
    int phases;          // 1 = phase A, 2 = phase B, 3 = both (one stream)
    long long e0, e1;    // element range (a z-slab: elements are z-major)
    cudaEvent_t ev[3];   // optional timing events: before A, after A, after B
};

// Precision combination ids: stored type / state arithmetic / flux arithmetic
enum Combo : int {
    kF32 = 0,      // float / float / float
    kF64 = 1,      // double / double / double
    kU64C32 = 2,   // double / float / float   (reference pipeline with u_real = f64, compute_real = f32)
    kU32C64 = 3,   // float / double / double
    kMixed = 4,    // double / double / float  (precision form: f64 state, RK and pressure; f32 fluxes)
};

// Work run between phase A and phase B of every RK stage (the learned
// closure): reads the stage's input state, may modify the RHS buffer.
using StageHook = cudaError_t (*)(void* user, const void* u_in, void* rhs, cudaStream_t s);

}  // namespace od

struct od_mlp;

namespace od {

// the learned closure's hook and its per-mesh preparation (od_closure.cu);
// closure_stage_features fills the parameters for phase A to write the
// features itself (false: the hook computes them), closure_network_hook then
// runs the network alone
cudaError_t closure_stage_hook(void* user, const void* u_in, void* rhs, cudaStream_t s);
bool closure_stage_features(void* user, StageFeatures* out);
cudaError_t closure_network_hook(void* user, const void* u_in, void* rhs, cudaStream_t s);
int closure_prepare(od_mlp* m, int nx, int ny, int nz, double lx, double ly, double lz, bool f64);

// Diagnostics (od_diag.cu): accumulates into d_vol6 / d_prof (zeroed by the caller).
cudaError_t launch_diag(const void* u, bool u_f64, int nx, int ny, int nz, double lx, double ly, double lz,
                        const TablesD& tab, double* d_vol6, double* d_prof, cudaStream_t s);

cudaError_t launch_stage_f32(const StageLaunch& L, cudaStream_t s);
cudaError_t launch_stage_f64(const StageLaunch& L, cudaStream_t s);
cudaError_t launch_stage_u64c32(const StageLaunch& L, cudaStream_t s);
cudaError_t launch_stage_u32c64(const StageLaunch& L, cudaStream_t s);
cudaError_t launch_stage_mixed(const StageLaunch& L, cudaStream_t s);

// Set the dynamic shared-memory limits of every kernel variant once per device.
cudaError_t prepare_kernels_f32();
cudaError_t prepare_kernels_f64();
cudaError_t prepare_kernels_u64c32();
cudaError_t prepare_kernels_u32c64();
cudaError_t prepare_kernels_mixed();

}  // namespace od
