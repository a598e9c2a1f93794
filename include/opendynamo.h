/*
 * opendynamo-b200 — C ABI of the B200 (sm_100a) FR P=3 compressible
 * Navier–Stokes step path.
 *
 * The reference (drunkseal/opendynamo) has no library boundary: its Rust host
 * NVRTC-compiles four CUDA sources and launches seven kernels by name
 * (src/solver.rs:432-461, 610-738). This header is the boundary that replaces
 * that source-level coupling. A host — the bundled C++ runner, the Python
 * package, or a Rust `solver.rs` through `extern "C"` — owns the step loop's
 * policy (labels, dumps, checkpoints; src/solver.rs:319-330, 745-818) and
 * calls these entry points for everything that touches the device.
 *
 * Conventions
 *  - Every function returns 0 on success or a negative OD_ERR_* code; the
 *    message of the last failure is kept per context (od_last_error). No
 *    exceptions cross the ABI.
 *  - State layout is the reference's (src/cuda/rhs.cu:352-361, README
 *    layout notes): 5 var-major planes rho, rho*u, rho*v, rho*w, E; inside a
 *    plane element-major blocks of 64 points, point = i + 4 j + 16 k,
 *    element = ex + nx*ey + nx*ny*ez. Values are of the u_real type.
 *  - All device work of a context is ordered on its own CUDA stream; calls
 *    on one context must come from one thread at a time.
 */
#ifndef OPENDYNAMO_H
#define OPENDYNAMO_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { OD_FLUX_SLAU2 = 0, OD_FLUX_AUSMPLUS = 1, OD_FLUX_RUSANOV = 2 };
enum { OD_F32 = 0, OD_F64 = 1 };
enum {
    OD_OK = 0,
    OD_ERR_ARG = -1,    /* invalid argument or unsupported combination */
    OD_ERR_CUDA = -2,   /* a CUDA call failed (see od_last_error) */
    OD_ERR_SIZE = -3,   /* buffer size does not match the mesh */
    OD_ERR_STATE = -4,  /* call out of order (e.g. no state set) */
    OD_ERR_IO = -5,     /* state-file read/write failure */
    OD_ERR_SCRATCH = -6 /* od_rhs_noalloc: the mesh needs more than OD_NOALLOC_SCRATCH_BYTES */
};

typedef struct od_ctx od_ctx;

/* Solver parameters. Mirrors the reference's config schema (src/config.rs)
 * plus the compile-time constants it hardcodes (src/cuda/constants.cuh). */
typedef struct od_params {
    int nx, ny, nz;                /* elements per axis ([mesh] nx ny nz) */
    double lx, ly, lz;             /* box extents; the reference stores them as f32 (config.rs:19-25) */
    int flux;                      /* OD_FLUX_* ([solver] flux_scheme) */
    int y_wall;                    /* 1 = slip walls at y = +-ly/2, 0 = periodic ([physics] y_boundary) */
    int u_real, q_real, rhs_real, compute_real; /* OD_F32 / OD_F64 ([precision] table) */
    int mixed;                     /* 1 = precision form: f64 state, RK and pressure recovery with
                                      f32 fluxes; requires u_real = f64, compute_real = f32 */
    int fast_math;                 /* 1 = approximate f32 division / square root, as the reference's
                                      default --use_fast_math build ([solver] fast_math); f64 unaffected */
    double mu;                     /* dynamic viscosity; reference constant 1.6e-4 (constants.cuh:42) */
    double forcing;                /* source added to the rho*u RHS; reference 1e-3 (rhs.cu:508) */
    int device;                    /* CUDA device ordinal */
    int ref_compat;                /* OD_COMPAT_* bits: reproduce reference arithmetic quirks (default 0) */
    int viscosity_model;           /* OD_VISC_CONSTANT (reference) or OD_VISC_SUTHERLAND (extension) */
    double t_ref, s_suth;          /* Sutherland reference temperature and constant, K ([physics] t_ref
                                      s_suth; defaults 273.15, 110.4) */
} od_params;

/* Viscosity models. The reference parses [physics] viscosity_model but its
 * kernels always use the constant MU_REF (constants.cuh:42); Sutherland's law
 * mu = mu * T^1.5 (1 + S) / (T + S), T = gamma p / rho, S = s_suth / t_ref,
 * is an extension selected explicitly. */
enum { OD_VISC_CONSTANT = 0, OD_VISC_SUTHERLAND = 1 };

/* ref_compat bits. OD_COMPAT_Y_SLICE_F32: the reference builds its y-face
 * gradient slices with __fmul_rn, a float intrinsic, also in its f64
 * pipeline (src/cuda/rhs.cu:145-160), which rounds those products and sums
 * to f32. With this bit an f64-compute run does the same, for bit-level
 * agreement with the reference's f64 results; without it the f64 pipeline
 * is f64 throughout (more accurate). */
enum { OD_COMPAT_Y_SLICE_F32 = 1 };

/* Reference defaults: SLAU2, slip walls, all f32, mu 1.6e-4 constant, forcing 1e-3. */
void od_default_params(od_params* p);

/* Layout checks for hosts that declare od_params themselves (a Rust
 * #[repr(C)] struct, ctypes): sizeof(od_params) as compiled into the
 * library, and the ABI version, raised whenever a struct of this header
 * changes its fields. No counterpart in the reference (its host and kernels
 * are compiled together, src/solver.rs:380-447). */
#define OD_ABI_VERSION 2
size_t od_params_size(void);
int od_abi_version(void);

/* Allocate device buffers and prepare the kernels.
 * Replaces: run_solver_generic setup — compile_module / load_kernels /
 * setup_fr_operators / allocate_buffers (src/solver.rs:147-159, 432-601). */
int od_create(const od_params* p, od_ctx** out);

/* Release everything the context owns. */
void od_destroy(od_ctx* ctx);

/* Bytes of one full state (5 planes of nx*ny*nz*64 u_real values). */
size_t od_state_bytes(const od_ctx* ctx);

/* Host -> device state upload (blocking).
 * Replaces: the initial-state upload stream.memcpy_htod (src/solver.rs:197-201). */
int od_set_state(od_ctx* ctx, const void* host, size_t bytes);

/* Device -> host state download (blocking w.r.t. the context's stream).
 * Replaces: the dump copy io_stream.memcpy_dtoh (src/solver.rs:757-759). */
int od_get_state(od_ctx* ctx, void* host, size_t bytes);

/* Asynchronous download: the state as of this point of the context's stream
 * goes to `host` (pinned for a truly asynchronous copy) on `stream`; the call
 * returns at once and later od_step calls may run meanwhile — the copy reads
 * a device snapshot taken on the context's stream. The data is in `host` once
 * `stream` has passed this point (synchronise it or an event on it). A null
 * stream makes it od_get_state. One snapshot per context: a second call
 * waits, on the device, for the first download to finish.
 * Replaces: the dump copy on the IO stream with its event hand-off
 * (src/solver.rs:161-175, 745-759). */
int od_get_state_async(od_ctx* ctx, void* host, size_t bytes, void* stream);

/* Asynchronous upload: `host` (pinned for a truly asynchronous copy) is
 * copied to a device staging buffer on `stream`, and the context's stream
 * takes it over as its state at this point of its order (a device copy); the
 * call returns at once. The upload may overlap steps enqueued earlier; it
 * waits, on the device, until the previous asynchronous upload has been taken
 * over. `host` must stay unchanged until `stream` has passed this point. A
 * null stream makes it od_set_state. With od_get_state_async on another
 * stream, a host pipelines independent runs: the next run's upload and the
 * last run's download overlap the steps in between.
 * Replaces: the initial-state upload stream.memcpy_htod (src/solver.rs:197-201),
 * for hosts that run many initial states back to back. */
int od_set_state_async(od_ctx* ctx, const void* host, size_t bytes, void* stream);

/* Same as above from / to device memory (stream-ordered, no host sync). */
int od_set_state_device(od_ctx* ctx, const void* dptr, size_t bytes);
int od_get_state_device(od_ctx* ctx, void* dptr, size_t bytes);

/* Enqueue n SSP-RK3 steps of size dt on the context's stream (asynchronous).
 * Pass dt exactly as the reference does: the configured f32 value widened.
 * Replaces: the per-step launch sequence launch_rhs_stage + launch_rk_stage
 * x 3 (src/solver.rs:262-317, 610-738). */
int od_step(od_ctx* ctx, int n_steps, double dt);

/* Full right-hand side (volume RHS + lifted face corrections) of the current
 * state into device memory of the u_real type (asynchronous).
 * Replaces: one launch_rhs_stage followed by the RHS+correction sum of
 * rk.cu:12-25, exposed for tests and the learned closure. */
int od_rhs(od_ctx* ctx, void* d_out, size_t bytes);

/* Wait for the context's stream. */
int od_sync(od_ctx* ctx);

/* The context's cudaStream_t (for events and stream-ordered interop). */
void* od_stream(od_ctx* ctx);

/* Kernel launches od_step enqueues per step (for launch accounting). */
int od_launches_per_step(const od_ctx* ctx);

/* Launch shape: elements per thread block of the phase-A kernel (2 or 4;
 * 16 threads per element) and of phase B: 8 or 16 with a thread per x-line
 * (all five variables), or 2 or 4 with a thread per x-line and variable (80
 * threads per element). Default 4 / 2 (fastest measured on B200). The
 * phase-B shape and the z-slab setting do not change results; the two
 * phase-A shapes are separate kernels and agree to round-off (the compiler
 * may contract a multiply-add differently). */
int od_set_launch_shape(od_ctx* ctx, int elems_per_block_a, int elems_per_block_b);

/* z-slab pipeline: each stage runs phase A slab by slab on the context's
 * stream and phase B of a slab on a second stream as soon as its z
 * neighbours are done, overlapping phase B's memory traffic with phase A's
 * arithmetic. slabs = 1 disables it, 0 restores the default (1: on B200 the
 * pipeline measured slower, phase A alone already fills every SM). Results
 * do not depend on it. */
int od_set_pipeline_slabs(od_ctx* ctx, int slabs);

/* ------------------------------------------------------------------------
 * z-slab domain decomposition: a mesh split along z over several contexts
 * (one per GPU, or several on one), exchanging one layer of halo per phase.
 * No counterpart in the reference (its solver runs one GPU).
 * ------------------------------------------------------------------------ */

/* Context for the z-layers z0 .. z1-1 of the mesh `params` (0 <= z0 < z1 <=
 * nz). It holds those layers plus a ghost layer below and above; its state
 * (od_state_bytes, od_set_state / od_get_state and the device variants) is
 * the owned layers only, 5 planes of nx*ny*64*(z1-z0) values. Element size
 * and Jacobians are those of the whole mesh, z is periodic across the slabs.
 * od_step, od_rhs, od_diagnostics and od_attach_closure are not available on
 * it: it steps stage by stage with od_slab_stage and the halo calls below. */
int od_create_slab(const od_params* params, int z0, int z1, od_ctx** out);

/* Phase A (phase 0) or phase B (phase 1) of SSP-RK3 stage `stage` (0..2) on
 * the owned layers, enqueued on the context's stream. One stage is:
 *   exchange kind 0 (the stage's input state), phase A,
 *   exchange kind 1 (the z-face records phase A wrote), phase B.
 * An exchange: od_slab_pack(dir 0) goes to the slab below, od_slab_pack(dir 1)
 * to the slab above; the receiver calls od_slab_unpack with the same dir
 * (dir 0: a message that travelled down, into the top ghost layer; dir 1: up,
 * into the bottom ghost layer). With one slab, its own messages return to it.
 * Results equal od_step on the whole mesh bit for bit. */
int od_slab_stage(od_ctx* ctx, int stage, int phase, double dt);

/* Bytes of one halo message: kind 0 = a z-layer of the state (5 x nx*ny*64
 * state values), kind 1 = the layer's z-face records (dir 0: nx*ny*80, dir 1:
 * nx*ny*64 compute-type values). 0 for invalid arguments. */
size_t od_slab_halo_bytes(const od_ctx* ctx, int kind, int dir);

/* Copy a halo message out of (pack) / into (unpack) the context: device
 * buffers of od_slab_halo_bytes, enqueued on `stream` (null: the context's
 * stream, ordered with its phases). */
int od_slab_pack(od_ctx* ctx, int stage, int kind, int dir, void* d_dst, void* stream);
int od_slab_unpack(od_ctx* ctx, int stage, int kind, int dir, const void* d_src, void* stream);

/* n SSP-RK3 steps of a whole decomposed mesh whose n slab contexts are all
 * in this process (slabs[r] holds the layers just below slabs[r+1]'s; z
 * periodic; one device or several): every exchange is a device copy
 * straight from a neighbour's boundary layer into the ghost layer it fills,
 * ordered across the slabs' streams by events, so the host enqueues a whole
 * step with no wait. Asynchronous (od_sync each slab). Results equal od_step
 * on the whole mesh bit for bit. No reference counterpart. */
int od_slabs_step(od_ctx* const* slabs, int n, int n_steps, double dt);

/* Per-kernel timing: when enabled, every stage records CUDA events around its
 * phase-A and phase-B kernels; od_timing sums the recorded intervals since the
 * last reset (synchronizes the stream). */
int od_set_timing(od_ctx* ctx, int enabled);
int od_timing(od_ctx* ctx, double* ms_phase_a, double* ms_phase_b, long long* n_stages);

/* Full right-hand side of a device-resident state without allocating
 * anything: no context, no cudaMalloc / cudaFree, no allocating library call.
 * No counterpart in the reference (its host allocates every buffer up front);
 * it serves callers that cannot allocate device memory when they need an RHS,
 * e.g. code inside another framework's step callback that owns the device
 * memory, or fixed-footprint loops. The caller passes the state (d_state, 5
 * planes of u_real) and the output (d_rhs, same size, not aliasing d_state) in
 * device memory; the result equals od_rhs on a context with the same params.
 * The kernels' only scratch, the per-face viscous and interface fluxes, lives
 * in one static device array of OD_NOALLOC_SCRATCH_BYTES per GPU (held until
 * exit), which limits the mesh to OD_NOALLOC_SCRATCH_BYTES /
 * (432 * sizeof(compute type)) elements (9709 in f32 compute, 4854 in f64);
 * larger meshes return
 * OD_ERR_SCRATCH. All calls share the array: calls whose kernels overlap on
 * the GPU race, so order them on one stream. The first call on a device looks
 * up the array's device address (cudaGetSymbolAddress) and sets the kernels'
 * shared-memory limits; make it before any stream capture. With CUDA's lazy
 * module loading that first call (per device and precision combination) is
 * also where the driver loads the kernels and places the array in device
 * memory, so it can take device memory: make it during initialisation,
 * outside any window in which allocation is forbidden; later calls allocate
 * nothing. Runs on
 * params->device (the caller's current device is restored) and enqueues on
 * `stream` (cudaStream_t, null = legacy default stream); returns before the
 * kernels finish. */
#define OD_NOALLOC_SCRATCH_BYTES (16u * 1024u * 1024u)
int od_rhs_noalloc(const od_params* params, const void* d_state, void* d_rhs, size_t bytes, void* stream);

/* Message of the last failure on this context ("" if none). */
const char* od_last_error(const od_ctx* ctx);

/* Diagnostics of the current state (synchronous). Gauss-Legendre quadrature
 * of the solution points; the vorticity uses element-local FR derivatives.
 *   vol6 = { int rho, int rho*u, int E, int 1/2 rho |u|^2,
 *            int 1/2 rho |curl u|^2, volume }
 *   prof (may be null; prof_len >= ny*4*8): x-z plane averages at the y of
 *   every solution-point row (row = 4*ey + j, bottom to top), 8 per row:
 *   <rho> <u> <v> <w> <u u> <v v> <w w> <u v>, u = rho*u / rho etc. The
 *   mean profile is <u>; Reynolds stresses are <u u> - <u><u> etc.
 * No reference counterpart (the reference reports only min/max of rho and
 * u at the end of a run, solver.rs:820-840); used for the precision-form
 * drift figures and the closure's evaluation. */
int od_diagnostics(od_ctx* ctx, double* vol6, double* prof, size_t prof_len);

/* ------------------------------------------------------------------------
 * Solver-native state files (HDF5; src/io.rs). Host-only, no device work.
 * A file holds /data/{rho,rhou,rhov,rhow,E} as 1-D datasets of nx*ny*nz*64
 * values of the state type, plus root attributes nx ny nz fr_order step
 * (u64), t lx ly lz (f64) and u_real ("f32"/"f64", fixed 3-byte ASCII).
 * The writer emits the HDF5 "earliest" format libhdf5 writes by default;
 * the reader accepts that format as libhdf5 writes it (continuation blocks,
 * multi-level chunk indexes). Errors are kept per thread (od_state_error).
 * ------------------------------------------------------------------------ */

/* Write a state file (atomically: <path>.tmp, then rename).
 * planes: 5 planes of the state type (u_f64 ? double : float), var-major as
 * the device holds them. compression: "none" (contiguous), "gzip1".."gzip9"
 * (262144-element chunks, shuffle + deflate), "blosc-lz4" (clevel 9) or
 * "blosc-zstd" (clevel 5) (HDF5 filter 32001, byte shuffle; needs
 * liblz4.so.1 / libzstd.so.1 at run time). lx, ly, lz: the f32 extents
 * widened, as the reference stores them.
 * Replaces: save_state_h5 (src/io.rs:59-136) and parse_compression
 * (src/io.rs:32-52); same file layout, attributes and error text. */
int od_state_save(const char* path, const void* planes, int u_f64, int nx, int ny, int nz,
                  unsigned long long step, double t, double lx, double ly, double lz,
                  const char* compression);

/* Read a state file's attributes (any pointer may be null). u_real4 receives
 * the precision tag, NUL-terminated. */
int od_state_info(const char* path, int* nx, int* ny, int* nz, int* fr_order,
                  unsigned long long* step, double* t, double* lx, double* ly, double* lz,
                  char* u_real4);

/* Validating load into planes_out (bytes = 5 * nx*ny*nz*64 * sizeof(state
 * type)): the file's mesh, fr_order (3) and u_real must match, else
 * OD_ERR_SIZE with the reference's message. Returns the file's step label
 * and time. Planes are read in their stored type: an f64 file loads exactly
 * (the reference reads every plane through f32, src/io.rs:221, so its f64
 * resume rounds; here it is exact).
 * Replaces: load_state_h5 (src/io.rs:163-234). */
int od_state_load(const char* path, void* planes_out, size_t bytes, int expect_u_f64,
                  int nx, int ny, int nz, unsigned long long* step, double* t);

/* Message of this thread's last state-file failure. */
const char* od_state_error(void);

/* ------------------------------------------------------------------------
 * Initial states (host only, no device work): the reference's IC generator
 * (scripts/make_initial_state.py:122-241) without Python, plus the
 * Taylor-Green vortex.
 * ------------------------------------------------------------------------ */
enum { OD_IC_CHANNEL = 0, OD_IC_UNIFORM = 1, OD_IC_TAYLOR_GREEN = 2 };

typedef struct od_ic_params {
    int nx, ny, nz;                /* elements per axis */
    double lx, ly, lz;             /* [mesh] extents as configured (rounded to f32 here, as the script does) */
    double mach_bulk;              /* [physics] mach_bulk (Taylor-Green: the velocity amplitude v0) */
    int initial_condition;         /* OD_IC_* ([physics] initial_condition; Taylor-Green is an extension) */
    double perturbation_amplitude; /* [physics] perturbation_amplitude (0: no trip) */
    int perturbation_modes;        /* [physics] perturbation_modes */
    int perturbation_seed;         /* [physics] perturbation_seed */
} od_ic_params;

/* Five planes (rho, rho*u, rho*v, rho*w, E) of nx*ny*nz*64 values (double if
 * u_f64, else float) into `planes` (bytes = 5 * nx*ny*nz*64 * size). Channel
 * and uniform states in the script's float32 arithmetic: without a trip
 * they equal the script's bit for bit. The trip's sines and cosines are
 * correctly rounded float32 values where the script takes numpy's (which
 * differ in about 15% of arguments), and its hash amplifies such a
 * difference, so a tripped state is a trip of the same construction and
 * amplitude, not the script's bits. Taylor-Green (double, on [0,lx]x[0,ly]x
 * [0,lz]): u = v0 sin x cos y cos z, v = -v0 cos x sin y cos z, w = 0,
 * rho = 1, p = 1/1.4 + v0^2/16 (cos 2x + cos 2y)(cos 2z + 2).
 * Replaces: initial_condition / apply_trip of scripts/make_initial_state.py
 * (:122-241). */
int od_make_initial_state(const od_ic_params* p, void* planes, size_t bytes, int u_f64);

/* ------------------------------------------------------------------------
 * Post-processing: the ParaView conversion of scripts/h5_to_xdmf.py.
 * ------------------------------------------------------------------------ */

/* Point fields of a state on the device (enqueued on `stream`): planes = 5
 * device planes of the state type, out = 7 device f32 arrays of
 * (4nx) x (4ny) x (4nz) points, row-major with z fastest — the reference's
 * to_tensor order (scripts/h5_to_xdmf.py:35-44): rho, rhou, rhov, rhow, E,
 * vel = sqrt(rhou^2 + rhov^2 + rhow^2) / max(rho, 1e-30) and
 * p = max(1e-7, 0.4 (E - 0.5 (rhou^2 + rhov^2 + rhow^2) / max(rho, 1e-30)))
 * (h5_to_xdmf.py:74-79), in f32 after rounding f64 planes to f32, with the
 * script's operation order. */
int od_point_fields(const void* planes, int u_f64, int nx, int ny, int nz, float* out, void* stream);

/* Point-field file: group /data with nfields 3-D f32 datasets n0 x n1 x n2
 * (row-major), chunk min(chunk, n) per dimension, compression as
 * od_state_save ("gzip4" in the conversion). */
int od_fields_save(const char* path, const float* fields, int nfields, const char* const* names,
                   long long n0, long long n1, long long n2, int chunk, const char* compression);

/* The .xmf text of a converted file (3DRectMesh of npx x npy x npz cells,
 * VXVYVZ axes linspace(0, L, n + 1), the 7 point fields as cell attributes
 * from <h5_name>:/data/<field>), h5_to_xdmf.py:87-123. Writes at most len
 * bytes (NUL-terminated) and returns the full length, or < 0. */
long long od_xdmf_text(char* buf, size_t len, const char* h5_name, int npx, int npy, int npz, double lx,
                       double ly, double lz, unsigned long long step, double t);

/* Convert one state file: <stem>.pv.h5 (the 7 point fields, chunks of 48,
 * shuffle + gzip 4) and <stem>.xmf beside it, computed on the current
 * device. out_h5 / out_xmf (may be null) receive the two paths. Returns 0,
 * or < 0 with the message in err.
 * Replaces: process() of scripts/h5_to_xdmf.py:47-143. */
int od_xdmf_convert(const char* src, char* out_h5, size_t out_h5_len, char* out_xmf, size_t out_xmf_len,
                    char* err, int err_len);

/* ------------------------------------------------------------------------
 * Run driver: the reference's run loop (src/solver.rs:139-374, 745-818) on
 * top of the entry points above. Loads [physics].initial_state, writes the
 * startup state as label S (the file's own label) at t = base_t, runs
 * n_steps SSP-RK3 steps, and after loop step k (0-based) with
 * k % save_freq == 0 or k == n_steps-1 writes <output_dir>/<prefix>_<u_real>
 * _<label:06>.h5 with label = S + k + 1 and t = base_t + (k + 1) * dt; the
 * same state also goes to checkpoint_<u_real>_<label:06>.h5 when
 * k == n_steps-1 or (checkpoint_freq > 0 and k % checkpoint_freq == 0).
 * Dumps are asynchronous: a device-side snapshot, a copy to one of three
 * pinned host buffers on a second stream and a host thread per file, so the
 * step loop waits only when all three buffers are in flight. As in the
 * reference, a failed file write is reported on stderr and the run
 * continues (counted in io_errors).
 * ------------------------------------------------------------------------ */
typedef struct od_run_opts {
    const char* initial_state;     /* [physics] initial_state (required) */
    long long n_steps;             /* [solver] n_steps */
    double dt;                     /* [solver] dt: the f32 value widened */
    long long save_freq;           /* [io] save_freq (> 0) */
    long long checkpoint_freq;     /* [io] checkpoint_freq (0 = final step only) */
    const char* compression;       /* [io] compression */
    const char* output_dir;        /* [io] output_dir (created if missing) */
    const char* prefix;            /* [io] prefix */
    int quiet;                     /* 1 = no progress lines on stdout */
} od_run_opts;

typedef struct od_run_result {
    unsigned long long start_label, final_label;
    double start_t, final_t;
    double seconds;                /* wall time of the step loop incl. waiting for the dumps */
    double ms_per_step;
    long long files_written, io_errors;
    float rho_min, rho_max, u_min, u_max; /* final physical-state report (f32, solver.rs:820-840) */
} od_run_result;

/* Run. err (may be null) receives the failure message. */
int od_run(const od_params* p, const od_run_opts* o, od_run_result* r, char* err, size_t err_len);

/* ------------------------------------------------------------------------
 * Ensembles (the batching form): independent boxes of uneven size, each with
 * its own extents, flux scheme, viscosity, forcing and time step, advanced
 * together in the f32 pipeline by ONE persistent launch per RK stage (phase
 * A of every box's elements, a grid barrier, phase B; or, in the dynamic
 * mode, tiles from a work queue with per-box phase-A counts instead of the
 * barrier) or, in the batched mode, two ordinary launches per stage over
 * every box's tiles; a step is replayed as a CUDA graph and the autotuner
 * picks the mode. Each box agrees with advancing it alone with
 * od_step to f32 round-off (same stage code; a few values differ in the last
 * bit where the compiler contracts multiply-adds differently); results are
 * deterministic and do not depend on the grid size or the graph. No
 * reference counterpart (the reference runs one box per process).
 * ------------------------------------------------------------------------ */
typedef struct od_ensemble od_ensemble;

typedef struct od_box {
    int nx, ny, nz;
    double lx, ly, lz;     /* f32 values widened */
    int flux;              /* OD_FLUX_* */
    int y_wall;            /* 1 = slip walls in y */
    double mu, forcing;    /* constant viscosity, rho*u source */
    double dt;             /* this box's time step (f32 value widened) */
} od_box;

int od_ensemble_create(const od_box* boxes, int nbox, int device, int fast_math, od_ensemble** out);
void od_ensemble_destroy(od_ensemble* e);
size_t od_ensemble_state_bytes(const od_ensemble* e, int box);
int od_ensemble_set_state(od_ensemble* e, int box, const void* host, size_t bytes);   /* f32 planes */
int od_ensemble_get_state(od_ensemble* e, int box, void* host, size_t bytes);
/* n SSP-RK3 steps of every box; waits for completion and reports a timed-out
 * grid barrier (the bounded wait's error flag) as OD_ERR_CUDA. */
int od_ensemble_step(od_ensemble* e, int n_steps);
/* The grid barrier's bounded wait: a block polls the arrival counter at most
 * spin_limit times (about 100 ns apart; 0 = the default 2^25, seconds) and
 * then sets the error flag and returns, skipping the rest of the stage;
 * od_ensemble_step then returns OD_ERR_CUDA and the states are undefined
 * until set again. extra_arrivals > 0 raises every barrier target by that
 * many arrivals, which no launch reaches: a wait that must run out, for
 * testing the error path without faulting or hanging the GPU. The call
 * also restarts the arrival counter and clears the error flag, so it is how
 * a host recovers after a timed-out barrier (od_ensemble_set_wait(e, 0, 0)).
 * No reference counterpart. */
int od_ensemble_set_wait(od_ensemble* e, long long spin_limit, int extra_arrivals);

/* Launch shape: elements per block (2 or 4; 16 threads each), blocks per SM
 * (0: all that are co-resident), CUDA graph on/off. blocks_per_sm =
 * OD_ENSEMBLE_BATCHED selects the batched mode instead of the persistent
 * launch: two ordinary launches per stage over the tiles of every box (phase
 * A at 4 elements per block, elems_per_block ignored; phase B with a thread
 * per element, variable and x-line), no grid barrier; od_ensemble_info then
 * reports blocks_per_sm = OD_ENSEMBLE_BATCHED and grid = the phase-A blocks. */
#define OD_ENSEMBLE_BATCHED (-1)
/* blocks_per_sm = OD_ENSEMBLE_DYNAMIC: one persistent launch per stage whose
 * blocks (all that are co-resident) take phase-A and phase-B tiles from a
 * ticket queue; a phase-B tile waits (bounded, od_ensemble_set_wait) only
 * for its own box's phase A, so there is no grid barrier. Up to 64 boxes;
 * elems_per_block ignored (4). */
#define OD_ENSEMBLE_DYNAMIC (-2)
int od_ensemble_set_shape(od_ensemble* e, int elems_per_block, int blocks_per_sm, int use_graph);
int od_ensemble_info(const od_ensemble* e, int* elems_per_block, int* blocks_per_sm, int* grid, int* graph);
/* Autotuner: times every candidate shape for trial_steps steps on the
 * ensemble itself (states restored afterwards), keeps the fastest; report
 * (may be null) receives one line per candidate. */
int od_ensemble_autotune(od_ensemble* e, int trial_steps, char* report, size_t report_len);
const char* od_ensemble_last_error(const od_ensemble* e);
void* od_ensemble_stream(od_ensemble* e);

/* BF16 tensor-core GEMM of the closure network (tcgen05, fp32 accumulation
 * in tensor memory): C[M x N] (+ bias[N]) = A[M x K] * B[N x K]^T, A and B
 * bf16 row-major in device memory, C fp32. M % 128 == 0, N % 64 == 0,
 * K % 64 == 0. Synchronous on `stream`. Exposed for tests; the closure uses
 * the same kernel with fused epilogues. No reference counterpart. */
int od_gemm_bf16(int M, int N, int K, const void* dA, const void* dB, float* dC, const float* dbias, void* stream);

/* Self-test of the bounded mbarrier wait that every tcgen05 kernel of the
 * closure uses (copies and MMAs signal mbarriers; a wait gives up after a
 * poll limit, sets the kernel's error flag and returns). One block on
 * `device`: a wait on a barrier nothing arrives on, with `limit` polls, must
 * give up (*first_completed = 0); after one arrival the same wait must
 * complete (*second_completed = 1). Synchronous. No reference counterpart. */
int od_mlp_wait_selftest(long long limit, int device, int* first_completed, int* second_completed);

/* ------------------------------------------------------------------------
 * Learned closure (no reference counterpart): a per-element MLP
 * 896 -> 256 -> 256 -> 256 -> 320 (GELU) whose output, scaled per variable,
 * is added to the RHS of an under-resolved coarse run. Inputs: 64 points x
 * (5 conserved + 9 velocity gradients du_i/dx_j) per element, standardised
 * with per-channel constants. BF16 weights and activations, fp32
 * accumulation on the tcgen05 tensor cores; fp32 master weights and Adam.
 * Parameters (flat fp32): W1 [256 x 896], b1 [256], W2 [256 x 256], b2,
 * W3 [256 x 256], b3, W4 [384 x 256], b4 [384] (rows 320..383 of the last
 * layer are padding and stay zero). Output column v*64 + p corrects
 * variable v at point p.
 * ------------------------------------------------------------------------ */
typedef struct od_mlp od_mlp;
int od_mlp_create(int max_rows, int device, od_mlp** out);
void od_mlp_destroy(od_mlp* m);
const char* od_mlp_last_error(const od_mlp* m);
long long od_mlp_param_count(const od_mlp* m);
int od_mlp_set_params(od_mlp* m, const float* host_params);   /* also resets Adam */
int od_mlp_get_params(od_mlp* m, float* host_params);
/* Y [rows x 384] fp32 = network(X [rows x 896] bf16), device pointers, rows % 128 == 0 */
int od_mlp_forward(od_mlp* m, const void* X, int rows, float* Y);
/* gradients (host, flat layout) of mean((Y - T)^2) over the first `valid`
 * rows and 320 columns; X, XT = X^T [896 x rows] bf16, T [rows x 384] fp32 */
int od_mlp_gradients(od_mlp* m, const void* X, const void* XT, const float* T, int rows, int valid, float* grads,
                     double* loss);
/* one Adam step (lr; betas 0.9, 0.999) on the rows `rows_host` of device
 * pools Xpool [n x 896] bf16 / Tpool [n x 320] bf16; loss = batch MSE */
int od_mlp_train_step(od_mlp* m, const void* Xpool, const void* Tpool, const long long* rows_host, int batch,
                      float lr, double* loss);
/* input standardisation (x - mean) / scale per channel (14) and output scale per variable (5) */
int od_mlp_set_scaling(od_mlp* m, const float* mean14, const float* scale14, const float* out_scale5);
/* Inference inside an attached f32 solver as one fused kernel per stage (on,
 * the default: all four layers per 128-element tile, activations kept in
 * shared memory, output added into the RHS) or as four GEMM launches (off).
 * Results agree to bf16 round-off of the same operands. */
int od_mlp_set_fused(od_mlp* m, int on);
/* Attach (m != null) or detach the network to a solver: every RK stage of
 * od_step then runs phase A, features of the stage's state (written by phase
 * A itself for the fused network with constant viscosity), the network,
 * rhs += out_scale * output, phase B. Needs an f32 state. The network must
 * outlive the attachment. */
int od_attach_closure(od_ctx* ctx, od_mlp* m);

/* Data kernels on caller-owned device memory, enqueued on `stream`:
 * L2 projection of a fine state (5 planes, mesh factor*nxc x factor*nyc x
 * factor*nzc) onto the coarse nxc x nyc x nzc P=3 basis (exact for the
 * piecewise-cubic fine field) ... */
int od_project(const void* src, int src_f64, int nxc, int nyc, int nzc, int factor, void* dst, int dst_f64,
               void* stream);
/* ... the network's standardised bf16 feature rows [nelem x 896] of a state ... */
int od_closure_features(const void* state, int u_f64, int nx, int ny, int nz, double lx, double ly, double lz,
                        const float* mean14, const float* scale14, void* X, void* stream);
/* ... and an fp32 -> bf16 conversion. */
int od_f32_to_bf16(const float* a, void* b, long long n, void* stream);

/* FR P=3 operator tables in double, as src/fr_math.rs:107-142 builds them:
 * points[4], D[16] (D[i*4+j] = l'_j(x_i)), extrap_left[4], extrap_right[4],
 * g_left'[4], g_right'[4]. */
int od_fr_tables(double* out36);

#ifdef __cplusplus
}
#endif

#endif /* OPENDYNAMO_H */
