// C ABI of the FR P=3 step path (declared in include/opendynamo.h).
//
// Owns the device buffers of one solver instance and enqueues the SSP-RK3
// stages (src/solver.rs:262-317) as phase-A / phase-B kernel pairs on its own
// stream. The RK scheme needs three state buffers here instead of the
// reference's two: a phase-A kernel reads its neighbours' state while other
// blocks write their results, so a stage never writes the buffer it reads.
//   stage 1: U0 -> U1        u1 = u0 + dt L(u0)
//   stage 2: U1 (+U0) -> U2  u2 = 3/4 u0 + 1/4 u1 + 1/4 dt L(u1)
//   stage 3: U2 (+U0) -> U0  u  = 1/3 u0 + 2/3 u2 + 2/3 dt L(u2)
// Stage 3 overwrites U0 element by element: each thread reads its own
// point of U0 before writing it, and no other block reads U0 in that stage.

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include <algorithm>

#include "../../include/opendynamo.h"
#include "od_launch.h"

namespace {

// ---- FR operator tables (src/fr_math.rs:3-142), computed on the host in double
double legendre(int p, double x) {
    if (p == 0) return 1.0;
    if (p == 1) return x;
    double a = 1.0, b = x, val = 0.0;
    for (int k = 2; k <= p; ++k) {
        val = ((2.0 * k - 1.0) * x * b - (k - 1.0) * a) / (double)k;
        a = b;
        b = val;
    }
    return val;
}

double dlegendre(int p, double x) {
    if (p == 0) return 0.0;
    return (double)p / (x * x - 1.0) * (x * legendre(p, x) - legendre(p - 1, x));
}

od::TablesD build_tables() {
    od::TablesD t;
    const int n = 4, p = 3;
    for (int i = 0; i < n; ++i) {
        double x = std::cos(M_PI * (i + 0.75) / (n + 0.5));  // Newton from the Chebyshev-like guess
        for (int it = 0; it < 100; ++it) {
            double step = legendre(n, x) / dlegendre(n, x);
            x -= step;
            if (std::fabs(step) < 1e-14) break;
        }
        t.pts[i] = x;
    }
    std::sort(t.pts, t.pts + n);
    for (int i = 0; i < n; ++i) {
        for (int j = 0; j < n; ++j) {
            if (i == j) {
                double s = 0.0;
                for (int k = 0; k < n; ++k)
                    if (k != i) s += 1.0 / (t.pts[i] - t.pts[k]);
                t.D[i * n + j] = s;
            } else {
                double num = 1.0, den = 1.0;
                for (int k = 0; k < n; ++k) {
                    if (k != i && k != j) num *= t.pts[i] - t.pts[k];
                    if (k != j) den *= t.pts[j] - t.pts[k];
                }
                t.D[i * n + j] = num / den;
            }
        }
    }
    for (int i = 0; i < n; ++i) {
        double l = 1.0, r = 1.0;
        for (int j = 0; j < n; ++j) {
            if (j == i) continue;
            l *= (-1.0 - t.pts[j]) / (t.pts[i] - t.pts[j]);
            r *= (1.0 - t.pts[j]) / (t.pts[i] - t.pts[j]);
        }
        t.eL[i] = l;
        t.eR[i] = r;
        double dp = dlegendre(p, t.pts[i]), dp1 = dlegendre(p + 1, t.pts[i]);
        t.gR[i] = 0.5 * (dp + dp1);
        t.gL[i] = 0.5 * -1.0 * (dp - dp1);  // (-1)^P with P = 3
    }
    return t;
}

struct Fns {
    cudaError_t (*launch)(const od::StageLaunch&, cudaStream_t);
    cudaError_t (*prepare)();
    bool p_double, c_double, s_double;
};

Fns combo_fns(od::Combo c) {
    switch (c) {
        case od::kF32: return {od::launch_stage_f32, od::prepare_kernels_f32, false, false, false};
        case od::kF64: return {od::launch_stage_f64, od::prepare_kernels_f64, true, true, true};
        case od::kU64C32: return {od::launch_stage_u64c32, od::prepare_kernels_u64c32, false, false, true};
        case od::kU32C64: return {od::launch_stage_u32c64, od::prepare_kernels_u32c64, true, true, false};
        default: return {od::launch_stage_mixed, od::prepare_kernels_mixed, true, false, true};
    }
}

// x evaluated as the given arithmetic type
double in_type(bool dbl, double x) { return dbl ? x : (double)(float)x; }

constexpr int kMaxSlabs = 64;

// Default z-slab count: 1 (no pipeline). Measured on B200 at 48^3 f32 and
// mixed, 4 to 24 slabs were 6-35% slower per stage than 1: phase A alone
// already keeps every SM resident, so phase-B blocks only compete with it,
// and each extra launch adds a partial wave.
int auto_slabs(const od_params&) { return 1; }

}  // namespace

namespace od {
TablesD host_fr_tables() { return build_tables(); }
}  // namespace od

struct od_ctx {
    od_params p{};
    od::Combo combo = od::kF32;
    Fns fns{};
    cudaStream_t stream = nullptr;
    cudaStream_t stream_b = nullptr;          // phase B of the z-slab pipeline
    int slabs = 1;                            // z-slabs per stage (1 = no pipeline)
    std::vector<cudaEvent_t> slab_ev;         // per-slab "phase A done" + the join event
    void* U[3] = {nullptr, nullptr, nullptr};
    void* fv = nullptr;
    void* rhs = nullptr;      // deferred RK combination: RHS between phase A and phase B
    size_t state_bytes = 0;
    size_t elem_size = 4;
    long long nelem = 0;
    od::TablesD tab{};
    double jac[3] = {0, 0, 0};
    int round_flags = 0;
    bool have_state = false;
    // launch shape: 4 elements per phase-A block; phase B with a thread per
    // (element, variable, x-line), 2 elements per block (B200, 48^3 f32: phase
    // B 0.122 ms against 0.128 with a thread per x-line and 8 elements, 0.136
    // with 16; phase A 2 vs 4 equal, 8 and 16 slower: 262.6 and 274.9 against
    // 260.4 us, the larger blocks' barriers cost more than their warps gain
    // from running close together in the code)
    int epb_a = 4, epb_b = 2;
    std::string err;
    bool timing = false;
    std::vector<cudaEvent_t> events;
    size_t ev_used = 0;
    long long n_stages = 0;
    od::StageHook hook = nullptr;   // learned closure between phase A and phase B
    void* hook_user = nullptr;
    // z-slab of a decomposed mesh (od_create_slab): the local mesh holds the
    // owned layers 1 .. nz-2 and a ghost layer below and above, which the
    // caller fills between the phases (od_slab_unpack)
    bool slab = false;
    int slab_z0 = 0, slab_z1 = 0, mesh_nz = 0;   // owned z-layers [z0, z1) of a mesh of mesh_nz layers
    cudaEvent_t ev_halo[2] = {nullptr, nullptr};   // od_slabs_step: stage input ready / face records ready
    size_t buf_bytes = 0;     // one state buffer (state_bytes: the owned part the caller sees)
    // od_get_state_async: device snapshot of the state and its two events
    void* snap = nullptr;
    cudaEvent_t ev_snap = nullptr, ev_copied = nullptr;
    // od_set_state_async: device staging buffer of an upload and its two events
    void* stage = nullptr;
    cudaEvent_t ev_staged = nullptr, ev_taken = nullptr;
};

namespace {

int fail(od_ctx* c, int code, const std::string& msg) {
    if (c) c->err = msg;
    return code;
}

int cuda_fail(od_ctx* c, cudaError_t e, const char* what) {
    return fail(c, OD_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// jac = 2 / (L / n) in the compute type (rk.cu:93-95), from the mesh p
void set_jac(od_ctx* c, const od_params* p) {
    const double L3[3] = {p->lx, p->ly, p->lz};
    const int n3[3] = {p->nx, p->ny, p->nz};
    for (int d = 0; d < 3; ++d) {
        if (c->fns.c_double)
            c->jac[d] = 2.0 / (L3[d] / (double)n3[d]);
        else
            c->jac[d] = (double)(2.0f / ((float)L3[d] / (float)n3[d]));
    }
}

// The caller-visible state of a context: all of U0, or for a slab its owned
// layers (5 planes of nx*ny*64 points per owned layer, var-major).
// to_ctx: other -> U0, else U0 -> other; kind: the copy direction.
cudaError_t copy_state(od_ctx* c, void* other, bool to_ctx, cudaMemcpyKind kind) {
    if (!c->slab) {
        return to_ctx ? cudaMemcpyAsync(c->U[0], other, c->state_bytes, kind, c->stream)
                      : cudaMemcpyAsync(other, c->U[0], c->state_bytes, kind, c->stream);
    }
    const size_t layer = (size_t)c->p.nx * c->p.ny * 64 * c->elem_size;
    const size_t owned = c->state_bytes / 5, plane = c->buf_bytes / 5;
    char* u = (char*)c->U[0] + layer;
    return to_ctx ? cudaMemcpy2DAsync(u, plane, other, owned, owned, 5, kind, c->stream)
                  : cudaMemcpy2DAsync(other, owned, u, plane, owned, 5, kind, c->stream);
}

int set_device(od_ctx* c) {
    cudaError_t e = cudaSetDevice(c->p.device);
    if (e != cudaSuccess) return cuda_fail(c, e, "cudaSetDevice");
    return OD_OK;
}

// One stage: phase A (+ phase B) with the given buffers and RK coefficients.
// The launch description of one stage on the context's buffers.
od::StageLaunch make_launch(od_ctx* c, const void* u_in, const void* u0, void* u_out, double ra, double rb,
                            double rc) {
    od::StageLaunch L{};
    L.u_in = u_in;
    L.u0 = u0;
    L.u_out = u_out;
    L.fv = c->fv;
    L.rhs = c->rhs;
    L.fast_math = c->p.fast_math != 0;
    L.nx = c->p.nx;
    L.ny = c->p.ny;
    L.nz = c->p.nz;
    L.y_wall = c->p.y_wall;
    L.nelem = c->nelem;
    L.tab = c->tab;
    for (int d = 0; d < 3; ++d) L.jac[d] = c->jac[d];
    L.ra = ra;
    L.rb = rb;
    L.rc = rc;
    L.mu = c->p.mu;
    L.forcing = c->p.forcing;
    L.suth = c->p.viscosity_model == OD_VISC_SUTHERLAND ? c->p.s_suth / c->p.t_ref : -1.0;
    L.flags = c->round_flags | (u0 ? 1 : 0);
    L.flux = c->p.flux;
    L.epb_a = c->epb_a;
    L.epb_b = c->epb_b;
    return L;
}

int enqueue_stage(od_ctx* c, const void* u_in, const void* u0, void* u_out, double ra, double rb, double rc) {
    od::StageLaunch L = make_launch(c, u_in, u0, u_out, ra, rb, rc);
    cudaEvent_t tev[3] = {nullptr, nullptr, nullptr};
    if (c->timing) {
        while (c->events.size() < c->ev_used + 3) {
            cudaEvent_t ev;
            cudaError_t e = cudaEventCreate(&ev);
            if (e != cudaSuccess) return cuda_fail(c, e, "cudaEventCreate");
            c->events.push_back(ev);
        }
        for (int q = 0; q < 3; ++q) tev[q] = c->events[c->ev_used + q];
        c->ev_used += 3;
    }
    const int K = c->slabs;
    if (c->hook) {
        // phase A leaves the RHS in c->rhs (and, f32 state with constant
        // viscosity, writes the closure's features); the hook corrects the
        // RHS; phase B finishes the stage
        L.e0 = 0;
        L.e1 = c->nelem;
        L.phases = 1;
        L.ev[0] = tev[0];
        L.ev[1] = tev[1];
        L.ev[2] = nullptr;
        od::StageFeatures sf;
        const bool feat = c->combo == od::kF32 && c->p.viscosity_model == OD_VISC_CONSTANT &&
                          od::closure_stage_features(c->hook_user, &sf);
        L.feat = feat ? &sf : nullptr;
        cudaError_t e = c->fns.launch(L, c->stream);
        L.feat = nullptr;
        if (e == cudaSuccess)
            e = feat ? od::closure_network_hook(c->hook_user, u_in, c->rhs, c->stream)
                     : c->hook(c->hook_user, u_in, c->rhs, c->stream);
        if (e == cudaSuccess) {
            L.phases = 2;
            L.ev[0] = L.ev[1] = nullptr;
            L.ev[2] = tev[2];
            e = c->fns.launch(L, c->stream);
        }
        if (e != cudaSuccess) return cuda_fail(c, e, "stage launch (closure)");
        c->n_stages++;
        return OD_OK;
    }
    if (K <= 1) {
        L.phases = 3;
        L.e0 = 0;
        L.e1 = c->nelem;
        for (int q = 0; q < 3; ++q) L.ev[q] = tev[q];
        cudaError_t e = c->fns.launch(L, c->stream);
        if (e != cudaSuccess) return cuda_fail(c, e, "stage launch");
        c->n_stages++;
        return OD_OK;
    }
    // z-slab pipeline: phase A of every slab back to back on the main stream;
    // phase B of slab k on the second stream once phase A of its z neighbours
    // (slabs k-1, k+1; z is periodic) is done, so phase B's HBM traffic
    // overlaps phase A's arithmetic and its inputs are still in L2. Slab 0
    // needs slab K-1 and goes last.
    const long long per_layer = (long long)c->p.nx * c->p.ny;
    auto bounds = [&](int k, long long& e0, long long& e1) {
        e0 = (long long)k * c->p.nz / K * per_layer;
        e1 = (long long)(k + 1) * c->p.nz / K * per_layer;
    };
    cudaError_t e;
    for (int k = 0; k < K; ++k) {
        L.phases = 1;
        bounds(k, L.e0, L.e1);
        L.ev[0] = k == 0 ? tev[0] : nullptr;
        L.ev[1] = k == K - 1 ? tev[1] : nullptr;
        L.ev[2] = nullptr;
        e = c->fns.launch(L, c->stream);
        if (e != cudaSuccess) return cuda_fail(c, e, "phase A launch");
        e = cudaEventRecord(c->slab_ev[k], c->stream);
        if (e != cudaSuccess) return cuda_fail(c, e, "cudaEventRecord");
    }
    for (int q = 1; q <= K; ++q) {
        const int k = q % K;
        const int need = k == 0 ? K - 1 : (k + 1 < K ? k + 1 : K - 1);
        e = cudaStreamWaitEvent(c->stream_b, c->slab_ev[need], 0);
        if (e != cudaSuccess) return cuda_fail(c, e, "cudaStreamWaitEvent");
        L.phases = 2;
        bounds(k, L.e0, L.e1);
        L.ev[0] = L.ev[1] = nullptr;
        L.ev[2] = q == K ? tev[2] : nullptr;
        e = c->fns.launch(L, c->stream_b);
        if (e != cudaSuccess) return cuda_fail(c, e, "phase B launch");
    }
    // join: the next stage (or any later call) starts after phase B everywhere
    e = cudaEventRecord(c->slab_ev[K], c->stream_b);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(c->stream, c->slab_ev[K], 0);
    if (e != cudaSuccess) return cuda_fail(c, e, "stream join");
    c->n_stages++;
    return OD_OK;
}

// Buffers and coefficients of SSP-RK3 stage k (0..2): U0 -> U1, (U0, U1) ->
// U2, (U0, U2) -> U0, coefficients evaluated in the state-arithmetic type
// (solver.rs:256, 275-316).
struct RkStage {
    const void* u_in;
    const void* u0;
    void* u_out;
    double ra, rb, rc;
};

RkStage rk_stage(od_ctx* c, int k, double dt) {
    const bool pd = c->fns.p_double;
    const double dtp = in_type(pd, dt);
    if (k == 0) return {c->U[0], nullptr, c->U[1], 0.0, 1.0, dtp};
    if (k == 1) return {c->U[1], c->U[0], c->U[2], 0.75, 0.25, in_type(pd, in_type(pd, 0.25) * dtp)};
    return {c->U[2], c->U[0], c->U[0], in_type(pd, 1.0 / 3.0), in_type(pd, 2.0 / 3.0),
            in_type(pd, in_type(pd, 2.0 / 3.0) * dtp)};
}

}  // namespace

extern "C" {

void od_default_params(od_params* p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->nx = p->ny = p->nz = 8;
    p->lx = (double)(4.0f * (float)M_PI);
    p->ly = 2.0;
    p->lz = (double)((4.0f / 3.0f) * (float)M_PI);
    p->flux = OD_FLUX_SLAU2;
    p->y_wall = 1;
    p->u_real = p->q_real = p->rhs_real = p->compute_real = OD_F32;
    p->fast_math = 1;
    p->mu = 1.6e-4;
    p->forcing = 1e-3;
    p->viscosity_model = OD_VISC_CONSTANT;
    p->t_ref = 273.15;
    p->s_suth = 110.4;
}

size_t od_params_size(void) { return sizeof(od_params); }

int od_abi_version(void) { return OD_ABI_VERSION; }

int od_fr_tables(double* out) {
    if (!out) return OD_ERR_ARG;
    od::TablesD t = build_tables();
    std::memcpy(out, t.pts, sizeof(t.pts));
    std::memcpy(out + 4, t.D, sizeof(t.D));
    std::memcpy(out + 20, t.eL, sizeof(t.eL));
    std::memcpy(out + 24, t.eR, sizeof(t.eR));
    std::memcpy(out + 28, t.gL, sizeof(t.gL));
    std::memcpy(out + 32, t.gR, sizeof(t.gR));
    return OD_OK;
}

int od_create(const od_params* p, od_ctx** out) {
    if (!p || !out) return OD_ERR_ARG;
    *out = nullptr;
    if (p->nx <= 0 || p->ny <= 0 || p->nz <= 0 || p->flux < 0 || p->flux > 2 || !(p->lx > 0) ||
        !(p->ly > 0) || !(p->lz > 0))
        return OD_ERR_ARG;
    if (p->viscosity_model != OD_VISC_CONSTANT &&
        (p->viscosity_model != OD_VISC_SUTHERLAND || !(p->t_ref > 0) || !(p->s_suth >= 0)))
        return OD_ERR_ARG;
    long long nelem = (long long)p->nx * p->ny * p->nz;
    if (nelem >= (1LL << 31)) return OD_ERR_ARG;   // element indices are 32-bit in the kernels
    od_ctx* c = new od_ctx();
    c->p = *p;
    c->nelem = nelem;
    if (p->mixed) {
        if (p->u_real != OD_F64 || p->compute_real != OD_F32) {
            delete c;
            return OD_ERR_ARG;
        }
        c->combo = od::kMixed;
    } else if (p->u_real == OD_F32) {
        c->combo = p->compute_real == OD_F32 ? od::kF32 : od::kU32C64;
    } else {
        c->combo = p->compute_real == OD_F64 ? od::kF64 : od::kU64C32;
    }
    c->fns = combo_fns(c->combo);
    c->elem_size = c->fns.s_double ? 8 : 4;
    c->state_bytes = (size_t)nelem * 64 * 5 * c->elem_size;
    // Q / RHS rounding only bites when they are narrower than the compute type
    if (c->fns.c_double && !p->mixed) {
        if (p->q_real == OD_F32) c->round_flags |= od::kRoundQ;
        if (p->rhs_real == OD_F32) c->round_flags |= od::kRoundRhs;
    }
    if (c->fns.c_double && (p->ref_compat & OD_COMPAT_Y_SLICE_F32)) c->round_flags |= od::kRefYSlice;
    c->tab = build_tables();
    c->buf_bytes = c->state_bytes;
    set_jac(c, p);
    int rc = set_device(c);
    if (rc) {
        *out = c;
        return rc;
    }
    cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream_b, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        *out = c;
        return cuda_fail(c, e, "cudaStreamCreate");
    }
    // events of the z-slab pipeline (one per slab + the join), timing disabled
    const int max_slabs = std::min(p->nz, kMaxSlabs);
    for (int k = 0; k <= max_slabs; ++k) {
        cudaEvent_t ev;
        e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
        if (e != cudaSuccess) {
            *out = c;
            return cuda_fail(c, e, "cudaEventCreate");
        }
        c->slab_ev.push_back(ev);
    }
    c->slabs = auto_slabs(*p);
    e = c->fns.prepare();
    if (e != cudaSuccess) {
        *out = c;
        return cuda_fail(c, e, "kernel attributes");
    }
    for (int b = 0; b < 3; ++b) {
        e = cudaMalloc(&c->U[b], c->buf_bytes);
        if (e != cudaSuccess) {
            *out = c;
            return cuda_fail(c, e, "cudaMalloc state");
        }
    }
    // An f32 state is rounded once per stage: the RK combination happens in
    // phase B, phase A hands over the unrounded RHS.
    if (!c->fns.s_double) {
        e = cudaMalloc(&c->rhs, c->buf_bytes);
        if (e != cudaSuccess) {
            *out = c;
            return cuda_fail(c, e, "cudaMalloc RHS buffer");
        }
    }
    // plus-face viscous fluxes [elem][3][4][16] + minus-face records F_I - 1/2 Fv [elem][3][5][16]
    const size_t fv_bytes = (size_t)nelem * od::kFaceWords * (c->fns.c_double ? 8 : 4);
    e = cudaMalloc(&c->fv, fv_bytes);
    if (e != cudaSuccess) {
        *out = c;
        return cuda_fail(c, e, "cudaMalloc face buffer");
    }
    e = cudaMemsetAsync(c->fv, 0, fv_bytes, c->stream);
    if (e != cudaSuccess) {
        *out = c;
        return cuda_fail(c, e, "cudaMemset");
    }
    *out = c;
    return OD_OK;
}

void od_destroy(od_ctx* c) {
    if (!c) return;
    cudaSetDevice(c->p.device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->stream_b) cudaStreamSynchronize(c->stream_b);
    for (auto ev : c->events) cudaEventDestroy(ev);
    for (auto ev : c->slab_ev) cudaEventDestroy(ev);
    for (auto ev : c->ev_halo)
        if (ev) cudaEventDestroy(ev);
    for (int b = 0; b < 3; ++b)
        if (c->U[b]) cudaFree(c->U[b]);
    if (c->fv) cudaFree(c->fv);
    if (c->rhs) cudaFree(c->rhs);
    // copies still running on the caller's streams
    if (c->ev_copied) cudaEventSynchronize(c->ev_copied);
    if (c->ev_staged) cudaEventSynchronize(c->ev_staged);
    if (c->snap) cudaFree(c->snap);
    if (c->ev_snap) cudaEventDestroy(c->ev_snap);
    if (c->ev_copied) cudaEventDestroy(c->ev_copied);
    if (c->stage) cudaFree(c->stage);
    if (c->ev_staged) cudaEventDestroy(c->ev_staged);
    if (c->ev_taken) cudaEventDestroy(c->ev_taken);
    if (c->stream_b) cudaStreamDestroy(c->stream_b);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

size_t od_state_bytes(const od_ctx* c) { return c ? c->state_bytes : 0; }

int od_set_state(od_ctx* c, const void* host, size_t bytes) {
    if (!c || !host) return OD_ERR_ARG;
    if (bytes != c->state_bytes) return fail(c, OD_ERR_SIZE, "state size does not match the mesh");
    if (int rc = set_device(c)) return rc;
    cudaError_t e = copy_state(c, const_cast<void*>(host), true, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "state upload");
    c->have_state = true;
    return OD_OK;
}

int od_get_state(od_ctx* c, void* host, size_t bytes) {
    if (!c || !host) return OD_ERR_ARG;
    if (bytes != c->state_bytes) return fail(c, OD_ERR_SIZE, "state size does not match the mesh");
    if (!c->have_state) return fail(c, OD_ERR_STATE, "no state set");
    if (int rc = set_device(c)) return rc;
    cudaError_t e = copy_state(c, host, false, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "state download");
    return OD_OK;
}

int od_get_state_async(od_ctx* c, void* host, size_t bytes, void* stream) {
    if (!stream) return od_get_state(c, host, bytes);
    if (!c || !host) return OD_ERR_ARG;
    if (bytes != c->state_bytes) return fail(c, OD_ERR_SIZE, "state size does not match the mesh");
    if (!c->have_state) return fail(c, OD_ERR_STATE, "no state set");
    if (int rc = set_device(c)) return rc;
    cudaError_t e = cudaSuccess;
    if (!c->snap) {
        void* buf = nullptr;
        e = cudaMalloc(&buf, c->state_bytes);
        if (e == cudaSuccess) c->snap = buf;
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_snap, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_copied, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventRecord(c->ev_copied, c->stream);
        if (e != cudaSuccess) {
            // leave nothing half made: the next call starts over
            if (c->ev_copied) cudaEventDestroy(c->ev_copied);
            if (c->ev_snap) cudaEventDestroy(c->ev_snap);
            if (c->snap) cudaFree(c->snap);
            c->ev_copied = c->ev_snap = nullptr;
            c->snap = nullptr;
            return cuda_fail(c, e, "state snapshot buffer");
        }
    }
    cudaStream_t s = (cudaStream_t)stream;
    // the compute stream: wait until the previous download has read the
    // snapshot, take a new one (a device copy), and carry on
    e = cudaStreamWaitEvent(c->stream, c->ev_copied, 0);
    if (e == cudaSuccess) e = copy_state(c, c->snap, false, cudaMemcpyDeviceToDevice);
    if (e == cudaSuccess) e = cudaEventRecord(c->ev_snap, c->stream);
    // the caller's stream: download the snapshot
    if (e == cudaSuccess) e = cudaStreamWaitEvent(s, c->ev_snap, 0);
    if (e == cudaSuccess) e = cudaMemcpyAsync(host, c->snap, bytes, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaEventRecord(c->ev_copied, s);
    if (e != cudaSuccess) return cuda_fail(c, e, "asynchronous state download");
    return OD_OK;
}

int od_set_state_async(od_ctx* c, const void* host, size_t bytes, void* stream) {
    if (!stream) return od_set_state(c, host, bytes);
    if (!c || !host) return OD_ERR_ARG;
    if (bytes != c->state_bytes) return fail(c, OD_ERR_SIZE, "state size does not match the mesh");
    if (int rc = set_device(c)) return rc;
    cudaError_t e = cudaSuccess;
    if (!c->stage) {
        void* buf = nullptr;
        e = cudaMalloc(&buf, c->state_bytes);
        if (e == cudaSuccess) c->stage = buf;
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_staged, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_taken, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventRecord(c->ev_taken, c->stream);
        if (e != cudaSuccess) {
            // leave nothing half made: the next call starts over
            if (c->ev_taken) cudaEventDestroy(c->ev_taken);
            if (c->ev_staged) cudaEventDestroy(c->ev_staged);
            if (c->stage) cudaFree(c->stage);
            c->ev_taken = c->ev_staged = nullptr;
            c->stage = nullptr;
            return cuda_fail(c, e, "state staging buffer");
        }
    }
    cudaStream_t s = (cudaStream_t)stream;
    // the caller's stream: once the previous upload has been taken over,
    // upload into the staging buffer
    e = cudaStreamWaitEvent(s, c->ev_taken, 0);
    if (e == cudaSuccess) e = cudaMemcpyAsync(c->stage, host, bytes, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaEventRecord(c->ev_staged, s);
    // the compute stream: take the staged state over at this point (a device copy)
    if (e == cudaSuccess) e = cudaStreamWaitEvent(c->stream, c->ev_staged, 0);
    if (e == cudaSuccess) e = copy_state(c, c->stage, true, cudaMemcpyDeviceToDevice);
    if (e == cudaSuccess) e = cudaEventRecord(c->ev_taken, c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "asynchronous state upload");
    c->have_state = true;
    return OD_OK;
}

int od_set_state_device(od_ctx* c, const void* dptr, size_t bytes) {
    if (!c || !dptr) return OD_ERR_ARG;
    if (bytes != c->state_bytes) return fail(c, OD_ERR_SIZE, "state size does not match the mesh");
    if (int rc = set_device(c)) return rc;
    cudaError_t e = copy_state(c, const_cast<void*>(dptr), true, cudaMemcpyDeviceToDevice);
    if (e != cudaSuccess) return cuda_fail(c, e, "state copy");
    c->have_state = true;
    return OD_OK;
}

int od_get_state_device(od_ctx* c, void* dptr, size_t bytes) {
    if (!c || !dptr) return OD_ERR_ARG;
    if (bytes != c->state_bytes) return fail(c, OD_ERR_SIZE, "state size does not match the mesh");
    if (!c->have_state) return fail(c, OD_ERR_STATE, "no state set");
    if (int rc = set_device(c)) return rc;
    cudaError_t e = copy_state(c, dptr, false, cudaMemcpyDeviceToDevice);
    if (e != cudaSuccess) return cuda_fail(c, e, "state copy");
    return OD_OK;
}

int od_step(od_ctx* c, int n_steps, double dt) {
    if (!c || n_steps < 0) return OD_ERR_ARG;
    if (!c->have_state) return fail(c, OD_ERR_STATE, "no state set");
    if (c->slab) return fail(c, OD_ERR_STATE, "a slab context steps through od_slab_stage");
    if (int rc = set_device(c)) return rc;
    for (int s = 0; s < n_steps; ++s)
        for (int k = 0; k < 3; ++k) {
            const RkStage r = rk_stage(c, k, dt);
            if (int rc = enqueue_stage(c, r.u_in, r.u0, r.u_out, r.ra, r.rb, r.rc)) return rc;
        }
    return OD_OK;
}

// ---- z-slab decomposition

int od_create_slab(const od_params* g, int z0, int z1, od_ctx** out) {
    if (!g || !out) return OD_ERR_ARG;
    *out = nullptr;
    if (z0 < 0 || z1 <= z0 || z1 > g->nz) return OD_ERR_ARG;
    od_params p = *g;
    p.nz = z1 - z0 + 2;   // owned layers + a ghost layer below and above
    if (int rc = od_create(&p, out)) return rc;
    od_ctx* c = *out;
    set_jac(c, g);        // element size of the whole mesh
    c->slab = true;
    c->slab_z0 = z0;
    c->slab_z1 = z1;
    c->mesh_nz = g->nz;
    c->state_bytes = (size_t)p.nx * p.ny * (size_t)(z1 - z0) * 64 * 5 * c->elem_size;
    return OD_OK;
}

int od_slab_stage(od_ctx* c, int stage, int phase, double dt) {
    if (!c) return OD_ERR_ARG;
    if (!c->slab) return fail(c, OD_ERR_STATE, "not a slab context (od_create_slab)");
    if (stage < 0 || stage > 2 || (phase != 0 && phase != 1))
        return fail(c, OD_ERR_ARG, "stage must be 0, 1 or 2 and phase 0 (A) or 1 (B)");
    if (!c->have_state) return fail(c, OD_ERR_STATE, "no state set");
    if (int rc = set_device(c)) return rc;
    const RkStage r = rk_stage(c, stage, dt);
    od::StageLaunch L = make_launch(c, r.u_in, r.u0, r.u_out, r.ra, r.rb, r.rc);
    const long long nxy = (long long)c->p.nx * c->p.ny;
    L.e0 = nxy;               // the owned layers only
    L.e1 = c->nelem - nxy;
    L.phases = phase == 0 ? 1 : 2;
    cudaError_t e = c->fns.launch(L, c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, phase == 0 ? "slab phase A" : "slab phase B");
    return OD_OK;
}

}  // extern "C"

namespace {

// One halo message inside a slab context: `rows` rows of `width` bytes,
// `pitch` bytes apart, starting at p. kind 0: the five planes of z-layer
// `layer` of RK stage `stage`'s input state; kind 1: the z-face records of
// the layer's elements — minus-face records F_I - Fv/2 (fi) or the plus-face
// viscous fluxes (fv), direction 2 of [elem][dir 3][var][16].
struct HaloBlock {
    char* p;
    size_t width, pitch, rows;
};

HaloBlock halo_block(od_ctx* c, int stage, int kind, int layer, bool fi) {
    const size_t nxy = (size_t)c->p.nx * c->p.ny;
    if (kind == 0) {
        const size_t w = nxy * 64 * c->elem_size;
        return {(char*)c->U[stage] + (size_t)layer * w, w, c->buf_bytes / 5, 5};
    }
    const size_t cw = c->fns.c_double ? 8 : 4;
    const size_t e0 = (size_t)layer * nxy;
    if (fi) {
        char* base = (char*)c->fv + (size_t)c->nelem * od::kFvWords * cw;
        return {base + ((e0 * 3 + 2) * 80) * cw, 80 * cw, 240 * cw, nxy};
    }
    return {(char*)c->fv + ((e0 * 3 + 2) * 64) * cw, 64 * cw, 192 * cw, nxy};
}

int halo_args(od_ctx* c, int stage, int kind, int dir) {
    if (!c) return OD_ERR_ARG;
    if (!c->slab) return fail(c, OD_ERR_STATE, "not a slab context (od_create_slab)");
    if (stage < 0 || stage > 2 || kind < 0 || kind > 1 || dir < 0 || dir > 1)
        return fail(c, OD_ERR_ARG, "stage 0..2, kind 0 (state) or 1 (face records), dir 0 (down) or 1 (up)");
    return set_device(c);
}

}  // namespace

extern "C" {

size_t od_slab_halo_bytes(const od_ctx* c, int kind, int dir) {
    if (!c || !c->slab || kind < 0 || kind > 1 || dir < 0 || dir > 1) return 0;
    const size_t nxy = (size_t)c->p.nx * c->p.ny;
    if (kind == 0) return 5 * nxy * 64 * c->elem_size;
    return nxy * (dir == 0 ? 80 : 64) * (c->fns.c_double ? 8 : 4);
}

int od_slab_pack(od_ctx* c, int stage, int kind, int dir, void* d_dst, void* stream) {
    if (int rc = halo_args(c, stage, kind, dir)) return rc;
    if (!d_dst) return OD_ERR_ARG;
    // down: the lowest owned layer (its minus-face records); up: the highest (plus-face viscous fluxes)
    const int layer = dir == 0 ? 1 : c->p.nz - 2;
    const HaloBlock b = halo_block(c, stage, kind, layer, dir == 0);
    cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
    cudaError_t e = cudaMemcpy2DAsync(d_dst, b.width, b.p, b.pitch, b.width, b.rows, cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess) return cuda_fail(c, e, "slab halo pack");
    return OD_OK;
}

int od_slab_unpack(od_ctx* c, int stage, int kind, int dir, const void* d_src, void* stream) {
    if (int rc = halo_args(c, stage, kind, dir)) return rc;
    if (!d_src) return OD_ERR_ARG;
    // a message that travelled down fills the top ghost layer, one that travelled up the bottom one
    const int layer = dir == 0 ? c->p.nz - 1 : 0;
    const HaloBlock b = halo_block(c, stage, kind, layer, dir == 0);
    cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
    cudaError_t e = cudaMemcpy2DAsync(b.p, b.pitch, d_src, b.width, b.width, b.rows, cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess) return cuda_fail(c, e, "slab halo unpack");
    return OD_OK;
}

}  // extern "C"

namespace {

// Two strided copies (`rows` rows of `width` bytes, pitches in bytes; every
// address, width and pitch a multiple of 16) in one launch: blockIdx.y picks
// the copy, the x blocks stride over its 16-byte words.
struct HaloCopy {
    const char* src;
    char* dst;
    size_t src_pitch, dst_pitch, width, rows;
};

__global__ void __launch_bounds__(256) halo_copy_kernel(const HaloCopy c0, const HaloCopy c1) {
    const HaloCopy& c = blockIdx.y == 0 ? c0 : c1;
    const size_t per_row = c.width / 16, total = per_row * c.rows;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const size_t r = i / per_row, w = i - r * per_row;
        *reinterpret_cast<uint4*>(c.dst + r * c.dst_pitch + 16 * w) =
            *reinterpret_cast<const uint4*>(c.src + r * c.src_pitch + 16 * w);
    }
}

// The two halo messages of one exchange into slab `to`, on to's stream: dir 0
// travels down (`above`'s lowest owned layer -> to's top ghost), dir 1 up
// (`below`'s highest owned layer -> to's bottom ghost). Slabs on the same
// device: one copy kernel; otherwise two peer copies (cudaMemcpy2DAsync).
cudaError_t slab_exchange(od_ctx* to, od_ctx* above, od_ctx* below, int stage, int kind) {
    const HaloBlock sa = halo_block(above, stage, kind, 1, true);
    const HaloBlock da = halo_block(to, stage, kind, to->p.nz - 1, true);
    const HaloBlock sb = halo_block(below, stage, kind, below->p.nz - 2, false);
    const HaloBlock db = halo_block(to, stage, kind, 0, false);
    if (above->p.device != to->p.device || below->p.device != to->p.device) {
        cudaError_t e = cudaMemcpy2DAsync(da.p, da.pitch, sa.p, sa.pitch, sa.width, sa.rows, cudaMemcpyDefault,
                                          to->stream);
        if (e != cudaSuccess) return e;
        return cudaMemcpy2DAsync(db.p, db.pitch, sb.p, sb.pitch, sb.width, sb.rows, cudaMemcpyDefault, to->stream);
    }
    const HaloCopy c0{sa.p, da.p, sa.pitch, da.pitch, sa.width, sa.rows};
    const HaloCopy c1{sb.p, db.p, sb.pitch, db.pitch, sb.width, sb.rows};
    const size_t words = std::max(sa.width * sa.rows, sb.width * sb.rows) / 16;
    const unsigned blocks = (unsigned)std::min<size_t>((words + 255) / 256, 148 * 4);
    halo_copy_kernel<<<dim3(blocks, 2), 256, 0, to->stream>>>(c0, c1);
    return cudaGetLastError();
}

}  // namespace

extern "C" {

int od_slabs_step(od_ctx* const* S, int n, int n_steps, double dt) {
    if (!S || n <= 0 || n_steps < 0) return OD_ERR_ARG;
    for (int r = 0; r < n; ++r) {
        od_ctx* c = S[r];
        if (!c) return OD_ERR_ARG;
        if (!c->slab) return fail(c, OD_ERR_STATE, "not a slab context (od_create_slab)");
        if (!c->have_state) return fail(c, OD_ERR_STATE, "no state set");
        const od_ctx* b = S[(r + 1) % n];
        const bool next_ok = r + 1 < n ? b->slab_z0 == c->slab_z1 : (b->slab_z0 == 0 && c->slab_z1 == c->mesh_nz);
        if (!b->slab || b->p.nx != c->p.nx || b->p.ny != c->p.ny || b->mesh_nz != c->mesh_nz ||
            b->combo != c->combo || !next_ok)
            return fail(c, OD_ERR_ARG, "slabs must be one mesh's z-slabs, in z order, covering every layer");
    }
    for (int r = 0; r < n; ++r) {
        od_ctx* c = S[r];
        if (int rc = set_device(c)) return rc;
        for (auto& ev : c->ev_halo) {
            if (ev) continue;
            cudaError_t e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
            if (e != cudaSuccess) return cuda_fail(c, e, "cudaEventCreate");
        }
    }
    // Per stage: every slab marks its stage input ready; each copies the two
    // state layers it needs from its neighbours once they are; phase A; the
    // same with the z-face records; phase B. A slab never runs more than one
    // phase ahead of its neighbours, so no buffer is overwritten while a
    // neighbour still copies from it.
    for (int it = 0; it < n_steps; ++it) {
        for (int k = 0; k < 3; ++k) {
            for (int kind = 0; kind < 2; ++kind) {
                for (int r = 0; r < n; ++r) {
                    od_ctx* c = S[r];
                    if (int rc = set_device(c)) return rc;
                    cudaError_t e = cudaEventRecord(c->ev_halo[kind], c->stream);
                    if (e != cudaSuccess) return cuda_fail(c, e, "cudaEventRecord");
                }
                for (int r = 0; r < n; ++r) {
                    od_ctx* c = S[r];
                    od_ctx* above = S[(r + 1) % n];
                    od_ctx* below = S[(r + n - 1) % n];
                    if (int rc = set_device(c)) return rc;
                    cudaError_t e = cudaStreamWaitEvent(c->stream, above->ev_halo[kind], 0);
                    if (e == cudaSuccess) e = cudaStreamWaitEvent(c->stream, below->ev_halo[kind], 0);
                    if (e == cudaSuccess) e = slab_exchange(c, above, below, k, kind);
                    if (e != cudaSuccess) return cuda_fail(c, e, "slab halo copy");
                    if (int rc = od_slab_stage(c, k, kind, dt)) return rc;
                }
            }
        }
    }
    return OD_OK;
}

int od_rhs(od_ctx* c, void* d_out, size_t bytes) {
    if (!c || !d_out) return OD_ERR_ARG;
    if (c->slab) return fail(c, OD_ERR_STATE, "not available on a slab context");
    if (bytes != c->state_bytes) return fail(c, OD_ERR_SIZE, "RHS size does not match the mesh");
    if (!c->have_state) return fail(c, OD_ERR_STATE, "no state set");
    if (d_out == c->U[0] || (c->rhs && d_out == c->rhs))
        return fail(c, OD_ERR_ARG, "RHS output must not alias the state");
    if (int rc = set_device(c)) return rc;
    return enqueue_stage(c, c->U[0], nullptr, d_out, 0.0, 0.0, 1.0);
}

int od_diagnostics(od_ctx* c, double* vol6, double* prof, size_t prof_len) {
    if (!c || !vol6) return OD_ERR_ARG;
    if (c->slab) return fail(c, OD_ERR_STATE, "not available on a slab context");
    if (!c->have_state) return fail(c, OD_ERR_STATE, "no state set");
    const size_t nprof = (size_t)c->p.ny * 4 * 8;
    if (prof && prof_len < nprof) return fail(c, OD_ERR_SIZE, "profile buffer smaller than ny*4*8");
    if (int rc = set_device(c)) return rc;
    double* d = nullptr;
    const size_t bytes = (6 + nprof) * sizeof(double);
    cudaError_t e = cudaMallocAsync((void**)&d, bytes, c->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(d, 0, bytes, c->stream);
    if (e == cudaSuccess)
        e = od::launch_diag(c->U[0], c->elem_size == 8, c->p.nx, c->p.ny, c->p.nz, c->p.lx, c->p.ly, c->p.lz,
                            c->tab, d, prof ? d + 6 : nullptr, c->stream);
    std::vector<double> h(6 + nprof);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), d, bytes, cudaMemcpyDeviceToHost, c->stream);
    if (d) cudaFreeAsync(d, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "diagnostics");
    std::copy(h.begin(), h.begin() + 6, vol6);
    if (prof) {
        const double area = c->p.lx * c->p.lz;
        for (size_t i = 0; i < nprof; ++i) prof[i] = h[6 + i] / area;
    }
    return OD_OK;
}

int od_attach_closure(od_ctx* c, od_mlp* m) {
    if (!c) return OD_ERR_ARG;
    if (c->slab && m) return fail(c, OD_ERR_STATE, "not available on a slab context");
    if (!m) {
        c->hook = nullptr;
        c->hook_user = nullptr;
        return OD_OK;
    }
    if (!c->rhs) return fail(c, OD_ERR_ARG, "the closure needs an f32 state (the RHS buffer between phases)");
    if (int rc = set_device(c)) return rc;
    if (int rc = od::closure_prepare(m, c->p.nx, c->p.ny, c->p.nz, c->p.lx, c->p.ly, c->p.lz, c->elem_size == 8))
        return fail(c, rc, od_mlp_last_error(m));
    c->hook = od::closure_stage_hook;
    c->hook_user = m;
    return OD_OK;
}

int od_sync(od_ctx* c) {
    if (!c) return OD_ERR_ARG;
    if (int rc = set_device(c)) return rc;
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "stream synchronize");
    return OD_OK;
}

void* od_stream(od_ctx* c) { return c ? (void*)c->stream : nullptr; }

int od_launches_per_step(const od_ctx* c) {
    if (!c) return 0;
    return 3 * 2 * (c->slabs > 1 && !c->hook ? c->slabs : 1);
}

int od_set_pipeline_slabs(od_ctx* c, int slabs) {
    if (!c) return OD_ERR_ARG;
    if (slabs == 0) {
        c->slabs = auto_slabs(c->p);
        return OD_OK;
    }
    if (slabs < 1 || slabs > std::min(c->p.nz, kMaxSlabs))
        return fail(c, OD_ERR_ARG, "slabs must be 0 (auto) or 1..min(nz, 64)");
    if (int rc = od_sync(c)) return rc;
    c->slabs = slabs;
    return OD_OK;
}

int od_set_launch_shape(od_ctx* c, int elems_per_block_a, int elems_per_block_b) {
    if (!c) return OD_ERR_ARG;
    if (elems_per_block_a != 2 && elems_per_block_a != 4)
        return fail(c, OD_ERR_ARG, "phase-A elements per block must be 2 or 4");
    if (elems_per_block_b != 2 && elems_per_block_b != 4 && elems_per_block_b != 8 && elems_per_block_b != 16)
        return fail(c, OD_ERR_ARG, "phase-B elements per block must be 8 or 16 (a thread per x-line) or 2 or 4 "
                                   "(a thread per x-line and variable)");
    c->epb_a = elems_per_block_a;
    c->epb_b = elems_per_block_b;
    return OD_OK;
}

int od_set_timing(od_ctx* c, int enabled) {
    if (!c) return OD_ERR_ARG;
    if (int rc = od_sync(c)) return rc;
    c->timing = enabled != 0;
    c->ev_used = 0;
    c->n_stages = 0;
    return OD_OK;
}

int od_timing(od_ctx* c, double* ms_a, double* ms_b, long long* n_stages) {
    if (!c) return OD_ERR_ARG;
    if (int rc = od_sync(c)) return rc;
    double a = 0, b = 0;
    for (size_t q = 0; q + 3 <= c->ev_used; q += 3) {
        float t1 = 0, t2 = 0;
        cudaError_t e = cudaEventElapsedTime(&t1, c->events[q], c->events[q + 1]);
        if (e == cudaSuccess) e = cudaEventElapsedTime(&t2, c->events[q + 1], c->events[q + 2]);
        if (e != cudaSuccess) return cuda_fail(c, e, "cudaEventElapsedTime");
        a += t1;
        b += t2;
    }
    if (ms_a) *ms_a = a;
    if (ms_b) *ms_b = b;
    if (n_stages) *n_stages = (long long)(c->ev_used / 3);
    c->ev_used = 0;
    return OD_OK;
}

const char* od_last_error(const od_ctx* c) { return c ? c->err.c_str() : "null context"; }

}  // extern "C"
