// Ensembles: many independent boxes (own mesh, extents, flux scheme,
// viscosity, time step) advanced together, f32 pipeline.
//
// One persistent cooperative launch per RK stage covers every box: the grid
// (sized to what is co-resident: blocks per SM x SM count) strides over the
// phase-A tiles of all boxes, meets at a grid barrier, then strides over the
// phase-B tiles. The batched mode runs the same tiles as two ordinary
// launches per stage (a block per tile), each phase at its own occupancy. The per-element work is the single-box stage code
// (stage_a_tile / stage_b_tile of od_stage.cuh) with the flux scheme chosen
// at run time, so every box agrees with advancing it alone with od_step to
// f32 round-off (the compiler contracts a few multiply-adds differently in
// this kernel: a handful of values per box differ in the last bit); for a
// given shape the result is deterministic. A step (three stage launches) is
// captured once as a CUDA graph and replayed.
//
// The grid barrier is a monotonically growing arrival counter: each launch
// adds exactly gridDim.x arrivals, a block waits for the next multiple. The
// wait is bounded: after kSpinLimit polls the block sets the error flag and
// returns without running phase B; the host reports the flag after the step.
// The cooperative launch guarantees co-residency, so the bound is a guard, not
// a schedule.
//
// The autotuner times each candidate shape (the batched mode; elements per
// block and blocks per SM of the persistent launch) on the ensemble itself
// for a few steps and keeps the fastest.

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/opendynamo.h"
#include "od_launch.h"
#include "od_stage.cuh"

namespace od {
TablesD host_fr_tables();
}

namespace {

using od::LPE;
using od::NE;
using od::NF;
using od::SlotA;
// FR tables of every box (identical) in constant memory; the stage code reads
// them through these proxies with compile-time offsets, as it reads kernel
// parameters in the single-box kernels.
__constant__ od::Tab<float> c_tab;

template <int W>
struct CTabArr {
    __device__ __forceinline__ float operator[](int i) const {
        if constexpr (W == 0)
            return c_tab.D[i];
        else if constexpr (W == 1)
            return c_tab.eL[i];
        else if constexpr (W == 2)
            return c_tab.eR[i];
        else if constexpr (W == 3)
            return c_tab.gL[i];
        else
            return c_tab.gR[i];
    }
};

struct CTab {
    CTabArr<0> D;
    CTabArr<1> eL;
    CTabArr<2> eR;
    CTabArr<3> gL;
    CTabArr<4> gR;
};

// per-box stage parameters (the fields the stage code reads; tables from c_tab)
struct StageA {
    using S_t = float;
    using P_t = float;
    using C_t = float;
    const float* u_in;
    const float* u0;
    float* u_out;
    float* fv;
    float* fi;
    od::Mesh m;
    CTab tp, tc;
    od::ScaledTab<float> sc;
    float jac[3];
    float ra, rb, rc;
    float mu, forcing, suth;
    float kappa;   // heat-flux coefficient of mu (od::heat_coeff_host)
    int flags;
    int flux;
    long long e0, e1;
};

struct StageB {
    using S_t = float;
    using P_t = float;
    using C_t = float;
    float* u_out;
    const float* rhs;
    const float* u_in;
    const float* u0;
    const float* fv;
    const float* fi;
    od::Mesh m;
    CTab tc;
    float jac[3];
    float ra, rb, rc;
    int flags;
    long long e0, e1;
};

// Grid-barrier state in device memory. spin_limit and extra_arrivals are
// set by od_ensemble_set_wait (0 = defaults): the polls a block makes before
// it gives up, and arrivals added to the barrier target (a target nothing
// reaches makes every wait run out: the error path's test).
struct GridSync {
    unsigned long long count;
    int err;
    int extra_arrivals;
    long long spin_limit;
};

constexpr long long kSpinLimit = 1LL << 25;

struct EnsBoxStage {
    StageA A;
    StageB B;
};

// Per-box parameters of the running stage in constant memory (ensembles of
// up to kConstBoxes boxes): the stage code then reads them as it reads
// kernel parameters in the single-box kernels, cached and known constant
// across barriers. Copied in before every stage launch (a node of the step
// graph), so ensembles on one device must not run concurrently.
constexpr int kConstBoxes = 64;
__constant__ EnsBoxStage c_boxes[kConstBoxes];

__device__ __forceinline__ unsigned long long ld_acquire(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ bool grid_barrier(GridSync* g) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned long long n = gridDim.x;
        const long long limit = g->spin_limit > 0 ? g->spin_limit : kSpinLimit;
        const unsigned long long old = atomicAdd(&g->count, 1ull);
        const unsigned long long target = (old / n + 1) * n + (unsigned long long)max(g->extra_arrivals, 0);
        int good = 1;
        for (long long it = 0;; ++it) {
            if (ld_acquire(&g->count) >= target) break;
            if (it >= limit || *(volatile int*)&g->err) {
                atomicExch(&g->err, 1);
                good = 0;
                break;
            }
            __nanosleep(100);
        }
        __threadfence();
        ok = good;
    }
    __syncthreads();
    return ok != 0;
}

template <class T>
__device__ __forceinline__ void block_copy(T* dst, const T* src) {
    static_assert(sizeof(T) % 4 == 0, "word copy");
    const int n = sizeof(T) / 4;
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        reinterpret_cast<int*>(dst)[i] = reinterpret_cast<const int*>(src)[i];
}

// 8 (EPB 4) or 16 (EPB 2) blocks per SM: 128 registers per thread, the
// occupancy of the single-box phase-A kernel (shared memory bounds both).
template <class M, int EPB, bool CP>
__global__ void __launch_bounds__(LPE * EPB, 16 / EPB * 2) ensemble_stage_kernel(const EnsBoxStage* __restrict__ boxes, int nbox,
                                                                   const long long* __restrict__ start_a,
                                                                   const long long* __restrict__ start_b,
                                                                   const int2* __restrict__ tile_map,
                                                                   const int2* __restrict__ tile_map_b,
                                                                   GridSync* sync) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ __align__(16) StageA As;
    const long long G = gridDim.x;
    // tile_map[t] = (box, tile inside the box); the entry of the next tile is
    // loaded while the current one is processed
    // phase A: tiles blockIdx.x, +G, +2G, ... of all boxes. At any moment the
    // grid works on a window of consecutive tiles, as the waves of a single-box
    // launch do, so the neighbours' state read by one tile is still in L2 from
    // the tiles around it (contiguous chunks per block measured 1.4x slower:
    // every neighbour read went to DRAM).
    {
        const long long total = start_a[nbox];
        int cur = -1;
        int2 info = blockIdx.x < total ? tile_map[blockIdx.x] : make_int2(0, 0);
        for (long long t = blockIdx.x; t < total; t += G) {
            const int2 next = t + G < total ? tile_map[t + G] : info;
            __syncthreads();  // the previous tile is done with the element slots (and As)
            if constexpr (CP) {
                od::stage_a_tile<M, od::kFluxRuntime, EPB>(c_boxes[info.x].A, smem_raw, info.y);
            } else {
                if (info.x != cur) {
                    block_copy(&As, &boxes[info.x].A);
                    cur = info.x;
                    __syncthreads();
                }
                od::stage_a_tile<M, od::kFluxRuntime, EPB>(As, smem_raw, info.y);
            }
            info = next;
        }
    }
    if (!grid_barrier(sync)) return;
    // phase B, same order. Its tiles are short, so the parameters of every box
    // are copied into the (now idle) element slots once, and the loop has no
    // block synchronisation.
    {
        const long long total = start_b[nbox];
        StageB* Bs = reinterpret_cast<StageB*>(smem_raw);
        const bool in_smem = !CP && (size_t)nbox * sizeof(StageB) <= sizeof(SlotA<float, float>) * EPB;
        if (in_smem) {
            for (int b = 0; b < nbox; ++b) block_copy(&Bs[b], &boxes[b].B);
            __syncthreads();
        }
        int2 info = blockIdx.x < total ? tile_map_b[blockIdx.x] : make_int2(0, 0);
        for (long long t = blockIdx.x; t < total; t += G) {
            const int2 next = t + G < total ? tile_map_b[t + G] : info;
            if constexpr (CP)
                od::stage_b_tile<EPB, true>(c_boxes[info.x].B, info.y);
            else if (in_smem)
                od::stage_b_tile<EPB, true>(Bs[info.x], info.y);
            else
                od::stage_b_tile<EPB, true>(boxes[info.x].B, info.y);
            info = next;
        }
    }
}

// Batched mode: two ordinary launches per stage over the tiles of every box.
// Phase A: one tile (EPB elements) per block, at the single-box kernel's
// occupancy. Phase B: a thread per (element, variable, x-line), two elements
// per block, as the single-box split kernel. Each launch fills the GPU
// however small the boxes are, and phase B runs at its own occupancy (the
// persistent kernel runs it at phase A's); the launches are graph nodes.
constexpr int kBatchEpbA = 4;
constexpr int kBatchEpbB = 2;

template <class M, bool CP>
__global__ void __launch_bounds__(LPE * kBatchEpbA, 32 / kBatchEpbA)
    ensemble_a_kernel(const EnsBoxStage* __restrict__ boxes, const int2* __restrict__ tile_map) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int2 info = tile_map[blockIdx.x];
    if constexpr (CP) {
        od::stage_a_tile<M, od::kFluxRuntime, kBatchEpbA>(c_boxes[info.x].A, smem_raw, info.y);
    } else {
        __shared__ __align__(16) StageA As;
        block_copy(&As, &boxes[info.x].A);
        __syncthreads();
        od::stage_a_tile<M, od::kFluxRuntime, kBatchEpbA>(As, smem_raw, info.y);
    }
}

template <bool CP>
__global__ void __launch_bounds__(LPE * od::NV * kBatchEpbB)
    ensemble_b_kernel(const EnsBoxStage* __restrict__ boxes, const int2* __restrict__ tile_map) {
    // reverse tile order: phase A's last writes are still in L2 (as the single-box phase B)
    const int2 info = tile_map[gridDim.x - 1 - blockIdx.x];
    const int g = threadIdx.x / LPE;
    const int v = g / kBatchEpbB;
    const long long e = (long long)info.y * kBatchEpbB + (g - v * kBatchEpbB);
    const int l = threadIdx.x & (LPE - 1);
    if constexpr (CP) {
        const StageB& B = c_boxes[info.x].B;
        if (e < B.e1) od::stage_b_var<false>(B, od::b_ctx(B, e, l), v);
    } else {
        __shared__ __align__(16) StageB Bs;
        block_copy(&Bs, &boxes[info.x].B);
        __syncthreads();
        if (e < Bs.e1) od::stage_b_var<false>(Bs, od::b_ctx(Bs, e, l), v);
    }
}

void* batched_a_ptr(bool fast, bool cp) {
    if (fast) return cp ? (void*)ensemble_a_kernel<od::MathFast, true> : (void*)ensemble_a_kernel<od::MathFast, false>;
    return cp ? (void*)ensemble_a_kernel<od::MathIeee, true> : (void*)ensemble_a_kernel<od::MathIeee, false>;
}

void* batched_b_ptr(bool cp) { return cp ? (void*)ensemble_b_kernel<true> : (void*)ensemble_b_kernel<false>; }

// Dynamic persistent mode: ONE launch per stage whose blocks take work items
// from a ticket counter in a fixed order: every box's phase-A tiles, and each
// box's phase-B tiles placed at least a grid's worth of items after the box's
// last phase-A tile. A phase-B tile waits (bounded) until its own box has
// finished phase A, counted per box, so there is no grid-wide barrier and the
// HBM-bound phase-B tiles of one box run on the same SMs as the issue-bound
// phase-A tiles of the next. Every block takes tickets until it draws one
// past the launch's items, so a launch consumes exactly items + grid tickets
// and ticket / (items + grid) is the launch's index: the per-box counters
// grow by the box's phase-A tile count per launch (targets need no reset
// between launches or graph replays). Deadlock-free without co-residency: a
// phase-B tile waits only for phase-A tiles that blocks already hold, and a
// phase-A tile never waits. Per-box parameters from constant memory (up to
// kConstBoxes boxes).
constexpr int kDynEpb = 4;
constexpr int kDynChunk = 4;   // tiles per work item (one ticket)

template <class M>
__global__ void __launch_bounds__(LPE * kDynEpb, 32 / kDynEpb)
    ensemble_dyn_kernel(const int4* __restrict__ items, int total, const int* __restrict__ tiles_a,
                        unsigned long long* adone, GridSync* sync) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int4 it;
    __shared__ int skip;
    const unsigned long long per = (unsigned long long)total + gridDim.x;
    for (;;) {
        __syncthreads();   // the previous item is done with the element slots and `it`
        if (threadIdx.x == 0) {
            const unsigned long long t = atomicAdd(&sync->count, 1ull);
            const unsigned long long item = t % per;
            it = item < (unsigned long long)total ? items[item] : make_int4(-1, 0, 0, 0);
            int bad = *(volatile int*)&sync->err;
            if (!bad && it.x >= 0 && it.z == 1) {
                // phase B of box it.x: wait for all its phase-A tiles of this launch
                const unsigned long long target = (t / per + 1) * (unsigned long long)tiles_a[it.x] +
                                                  (unsigned long long)max(sync->extra_arrivals, 0);
                const long long limit = sync->spin_limit > 0 ? sync->spin_limit : kSpinLimit;
                for (long long n = 0; ld_acquire(&adone[it.x]) < target; ++n) {
                    if (n >= limit || *(volatile int*)&sync->err) {
                        atomicExch(&sync->err, 1);
                        bad = 1;
                        break;
                    }
                    __nanosleep(64);
                }
                __threadfence();
            }
            skip = bad;
        }
        __syncthreads();
        const int4 w = it;
        if (w.x < 0) break;   // past the launch's items (after an error too: tickets stay counted)
        if (skip) continue;
        if (w.z == 0) {
            for (int k = 0; k < w.w; ++k) {
                if (k) __syncthreads();   // the previous tile is done with the element slots
                od::stage_a_tile<M, od::kFluxRuntime, kDynEpb>(c_boxes[w.x].A, smem_raw, w.y + k);
            }
            __threadfence();   // this thread's records and RHS before the box's count
            __syncthreads();
            if (threadIdx.x == 0) atomicAdd(&adone[w.x], (unsigned long long)w.w);
        } else {
            for (int k = 0; k < w.w; ++k) od::stage_b_tile<kDynEpb, true>(c_boxes[w.x].B, w.y + k);
        }
    }
}

void* dyn_ptr(bool fast) {
    return fast ? (void*)ensemble_dyn_kernel<od::MathFast> : (void*)ensemble_dyn_kernel<od::MathIeee>;
}

template <class M, int EPB>
void* kernel_ptr(bool cp) {
    return cp ? (void*)ensemble_stage_kernel<M, EPB, true> : (void*)ensemble_stage_kernel<M, EPB, false>;
}

void* pick_kernel(bool fast, int epb, bool cp) {
    if (fast) return epb == 2 ? kernel_ptr<od::MathFast, 2>(cp) : kernel_ptr<od::MathFast, 4>(cp);
    return epb == 2 ? kernel_ptr<od::MathIeee, 2>(cp) : kernel_ptr<od::MathIeee, 4>(cp);
}

size_t dyn_smem(int epb) { return sizeof(SlotA<float, float>) * (size_t)epb; }

}  // namespace

struct od_ensemble {
    std::vector<od_box> box;
    int device = 0;
    bool fast = true;
    cudaStream_t stream = nullptr;
    int nsm = 0;
    // device memory
    void* pool = nullptr;
    std::vector<float*> U[3];
    std::vector<float*> rhs, fv;
    std::vector<long long> nelem;
    EnsBoxStage* d_stage[3] = {nullptr, nullptr, nullptr};
    long long* d_start_a = nullptr;  // per EPB choice: rebuilt by set_shape
    long long* d_start_b = nullptr;
    int2* d_tile_map = nullptr;      // (box, tile in box) of every phase-A tile (sized for 2 elements per tile)
    int2* d_tile_map_b = nullptr;    // the same for the phase-B tiles
    GridSync* d_sync = nullptr;
    // shape; batched: two ordinary launches per stage instead of the persistent one;
    // dynamic: one launch per stage, work items and per-box phase-A counts
    int epb = 4, bps = 0, grid = 0;
    bool batched = false, dynamic = false;
    long long tiles_a = 0, tiles_b = 0;
    int4* d_items = nullptr;            // dynamic mode: (box, first tile, phase, tiles) in issue order
    int n_items = 0;
    int* d_tiles_box = nullptr;         // phase-A tiles per box
    unsigned long long* d_adone = nullptr;   // phase-A tiles done per box (monotonic)
    bool use_graph = true, graph_ok = false;
    cudaGraphExec_t exec = nullptr;
    std::string err;
    long long steps_done = 0;
};

namespace {

int efail(od_ensemble* e, int code, const std::string& m) {
    if (e) e->err = m;
    return code;
}

int ecuda(od_ensemble* e, cudaError_t c, const char* what) {
    return efail(e, OD_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(c));
}

// RK stage parameters of every box for the current shape
int build_stage_params(od_ensemble* E) {
    const od::TablesD tab = od::host_fr_tables();
    od::Tab<float> tables_f;
    for (int i = 0; i < 16; ++i) tables_f.D[i] = (float)tab.D[i];
    for (int i = 0; i < 4; ++i) {
        tables_f.eL[i] = (float)tab.eL[i];
        tables_f.eR[i] = (float)tab.eR[i];
        tables_f.gL[i] = (float)tab.gL[i];
        tables_f.gR[i] = (float)tab.gR[i];
    }
    const int nb = (int)E->box.size();
    std::vector<EnsBoxStage> h(nb);
    std::vector<long long> sa(nb + 1, 0), sb(nb + 1, 0);
    const int eb = E->batched ? kBatchEpbB : E->epb;
    for (int b = 0; b < nb; ++b) {
        sa[b + 1] = sa[b] + (E->nelem[b] + E->epb - 1) / E->epb;
        sb[b + 1] = sb[b] + (E->nelem[b] + eb - 1) / eb;
    }
    E->tiles_a = sa[nb];
    E->tiles_b = sb[nb];
    if (E->dynamic) {
        // issue order: phase-A tiles box by box; a box's phase-B tiles once at
        // least a grid's worth of phase-A items follow its last phase-A tile
        std::vector<int4> items;
        items.reserve((size_t)(sa[nb] + sb[nb]));
        std::vector<std::pair<int, long long>> pending;   // (box, phase-A items issued when it ended)
        size_t head = 0;
        long long na = 0;
        // an item: (box, first tile, phase, tiles), up to kDynChunk tiles of one box and phase
        auto emit_b = [&](int b) {
            const long long n = sb[b + 1] - sb[b];
            for (long long t = 0; t < n; t += kDynChunk)
                items.push_back(make_int4(b, (int)t, 1, (int)std::min<long long>(kDynChunk, n - t)));
        };
        std::vector<int> tiles_box(nb);
        for (int b = 0; b < nb; ++b) {
            const long long n = sa[b + 1] - sa[b];
            tiles_box[b] = (int)n;
            for (long long t = 0; t < n; t += kDynChunk) {
                items.push_back(make_int4(b, (int)t, 0, (int)std::min<long long>(kDynChunk, n - t)));
                ++na;
                while (head < pending.size() && na - pending[head].second >= E->grid) emit_b(pending[head++].first);
            }
            pending.push_back({b, na});
        }
        while (head < pending.size()) emit_b(pending[head++].first);
        if (E->d_items) cudaFree(E->d_items);
        E->d_items = nullptr;
        E->n_items = (int)items.size();
        cudaError_t c = cudaMalloc(&E->d_items, sizeof(int4) * items.size());
        if (c == cudaSuccess)
            c = cudaMemcpy(E->d_items, items.data(), sizeof(int4) * items.size(), cudaMemcpyHostToDevice);
        if (c == cudaSuccess)
            c = cudaMemcpy(E->d_tiles_box, tiles_box.data(), sizeof(int) * nb, cudaMemcpyHostToDevice);
        if (c != cudaSuccess) return ecuda(E, c, "dynamic work items");
    }
    for (int s = 0; s < 3; ++s) {
        for (int b = 0; b < nb; ++b) {
            const od_box& x = E->box[b];
            StageA& A = h[b].A;
            std::memset(&A, 0, sizeof A);
            const float dt = (float)x.dt;
            // stage coefficients in f32 (od_step, src/solver.rs:275-316)
            const float ra[3] = {0.0f, 0.75f, (float)(1.0 / 3.0)};
            const float rb[3] = {1.0f, 0.25f, (float)(2.0 / 3.0)};
            const float rc[3] = {dt, 0.25f * dt, (float)(2.0 / 3.0) * dt};
            float* in[3] = {E->U[0][b], E->U[1][b], E->U[2][b]};
            float* out[3] = {E->U[1][b], E->U[2][b], E->U[0][b]};
            A.u_in = in[s];
            A.u0 = s == 0 ? nullptr : E->U[0][b];
            A.u_out = E->rhs[b];
            A.fv = E->fv[b];
            A.fi = E->fv[b] + E->nelem[b] * od::kFvWords;
            A.m.nx = x.nx;
            A.m.ny = x.ny;
            A.m.nz = x.nz;
            A.m.y_wall = x.y_wall;
            A.m.nelem = E->nelem[b];
            od::mesh_set_div(A.m);
            A.m.npts = E->nelem[b] * NE;
            const double L3[3] = {x.lx, x.ly, x.lz};
            const int n3[3] = {x.nx, x.ny, x.nz};
            for (int d = 0; d < 3; ++d) A.jac[d] = 2.0f / ((float)L3[d] / (float)n3[d]);
            A.sc = od::scale_tab<float>(tables_f, A.jac);
            A.ra = ra[s];
            A.rb = rb[s];
            A.rc = rc[s];
            A.mu = (float)x.mu;
            A.kappa = od::heat_coeff_host<float>(A.mu);
            A.forcing = (float)x.forcing;
            A.suth = -1.0f;
            A.flags = od::kDeferRK | (s == 0 ? 0 : od::kHasU0);
            A.flux = x.flux;
            A.e0 = 0;
            A.e1 = E->nelem[b];
            StageB& B = h[b].B;
            std::memset(&B, 0, sizeof B);
            B.u_out = out[s];
            B.rhs = E->rhs[b];
            B.u_in = in[s];
            B.u0 = A.u0;
            B.fv = A.fv;
            B.fi = A.fi;
            B.m = A.m;
            for (int d = 0; d < 3; ++d) B.jac[d] = A.jac[d];
            B.ra = A.ra;
            B.rb = A.rb;
            B.rc = A.rc;
            B.flags = A.flags;
            B.e0 = 0;
            B.e1 = E->nelem[b];
        }
        cudaError_t c = cudaMemcpy(E->d_stage[s], h.data(), sizeof(EnsBoxStage) * nb, cudaMemcpyHostToDevice);
        if (c != cudaSuccess) return ecuda(E, c, "stage parameters");
    }
    cudaError_t c = cudaMemcpyToSymbol(c_tab, &tables_f, sizeof tables_f);
    if (c == cudaSuccess) c = cudaMemcpy(E->d_start_a, sa.data(), sizeof(long long) * (nb + 1), cudaMemcpyHostToDevice);
    if (c == cudaSuccess) c = cudaMemcpy(E->d_start_b, sb.data(), sizeof(long long) * (nb + 1), cudaMemcpyHostToDevice);
    std::vector<int2> ta((size_t)sa[nb]), tb((size_t)sb[nb]);
    for (int b = 0; b < nb; ++b) {
        for (long long t = sa[b]; t < sa[b + 1]; ++t) ta[(size_t)t] = make_int2(b, (int)(t - sa[b]));
        for (long long t = sb[b]; t < sb[b + 1]; ++t) tb[(size_t)t] = make_int2(b, (int)(t - sb[b]));
    }
    if (c == cudaSuccess) c = cudaMemcpy(E->d_tile_map, ta.data(), sizeof(int2) * ta.size(), cudaMemcpyHostToDevice);
    if (c == cudaSuccess) c = cudaMemcpy(E->d_tile_map_b, tb.data(), sizeof(int2) * tb.size(), cudaMemcpyHostToDevice);
    if (c != cudaSuccess) return ecuda(E, c, "tile tables");
    return OD_OK;
}

cudaError_t launch_stage(od_ensemble* E, int s) {
    int nbox = (int)E->box.size();
    const bool cp = nbox <= kConstBoxes;
    if (cp) {
        cudaError_t c = cudaMemcpyToSymbolAsync(c_boxes, E->d_stage[s], sizeof(EnsBoxStage) * nbox, 0,
                                                cudaMemcpyDeviceToDevice, E->stream);
        if (c != cudaSuccess) return c;
    }
    if (E->dynamic) {
        void* args[] = {(void*)&E->d_items, (void*)&E->n_items, (void*)&E->d_tiles_box, (void*)&E->d_adone,
                        (void*)&E->d_sync};
        return cudaLaunchKernel(dyn_ptr(E->fast), dim3((unsigned)E->grid), dim3(LPE * kDynEpb), args,
                                dyn_smem(kDynEpb), E->stream);
    }
    if (E->batched) {
        void* args_a[] = {(void*)&E->d_stage[s], (void*)&E->d_tile_map};
        cudaError_t c = cudaLaunchKernel(batched_a_ptr(E->fast, cp), dim3((unsigned)E->tiles_a),
                                         dim3(LPE * kBatchEpbA), args_a, dyn_smem(kBatchEpbA), E->stream);
        if (c != cudaSuccess) return c;
        void* args_b[] = {(void*)&E->d_stage[s], (void*)&E->d_tile_map_b};
        return cudaLaunchKernel(batched_b_ptr(cp), dim3((unsigned)E->tiles_b), dim3(LPE * od::NV * kBatchEpbB),
                                args_b, 0, E->stream);
    }
    void* fn = pick_kernel(E->fast, E->epb, cp);
    void* args[] = {(void*)&E->d_stage[s], (void*)&nbox, (void*)&E->d_start_a, (void*)&E->d_start_b,
                    (void*)&E->d_tile_map, (void*)&E->d_tile_map_b,
                    (void*)&E->d_sync};
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)E->grid);
    cfg.blockDim = dim3((unsigned)(LPE * E->epb));
    cfg.dynamicSmemBytes = dyn_smem(E->epb);
    cfg.stream = E->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelExC(&cfg, fn, args);
}

void drop_graph(od_ensemble* E) {
    if (E->exec) cudaGraphExecDestroy(E->exec);
    E->exec = nullptr;
    E->graph_ok = false;
}

// set the launch shape; blocks_per_sm <= 0 = as many as are co-resident,
// OD_ENSEMBLE_BATCHED = two ordinary launches per stage (phase A at 4
// elements per block)
int apply_shape(od_ensemble* E, int epb, int bps, bool use_graph) {
    const bool batched = bps == OD_ENSEMBLE_BATCHED;
    const bool dynamic = bps == OD_ENSEMBLE_DYNAMIC;
    if (batched) epb = kBatchEpbA;
    if (dynamic) epb = kDynEpb;
    if (bps < 0 && !batched && !dynamic) return efail(E, OD_ERR_ARG, "unknown launch mode");
    if (epb != 2 && epb != 4) return efail(E, OD_ERR_ARG, "elements per block must be 2 or 4");
    const bool cp = E->box.size() <= (size_t)kConstBoxes;
    if (dynamic && !cp) return efail(E, OD_ERR_ARG, "the dynamic mode takes at most 64 boxes");
    void* fn = dynamic ? dyn_ptr(E->fast) : batched ? batched_a_ptr(E->fast, cp) : pick_kernel(E->fast, epb, cp);
    cudaError_t c = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn_smem(epb));
    if (c != cudaSuccess) return ecuda(E, c, "cudaFuncSetAttribute");
    int maxb = 0;
    c = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&maxb, fn, LPE * epb, dyn_smem(epb));
    if (c != cudaSuccess) return ecuda(E, c, "occupancy");
    if (maxb <= 0) return efail(E, OD_ERR_CUDA, "ensemble kernel cannot be resident");
    if (dynamic || (!batched && (bps <= 0 || bps > maxb))) bps = maxb;
    drop_graph(E);
    const bool rebuild = epb != E->epb || batched != E->batched || dynamic != E->dynamic || dynamic ||
                         !E->d_stage[0];
    E->epb = epb;
    E->batched = batched;
    E->dynamic = dynamic;
    E->use_graph = use_graph;
    E->grid = bps * E->nsm;   // the dynamic mode's item order depends on it
    if (rebuild) {
        if (int rc = build_stage_params(E)) return rc;
    }
    E->bps = batched ? OD_ENSEMBLE_BATCHED : dynamic ? OD_ENSEMBLE_DYNAMIC : bps;
    if (batched) E->grid = (int)E->tiles_a;
    // a new grid size restarts the arrival / ticket counter and the per-box counts
    c = cudaMemsetAsync(E->d_sync, 0, sizeof(GridSync), E->stream);
    if (c == cudaSuccess) c = cudaMemsetAsync(E->d_adone, 0, sizeof(unsigned long long) * E->box.size(), E->stream);
    if (c == cudaSuccess) c = cudaStreamSynchronize(E->stream);
    if (c != cudaSuccess) return ecuda(E, c, "barrier reset");
    if (use_graph) {
        cudaGraph_t g = nullptr;
        c = cudaStreamBeginCapture(E->stream, cudaStreamCaptureModeThreadLocal);
        if (c == cudaSuccess) {
            cudaError_t lc = cudaSuccess;
            for (int s = 0; s < 3 && lc == cudaSuccess; ++s) lc = launch_stage(E, s);
            c = cudaStreamEndCapture(E->stream, &g);
            if (lc != cudaSuccess) c = lc;
        }
        if (c == cudaSuccess) c = cudaGraphInstantiate(&E->exec, g, 0);
        if (g) cudaGraphDestroy(g);
        if (c != cudaSuccess) {
            cudaGetLastError();
            E->exec = nullptr;
            E->graph_ok = false;  // direct launches instead
        } else {
            E->graph_ok = true;
        }
    }
    return OD_OK;
}

int enqueue_steps(od_ensemble* E, int n) {
    for (int i = 0; i < n; ++i) {
        cudaError_t c;
        if (E->graph_ok) {
            c = cudaGraphLaunch(E->exec, E->stream);
        } else {
            c = cudaSuccess;
            for (int s = 0; s < 3 && c == cudaSuccess; ++s) c = launch_stage(E, s);
        }
        if (c != cudaSuccess) return ecuda(E, c, "ensemble step");
    }
    E->steps_done += n;
    return OD_OK;
}

int check_sync_flag(od_ensemble* E) {
    GridSync h;
    cudaError_t c = cudaMemcpyAsync(&h, E->d_sync, sizeof h, cudaMemcpyDeviceToHost, E->stream);
    if (c == cudaSuccess) c = cudaStreamSynchronize(E->stream);
    if (c != cudaSuccess) return ecuda(E, c, "ensemble step");
    if (h.err)
        return efail(E, OD_ERR_CUDA, E->dynamic ? "ensemble phase-B wait timed out (a box's phase A never completed)"
                                                : "ensemble grid barrier timed out (blocks not co-resident)");
    return OD_OK;
}

}  // namespace

extern "C" {

int od_ensemble_create(const od_box* boxes, int nbox, int device, int fast_math, od_ensemble** out) {
    if (!boxes || nbox <= 0 || !out) return OD_ERR_ARG;
    *out = nullptr;
    for (int b = 0; b < nbox; ++b) {
        const od_box& x = boxes[b];
        if (x.nx <= 0 || x.ny <= 0 || x.nz <= 0 || !(x.lx > 0) || !(x.ly > 0) || !(x.lz > 0) || x.flux < 0 ||
            x.flux > 2 || !(x.dt > 0) || !(x.mu >= 0))
            return OD_ERR_ARG;
    }
    od_ensemble* E = new od_ensemble();
    E->box.assign(boxes, boxes + nbox);
    E->device = device;
    E->fast = fast_math != 0;
    cudaError_t c = cudaSetDevice(device);
    if (c == cudaSuccess) c = cudaStreamCreateWithFlags(&E->stream, cudaStreamNonBlocking);
    if (c == cudaSuccess) c = cudaDeviceGetAttribute(&E->nsm, cudaDevAttrMultiProcessorCount, device);
    int coop = 0;
    if (c == cudaSuccess) c = cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device);
    if (c != cudaSuccess || !coop) {
        *out = E;
        return c != cudaSuccess ? ecuda(E, c, "device setup") : efail(E, OD_ERR_CUDA, "no cooperative launch");
    }
    size_t total = 0;
    std::vector<size_t> off(nbox);
    auto align = [](size_t x) { return (x + 255) & ~(size_t)255; };
    for (int b = 0; b < nbox; ++b) {
        const long long ne = (long long)boxes[b].nx * boxes[b].ny * boxes[b].nz;
        E->nelem.push_back(ne);
        off[b] = total;
        const size_t st = (size_t)ne * NE * 5 * sizeof(float);
        total += 4 * align(st) + align((size_t)ne * od::kFaceWords * sizeof(float));
    }
    c = cudaMalloc(&E->pool, total);
    if (c == cudaSuccess) c = cudaMemset(E->pool, 0, total);
    for (int s = 0; s < 3 && c == cudaSuccess; ++s) c = cudaMalloc(&E->d_stage[s], sizeof(EnsBoxStage) * nbox);
    if (c == cudaSuccess) c = cudaMalloc(&E->d_start_a, sizeof(long long) * (nbox + 1));
    if (c == cudaSuccess) c = cudaMalloc(&E->d_start_b, sizeof(long long) * (nbox + 1));
    long long max_tiles = 0;
    for (int b = 0; b < nbox; ++b) max_tiles += (E->nelem[b] + 1) / 2;
    if (c == cudaSuccess) c = cudaMalloc(&E->d_tile_map, sizeof(int2) * (size_t)max_tiles);
    if (c == cudaSuccess) c = cudaMalloc(&E->d_tile_map_b, sizeof(int2) * (size_t)max_tiles);
    if (c == cudaSuccess) c = cudaMalloc(&E->d_sync, sizeof(GridSync));
    if (c == cudaSuccess) c = cudaMalloc(&E->d_tiles_box, sizeof(int) * nbox);
    if (c == cudaSuccess) c = cudaMalloc(&E->d_adone, sizeof(unsigned long long) * nbox);
    if (c != cudaSuccess) {
        *out = E;
        return ecuda(E, c, "allocation");
    }
    for (int b = 0; b < nbox; ++b) {
        char* p = (char*)E->pool + off[b];
        const size_t st = align((size_t)E->nelem[b] * NE * 5 * sizeof(float));
        for (int k = 0; k < 3; ++k) E->U[k].push_back((float*)(p + k * st));
        E->rhs.push_back((float*)(p + 3 * st));
        E->fv.push_back((float*)(p + 4 * st));
    }
    *out = E;
    E->epb = 0;  // forces the parameter build
    return apply_shape(E, 4, OD_ENSEMBLE_BATCHED, true);   // the faster mode on B200 at every size measured
}

void od_ensemble_destroy(od_ensemble* E) {
    if (!E) return;
    cudaSetDevice(E->device);
    drop_graph(E);
    if (E->stream) cudaStreamSynchronize(E->stream);
    for (int s = 0; s < 3; ++s)
        if (E->d_stage[s]) cudaFree(E->d_stage[s]);
    if (E->d_start_a) cudaFree(E->d_start_a);
    if (E->d_start_b) cudaFree(E->d_start_b);
    if (E->d_tile_map) cudaFree(E->d_tile_map);
    if (E->d_tile_map_b) cudaFree(E->d_tile_map_b);
    if (E->d_sync) cudaFree(E->d_sync);
    if (E->d_items) cudaFree(E->d_items);
    if (E->d_tiles_box) cudaFree(E->d_tiles_box);
    if (E->d_adone) cudaFree(E->d_adone);
    if (E->pool) cudaFree(E->pool);
    if (E->stream) cudaStreamDestroy(E->stream);
    delete E;
}

size_t od_ensemble_state_bytes(const od_ensemble* E, int b) {
    if (!E || b < 0 || b >= (int)E->box.size()) return 0;
    return (size_t)E->nelem[b] * NE * 5 * sizeof(float);
}

int od_ensemble_set_state(od_ensemble* E, int b, const void* host, size_t bytes) {
    if (!E || !host || b < 0 || b >= (int)E->box.size()) return OD_ERR_ARG;
    if (bytes != od_ensemble_state_bytes(E, b)) return efail(E, OD_ERR_SIZE, "state size does not match the box");
    cudaSetDevice(E->device);
    cudaError_t c = cudaMemcpyAsync(E->U[0][b], host, bytes, cudaMemcpyHostToDevice, E->stream);
    if (c == cudaSuccess) c = cudaStreamSynchronize(E->stream);
    if (c != cudaSuccess) return ecuda(E, c, "set state");
    return OD_OK;
}

int od_ensemble_get_state(od_ensemble* E, int b, void* host, size_t bytes) {
    if (!E || !host || b < 0 || b >= (int)E->box.size()) return OD_ERR_ARG;
    if (bytes != od_ensemble_state_bytes(E, b)) return efail(E, OD_ERR_SIZE, "state size does not match the box");
    cudaSetDevice(E->device);
    cudaError_t c = cudaMemcpyAsync(host, E->U[0][b], bytes, cudaMemcpyDeviceToHost, E->stream);
    if (c == cudaSuccess) c = cudaStreamSynchronize(E->stream);
    if (c != cudaSuccess) return ecuda(E, c, "get state");
    return OD_OK;
}

int od_ensemble_step(od_ensemble* E, int n) {
    if (!E || n < 0) return OD_ERR_ARG;
    cudaSetDevice(E->device);
    if (int rc = enqueue_steps(E, n)) return rc;
    return check_sync_flag(E);
}

int od_ensemble_set_wait(od_ensemble* E, long long spin_limit, int extra_arrivals) {
    if (!E || spin_limit < 0 || extra_arrivals < 0) return OD_ERR_ARG;
    cudaSetDevice(E->device);
    GridSync h{};
    h.spin_limit = spin_limit;
    h.extra_arrivals = extra_arrivals;
    // restarts the arrival / ticket counter and the per-box counts and clears
    // a timed-out wait's error flag
    cudaError_t c = cudaMemcpyAsync(E->d_sync, &h, sizeof h, cudaMemcpyHostToDevice, E->stream);
    if (c == cudaSuccess) c = cudaMemsetAsync(E->d_adone, 0, sizeof(unsigned long long) * E->box.size(), E->stream);
    if (c == cudaSuccess) c = cudaStreamSynchronize(E->stream);
    if (c != cudaSuccess) return ecuda(E, c, "od_ensemble_set_wait");
    return OD_OK;
}

int od_ensemble_set_shape(od_ensemble* E, int epb, int blocks_per_sm, int use_graph) {
    if (!E) return OD_ERR_ARG;
    cudaSetDevice(E->device);
    return apply_shape(E, epb, blocks_per_sm, use_graph != 0);
}

int od_ensemble_info(const od_ensemble* E, int* epb, int* blocks_per_sm, int* grid, int* graph) {
    if (!E) return OD_ERR_ARG;
    if (epb) *epb = E->epb;
    if (blocks_per_sm) *blocks_per_sm = E->bps;
    if (grid) *grid = E->grid;
    if (graph) *graph = E->graph_ok ? 1 : 0;
    return OD_OK;
}

// Times every candidate shape for trial_steps steps (after one warm-up step)
// on a scratch copy of the states, keeps the fastest and restores the states.
int od_ensemble_autotune(od_ensemble* E, int trial_steps, char* report, size_t report_len) {
    if (!E || trial_steps <= 0) return OD_ERR_ARG;
    cudaSetDevice(E->device);
    const int nb = (int)E->box.size();
    std::vector<void*> save(nb, nullptr);
    cudaError_t c = cudaSuccess;
    for (int b = 0; b < nb && c == cudaSuccess; ++b) {
        c = cudaMalloc(&save[b], od_ensemble_state_bytes(E, b));
        if (c == cudaSuccess)
            c = cudaMemcpyAsync(save[b], E->U[0][b], od_ensemble_state_bytes(E, b), cudaMemcpyDeviceToDevice,
                                E->stream);
    }
    if (c != cudaSuccess) {
        for (void* p : save)
            if (p) cudaFree(p);
        return ecuda(E, c, "autotune scratch");
    }
    std::string rep;
    double best = 1e30;
    int best_epb = 4, best_bps = 0;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int rc = OD_OK;
    for (int epb : {2, 4}) {
        void* fn = pick_kernel(E->fast, epb, E->box.size() <= (size_t)kConstBoxes);
        cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn_smem(epb));
        int maxb = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&maxb, fn, LPE * epb, dyn_smem(epb));
        std::vector<int> cands;
        for (int b = maxb; b >= 1; b = b > 2 ? b * 3 / 4 : b - 1) cands.push_back(b);
        if (epb == kBatchEpbA) cands.insert(cands.begin(), OD_ENSEMBLE_BATCHED);
        if (epb == kDynEpb && E->box.size() <= (size_t)kConstBoxes) cands.insert(cands.begin(), OD_ENSEMBLE_DYNAMIC);
        for (int bps : cands) {
            if ((rc = apply_shape(E, epb, bps, true))) break;
            if ((rc = enqueue_steps(E, 1))) break;
            cudaEventRecord(e0, E->stream);
            if ((rc = enqueue_steps(E, trial_steps))) break;
            cudaEventRecord(e1, E->stream);
            if ((rc = check_sync_flag(E))) break;
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            char line[128];
            if (E->dynamic)
                std::snprintf(line, sizeof line, "dynamic (one launch per stage, %d items, grid %d) graph=%d: %.4f ms/step\n",
                              E->n_items, E->grid, E->graph_ok ? 1 : 0, ms / trial_steps);
            else if (E->batched)
                std::snprintf(line, sizeof line, "batched (two launches per stage, %lld + %lld blocks) graph=%d: %.4f ms/step\n",
                              E->tiles_a, E->tiles_b, E->graph_ok ? 1 : 0, ms / trial_steps);
            else
                std::snprintf(line, sizeof line, "epb=%d blocks/SM=%d grid=%d graph=%d: %.4f ms/step\n", epb, bps,
                              E->grid, E->graph_ok ? 1 : 0, ms / trial_steps);
            rep += line;
            if (ms < best) {
                best = ms;
                best_epb = epb;
                best_bps = bps;
            }
            // restore the states between trials
            for (int b = 0; b < nb; ++b)
                cudaMemcpyAsync(E->U[0][b], save[b], od_ensemble_state_bytes(E, b), cudaMemcpyDeviceToDevice,
                                E->stream);
        }
        if (rc) break;
    }
    for (int b = 0; b < nb; ++b) {
        cudaMemcpyAsync(E->U[0][b], save[b], od_ensemble_state_bytes(E, b), cudaMemcpyDeviceToDevice, E->stream);
    }
    cudaStreamSynchronize(E->stream);
    for (void* p : save) cudaFree(p);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    E->steps_done = 0;
    rc = apply_shape(E, best_epb, best_bps, true);
    char line[128];
    if (best_bps == OD_ENSEMBLE_BATCHED)
        std::snprintf(line, sizeof line, "chosen: batched\n");
    else if (best_bps == OD_ENSEMBLE_DYNAMIC)
        std::snprintf(line, sizeof line, "chosen: dynamic\n");
    else
        std::snprintf(line, sizeof line, "chosen: epb=%d blocks/SM=%d\n", best_epb, best_bps);
    rep += line;
    if (report && report_len) {
        std::strncpy(report, rep.c_str(), report_len - 1);
        report[report_len - 1] = 0;
    }
    return rc;
}

const char* od_ensemble_last_error(const od_ensemble* E) { return E ? E->err.c_str() : ""; }

void* od_ensemble_stream(od_ensemble* E) { return E ? (void*)E->stream : nullptr; }

}  // extern "C"
