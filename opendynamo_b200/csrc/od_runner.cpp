// Run driver over the public C ABI: the reference's run loop
// (src/solver.rs:139-374) with its dump / checkpoint pipeline
// (src/solver.rs:161-175, 745-818).
//
// Dump pipeline, per dump:
//   compute stream : od_get_state_device -> snapshot slot k (device copy of
//                    the state; the next step may overwrite the state in
//                    place), event "snap_k"
//   io stream      : waits snap_k, copies slot k to pinned host buffer k,
//                    event "host_k"
//   host thread    : waits host_k, writes the dump (and checkpoint), returns
//                    slot k to the pool
// Three slots, as the reference's three pinned buffers: the step loop
// blocks only when all three are in flight.

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <filesystem>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "opendynamo.h"

namespace {

constexpr int kSlots = 3;

struct Pool {
    std::mutex m;
    std::condition_variable cv;
    std::deque<int> free;
    int take() {
        std::unique_lock<std::mutex> lk(m);
        cv.wait(lk, [&] { return !free.empty(); });
        int k = free.front();
        free.pop_front();
        return k;
    }
    void give(int k) {
        {
            std::lock_guard<std::mutex> lk(m);
            free.push_back(k);
        }
        cv.notify_one();
    }
};

std::string file_name(const std::string& dir, const std::string& prefix, const char* kind,
                      unsigned long long label) {
    char buf[64];
    std::snprintf(buf, sizeof buf, "_%s_%06llu.h5", kind, label);
    return (std::filesystem::path(dir) / (prefix + buf)).string();
}

void set_err(char* err, size_t n, const std::string& s) {
    if (err && n) {
        std::strncpy(err, s.c_str(), n - 1);
        err[n - 1] = 0;
    }
}

// physical_state_report (src/solver.rs:820-840): min/max of rho and u = rho*u/rho in f32
template <class T>
void state_report(const T* s, size_t npts, od_run_result* r) {
    float rmin = 3.4028235e38f, rmax = -3.4028235e38f, umin = 3.4028235e38f, umax = -3.4028235e38f;
    for (size_t i = 0; i < npts; ++i) {
        const float rho = (float)s[i];
        const float u = (float)s[npts + i] / rho;
        rmin = std::min(rmin, rho);
        rmax = std::max(rmax, rho);
        umin = std::min(umin, u);
        umax = std::max(umax, u);
    }
    r->rho_min = rmin;
    r->rho_max = rmax;
    r->u_min = umin;
    r->u_max = umax;
}

}  // namespace

extern "C" int od_run(const od_params* p, const od_run_opts* o, od_run_result* r, char* err, size_t err_len) {
    if (!p || !o || !r) {
        set_err(err, err_len, "null argument");
        return OD_ERR_ARG;
    }
    std::memset(r, 0, sizeof *r);
    if (!o->initial_state) {
        set_err(err, err_len,
                "[physics].initial_state is required: point it at a solver state file (a fresh IC, or a "
                "checkpoint <output_dir>/checkpoint_..._.h5 to resume from).");
        return OD_ERR_ARG;
    }
    if (o->save_freq <= 0 || o->n_steps < 0 || o->checkpoint_freq < 0) {
        set_err(err, err_len, "save_freq must be > 0, n_steps and checkpoint_freq >= 0");
        return OD_ERR_ARG;
    }
    const std::string comp = o->compression ? o->compression : "blosc-lz4";
    const std::string out_dir = o->output_dir ? o->output_dir : "output";
    const std::string prefix = o->prefix ? o->prefix : "flow";
    const bool quiet = o->quiet != 0;
    const bool f64 = p->u_real == OD_F64;
    const char* kind = f64 ? "f64" : "f32";

    od_ctx* ctx = nullptr;
    int rc = od_create(p, &ctx);
    if (rc) {
        set_err(err, err_len, std::string("od_create: ") + (ctx ? od_last_error(ctx) : ""));
        if (ctx) od_destroy(ctx);
        return rc;
    }
    const size_t bytes = od_state_bytes(ctx);
    const size_t npts = (size_t)p->nx * p->ny * p->nz * 64;
    if (!quiet)
        std::printf("Allocating device memory for %zu elements, total DOFs: %zu\n", npts / 64, npts);

    // device snapshots + pinned host buffers + streams / events
    void* snap[kSlots] = {};
    void* host[kSlots] = {};
    cudaEvent_t ev_snap[kSlots] = {}, ev_host[kSlots] = {};
    cudaStream_t io_stream = nullptr;
    std::vector<std::thread> threads;
    Pool pool;
    std::mutex io_m;
    long long written = 0, io_errors = 0;
    int final_slot = -1;
    int prev_dev = 0;
    cudaGetDevice(&prev_dev);
    auto cleanup = [&]() {
        for (auto& t : threads)
            if (t.joinable()) t.join();
        for (int k = 0; k < kSlots; ++k) {
            if (snap[k]) cudaFree(snap[k]);
            if (host[k]) cudaFreeHost(host[k]);
            if (ev_snap[k]) cudaEventDestroy(ev_snap[k]);
            if (ev_host[k]) cudaEventDestroy(ev_host[k]);
        }
        if (io_stream) cudaStreamDestroy(io_stream);
        od_destroy(ctx);
        cudaSetDevice(prev_dev);
    };
    auto cuda_fail = [&](cudaError_t e, const char* what) {
        set_err(err, err_len, std::string(what) + ": " + cudaGetErrorString(e));
        cleanup();
        return OD_ERR_CUDA;
    };
    cudaSetDevice(p->device);
    for (int k = 0; k < kSlots; ++k) {
        cudaError_t e = cudaMalloc(&snap[k], bytes);
        if (e == cudaSuccess) e = cudaMallocHost(&host[k], bytes);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev_snap[k], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev_host[k], cudaEventDisableTiming);
        if (e != cudaSuccess) return cuda_fail(e, "allocating dump buffers");
        pool.free.push_back(k);
    }
    if (cudaError_t e = cudaStreamCreateWithFlags(&io_stream, cudaStreamNonBlocking)) return cuda_fail(e, "io stream");
    cudaStream_t stream = (cudaStream_t)od_stream(ctx);

    // initial state (solver.rs:186-226)
    if (!quiet) std::printf("Loading initial state from %s ...\n", o->initial_state);
    unsigned long long base_label = 0;
    double base_t = 0.0;
    rc = od_state_load(o->initial_state, host[0], bytes, f64 ? 1 : 0, p->nx, p->ny, p->nz, &base_label, &base_t);
    if (rc) {
        set_err(err, err_len, od_state_error());
        cleanup();
        return rc;
    }
    rc = od_set_state(ctx, host[0], bytes);
    if (rc) {
        set_err(err, err_len, od_last_error(ctx));
        cleanup();
        return rc;
    }
    if (!quiet) std::printf("Initial state loaded: label %llu (t = %.6f).\n", base_label, base_t);
    r->start_label = base_label;
    r->start_t = base_t;
    std::error_code fec;
    std::filesystem::create_directories(out_dir, fec);
    if (fec) {
        set_err(err, err_len, "cannot create output_dir " + out_dir + ": " + fec.message());
        cleanup();
        return OD_ERR_IO;
    }
    // startup state as label base at t = base_t (solver.rs:228-256), synchronous
    rc = od_state_save(file_name(out_dir, prefix, kind, base_label).c_str(), host[0], f64 ? 1 : 0, p->nx, p->ny,
                       p->nz, base_label, base_t, p->lx, p->ly, p->lz, comp.c_str());
    if (rc) {
        set_err(err, err_len, od_state_error());
        cleanup();
        return rc;
    }
    ++written;

    if (!quiet) std::printf("Starting RK3 explicit time integration...\n");
    const auto t0 = std::chrono::steady_clock::now();
    const long long n = o->n_steps;
    for (long long step = 0; step < n; ++step) {
        rc = od_step(ctx, 1, o->dt);
        if (rc) break;
        if (step % o->save_freq != 0 && step != n - 1) continue;
        const int k = pool.take();
        rc = od_get_state_device(ctx, snap[k], bytes);
        if (rc) break;
        cudaError_t e = cudaEventRecord(ev_snap[k], stream);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(io_stream, ev_snap[k], 0);
        if (e == cudaSuccess) e = cudaMemcpyAsync(host[k], snap[k], bytes, cudaMemcpyDeviceToHost, io_stream);
        if (e == cudaSuccess) e = cudaEventRecord(ev_host[k], io_stream);
        if (e != cudaSuccess) {
            for (auto& t : threads) t.join();
            threads.clear();
            return cuda_fail(e, "dump copy");
        }
        // labels count completed steps (solver.rs:787-793)
        const unsigned long long label = base_label + (unsigned long long)step + 1;
        const double t = base_t + ((double)step + 1.0) * o->dt;
        const bool ckpt = step == n - 1 || (o->checkpoint_freq > 0 && step % o->checkpoint_freq == 0);
        const bool last = step == n - 1;
        if (last) final_slot = k;
        const std::string dump = file_name(out_dir, prefix, kind, label);
        const std::string cpt = file_name(out_dir, "checkpoint", kind, label);
        threads.emplace_back([&, k, label, t, ckpt, last, dump, cpt]() {
            int wrc = 0;
            std::string msg;
            cudaError_t se = cudaEventSynchronize(ev_host[k]);
            if (se != cudaSuccess) {
                wrc = OD_ERR_CUDA;
                msg = cudaGetErrorString(se);
            }
            int nfiles = 0;
            if (!wrc) {
                wrc = od_state_save(dump.c_str(), host[k], f64 ? 1 : 0, p->nx, p->ny, p->nz, label, t, p->lx, p->ly,
                                    p->lz, comp.c_str());
                if (!wrc) ++nfiles;
                if (!wrc && ckpt) {
                    wrc = od_state_save(cpt.c_str(), host[k], f64 ? 1 : 0, p->nx, p->ny, p->nz, label, t, p->lx,
                                        p->ly, p->lz, comp.c_str());
                    if (!wrc) ++nfiles;
                }
                if (wrc) msg = od_state_error();
            }
            {
                std::lock_guard<std::mutex> lk(io_m);
                written += nfiles;
                if (wrc) {
                    ++io_errors;
                    std::fprintf(stderr, "IO task failed: %s\n", msg.c_str());
                }
            }
            if (!last) pool.give(k);  // the final slot is kept for the state report
        });
    }
    if (rc) {
        set_err(err, err_len, od_last_error(ctx));
        cleanup();
        return rc;
    }
    cudaStreamSynchronize(io_stream);
    for (auto& th : threads) th.join();
    threads.clear();
    cudaError_t e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return cuda_fail(e, "step loop");
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    r->seconds = secs;
    r->ms_per_step = n > 0 ? secs * 1000.0 / (double)n : 0.0;
    r->final_label = base_label + (unsigned long long)n;
    r->final_t = n > 0 ? base_t + (double)n * o->dt : base_t;
    if (!quiet) {
        std::printf("Simulation finished in %.3f seconds.\n", secs);
        std::printf("Time per step: %.3f ms\n", r->ms_per_step);
    }
    // final report from the last dump's buffer, else a fresh copy (solver.rs:356-370)
    int slot = final_slot;
    if (slot < 0) {
        slot = 0;
        rc = od_get_state(ctx, host[0], bytes);
        if (rc) {
            set_err(err, err_len, od_last_error(ctx));
            cleanup();
            return rc;
        }
    }
    if (f64)
        state_report((const double*)host[slot], npts, r);
    else
        state_report((const float*)host[slot], npts, r);
    if (!quiet) {
        std::printf("Physical State Check (Final):\n");
        std::printf("  Rho: [%.5f, %.5f]\n", r->rho_min, r->rho_max);
        std::printf("  U:   [%.5f, %.5f]\n", r->u_min, r->u_max);
        std::fflush(stdout);
    }
    r->files_written = written;
    r->io_errors = io_errors;
    cleanup();
    return OD_OK;
}
