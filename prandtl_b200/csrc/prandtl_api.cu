// prandtl_api.cu -- host side of the C ABI (include/prandtl_b200.h).
//
// Owns the per-mesh device state: geometry and neighbour tables, the 1D
// operator tables, scratch (NS gradients, RK registers, staging) and one CUDA
// stream.  All waits are bounded by the configured timeout.
#include <cuda_runtime.h>

#include <unistd.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/prandtl_b200.h"
#include "dgsem_kernels.cuh"
#include "host_common.hpp"

using namespace prandtl;
using namespace prandtl::host;

namespace {
// Host-pointer transfers above kStageMin bytes go through a pinned ring of
// kStageSlots chunks: host threads copy a chunk between the caller's pageable
// buffer and a pinned slot while the DMA engine moves the previous one.
constexpr size_t kStageChunk = size_t(8) << 20;
constexpr int kStageSlots = 4;
constexpr size_t kStageMin = size_t(4) << 20;
// host threads per chunk copy: filling pinned slots from the caller's buffer
// (H2D) gains nothing past 8, emptying them (D2H) up to 12 (measured on a
// 16-core host: 84 MB in 3.0 / 2.1 ms)
constexpr int kCopyPartsH2D = 8, kCopyPartsD2H = 12;
}   // namespace

struct prandtl_handle {
    int dim = 0, order = 0, Np = 0, nd = 0, nf = 0, E = 0, F = 0;
    long long Ndof = 0;
    prandtl_config cfg{};
    PhysParams P{};
    OpTables T{};
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    cudaEvent_t done = nullptr;
    // device memory
    double *d_geo = nullptr;
    int4 *d_nbr = nullptr;
    double *d_fnor = nullptr;
    double *d_in = nullptr, *d_out = nullptr;     // staging / ping-pong states
    double *d_rk1 = nullptr, *d_rk2 = nullptr;    // RK registers
    double *d_grad = nullptr;                     // NS primitive gradients (FP64 path)
    float *d_grad32 = nullptr;                    // NS primitive gradients (FP32-bulk form)
    double *d_alpha = nullptr;
    unsigned long long *d_lambda = nullptr;
    unsigned int *d_health = nullptr;             // sticky state-check bits of the RK stages
    unsigned int *h_health = nullptr;             // pinned host copy of d_health
    BcDev *d_bcs = nullptr;                       // boundary conditions
    // axisymmetric form: node coordinates [2][Ndof], axis-node flags, and the
    // state U recovered from the r-weighted RK state before each RHS
    double *d_xy = nullptr;
    unsigned char *d_axis = nullptr;
    double *d_U = nullptr;
    double *d_budget = nullptr;                   // budget partials [BUDGET_BLOCKS][12] + totals [12]
    // non-affine elements: per-node geometry [dim*dim + 1][Ndof], per-face-node
    // normals [F][Np^(dim-1)][dim], subcell interface normals (blending)
    double *d_ngeo = nullptr, *d_fnn = nullptr, *d_snor = nullptr;
    // prandtl_step's launch graph: kGraphSteps steps of one scheme on one state
    // buffer with one dt, captured on cap_stream and replayed on `stream`
    cudaStream_t cap_stream = nullptr;
    cudaGraphExec_t step_graph = nullptr;
    double *graph_x = nullptr;
    double graph_dt = 0.0;
    int graph_scheme = -1;
    long long graph_launches = 0;        // kernels per replay
    size_t bytes = 0;
    long long launches = 0;
    // optional per-kernel CUDA-event timing (prandtl_profile)
    bool profiling = false;
    std::vector<cudaEvent_t> ev_pool;
    struct Rec { int kernel; cudaEvent_t a, b; };
    std::vector<Rec> recs;
    double prof_ms[PRANDTL_NUM_KERNELS] = {0};
    long long prof_n[PRANDTL_NUM_KERNELS] = {0};
    // pinned staging ring for host-pointer transfers (allocated at the first
    // transfer above kStageMin bytes; null when pinned memory was refused)
    char *h_stage = nullptr;
    bool stage_tried = false;
    cudaEvent_t stage_ev[kStageSlots] = {};
    bool stage_pending[kStageSlots] = {};
    std::string err;
    std::mutex mu;
};

namespace {

// memcpy split over a small persistent pool of host threads (one call at a
// time; a process forked after the pool started copies on its calling thread,
// since the workers do not exist there).  The pool is never destroyed: its
// workers sleep on a condition variable until the process ends, and a forked
// child never joins threads it does not have.
class CopyPool {
  public:
    static CopyPool &get() {
        static CopyPool *pool = new CopyPool();
        return *pool;
    }
    // max_parts: how many threads (the caller included) share the copy
    void copy(void *dst, const void *src, size_t n, int max_parts) {
        if (n < (size_t(1) << 20) || workers_ == 0 || getpid() != pid_ || max_parts < 2) {
            std::memcpy(dst, src, n);
            return;
        }
        std::lock_guard<std::mutex> call(call_mu_);
        const int parts = std::min(workers_ + 1, max_parts);
        {
            std::lock_guard<std::mutex> lk(mu_);
            dst_ = static_cast<char *>(dst);
            src_ = static_cast<const char *>(src);
            n_ = n;
            parts_ = parts;
            pending_ = parts - 1;
            ++gen_;
        }
        cv_.notify_all();
        part(0);
        std::unique_lock<std::mutex> lk(mu_);
        done_cv_.wait(lk, [&] { return pending_ == 0; });
    }
  private:
    CopyPool() : pid_(getpid()) {
        const unsigned hw = std::thread::hardware_concurrency();
        const int n = (int)std::min(12u, hw > 1 ? hw * 3 / 4 : 1u) - 1;
        for (int i = 1; i <= n; ++i) {
            std::thread t([this, i] { loop(i); });
            t.detach();
            ++workers_;
        }
    }
    void part(int i) {
        // 64-byte aligned split points
        const size_t per = (n_ / parts_ + 63) / 64 * 64;
        const size_t b = std::min(n_, per * i), e = std::min(n_, per * (i + 1));
        if (e > b) std::memcpy(dst_ + b, src_ + b, e - b);
    }
    void loop(int i) {
        unsigned seen = 0;
        for (;;) {
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [&] { return gen_ != seen; });
                seen = gen_;
                if (i >= parts_) continue;   // not one of this copy's parts
            }
            part(i);
            std::lock_guard<std::mutex> lk(mu_);
            if (--pending_ == 0) done_cv_.notify_one();
        }
    }
    int workers_ = 0;
    std::mutex call_mu_, mu_;
    std::condition_variable cv_, done_cv_;
    unsigned gen_ = 0;
    int pending_ = 0, parts_ = 1;
    char *dst_ = nullptr;
    const char *src_ = nullptr;
    size_t n_ = 0;
    pid_t pid_;
};

thread_local char g_unbound_error[512];

prandtl_status fail(prandtl_handle *h, prandtl_status st, const std::string &msg) {
    if (h) h->err = msg;
    else set_unbound_error(msg.c_str());
    return st;
}

prandtl_status cuda_fail(prandtl_handle *h, cudaError_t e, const char *what) {
    std::string msg = std::string(what) + ": " + cudaGetErrorString(e);
    return fail(h, e == cudaErrorMemoryAllocation ? PRANDTL_ENOMEM : PRANDTL_ECUDA, msg);
}

#define CK(h, call, what)                                   \
    do {                                                    \
        cudaError_t _e = (call);                            \
        if (_e != cudaSuccess) return cuda_fail(h, _e, what); \
    } while (0)

prandtl_status wait_stream(prandtl_handle *h) {
    cudaError_t e = cudaEventRecord(h->done, h->stream);
    if (e != cudaSuccess) return cuda_fail(h, e, "cudaEventRecord");
    const double limit = h->cfg.timeout_s > 0 ? h->cfg.timeout_s : 120.0;
    const auto t0 = std::chrono::steady_clock::now();
    for (;;) {
        e = cudaEventQuery(h->done);
        if (e == cudaSuccess) return PRANDTL_OK;
        if (e != cudaErrorNotReady) return cuda_fail(h, e, "device work failed");
        const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (el > limit) return fail(h, PRANDTL_ETIMEDOUT, "wait for the handle's stream timed out");
        poll_pause(el);
    }
}

// Waits (bounded by the handle's timeout) for one event.
prandtl_status wait_event(prandtl_handle *h, cudaEvent_t ev) {
    const double limit = h->cfg.timeout_s > 0 ? h->cfg.timeout_s : 120.0;
    const auto t0 = std::chrono::steady_clock::now();
    for (;;) {
        const cudaError_t e = cudaEventQuery(ev);
        if (e == cudaSuccess) return PRANDTL_OK;
        if (e != cudaErrorNotReady) return cuda_fail(h, e, "device work failed");
        const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (el > limit) return fail(h, PRANDTL_ETIMEDOUT, "wait for a staged copy timed out");
        poll_pause(el);
    }
}

// The pinned staging ring, allocated once per handle; false when pinned host
// memory is refused (the transfers then go straight from pageable memory).
bool stage_ready(prandtl_handle *h) {
    if (h->h_stage) return true;
    if (h->stage_tried) return false;
    h->stage_tried = true;
    void *p = nullptr;
    if (cudaHostAlloc(&p, kStageChunk * kStageSlots, cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    for (int k = 0; k < kStageSlots; ++k) {
        if (cudaEventCreateWithFlags(&h->stage_ev[k], cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            for (int j = 0; j < k; ++j) cudaEventDestroy(h->stage_ev[j]);
            cudaFreeHost(p);
            return false;
        }
    }
    h->h_stage = static_cast<char *>(p);
    return true;
}

// Pinned slot k before the host writes into it: its last DMA has finished.
prandtl_status stage_slot_free(prandtl_handle *h, int k) {
    if (!h->stage_pending[k]) return PRANDTL_OK;
    prandtl_status st = wait_event(h, h->stage_ev[k]);
    if (st == PRANDTL_OK) h->stage_pending[k] = false;
    return st;
}

// Host (pageable) -> device on the handle's stream.  Large transfers are
// chunked through the pinned ring: the host threads fill slot k while the DMA
// of slot k-1 runs.  Returns with the DMAs enqueued (not finished).
prandtl_status copy_h2d(prandtl_handle *h, void *dst, const void *src, size_t bytes) {
    if (bytes < kStageMin || !stage_ready(h)) {
        CK(h, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, h->stream), "H2D");
        return PRANDTL_OK;
    }
    const char *s = static_cast<const char *>(src);
    char *d = static_cast<char *>(dst);
    for (size_t off = 0, c = 0; off < bytes; off += kStageChunk, ++c) {
        const int k = (int)(c % kStageSlots);
        const size_t n = std::min(kStageChunk, bytes - off);
        prandtl_status st = stage_slot_free(h, k);
        if (st != PRANDTL_OK) return st;
        char *slot = h->h_stage + (size_t)k * kStageChunk;
        CopyPool::get().copy(slot, s + off, n, kCopyPartsH2D);
        CK(h, cudaMemcpyAsync(d + off, slot, n, cudaMemcpyHostToDevice, h->stream), "H2D chunk");
        CK(h, cudaEventRecord(h->stage_ev[k], h->stream), "cudaEventRecord");
        h->stage_pending[k] = true;
    }
    return PRANDTL_OK;
}

// Device -> host (pageable) after the work already on the handle's stream.
// Small transfers are only enqueued (the caller's next stream wait completes
// them); large ones cross the pinned ring, the host threads emptying slot k
// while later DMAs run, and are in the caller's buffer on return.
prandtl_status copy_d2h(prandtl_handle *h, void *dst, const void *src, size_t bytes) {
    if (bytes < kStageMin || !stage_ready(h)) {
        CK(h, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, h->stream), "D2H");
        return PRANDTL_OK;
    }
    const char *s = static_cast<const char *>(src);
    char *d = static_cast<char *>(dst);
    const size_t nchunks = (bytes + kStageChunk - 1) / kStageChunk;
    auto issue = [&](size_t c) -> prandtl_status {
        const int k = (int)(c % kStageSlots);
        const size_t off = c * kStageChunk, n = std::min(kStageChunk, bytes - off);
        prandtl_status st = stage_slot_free(h, k);
        if (st != PRANDTL_OK) return st;
        CK(h, cudaMemcpyAsync(h->h_stage + (size_t)k * kStageChunk, s + off, n, cudaMemcpyDeviceToHost, h->stream),
           "D2H chunk");
        CK(h, cudaEventRecord(h->stage_ev[k], h->stream), "cudaEventRecord");
        h->stage_pending[k] = true;
        return PRANDTL_OK;
    };
    for (size_t c = 0; c < nchunks && c < (size_t)kStageSlots; ++c) {
        prandtl_status st = issue(c);
        if (st != PRANDTL_OK) return st;
    }
    for (size_t c = 0; c < nchunks; ++c) {
        const int k = (int)(c % kStageSlots);
        const size_t off = c * kStageChunk, n = std::min(kStageChunk, bytes - off);
        prandtl_status st = stage_slot_free(h, k);
        if (st != PRANDTL_OK) return st;
        CopyPool::get().copy(d + off, h->h_stage + (size_t)k * kStageChunk, n, kCopyPartsD2H);
        if (c + kStageSlots < nchunks && (st = issue(c + kStageSlots)) != PRANDTL_OK) return st;
    }
    return PRANDTL_OK;
}

// Copies the sticky state-check flag to the pinned host word, waits (bounded),
// clears the device flag and reports PRANDTL_ENONFINITE when it was set.
prandtl_status wait_and_report_health(prandtl_handle *h) {
    cudaError_t e = cudaMemcpyAsync(h->h_health, h->d_health, sizeof(unsigned int), cudaMemcpyDeviceToHost,
                                    h->stream);
    if (e != cudaSuccess) return cuda_fail(h, e, "D2H state check flag");
    e = cudaMemsetAsync(h->d_health, 0, sizeof(unsigned int), h->stream);
    if (e != cudaSuccess) return cuda_fail(h, e, "clear state check flag");
    prandtl_status st = wait_stream(h);
    if (st != PRANDTL_OK) return st;
    const unsigned bits = *h->h_health;
    *h->h_health = 0u;
    if (bits) return fail(h, PRANDTL_ENONFINITE, health_text(bits));
    return PRANDTL_OK;
}

// Event pair around one launch when profiling; returns the stop event or null.
cudaEvent_t prof_begin(prandtl_handle *h, int kernel) {
    if (!h->profiling || h->ev_pool.size() < 2 || h->recs.size() >= 8192) return nullptr;
    cudaEvent_t a = h->ev_pool.back(); h->ev_pool.pop_back();
    cudaEvent_t b = h->ev_pool.back(); h->ev_pool.pop_back();
    cudaEventRecord(a, h->stream);
    h->recs.push_back({kernel, a, b});
    return b;
}
void prof_end(prandtl_handle *h, cudaEvent_t b) {
    if (b) cudaEventRecord(b, h->stream);
}

MeshDev mesh_dev(const prandtl_handle *h) {
    MeshDev m;
    m.geo = h->d_geo;
    m.nbr = h->d_nbr;
    m.fnor = h->d_fnor;
    m.E = h->E;
    m.Ndof = h->Ndof;
    m.bcs = h->d_bcs;
    m.rad = h->d_xy ? h->d_xy + h->Ndof : nullptr;
    m.axis = h->d_axis;
    m.ngeo = h->d_ngeo;
    m.fnn = h->d_fnn;
    m.snor = h->d_snor;
    return m;
}

// One RHS evaluation of `u` with the given epilogue.
prandtl_status run_rhs(prandtl_handle *h, const double *u, RhsArgs a) {
    const MeshDev m = mesh_dev(h);
    a.u = u;
    if (h->d_U) {   // axisymmetric: fluxes of U, the RK update of r U (DGSEMOperator::Mult)
        cudaError_t e = launch_axi_recover(u, h->d_U, h->d_xy, h->d_axis, h->Ndof, h->nd,
                                           h->cfg.axis_rho_floor > 0.0 ? h->cfg.axis_rho_floor : 1e-12,
                                           h->stream);
        if (e != cudaSuccess) return cuda_fail(h, e, "axisymmetric recovery launch");
        h->launches++;
        a.u = h->d_U;
        a.u_rk = u;
    }
    const bool ns = h->cfg.parabolic != 0;
    const bool fp32 = h->cfg.precision == 1;
    if (ns) {
        LiftArgs la{u, h->d_grad, h->d_grad32};
        cudaEvent_t pe = prof_begin(h, PRANDTL_KERNEL_LIFT);
        cudaError_t e = fp32 ? launch_lift_fp32(h->dim, h->order, m, la, h->P, h->T, h->stream)
                             : launch_lift(h->dim, h->order, m, la, h->P, h->T, h->stream);
        prof_end(h, pe);
        if (e != cudaSuccess) return cuda_fail(h, e, "lift kernel launch");
        h->launches++;
        a.grad = h->d_grad;
        a.grad32 = h->d_grad32;
    }
    a.alpha = h->cfg.blending ? h->d_alpha : nullptr;
    cudaEvent_t pe = prof_begin(h, PRANDTL_KERNEL_RHS);
    cudaError_t e = fp32 ? launch_rhs_fp32(h->dim, h->order, ns, m, a, h->P, h->T, h->stream)
                         : launch_rhs(h->dim, h->order, ns, m, a, h->P, h->T, h->stream);
    prof_end(h, pe);
    if (e != cudaSuccess) return cuda_fail(h, e, "rhs kernel launch");
    h->launches++;
    return PRANDTL_OK;
}

void free_all(prandtl_handle *h) {
    cudaFree(h->d_geo);
    cudaFree(h->d_nbr);
    cudaFree(h->d_fnor);
    cudaFree(h->d_in);
    cudaFree(h->d_out);
    cudaFree(h->d_rk1);
    cudaFree(h->d_rk2);
    cudaFree(h->d_grad);
    cudaFree(h->d_grad32);
    cudaFree(h->d_alpha);
    cudaFree(h->d_lambda);
    cudaFree(h->d_health);
    if (h->h_health) cudaFreeHost(h->h_health);
    cudaFree(h->d_bcs);
    cudaFree(h->d_xy);
    cudaFree(h->d_axis);
    cudaFree(h->d_U);
    cudaFree(h->d_budget);
    cudaFree(h->d_ngeo);
    cudaFree(h->d_fnn);
    cudaFree(h->d_snor);
    if (h->h_stage) {
        for (int k = 0; k < kStageSlots; ++k) cudaEventDestroy(h->stage_ev[k]);
        cudaFreeHost(h->h_stage);
        h->h_stage = nullptr;
    }
    if (h->step_graph) cudaGraphExecDestroy(h->step_graph);
    if (h->cap_stream) cudaStreamDestroy(h->cap_stream);
    if (h->done) cudaEventDestroy(h->done);
    for (auto &r : h->recs) { cudaEventDestroy(r.a); cudaEventDestroy(r.b); }
    for (auto ev : h->ev_pool) cudaEventDestroy(ev);
    h->recs.clear();
    h->ev_pool.clear();
    if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
}

// The stage launches of `nsteps` steps on the device state x: SSP-RK3 (Shu-Osher,
// x -> y1 -> y2 -> x) or LSRK4(5) (2N storage, ping-pong with the state back in
// x at the end).  Every stage ORs its state check into the handle's flag.
prandtl_status enqueue_steps(prandtl_handle *h, double *x, double dt, int scheme, int nsteps) {
    prandtl_status st = PRANDTL_OK;
    if (scheme == PRANDTL_RK3SSP) {
        double *y1 = h->d_rk1, *y2 = h->d_rk2;
        for (int s = 0; s < nsteps && st == PRANDTL_OK; ++s) {
            RhsArgs a{};
            a.dt = dt;
            a.x0 = x;
            a.health = h->d_health;
            a.mode = EPI_SSP1; a.u_out = y1;
            if ((st = run_rhs(h, x, a)) != PRANDTL_OK) break;
            a.mode = EPI_SSP2; a.u_out = y2;
            if ((st = run_rhs(h, y1, a)) != PRANDTL_OK) break;
            a.mode = EPI_SSP3; a.u_out = x;
            st = run_rhs(h, y2, a);
        }
        return st;
    }
    static const double A[5] = {0.0, -567301805773.0 / 1357537059087.0,
                                -2404267990393.0 / 2016746695238.0,
                                -3550918686646.0 / 2091501179385.0,
                                -1275806237668.0 / 842570457699.0};
    static const double B[5] = {1432997174477.0 / 9575080441755.0,
                                5161836677717.0 / 13612068292357.0,
                                1720146321549.0 / 2090206949498.0,
                                3134564353537.0 / 4481467310338.0,
                                2277821191437.0 / 14882151754819.0};
    double *cur = x, *other = (x == h->d_in) ? h->d_out : h->d_rk2;
    double *du = h->d_rk1;
    for (int s = 0; s < nsteps && st == PRANDTL_OK; ++s)
        for (int k = 0; k < 5; ++k) {
            RhsArgs a{};
            a.mode = EPI_LSRK;
            a.health = h->d_health;
            a.dt = dt;
            a.rkA = A[k];
            a.rkB = B[k];
            a.du = du;
            a.u_out = other;
            if ((st = run_rhs(h, cur, a)) != PRANDTL_OK) break;
            std::swap(cur, other);
        }
    if (st == PRANDTL_OK && cur != x)
        CK(h, cudaMemcpyAsync(x, cur, (size_t)h->nf * h->Ndof * sizeof(double), cudaMemcpyDeviceToDevice,
                              h->stream), "copy result");
    return st;
}

// Steps per captured graph: even, so that LSRK's ping-pong ends in x.
constexpr int kGraphSteps = 4;

// The handle's step graph for (x, dt, scheme), captured on its capture stream
// the first time (and whenever one of them changes).
prandtl_status step_graph_for(prandtl_handle *h, double *x, double dt, int scheme) {
    if (h->step_graph && h->graph_x == x && h->graph_dt == dt && h->graph_scheme == scheme) return PRANDTL_OK;
    if (h->step_graph) cudaGraphExecDestroy(h->step_graph);
    h->step_graph = nullptr;
    const cudaStream_t run = h->stream;
    const long long before = h->launches;
    h->stream = h->cap_stream;
    // relaxed: the first launch of a kernel on this device may set its
    // shared-memory attribute (a host-side call) while the stream captures
    cudaError_t e = cudaStreamBeginCapture(h->cap_stream, cudaStreamCaptureModeRelaxed);
    prandtl_status st = e == cudaSuccess ? enqueue_steps(h, x, dt, scheme, kGraphSteps) : PRANDTL_OK;
    cudaGraph_t g = nullptr;
    const cudaError_t e2 = e == cudaSuccess ? cudaStreamEndCapture(h->cap_stream, &g) : e;
    h->stream = run;
    h->graph_launches = h->launches - before;
    h->launches = before;
    if (st != PRANDTL_OK) {
        if (g) cudaGraphDestroy(g);
        return st;
    }
    if (e2 != cudaSuccess) return cuda_fail(h, e2, "capture step graph");
    e = cudaGraphInstantiate(&h->step_graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        h->step_graph = nullptr;
        return cuda_fail(h, e, "instantiate step graph");
    }
    h->graph_x = x;
    h->graph_dt = dt;
    h->graph_scheme = scheme;
    return PRANDTL_OK;
}

template <typename T>
prandtl_status dalloc(prandtl_handle *h, T **p, size_t count, const char *what) {
    cudaError_t e = cudaMalloc((void **)p, count * sizeof(T));
    if (e != cudaSuccess) { *p = nullptr; return cuda_fail(h, e, what); }
    h->bytes += count * sizeof(T);
    return PRANDTL_OK;
}

}   // namespace

extern "C" {

void prandtl_config_default(prandtl_config *c) {
    if (!c) return;
    std::memset(c, 0, sizeof(*c));
    c->gamma = 1.4;
    c->Pr = 0.72;
    c->mu = 0.02;
    c->R_gas = 287.05;
    c->alpha_max = 0.5;
    c->alpha_min = 0.001;
    c->surface_dissipation = 1;
    c->timeout_s = 120.0;
}

prandtl_status prandtl_create(const prandtl_mesh_desc *md, const prandtl_config *cfg,
                              prandtl_handle **out) {
    set_unbound_error("");
    if (!out) return fail(nullptr, PRANDTL_EINVAL, "out is NULL");
    *out = nullptr;
    if (!md || !cfg) return fail(nullptr, PRANDTL_EINVAL, "mesh or config is NULL");
    if (cfg->precision != 0 && cfg->precision != 1)
        return fail(nullptr, PRANDTL_EUNSUPPORTED, "precision must be 0 (FP64) or 1 (FP32 bulk)");
    if (!(cfg->gamma > 1.0) || !(cfg->Pr > 0.0)) return fail(nullptr, PRANDTL_EINVAL, "bad gamma/Pr");
    if (cfg->axisymmetric && (md->dim != 2 || cfg->parabolic))
        return fail(nullptr, PRANDTL_EUNSUPPORTED, "the axisymmetric form is 2D Euler");
    if (cfg->axisymmetric && !cfg->node_coords)
        return fail(nullptr, PRANDTL_EINVAL, "the axisymmetric form needs node_coords");

    const int dim = md->dim, E = md->num_elements, F = md->num_faces;
    std::vector<int4> nbr;
    {
        std::string msg;
        prandtl_status vst = check_bcs(cfg, md->dim, msg);
        if (vst == PRANDTL_OK) vst = validate_mesh(md, nbr, msg, cfg->num_bcs);
        if (vst == PRANDTL_OK) vst = check_viscous_bcs(md, cfg, msg);
        if (vst == PRANDTL_OK) vst = check_curved(md, msg);
        if (vst == PRANDTL_OK && mesh_curved(md) && cfg->precision != 0 && cfg->parabolic) {
            msg = "non-affine Navier-Stokes runs in the FP64 form only (precision 0); FP32 bulk takes Euler";
            vst = PRANDTL_EUNSUPPORTED;
        }
        if (vst == PRANDTL_OK && cfg->parabolic && cfg->quirks != 0)
            vst = mesh_curved(md) ? check_face_node_normals(md, msg) : check_face_normals(md, msg);
        if (vst != PRANDTL_OK) return fail(nullptr, vst, msg);
    }

    int ndev = 0;
    cudaError_t ce = cudaGetDeviceCount(&ndev);
    if (ce != cudaSuccess || ndev == 0)
        return fail(nullptr, PRANDTL_ECUDA, std::string("no CUDA device: ") + cudaGetErrorString(ce));

    prandtl_handle *h = new prandtl_handle();
    h->dim = dim;
    h->order = md->order;
    h->Np = md->order + 1;
    h->nd = 1;
    for (int d = 0; d < dim; ++d) h->nd *= h->Np;
    h->nf = dim + 2;
    h->E = E;
    h->F = F;
    h->Ndof = (long long)E * h->nd;
    h->cfg = *cfg;
    h->cfg.bcs = nullptr;   // the caller's table is copied to the device below
    h->cfg.node_coords = nullptr;   // likewise the axisymmetric node coordinates
    if (h->cfg.timeout_s <= 0) h->cfg.timeout_s = 120.0;
    build_tables(md->order, h->T);
    build_phys(h->cfg, md->order, h->P);
    cudaGetDevice(&h->device);

    auto bail = [&](prandtl_status st) {
        set_unbound_error(h->err.c_str());
        free_all(h);
        delete h;
        return st;
    };
    prandtl_status st;
    if ((ce = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking)) != cudaSuccess)
        return bail(cuda_fail(h, ce, "cudaStreamCreate"));
    h->own_stream = true;
    if ((ce = cudaEventCreateWithFlags(&h->done, cudaEventDisableTiming)) != cudaSuccess)
        return bail(cuda_fail(h, ce, "cudaEventCreate"));
    if ((ce = cudaStreamCreateWithFlags(&h->cap_stream, cudaStreamNonBlocking)) != cudaSuccess)
        return bail(cuda_fail(h, ce, "cudaStreamCreate (capture)"));
    const size_t S = (size_t)h->nf * h->Ndof;
    const int GEO = dim * dim + 1;
    if ((st = dalloc(h, &h->d_geo, (size_t)E * GEO, "geometry")) != PRANDTL_OK) return bail(st);
    if ((st = dalloc(h, &h->d_nbr, nbr.size(), "neighbours")) != PRANDTL_OK) return bail(st);
    if ((st = dalloc(h, &h->d_fnor, (size_t)(F > 0 ? F : 1) * dim, "normals")) != PRANDTL_OK) return bail(st);
    if ((st = dalloc(h, &h->d_in, S, "state in")) != PRANDTL_OK) return bail(st);
    if ((st = dalloc(h, &h->d_out, S, "state out")) != PRANDTL_OK) return bail(st);
    if ((st = dalloc(h, &h->d_rk1, S, "rk register 1")) != PRANDTL_OK) return bail(st);
    if ((st = dalloc(h, &h->d_rk2, S, "rk register 2")) != PRANDTL_OK) return bail(st);
    if (cfg->parabolic && cfg->precision == 0 && (st = dalloc(h, &h->d_grad, (size_t)dim * S, "gradients")) != PRANDTL_OK)
        return bail(st);
    if (cfg->parabolic && cfg->precision == 1 && (st = dalloc(h, &h->d_grad32, (size_t)dim * S, "gradients")) != PRANDTL_OK)
        return bail(st);
    if ((st = dalloc(h, &h->d_alpha, (size_t)E, "alpha")) != PRANDTL_OK) return bail(st);
    if ((st = dalloc(h, &h->d_lambda, 1, "lambda")) != PRANDTL_OK) return bail(st);
    if ((st = dalloc(h, &h->d_health, 1, "state check flag")) != PRANDTL_OK) return bail(st);
    if ((ce = cudaMemset(h->d_health, 0, sizeof(unsigned int))) != cudaSuccess)
        return bail(cuda_fail(h, ce, "memset state check flag"));
    if ((ce = cudaMallocHost(&h->h_health, sizeof(unsigned int))) != cudaSuccess)
        return bail(cuda_fail(h, ce, "pinned state check flag"));
    *h->h_health = 0u;
    if ((st = dalloc(h, &h->d_budget, (size_t)(BUDGET_BLOCKS + 1) * 12, "budgets")) != PRANDTL_OK) return bail(st);
    const std::vector<BcDev> bcs = device_bcs(cfg, md->dim);
    if (!bcs.empty()) {
        if ((st = dalloc(h, &h->d_bcs, bcs.size(), "boundary conditions")) != PRANDTL_OK) return bail(st);
        if ((ce = cudaMemcpy(h->d_bcs, bcs.data(), bcs.size() * sizeof(BcDev), cudaMemcpyHostToDevice)) != cudaSuccess)
            return bail(cuda_fail(h, ce, "upload boundary conditions"));
    }

    const std::vector<double> geo = geometry_rows(md);
    if ((ce = cudaMemcpy(h->d_geo, geo.data(), geo.size() * sizeof(double), cudaMemcpyHostToDevice)) != cudaSuccess)
        return bail(cuda_fail(h, ce, "upload geometry"));
    if ((ce = cudaMemcpy(h->d_nbr, nbr.data(), nbr.size() * sizeof(int4), cudaMemcpyHostToDevice)) != cudaSuccess)
        return bail(cuda_fail(h, ce, "upload neighbours"));
    if (F > 0 && (ce = cudaMemcpy(h->d_fnor, md->face_nor, (size_t)F * dim * sizeof(double),
                                  cudaMemcpyHostToDevice)) != cudaSuccess)
        return bail(cuda_fail(h, ce, "upload normals"));
    if ((ce = cudaMemset(h->d_alpha, 0, (size_t)E * sizeof(double))) != cudaSuccess)
        return bail(cuda_fail(h, ce, "memset alpha"));
    if (mesh_curved(md)) {   // per-node geometry of non-affine elements
        const std::vector<double> ng = node_geometry_soa(md);
        const size_t nfn_all = (size_t)(F > 0 ? F : 1) * (h->nd / h->Np) * dim;
        if ((st = dalloc(h, &h->d_ngeo, ng.size(), "node geometry")) != PRANDTL_OK) return bail(st);
        if ((st = dalloc(h, &h->d_fnn, nfn_all, "face node normals")) != PRANDTL_OK) return bail(st);
        if ((ce = cudaMemcpy(h->d_ngeo, ng.data(), ng.size() * sizeof(double), cudaMemcpyHostToDevice)) != cudaSuccess)
            return bail(cuda_fail(h, ce, "upload node geometry"));
        if (F > 0 && (ce = cudaMemcpy(h->d_fnn, md->face_node_nor, (size_t)F * (h->nd / h->Np) * dim * sizeof(double),
                                      cudaMemcpyHostToDevice)) != cudaSuccess)
            return bail(cuda_fail(h, ce, "upload face node normals"));
        if (cfg->blending) {
            const std::vector<double> sn = subcell_normals(md, h->T);
            if ((st = dalloc(h, &h->d_snor, sn.size(), "subcell normals")) != PRANDTL_OK) return bail(st);
            if ((ce = cudaMemcpy(h->d_snor, sn.data(), sn.size() * sizeof(double), cudaMemcpyHostToDevice)) != cudaSuccess)
                return bail(cuda_fail(h, ce, "upload subcell normals"));
        }
    }
    if (cfg->axisymmetric) {
        // DGSEMOperator::BuildAxisIndexFromMarker (DGSEMOperator.cpp:482-518):
        // nodes at |r| <= 1e-14 of the elements on axis boundary faces
        std::vector<unsigned char> axis((size_t)h->Ndof, 0);
        for (int f = 0; f < F; ++f) {
            const int *fe = md->face_elems + 4 * f;
            if (fe[2] >= 0 || cfg->bcs[fe[3]].type != PRANDTL_BC_AXIS) continue;
            for (int n = 0; n < h->nd; ++n) {
                const long long g = (long long)fe[0] * h->nd + n;
                if (std::abs(cfg->node_coords[h->Ndof + g]) <= 1e-14) axis[(size_t)g] = 1;
            }
        }
        if ((st = dalloc(h, &h->d_xy, (size_t)2 * h->Ndof, "node coordinates")) != PRANDTL_OK) return bail(st);
        if ((st = dalloc(h, &h->d_axis, (size_t)h->Ndof, "axis nodes")) != PRANDTL_OK) return bail(st);
        if ((st = dalloc(h, &h->d_U, S, "recovered state")) != PRANDTL_OK) return bail(st);
        if ((ce = cudaMemcpy(h->d_xy, cfg->node_coords, (size_t)2 * h->Ndof * sizeof(double),
                             cudaMemcpyHostToDevice)) != cudaSuccess)
            return bail(cuda_fail(h, ce, "upload node coordinates"));
        if ((ce = cudaMemcpy(h->d_axis, axis.data(), axis.size(), cudaMemcpyHostToDevice)) != cudaSuccess)
            return bail(cuda_fail(h, ce, "upload axis nodes"));
    }
    *out = h;
    return PRANDTL_OK;
}

prandtl_status prandtl_destroy(prandtl_handle *h) {
    if (!h) return PRANDTL_EINVAL;
    {
        std::lock_guard<std::mutex> lk(h->mu);
        cudaSetDevice(h->device);
        if (h->stream) wait_stream(h);
        free_all(h);
    }
    delete h;
    return PRANDTL_OK;
}

prandtl_status prandtl_rhs(prandtl_handle *h, const double *u, double *dudt, double t,
                           double *lambda_max, int ptr_flags) {
    (void)t;
    if (!h || !u || !dudt) return h ? fail(h, PRANDTL_EINVAL, "null pointer") : PRANDTL_EINVAL;
    std::lock_guard<std::mutex> lk(h->mu);
    h->err.clear();
    CK(h, cudaSetDevice(h->device), "cudaSetDevice");
    const size_t bytes = (size_t)h->nf * h->Ndof * sizeof(double);
    const bool dev = (ptr_flags & PRANDTL_PTR_DEVICE) != 0;
    const double *u_d = u;
    double *dudt_d = dudt;
    if (!dev) {
        prandtl_status st = copy_h2d(h, h->d_in, u, bytes);
        if (st != PRANDTL_OK) return st;
        u_d = h->d_in;
        dudt_d = h->d_out;
    }
    if (lambda_max) CK(h, cudaMemsetAsync(h->d_lambda, 0, sizeof(unsigned long long), h->stream), "memset");
    RhsArgs a{};
    a.dudt = dudt_d;
    a.lambda = lambda_max ? h->d_lambda : nullptr;
    a.mode = EPI_STORE;
    prandtl_status st = run_rhs(h, u_d, a);
    if (st != PRANDTL_OK) return st;
    unsigned long long lam_bits = 0;
    if (!dev && (st = copy_d2h(h, dudt, h->d_out, bytes)) != PRANDTL_OK) return st;
    if (lambda_max)
        CK(h, cudaMemcpyAsync(&lam_bits, h->d_lambda, sizeof(lam_bits), cudaMemcpyDeviceToHost, h->stream), "D2H lambda");
    if (!dev || lambda_max) {
        st = wait_stream(h);
        if (st != PRANDTL_OK) return st;
    }
    if (lambda_max) {
        double v;
        std::memcpy(&v, &lam_bits, sizeof(v));
        *lambda_max = v;
    }
    return PRANDTL_OK;
}

prandtl_status prandtl_step(prandtl_handle *h, double *u, double t, double dt, int scheme,
                            int nsteps, int ptr_flags) {
    (void)t;
    if (!h || !u) return h ? fail(h, PRANDTL_EINVAL, "null pointer") : PRANDTL_EINVAL;
    if (nsteps < 0 || !(std::isfinite(dt))) return fail(h, PRANDTL_EINVAL, "bad nsteps/dt");
    if (scheme != PRANDTL_RK3SSP && scheme != PRANDTL_LSRK45) return fail(h, PRANDTL_EINVAL, "unknown scheme");
    std::lock_guard<std::mutex> lk(h->mu);
    h->err.clear();
    CK(h, cudaSetDevice(h->device), "cudaSetDevice");
    const size_t bytes = (size_t)h->nf * h->Ndof * sizeof(double);
    const bool dev = (ptr_flags & PRANDTL_PTR_DEVICE) != 0;
    double *x = u;
    prandtl_status st = PRANDTL_OK;
    if (!dev) {
        if ((st = copy_h2d(h, h->d_in, u, bytes)) != PRANDTL_OK) return st;
        x = h->d_in;
    }
    int left = nsteps;
    // long runs replay a captured graph of kGraphSteps steps (one launch per
    // replay instead of one per kernel); the remainder runs launch by launch
    if (!h->profiling && nsteps >= 2 * kGraphSteps) {
        st = step_graph_for(h, x, dt, scheme);
        for (; st == PRANDTL_OK && left >= kGraphSteps; left -= kGraphSteps) {
            cudaError_t e = cudaGraphLaunch(h->step_graph, h->stream);
            if (e != cudaSuccess) st = cuda_fail(h, e, "step graph launch");
            else h->launches += h->graph_launches;
        }
    }
    if (st == PRANDTL_OK) st = enqueue_steps(h, x, dt, scheme, left);
    if (st != PRANDTL_OK) return st;
    if (!dev) {
        if ((st = copy_d2h(h, u, x, bytes)) != PRANDTL_OK) return st;
        st = wait_and_report_health(h);
    }
    return st;
}

prandtl_status prandtl_get_alpha(prandtl_handle *h, double *alpha, int ptr_flags) {
    if (!h || !alpha) return h ? fail(h, PRANDTL_EINVAL, "null pointer") : PRANDTL_EINVAL;
    std::lock_guard<std::mutex> lk(h->mu);
    CK(h, cudaSetDevice(h->device), "cudaSetDevice");
    const bool dev = (ptr_flags & PRANDTL_PTR_DEVICE) != 0;
    CK(h, cudaMemcpyAsync(alpha, h->d_alpha, (size_t)h->E * sizeof(double),
                          dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, h->stream),
       "copy alpha");
    return wait_stream(h);
}

prandtl_status prandtl_recover_state(prandtl_handle *h, const double *rU, double *U, int ptr_flags) {
    if (!h || !rU || !U) return h ? fail(h, PRANDTL_EINVAL, "null pointer") : PRANDTL_EINVAL;
    std::lock_guard<std::mutex> lk(h->mu);
    h->err.clear();
    if (!h->d_U) return fail(h, PRANDTL_EUNSUPPORTED, "not an axisymmetric operator");
    CK(h, cudaSetDevice(h->device), "cudaSetDevice");
    const size_t bytes = (size_t)h->nf * h->Ndof * sizeof(double);
    const bool dev = (ptr_flags & PRANDTL_PTR_DEVICE) != 0;
    const double *src = rU;
    if (!dev) {
        CK(h, cudaMemcpyAsync(h->d_in, rU, bytes, cudaMemcpyHostToDevice, h->stream), "H2D rU");
        src = h->d_in;
    }
    CK(h, launch_axi_recover(src, dev ? U : h->d_out, h->d_xy, h->d_axis, h->Ndof, h->nd,
                             h->cfg.axis_rho_floor > 0.0 ? h->cfg.axis_rho_floor : 1e-12, h->stream),
       "axisymmetric recovery launch");
    h->launches++;
    if (!dev) CK(h, cudaMemcpyAsync(U, h->d_out, bytes, cudaMemcpyDeviceToHost, h->stream), "D2H U");
    return wait_stream(h);
}

prandtl_status prandtl_budgets(prandtl_handle *h, const double *u, const double *dudt, double *out, int ptr_flags) {
    if (!h || !u || !out) return h ? fail(h, PRANDTL_EINVAL, "null pointer") : PRANDTL_EINVAL;
    std::lock_guard<std::mutex> lk(h->mu);
    h->err.clear();
    if (h->d_U) return fail(h, PRANDTL_EUNSUPPORTED, "budgets are defined for the planar forms");
    CK(h, cudaSetDevice(h->device), "cudaSetDevice");
    const size_t bytes = (size_t)h->nf * h->Ndof * sizeof(double);
    const bool dev = (ptr_flags & PRANDTL_PTR_DEVICE) != 0;
    const double *ud = u, *dd = dudt;
    if (!dev) {
        CK(h, cudaMemcpyAsync(h->d_in, u, bytes, cudaMemcpyHostToDevice, h->stream), "H2D u");
        ud = h->d_in;
        if (dudt) {
            CK(h, cudaMemcpyAsync(h->d_out, dudt, bytes, cudaMemcpyHostToDevice, h->stream), "H2D dudt");
            dd = h->d_out;
        }
    }
    double *tot = h->d_budget + (size_t)BUDGET_BLOCKS * 12;
    const double *ndetj = h->d_ngeo ? h->d_ngeo + (size_t)(h->dim * h->dim) * h->Ndof : nullptr;
    CK(h, launch_budgets(ud, dd, h->d_geo, ndetj, h->T.w, h->dim, h->Np, h->E, h->cfg.gamma, h->d_budget, tot,
                         h->stream),
       "budget kernel launch");
    h->launches += 2;
    double buf[12];
    CK(h, cudaMemcpyAsync(buf, tot, sizeof(buf), cudaMemcpyDeviceToHost, h->stream), "D2H budgets");
    prandtl_status st = wait_stream(h);
    if (st != PRANDTL_OK) return st;
    // device slots: conserved [0..4], entropy [5], rates [6..10], entropy rate [11]
    const int nf = h->nf;
    for (int f = 0; f < nf; ++f) {
        out[f] = buf[f];
        out[nf + 1 + f] = dudt ? buf[6 + f] : 0.0;
    }
    out[nf] = buf[5];
    out[2 * nf + 1] = dudt ? buf[11] : 0.0;
    return PRANDTL_OK;
}

double prandtl_cfl_dt(double cfl, double hmin, double lambda_max, int order) {
    return cfl * hmin / (lambda_max * std::pow(order + 1, 2));
}

prandtl_status prandtl_set_stream(prandtl_handle *h, void *cuda_stream) {
    if (!h) return PRANDTL_EINVAL;
    std::lock_guard<std::mutex> lk(h->mu);
    if (h->own_stream && h->stream) {
        prandtl_status st = wait_stream(h);
        if (st != PRANDTL_OK) return st;
        cudaStreamDestroy(h->stream);
    }
    h->stream = (cudaStream_t)cuda_stream;
    h->own_stream = false;
    return PRANDTL_OK;
}

prandtl_status prandtl_synchronize(prandtl_handle *h) {
    if (!h) return PRANDTL_EINVAL;
    std::lock_guard<std::mutex> lk(h->mu);
    h->err.clear();
    CK(h, cudaSetDevice(h->device), "cudaSetDevice");
    return wait_and_report_health(h);
}

long long prandtl_kernel_launches(const prandtl_handle *h) { return h ? h->launches : 0; }

prandtl_status prandtl_profile(prandtl_handle *h, int enable) {
    if (!h) return PRANDTL_EINVAL;
    std::lock_guard<std::mutex> lk(h->mu);
    CK(h, cudaSetDevice(h->device), "cudaSetDevice");
    if (enable && h->ev_pool.empty() && h->recs.empty()) {
        for (int i = 0; i < 2 * 8192; ++i) {
            cudaEvent_t ev;
            CK(h, cudaEventCreate(&ev), "cudaEventCreate");
            h->ev_pool.push_back(ev);
        }
    }
    h->profiling = enable != 0;
    return PRANDTL_OK;
}

prandtl_status prandtl_profile_read(prandtl_handle *h, int kernel, double *total_ms, long long *launches) {
    if (!h || kernel < 0 || kernel >= PRANDTL_NUM_KERNELS) return PRANDTL_EINVAL;
    std::lock_guard<std::mutex> lk(h->mu);
    prandtl_status st = wait_stream(h);
    if (st != PRANDTL_OK) return st;
    for (auto &r : h->recs) {
        float ms = 0.f;
        CK(h, cudaEventElapsedTime(&ms, r.a, r.b), "cudaEventElapsedTime");
        h->prof_ms[r.kernel] += ms;
        h->prof_n[r.kernel] += 1;
        h->ev_pool.push_back(r.a);
        h->ev_pool.push_back(r.b);
    }
    h->recs.clear();
    if (total_ms) *total_ms = h->prof_ms[kernel];
    if (launches) *launches = h->prof_n[kernel];
    return PRANDTL_OK;
}

prandtl_status prandtl_profile_reset(prandtl_handle *h) {
    if (!h) return PRANDTL_EINVAL;
    double ms;
    long long n;
    prandtl_status st = prandtl_profile_read(h, 0, &ms, &n);
    if (st != PRANDTL_OK) return st;
    std::lock_guard<std::mutex> lk(h->mu);
    for (int k = 0; k < PRANDTL_NUM_KERNELS; ++k) { h->prof_ms[k] = 0.0; h->prof_n[k] = 0; }
    return PRANDTL_OK;
}

size_t prandtl_device_bytes(const prandtl_handle *h) { return h ? h->bytes : 0; }

const char *prandtl_last_error(const prandtl_handle *h) {
    return h ? h->err.c_str() : unbound_error();
}

const char *prandtl_version(void) { return "prandtl_b200 0.2 (sm_100a, FP64 + FP32-bulk)"; }

}   // extern "C"

namespace prandtl {
namespace host {
void set_unbound_error(const char *msg) {
    std::snprintf(g_unbound_error, sizeof(g_unbound_error), "%s", msg ? msg : "");
}
const char *unbound_error() { return g_unbound_error; }
}   // namespace host
}   // namespace prandtl
