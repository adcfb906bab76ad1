// prandtl_batch.cu -- host side of batches (prandtl_batch_* in the C ABI).
//
// A batch owns one device arena in which every admitted solve gets one block:
// three RK state buffers, NS gradients, the blending field and its mesh
// tables.  Solves of the same (dim, order, physics) form a class; a class
// keeps the solve ids and the padded element prefix over them in device
// memory, which the persistent batch kernels walk.  One step is the stage
// sequence (per stage and class: lifting, then RHS + fused stage update) and a
// step-end kernel; it is captured once per class set in a CUDA graph and
// replayed, so admissions and retirements between advances only rewrite the
// small device tables.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <deque>
#include <iterator>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "../../include/prandtl_b200.h"
#include "dgsem_kernels.cuh"
#include "host_common.hpp"

using namespace prandtl;
using namespace prandtl::host;

namespace {

constexpr size_t ALIGN = 256;
size_t align_up(size_t x) { return (x + ALIGN - 1) / ALIGN * ALIGN; }

// Carpenter & Kennedy (1994) 5-stage 2N-storage RK4, solution 3.
const double LSRK_A[5] = {0.0, -567301805773.0 / 1357537059087.0, -2404267990393.0 / 2016746695238.0,
                          -3550918686646.0 / 2091501179385.0, -1275806237668.0 / 842570457699.0};
const double LSRK_B[5] = {1432997174477.0 / 9575080441755.0, 5161836677717.0 / 13612068292357.0,
                          1720146321549.0 / 2090206949498.0, 3134564353537.0 / 4481467310338.0,
                          2277821191437.0 / 14882151754819.0};

// First-fit allocator over [0, size): free ranges by offset, merged on release.
class Arena {
public:
    void reset(size_t size) {
        free_.clear();
        if (size) free_[0] = size;
    }
    bool alloc(size_t n, size_t *off) {
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < n) continue;
            *off = it->first;
            const size_t rest = it->second - n, at = it->first + n;
            free_.erase(it);
            if (rest) free_[at] = rest;
            return true;
        }
        return false;
    }
    void release(size_t off, size_t n) {
        auto it = free_.emplace(off, n).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
    size_t largest() const {
        size_t m = 0;
        for (const auto &kv : free_) m = std::max(m, kv.second);
        return m;
    }

private:
    std::map<size_t, size_t> free_;
};

// Byte offsets of one solve's arrays inside its arena block.
struct Layout {
    size_t u[3], grad, alpha, geo, nbr, fnor, bcs, total;
};

Layout solve_layout(int dim, int order, int E, int F, bool ns, bool blending, bool fp32, int num_bcs = 0) {
    long long nd = 1;
    for (int d = 0; d < dim; ++d) nd *= order + 1;
    const size_t Ndof = (size_t)E * nd, nf = dim + 2;
    const size_t S = nf * Ndof * sizeof(double);
    Layout L{};
    size_t o = 0;
    for (int k = 0; k < 3; ++k) { L.u[k] = o; o += align_up(S); }
    L.grad = o;
    if (ns) o += align_up((size_t)dim * nf * Ndof * (fp32 ? sizeof(float) : sizeof(double)));
    L.alpha = o;
    if (blending) o += align_up((size_t)E * sizeof(double));
    L.geo = o;
    o += align_up((size_t)E * (dim * dim + 1) * sizeof(double));
    L.nbr = o;
    o += align_up((size_t)E * 2 * dim * sizeof(int4));
    L.fnor = o;
    o += align_up((size_t)std::max(F, 1) * dim * sizeof(double));
    L.bcs = o;
    o += align_up((size_t)std::max(num_bcs, 0) * sizeof(BcDev));
    L.total = o;
    return L;
}

int class_key(int dim, int order, bool ns, bool vc) { return ((dim * 16 + order) * 2 + (ns ? 1 : 0)) * 2 + (vc ? 1 : 0); }

struct Solve {
    bool used = false;
    int dim = 0, order = 0, key = 0, E = 0, nf = 0;
    bool ns = false;
    double gamma = 1.4;
    long long Ndof = 0;
    size_t off = 0;
    Layout L{};
};

constexpr int MAX_VARIANTS = 8;

struct Class {
    int dim = 0, order = 0;
    bool ns = false, vc = false;   // vc: NS with contravariant viscous fluxes (quirks = 1)
    OpTables T{};
    std::vector<int> ids;        // slot -> solve id
    int *d_buf = nullptr;        // ids[cap] | prefix[cap + 1] | hdr[4]
    BatchClassDev dev{};
    int variant = 0;
    BatchKernelInfo rinfo[MAX_VARIANTS]{};
    BatchKernelInfo linfo{};
    double ms[MAX_VARIANTS];
    double lift_ms = -1.0;
    // tuning inside the steps: summed ms per RHS launch of each timed shape,
    // the shapes timed so far (bitmask), summed lifting ms and launches
    double tune_ms[MAX_VARIANTS];
    unsigned tune_seen = 0;
    double tune_lift_ms = 0.0;
    int tune_lift_n = 0;
    bool tables_dirty = true;    // ids / prefix / header differ from the device copy
};

// Pinned ring for the small per-solve uploads of an admission (geometry rows,
// neighbour table, normals, boundary conditions, solve record): the host
// copies a blob into the ring and the DMA runs behind the next admission's
// host work instead of stalling the stream as a pageable copy does.
constexpr size_t kUpRing = size_t(32) << 20;
struct UpSegment {
    size_t begin, end;
    cudaEvent_t ev;
};

}   // namespace

struct prandtl_batch {
    prandtl_batch_config cfg{};
    int device = 0, num_sms = 0, cap = 0, nvar = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr, ev0 = nullptr, ev1 = nullptr;
    char *arena = nullptr;
    size_t arena_bytes = 0;
    Arena alloc;
    BatchInst *d_tab = nullptr;
    int *d_live = nullptr;       // live ids [cap] | count
    int *d_left = nullptr;       // steps left per solve id, written by the step-end kernel
    int *h_left = nullptr;       // pinned copy
    double *d_budget = nullptr;  // budget partials [BUDGET_BLOCKS][12] + totals [12]
    std::vector<Solve> solves;
    std::vector<int> free_ids;
    std::vector<int> live;
    std::map<int, Class> classes;
    cudaGraphExec_t g_many = nullptr, g_one = nullptr;
    bool graph_dirty = true;
    int tune_left = 0;                 // steps of tuning inside the next advances
    std::vector<cudaEvent_t> tev;      // their per-launch events
    bool live_dirty = true;            // live list differs from the device copy
    char *up_ring = nullptr;           // pinned upload ring (kUpRing bytes), null if refused
    bool up_tried = false;
    size_t up_head = 0;
    std::deque<UpSegment> up_pending;  // ring ranges whose DMA may still run
    std::vector<cudaEvent_t> up_free;  // spare events
    BatchInst *h_tab = nullptr;        // pinned copy of the solve records (read_many)
    long long launches = 0;
    size_t bytes = 0;
    std::string err;
    std::mutex mu;
};

namespace {

thread_local std::string g_batch_create_error;

prandtl_status bfail(prandtl_batch *b, prandtl_status st, const std::string &msg) {
    if (b) b->err = msg;
    else g_batch_create_error = msg;
    return st;
}
prandtl_status bcuda(prandtl_batch *b, cudaError_t e, const char *what) {
    return bfail(b, e == cudaErrorMemoryAllocation ? PRANDTL_ENOMEM : PRANDTL_ECUDA,
                 std::string(what) + ": " + cudaGetErrorString(e));
}
#define BCK(b, call, what)                                  \
    do {                                                    \
        cudaError_t _e = (call);                            \
        if (_e != cudaSuccess) return bcuda(b, _e, what);   \
    } while (0)

prandtl_status bwait(prandtl_batch *b) {
    cudaError_t e = cudaEventRecord(b->done, b->stream);
    if (e != cudaSuccess) return bcuda(b, e, "cudaEventRecord");
    const double limit = b->cfg.timeout_s > 0 ? b->cfg.timeout_s : 120.0;
    const auto t0 = std::chrono::steady_clock::now();
    for (;;) {
        e = cudaEventQuery(b->done);
        if (e == cudaSuccess) return PRANDTL_OK;
        if (e != cudaErrorNotReady) return bcuda(b, e, "device work failed");
        const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (el > limit) return bfail(b, PRANDTL_ETIMEDOUT, "wait for the batch's stream timed out");
        poll_pause(el);
    }
}

int stages_of(int scheme) { return scheme == PRANDTL_LSRK45 ? 5 : 3; }

BatchStage stage_of(int scheme, int k) {
    BatchStage st{};
    st.scheme = scheme == PRANDTL_LSRK45 ? BATCH_LSRK45 : BATCH_SSPRK3;
    st.stage = k;
    if (scheme == PRANDTL_LSRK45) {
        st.rkA = LSRK_A[k];
        st.rkB = LSRK_B[k];
    }
    return st;
}

prandtl_status upload_class(prandtl_batch *b, Class &c) {
    const int n = (int)c.ids.size();
    std::vector<int> prefix(n + 1, 0);
    for (int s = 0; s < n; ++s) {
        const int E = b->solves[c.ids[s]].E;
        prefix[s + 1] = prefix[s] + (E + BATCH_CHUNK - 1) / BATCH_CHUNK * BATCH_CHUNK;
    }
    const int hdr[4] = {n, prefix[n], 0, 0};
    int *ids = c.d_buf, *pre = c.d_buf + b->cap, *h = c.d_buf + 2 * b->cap + 1;
    if (n > 0) BCK(b, cudaMemcpyAsync(ids, c.ids.data(), n * sizeof(int), cudaMemcpyHostToDevice, b->stream), "class ids");
    BCK(b, cudaMemcpyAsync(pre, prefix.data(), (n + 1) * sizeof(int), cudaMemcpyHostToDevice, b->stream), "class prefix");
    BCK(b, cudaMemcpyAsync(h, hdr, sizeof(hdr), cudaMemcpyHostToDevice, b->stream), "class header");
    return PRANDTL_OK;
}

prandtl_status upload_live(prandtl_batch *b) {
    const int n = (int)b->live.size();
    if (n > 0)
        BCK(b, cudaMemcpyAsync(b->d_live, b->live.data(), n * sizeof(int), cudaMemcpyHostToDevice, b->stream), "live ids");
    BCK(b, cudaMemcpyAsync(b->d_live + b->cap, &n, sizeof(int), cudaMemcpyHostToDevice, b->stream), "live count");
    return PRANDTL_OK;
}

// The class tables and the live list the launches read, uploaded once before
// the next launches instead of at every admission or removal.
prandtl_status flush_tables(prandtl_batch *b) {
    for (auto &kv : b->classes) {
        if (!kv.second.tables_dirty) continue;
        prandtl_status st = upload_class(b, kv.second);
        if (st != PRANDTL_OK) return st;
        kv.second.tables_dirty = false;
    }
    if (b->live_dirty) {
        prandtl_status st = upload_live(b);
        if (st != PRANDTL_OK) return st;
        b->live_dirty = false;
    }
    return PRANDTL_OK;
}

// Waits (bounded by the batch's timeout) for one event.
prandtl_status bwait_event(prandtl_batch *b, cudaEvent_t ev) {
    const double limit = b->cfg.timeout_s > 0 ? b->cfg.timeout_s : 120.0;
    const auto t0 = std::chrono::steady_clock::now();
    for (;;) {
        const cudaError_t e = cudaEventQuery(ev);
        if (e == cudaSuccess) return PRANDTL_OK;
        if (e != cudaErrorNotReady) return bcuda(b, e, "device work failed");
        const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (el > limit) return bfail(b, PRANDTL_ETIMEDOUT, "wait for an upload timed out");
        poll_pause(el);
    }
}

// Host -> device upload of n bytes for an admission, on the batch stream.
// Blobs up to a quarter of the ring go through it (ranges still being read
// by their DMA are waited for first); larger ones, or all of them when pinned
// memory was refused, are copied directly.
prandtl_status up_copy(prandtl_batch *b, void *dst, const void *src, size_t n) {
    if (n == 0) return PRANDTL_OK;
    if (!b->up_ring && !b->up_tried) {
        b->up_tried = true;
        void *p = nullptr;
        if (cudaHostAlloc(&p, kUpRing, cudaHostAllocDefault) == cudaSuccess) b->up_ring = static_cast<char *>(p);
        else cudaGetLastError();
    }
    if (!b->up_ring || n > kUpRing / 4) {
        BCK(b, cudaMemcpyAsync(dst, src, n, cudaMemcpyHostToDevice, b->stream), "upload");
        return PRANDTL_OK;
    }
    const size_t need = (n + 255) / 256 * 256;
    if (b->up_head + need > kUpRing) b->up_head = 0;
    const size_t lo = b->up_head, hi = lo + need;
    for (auto it = b->up_pending.begin(); it != b->up_pending.end();) {
        const bool overlap = it->begin < hi && lo < it->end;
        const cudaError_t q = overlap ? cudaErrorNotReady : cudaEventQuery(it->ev);
        if (!overlap && q != cudaSuccess) {
            if (q != cudaErrorNotReady) return bcuda(b, q, "device work failed");
            ++it;
            continue;
        }
        if (overlap) {
            prandtl_status st = bwait_event(b, it->ev);
            if (st != PRANDTL_OK) return st;
        }
        b->up_free.push_back(it->ev);
        it = b->up_pending.erase(it);
    }
    std::memcpy(b->up_ring + lo, src, n);
    BCK(b, cudaMemcpyAsync(dst, b->up_ring + lo, n, cudaMemcpyHostToDevice, b->stream), "upload");
    cudaEvent_t ev = nullptr;
    if (!b->up_free.empty()) {
        ev = b->up_free.back();
        b->up_free.pop_back();
    } else {
        BCK(b, cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "upload event");
    }
    const cudaError_t e = cudaEventRecord(ev, b->stream);
    if (e != cudaSuccess) {
        b->up_free.push_back(ev);
        return bcuda(b, e, "cudaEventRecord");
    }
    b->up_pending.push_back({lo, hi, ev});
    b->up_head = hi;
    return PRANDTL_OK;
}

prandtl_status get_class(prandtl_batch *b, int dim, int order, bool ns, bool vc, Class **out) {
    const int key = class_key(dim, order, ns, vc);
    auto it = b->classes.find(key);
    if (it != b->classes.end()) { *out = &it->second; return PRANDTL_OK; }
    Class c;
    c.dim = dim;
    c.order = order;
    c.ns = ns;
    c.vc = vc;
    build_tables(order, c.T);
    const bool fp32 = b->cfg.precision == 1;
    int first_ok = -1;
    for (int v = 0; v < b->nvar; ++v) {
        c.ms[v] = -1.0;
        BCK(b, batch_prepare_rhs(dim, order, ns, vc, fp32, v, &c.rinfo[v]), "prepare batch rhs kernel");
        if (c.rinfo[v].blocks_per_sm > 0 && first_ok < 0) first_ok = v;
    }
    if (first_ok < 0) return bfail(b, PRANDTL_EUNSUPPORTED, "no RHS launch shape fits this device");
    c.variant = first_ok;
    if (ns) {
        BCK(b, batch_prepare_lift(dim, order, vc, fp32, &c.linfo), "prepare batch lift kernel");
        if (c.linfo.blocks_per_sm <= 0) return bfail(b, PRANDTL_EUNSUPPORTED, "lift kernel does not fit this device");
    }
    const size_t words = 2 * (size_t)b->cap + 5;
    BCK(b, cudaMalloc(&c.d_buf, words * sizeof(int)), "class tables");
    b->bytes += words * sizeof(int);
    c.dev.tab = b->d_tab;
    c.dev.ids = c.d_buf;
    c.dev.prefix = c.d_buf + b->cap;
    c.dev.hdr = c.d_buf + 2 * b->cap + 1;
    Class &ref = b->classes.emplace(key, c).first->second;
    ref.tables_dirty = true;
    b->graph_dirty = true;
    *out = &ref;
    return PRANDTL_OK;
}

// The launches of one step (all stages, all classes) and the step-end kernel.
prandtl_status enqueue_step(prandtl_batch *b, cudaStream_t s) {
    const bool fp32 = b->cfg.precision == 1;
    const int scheme = b->cfg.scheme;
    for (int k = 0; k < stages_of(scheme); ++k) {
        const BatchStage st = stage_of(scheme, k);
        for (auto &kv : b->classes) {
            Class &c = kv.second;
            if (c.ns) {
                const int grid = c.linfo.blocks_per_sm * b->num_sms;
                BCK(b, batch_launch_lift(c.dim, c.order, c.vc, fp32, grid, c.dev, st, c.T, s), "batch lift launch");
            }
            const int grid = c.rinfo[c.variant].blocks_per_sm * b->num_sms;
            BCK(b, batch_launch_rhs(c.dim, c.order, c.ns, c.vc, fp32, c.variant, grid, c.dev, st, c.T, s),
                "batch rhs launch");
        }
    }
    BCK(b, batch_launch_step_end(b->d_tab, b->d_live, b->d_live + b->cap,
                                 scheme == PRANDTL_LSRK45 ? 1 : 0, b->d_left, s),
        "batch step-end launch");
    return PRANDTL_OK;
}

// One step of tuning inside the advance: every class with resident solves
// runs RHS launch shape v (where it fits; else its current shape), and each
// lifting and RHS launch is bracketed by events.  The host waits for the step
// (bounded by the batch's timeout) and records the class's mean ms per RHS
// launch of the step for shape v.  The shapes give bit-identical results, so
// which shape a step ran does not change the solves.
prandtl_status tune_step(prandtl_batch *b, int v) {
    const bool fp32 = b->cfg.precision == 1;
    const int scheme = b->cfg.scheme, K = stages_of(scheme);
    const size_t need = (size_t)4 * K * b->classes.size();
    while (b->tev.size() < need) {
        cudaEvent_t e = nullptr;
        BCK(b, cudaEventCreate(&e), "tuning event");
        b->tev.push_back(e);
    }
    size_t q = 0;
    for (int k = 0; k < K; ++k) {
        const BatchStage st = stage_of(scheme, k);
        for (auto &kv : b->classes) {
            Class &c = kv.second;
            if (c.ns) {
                const int grid = c.linfo.blocks_per_sm * b->num_sms;
                BCK(b, cudaEventRecord(b->tev[q], b->stream), "event");
                BCK(b, batch_launch_lift(c.dim, c.order, c.vc, fp32, grid, c.dev, st, c.T, b->stream),
                    "batch lift launch");
                BCK(b, cudaEventRecord(b->tev[q + 1], b->stream), "event");
            }
            const int cv = c.rinfo[v].blocks_per_sm > 0 ? v : c.variant;
            const int grid = c.rinfo[cv].blocks_per_sm * b->num_sms;
            BCK(b, cudaEventRecord(b->tev[q + 2], b->stream), "event");
            BCK(b, batch_launch_rhs(c.dim, c.order, c.ns, c.vc, fp32, cv, grid, c.dev, st, c.T, b->stream),
                "batch rhs launch");
            BCK(b, cudaEventRecord(b->tev[q + 3], b->stream), "event");
            q += 4;
        }
    }
    BCK(b, batch_launch_step_end(b->d_tab, b->d_live, b->d_live + b->cap,
                                 scheme == PRANDTL_LSRK45 ? 1 : 0, b->d_left, b->stream),
        "batch step-end launch");
    prandtl_status st = bwait(b);
    if (st != PRANDTL_OK) return st;
    q = 0;
    for (int k = 0; k < K; ++k) {
        for (auto &kv : b->classes) {
            Class &c = kv.second;
            float ms = 0.f;
            if (c.ns && !c.ids.empty()) {
                BCK(b, cudaEventElapsedTime(&ms, b->tev[q], b->tev[q + 1]), "event time");
                c.tune_lift_ms += ms;
                ++c.tune_lift_n;
            }
            if (c.rinfo[v].blocks_per_sm > 0 && !c.ids.empty()) {
                BCK(b, cudaEventElapsedTime(&ms, b->tev[q + 2], b->tev[q + 3]), "event time");
                if (k == 0) c.tune_ms[v] = 0.0;
                c.tune_ms[v] += ms / K;
                if (k == K - 1) c.tune_seen |= 1u << v;
            }
            q += 4;
        }
    }
    return PRANDTL_OK;
}

// End of tuning inside the advances: each class keeps its fastest timed shape
// (its current one when none was timed) and the step graphs are rebuilt.
void tune_finish(prandtl_batch *b) {
    for (auto &kv : b->classes) {
        Class &c = kv.second;
        int best = c.variant;
        double best_ms = 1e300;
        for (int v = 0; v < b->nvar; ++v) {
            c.ms[v] = (c.tune_seen >> v) & 1u ? c.tune_ms[v] : -1.0;
            if (c.ms[v] >= 0.0 && c.ms[v] < best_ms) { best_ms = c.ms[v]; best = v; }
        }
        if (c.tune_lift_n > 0) c.lift_ms = c.tune_lift_ms / c.tune_lift_n;
        if (best != c.variant) b->graph_dirty = true;
        c.variant = best;
    }
}

long long launches_per_step(const prandtl_batch *b) {
    long long n = 0;
    for (const auto &kv : b->classes) n += kv.second.ns ? 2 : 1;
    return n * stages_of(b->cfg.scheme) + 1;
}

void drop_graphs(prandtl_batch *b) {
    if (b->g_many) cudaGraphExecDestroy(b->g_many);
    if (b->g_one) cudaGraphExecDestroy(b->g_one);
    b->g_many = b->g_one = nullptr;
}

prandtl_status capture(prandtl_batch *b, int steps, cudaGraphExec_t *exec) {
    BCK(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
    prandtl_status st = PRANDTL_OK;
    for (int s = 0; s < steps && st == PRANDTL_OK; ++s) st = enqueue_step(b, b->stream);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(b->stream, &g);
    if (st != PRANDTL_OK) {
        if (g) cudaGraphDestroy(g);
        return st;
    }
    if (e != cudaSuccess) return bcuda(b, e, "end capture");
    e = cudaGraphInstantiate(exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return bcuda(b, e, "instantiate graph");
    return PRANDTL_OK;
}

prandtl_status rebuild_graphs(prandtl_batch *b) {
    drop_graphs(b);
    prandtl_status st = capture(b, b->cfg.steps_per_graph, &b->g_many);
    if (st != PRANDTL_OK) return st;
    st = capture(b, 1, &b->g_one);
    if (st != PRANDTL_OK) return st;
    b->graph_dirty = false;
    return PRANDTL_OK;
}

void free_batch(prandtl_batch *b) {
    drop_graphs(b);
    for (cudaEvent_t e : b->tev) cudaEventDestroy(e);
    b->tev.clear();
    for (auto &kv : b->classes) cudaFree(kv.second.d_buf);
    b->classes.clear();
    for (auto &g : b->up_pending) cudaEventDestroy(g.ev);
    b->up_pending.clear();
    for (cudaEvent_t e : b->up_free) cudaEventDestroy(e);
    b->up_free.clear();
    if (b->up_ring) cudaFreeHost(b->up_ring);
    b->up_ring = nullptr;
    if (b->h_tab) cudaFreeHost(b->h_tab);
    b->h_tab = nullptr;
    cudaFree(b->arena);
    cudaFree(b->d_tab);
    cudaFree(b->d_live);
    cudaFree(b->d_left);
    if (b->h_left) cudaFreeHost(b->h_left);
    cudaFree(b->d_budget);
    if (b->done) cudaEventDestroy(b->done);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->stream) cudaStreamDestroy(b->stream);
}

}   // namespace

namespace prandtl {
namespace host {
// Room for one more solve of `bytes` (arena range and a table slot); the
// serving loop asks before it tries an admission.
bool batch_has_room(prandtl_batch *b, size_t bytes) {
    std::lock_guard<std::mutex> lk(b->mu);
    return !b->free_ids.empty() && b->alloc.largest() >= bytes;
}
}   // namespace host
}   // namespace prandtl

extern "C" {

void prandtl_batch_config_default(prandtl_batch_config *c) {
    if (!c) return;
    std::memset(c, 0, sizeof(*c));
    c->precision = 0;
    c->scheme = PRANDTL_LSRK45;
    c->max_solves = 4096;
    c->steps_per_graph = 4;
    c->use_graph = 1;
    c->timeout_s = 120.0;
}

prandtl_status prandtl_batch_create(const prandtl_batch_config *cin, prandtl_batch **out) {
    g_batch_create_error.clear();
    if (!out || !cin) return bfail(nullptr, PRANDTL_EINVAL, "null argument");
    *out = nullptr;
    prandtl_batch_config c = *cin;
    if (c.precision != 0 && c.precision != 1)
        return bfail(nullptr, PRANDTL_EUNSUPPORTED, "precision must be 0 (FP64) or 1 (FP32 bulk)");
    if (c.scheme != PRANDTL_LSRK45 && c.scheme != PRANDTL_RK3SSP)
        return bfail(nullptr, PRANDTL_EINVAL, "unknown scheme");
    if (c.max_solves <= 0) c.max_solves = 4096;
    if (c.max_solves > (1 << 20)) return bfail(nullptr, PRANDTL_EINVAL, "max_solves too large");
    if (c.steps_per_graph <= 0) c.steps_per_graph = 4;
    if (c.timeout_s <= 0) c.timeout_s = 120.0;
    int ndev = 0;
    cudaError_t ce = cudaGetDeviceCount(&ndev);
    if (ce != cudaSuccess || ndev == 0)
        return bfail(nullptr, PRANDTL_ECUDA, std::string("no CUDA device: ") + cudaGetErrorString(ce));

    prandtl_batch *b = new prandtl_batch();
    b->cfg = c;
    b->cap = c.max_solves;
    b->nvar = std::min(batch_num_variants(), MAX_VARIANTS);
    auto bail = [&](prandtl_status st) {
        g_batch_create_error = b->err;
        free_batch(b);
        delete b;
        return st;
    };
    cudaGetDevice(&b->device);
    if ((ce = cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, b->device)) != cudaSuccess)
        return bail(bcuda(b, ce, "device attribute"));
    if ((ce = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking)) != cudaSuccess)
        return bail(bcuda(b, ce, "cudaStreamCreate"));
    if ((ce = cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming)) != cudaSuccess ||
        (ce = cudaEventCreate(&b->ev0)) != cudaSuccess || (ce = cudaEventCreate(&b->ev1)) != cudaSuccess)
        return bail(bcuda(b, ce, "cudaEventCreate"));
    size_t arena = c.arena_bytes;
    if (arena == 0) {
        size_t fr = 0, tot = 0;
        if ((ce = cudaMemGetInfo(&fr, &tot)) != cudaSuccess) return bail(bcuda(b, ce, "cudaMemGetInfo"));
        arena = fr / 2;
    }
    arena = arena / ALIGN * ALIGN;
    if ((ce = cudaMalloc(&b->arena, arena)) != cudaSuccess) return bail(bcuda(b, ce, "arena"));
    b->arena_bytes = arena;
    b->alloc.reset(arena);
    if ((ce = cudaMalloc(&b->d_tab, (size_t)b->cap * sizeof(BatchInst))) != cudaSuccess)
        return bail(bcuda(b, ce, "solve table"));
    if ((ce = cudaMemset(b->d_tab, 0, (size_t)b->cap * sizeof(BatchInst))) != cudaSuccess)
        return bail(bcuda(b, ce, "solve table"));
    if ((ce = cudaMalloc(&b->d_live, ((size_t)b->cap + 1) * sizeof(int))) != cudaSuccess)
        return bail(bcuda(b, ce, "live list"));
    if ((ce = cudaMalloc(&b->d_left, (size_t)b->cap * sizeof(int))) != cudaSuccess)
        return bail(bcuda(b, ce, "steps-left table"));
    if ((ce = cudaMemset(b->d_left, 0, (size_t)b->cap * sizeof(int))) != cudaSuccess)
        return bail(bcuda(b, ce, "steps-left table"));
    if ((ce = cudaMallocHost(&b->h_left, (size_t)b->cap * sizeof(int))) != cudaSuccess)
        return bail(bcuda(b, ce, "pinned steps-left"));
    if ((ce = cudaMalloc(&b->d_budget, (size_t)(BUDGET_BLOCKS + 1) * 12 * sizeof(double))) != cudaSuccess)
        return bail(bcuda(b, ce, "budgets"));
    b->bytes = arena + (size_t)b->cap * (sizeof(BatchInst) + 2 * sizeof(int)) + sizeof(int);
    b->solves.resize(b->cap);
    for (int q = b->cap - 1; q >= 0; --q) b->free_ids.push_back(q);
    prandtl_status st = upload_live(b);
    if (st != PRANDTL_OK) return bail(st);
    if ((st = bwait(b)) != PRANDTL_OK) return bail(st);
    *out = b;
    return PRANDTL_OK;
}

prandtl_status prandtl_batch_destroy(prandtl_batch *b) {
    if (!b) return PRANDTL_EINVAL;
    {
        std::lock_guard<std::mutex> lk(b->mu);
        cudaSetDevice(b->device);
        bwait(b);
        free_batch(b);
    }
    delete b;
    return PRANDTL_OK;
}

prandtl_status prandtl_batch_footprint(prandtl_batch *b, const prandtl_mesh_desc *md, const prandtl_config *cfg,
                                       size_t *bytes) {
    if (!b || !md || !cfg || !bytes) return b ? bfail(b, PRANDTL_EINVAL, "null argument") : PRANDTL_EINVAL;
    if ((md->dim != 2 && md->dim != 3) || !order_supported(md->dim, md->order) || md->num_elements <= 0)
        return bfail(b, PRANDTL_EUNSUPPORTED, "unsupported mesh");
    const Layout L = solve_layout(md->dim, md->order, md->num_elements, md->num_faces, cfg->parabolic != 0,
                                  cfg->blending != 0, b->cfg.precision == 1, cfg->num_bcs);
    *bytes = L.total;
    return PRANDTL_OK;
}

}   // extern "C"

namespace {

// Host-side preparation of one admission, touching no batch state: the
// argument and mesh checks, the neighbour table and the geometry rows.  The
// preparations of different solves are independent, so
// prandtl_batch_add_many runs them on several host threads.  A Prep is
// reused across admissions: its tables keep their capacity, so admissions do
// not fault in fresh host pages for them (page faults, serialised in the
// kernel, were most of a large admission's host time).
struct Prep {
    prandtl_status st = PRANDTL_OK;
    std::string msg;
    std::vector<int4> nbr;
    std::vector<double> geo;
    // tables of a very large mesh are not kept for the next admission
    void trim() {
        if (nbr.capacity() * sizeof(int4) + geo.capacity() * sizeof(double) > (size_t(64) << 20)) {
            std::vector<int4>().swap(nbr);
            std::vector<double>().swap(geo);
        }
    }
};

void prep_solve(const prandtl_mesh_desc *md, const prandtl_config *cfg, const prandtl_solve_desc *sd, Prep &p) {
    p.st = PRANDTL_OK;
    p.msg.clear();
    if (sd->nsteps < 0 || !std::isfinite(sd->dt) || (sd->nsteps > 0 && !(sd->dt > 0.0)) ||
        !std::isfinite(sd->cfl) || (sd->cfl > 0.0 && !(sd->hmin > 0.0)) || !std::isfinite(sd->t_final) ||
        sd->t_final < 0.0) {
        p.st = PRANDTL_EINVAL;
        p.msg = "bad solve description (dt, cfl, hmin, nsteps, t_final)";
        return;
    }
    if (!(cfg->gamma > 1.0) || !(cfg->Pr > 0.0)) {
        p.st = PRANDTL_EINVAL;
        p.msg = "bad gamma/Pr";
        return;
    }
    prandtl_status st = check_bcs(cfg, md->dim, p.msg);
    if (st == PRANDTL_OK) st = validate_mesh(md, p.nbr, p.msg, cfg->num_bcs);
    if (st == PRANDTL_OK) st = check_viscous_bcs(md, cfg, p.msg);
    if (st == PRANDTL_OK && cfg->axisymmetric) {
        st = PRANDTL_EUNSUPPORTED;
        p.msg = "the axisymmetric form runs on a prandtl_create operator, not in a batch";
    }
    if (st == PRANDTL_OK && (md->node_adj || md->node_detj || md->face_node_nor)) {
        st = PRANDTL_EUNSUPPORTED;
        p.msg = "non-affine elements run on a prandtl_create FP64 operator, not in a batch";
    }
    if (st == PRANDTL_OK && cfg->parabolic && cfg->quirks != 0) st = check_face_normals(md, p.msg);
    if (st == PRANDTL_OK) geometry_rows_into(md, p.geo);
    p.st = st;
}

// Admission of a prepared solve (the batch's mutex held).
prandtl_status admit_prepared(prandtl_batch *b, const prandtl_mesh_desc *md, const prandtl_config *cfg,
                              const double *u0, int ptr_flags, const prandtl_solve_desc *sd, Prep &p, int *id) {
    if (p.st != PRANDTL_OK) return bfail(b, p.st, p.msg);
    prandtl_status st = PRANDTL_OK;
    const std::vector<int4> &nbr = p.nbr;
    BCK(b, cudaSetDevice(b->device), "cudaSetDevice");
    const int dim = md->dim, order = md->order, E = md->num_elements, F = md->num_faces;
    const bool ns = cfg->parabolic != 0, fp32 = b->cfg.precision == 1, blend = cfg->blending != 0;
    const bool vc = ns && cfg->quirks != 0;
    const Layout L = solve_layout(dim, order, E, F, ns, blend, fp32, cfg->num_bcs);
    if (b->free_ids.empty()) return bfail(b, PRANDTL_ENOMEM, "solve table full");
    Class *c = nullptr;
    if ((st = get_class(b, dim, order, ns, vc, &c)) != PRANDTL_OK) return st;
    size_t off = 0;
    if (!b->alloc.alloc(L.total, &off))
        return bfail(b, PRANDTL_ENOMEM, "arena has no room: need " + std::to_string(L.total) +
                                            " bytes, largest free range " + std::to_string(b->alloc.largest()));
    const int sid = b->free_ids.back();
    char *base = b->arena + off;
    Solve s;
    s.used = true;
    s.dim = dim;
    s.order = order;
    s.ns = ns;
    s.key = class_key(dim, order, ns, vc);
    s.E = E;
    s.nf = dim + 2;
    s.gamma = cfg->gamma;
    s.Ndof = (long long)E;
    for (int d = 0; d < dim; ++d) s.Ndof *= order + 1;
    s.off = off;
    s.L = L;
    auto undo = [&](prandtl_status r) {
        b->alloc.release(off, L.total);
        return r;
    };
    const std::vector<double> &geo = p.geo;
    const size_t S = (size_t)s.nf * s.Ndof * sizeof(double);
    cudaError_t e;
    if ((st = up_copy(b, base + L.geo, geo.data(), geo.size() * sizeof(double))) != PRANDTL_OK ||
        (st = up_copy(b, base + L.nbr, nbr.data(), nbr.size() * sizeof(int4))) != PRANDTL_OK ||
        (F > 0 && (st = up_copy(b, base + L.fnor, md->face_nor, (size_t)F * dim * sizeof(double))) != PRANDTL_OK))
        return undo(st);
    if ((e = cudaMemcpyAsync(base + L.u[0], u0, S,
                             (ptr_flags & PRANDTL_PTR_DEVICE) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                             b->stream)) != cudaSuccess ||
        (blend && (e = cudaMemsetAsync(base + L.alpha, 0, (size_t)E * sizeof(double), b->stream)) != cudaSuccess))
        return undo(bcuda(b, e, "upload solve"));
    const std::vector<BcDev> bcs = device_bcs(cfg, md->dim);
    if (!bcs.empty() && (st = up_copy(b, base + L.bcs, bcs.data(), bcs.size() * sizeof(BcDev))) != PRANDTL_OK)
        return undo(st);
    BatchInst I;
    std::memset(&I, 0, sizeof(I));
    build_phys(*cfg, order, I.P);
    I.geo = reinterpret_cast<const double *>(base + L.geo);
    I.nbr = reinterpret_cast<const int4 *>(base + L.nbr);
    I.fnor = reinterpret_cast<const double *>(base + L.fnor);
    for (int k = 0; k < 3; ++k) I.u[k] = reinterpret_cast<double *>(base + L.u[k]);
    I.grad = ns ? (void *)(base + L.grad) : nullptr;
    I.alpha = blend ? reinterpret_cast<double *>(base + L.alpha) : nullptr;
    I.bcs = bcs.empty() ? nullptr : reinterpret_cast<const BcDev *>(base + L.bcs);
    I.Ndof = s.Ndof;
    I.E = E;
    I.order = order;
    I.dt = sd->t_final > 0.0 ? std::min(sd->dt, sd->t_final) : sd->dt;
    I.t = 0.0;
    I.t_final = sd->t_final > 0.0 ? sd->t_final : 0.0;
    I.cfl = sd->cfl > 0.0 ? sd->cfl : 0.0;
    I.hmin = sd->hmin;
    I.steps_left = sd->nsteps;
    const int left = sd->nsteps;
    if ((st = up_copy(b, b->d_tab + sid, &I, sizeof(I))) != PRANDTL_OK ||
        (st = up_copy(b, b->d_left + sid, &left, sizeof(int))) != PRANDTL_OK)
        return undo(st);
    // the work prefix is built from the solve records: record this one first;
    // the class tables and the live list go up before the next launches
    b->solves[sid] = s;
    c->ids.push_back(sid);
    b->live.push_back(sid);
    c->tables_dirty = true;
    b->live_dirty = true;
    b->free_ids.pop_back();
    *id = sid;
    return PRANDTL_OK;
}

}   // namespace

extern "C" {

prandtl_status prandtl_batch_add(prandtl_batch *b, const prandtl_mesh_desc *md, const prandtl_config *cfg,
                                 const double *u0, int ptr_flags, const prandtl_solve_desc *sd, int *id) {
    if (!b) return PRANDTL_EINVAL;
    if (!md || !cfg || !u0 || !sd || !id) return bfail(b, PRANDTL_EINVAL, "null argument");
    thread_local Prep p;
    prep_solve(md, cfg, sd, p);
    std::lock_guard<std::mutex> lk(b->mu);
    b->err.clear();
    const prandtl_status st = admit_prepared(b, md, cfg, u0, ptr_flags, sd, p, id);
    p.trim();
    return st;
}

prandtl_status prandtl_batch_add_many(prandtl_batch *b, int n, const prandtl_mesh_desc *const *mds,
                                      const prandtl_config *const *cfgs, const double *const *u0s, int ptr_flags,
                                      const prandtl_solve_desc *sds, int *ids) {
    if (!b) return PRANDTL_EINVAL;
    if (n < 0 || (n > 0 && (!mds || !cfgs || !u0s || !sds || !ids))) return bfail(b, PRANDTL_EINVAL, "null argument");
    for (int k = 0; k < n; ++k) {
        ids[k] = -1;
        if (!mds[k] || !cfgs[k] || !u0s[k]) return bfail(b, PRANDTL_EINVAL, "null argument");
    }
    // windows of solves: prepared on host threads, then admitted in order
    constexpr int kWindow = 64;
    const unsigned hw = std::thread::hardware_concurrency();
    const int threads = (int)std::max(1u, std::min(16u, hw / 2));
    // the calling thread's buffers; the worker threads reach them through this
    // reference (inside a worker, the thread_local name is that worker's own)
    thread_local std::vector<Prep> tl_preps;
    std::vector<Prep> &preps = tl_preps;
    if (preps.size() < (size_t)kWindow) preps.resize(kWindow);
    for (int k0 = 0; k0 < n; k0 += kWindow) {
        const int k1 = std::min(n, k0 + kWindow);
        std::atomic<int> next{k0};
        auto work = [&] {
            for (int k = next.fetch_add(1); k < k1; k = next.fetch_add(1)) {
                try {
                    prep_solve(mds[k], cfgs[k], &sds[k], preps[k - k0]);
                } catch (const std::bad_alloc &) {   // host memory for the tables
                    preps[k - k0].st = PRANDTL_ENOMEM;
                    preps[k - k0].msg = "host memory for the mesh tables";
                }
            }
        };
        std::vector<std::thread> pool;
        for (int t = 1; t < std::min(threads, k1 - k0); ++t) pool.emplace_back(work);
        work();
        for (auto &t : pool) t.join();
        std::lock_guard<std::mutex> lk(b->mu);
        b->err.clear();
        for (int k = k0; k < k1; ++k) {
            prandtl_status st = admit_prepared(b, mds[k], cfgs[k], u0s[k], ptr_flags, &sds[k], preps[k - k0], &ids[k]);
            if (st != PRANDTL_OK) {
                b->err = "solve " + std::to_string(k) + ": " + b->err;
                for (auto &q : preps) q.trim();
                return st;
            }
        }
        for (int k = k0; k < k1; ++k) preps[k - k0].trim();
    }
    return PRANDTL_OK;
}

prandtl_status prandtl_batch_advance(prandtl_batch *b, int nsteps) {
    if (!b) return PRANDTL_EINVAL;
    if (nsteps < 0) return bfail(b, PRANDTL_EINVAL, "negative step count");
    std::lock_guard<std::mutex> lk(b->mu);
    b->err.clear();
    if (nsteps == 0 || b->classes.empty()) return PRANDTL_OK;
    BCK(b, cudaSetDevice(b->device), "cudaSetDevice");
    if (prandtl_status fs = flush_tables(b); fs != PRANDTL_OK) return fs;
    const long long per_step = launches_per_step(b);
    while (nsteps > 0 && b->tune_left > 0) {   // tuning inside the first steps
        prandtl_status st = tune_step(b, b->nvar - b->tune_left);
        if (st != PRANDTL_OK) return st;
        b->launches += per_step;
        --nsteps;
        if (--b->tune_left == 0) {
            tune_finish(b);
            // capture the tuned shapes' graphs now rather than in the next call
            if (b->cfg.use_graph && b->graph_dirty) {
                prandtl_status gs = rebuild_graphs(b);
                if (gs != PRANDTL_OK) return gs;
            }
        }
    }
    if (nsteps == 0) return PRANDTL_OK;
    if (!b->cfg.use_graph) {
        for (int s = 0; s < nsteps; ++s) {
            prandtl_status st = enqueue_step(b, b->stream);
            if (st != PRANDTL_OK) return st;
        }
    } else {
        if (b->graph_dirty) {
            prandtl_status st = rebuild_graphs(b);
            if (st != PRANDTL_OK) return st;
        }
        int left = nsteps;
        const int S = b->cfg.steps_per_graph;
        while (left >= S) {
            BCK(b, cudaGraphLaunch(b->g_many, b->stream), "graph launch");
            left -= S;
        }
        while (left > 0) {
            BCK(b, cudaGraphLaunch(b->g_one, b->stream), "graph launch");
            --left;
        }
    }
    b->launches += per_step * nsteps;
    return PRANDTL_OK;
}

prandtl_status prandtl_batch_sync(prandtl_batch *b) {
    if (!b) return PRANDTL_EINVAL;
    std::lock_guard<std::mutex> lk(b->mu);
    BCK(b, cudaSetDevice(b->device), "cudaSetDevice");
    return bwait(b);
}

prandtl_status prandtl_batch_finished(prandtl_batch *b, int *ids, int cap, int *count) {
    if (!b) return PRANDTL_EINVAL;
    if (!count || (cap > 0 && !ids)) return bfail(b, PRANDTL_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(b->mu);
    BCK(b, cudaSetDevice(b->device), "cudaSetDevice");
    BCK(b, cudaMemcpyAsync(b->h_left, b->d_left, (size_t)b->cap * sizeof(int), cudaMemcpyDeviceToHost, b->stream),
        "D2H steps left");
    prandtl_status st = bwait(b);
    if (st != PRANDTL_OK) return st;
    int n = 0;
    for (int q = 0; q < b->cap; ++q)
        if (b->solves[q].used && b->h_left[q] <= 0) {
            if (n < cap) ids[n] = q;
            ++n;
        }
    *count = n;
    return PRANDTL_OK;
}

prandtl_status prandtl_batch_query(prandtl_batch *b, int id, int *steps_left, int *steps_done, double *dt,
                                   double *lambda_max) {
    if (!b) return PRANDTL_EINVAL;
    std::lock_guard<std::mutex> lk(b->mu);
    if (id < 0 || id >= b->cap || !b->solves[id].used) return bfail(b, PRANDTL_EINVAL, "unknown solve id");
    BCK(b, cudaSetDevice(b->device), "cudaSetDevice");
    BatchInst I;
    BCK(b, cudaMemcpyAsync(&I, b->d_tab + id, sizeof(I), cudaMemcpyDeviceToHost, b->stream), "D2H solve record");
    prandtl_status st = bwait(b);
    if (st != PRANDTL_OK) return st;
    if (steps_left) *steps_left = I.steps_left;
    if (steps_done) *steps_done = I.steps_done;
    if (dt) *dt = I.dt;
    if (lambda_max) {
        double v;
        std::memcpy(&v, &I.lambda_last, sizeof(v));
        *lambda_max = v;
    }
    if (I.health) return bfail(b, PRANDTL_ENONFINITE, "solve " + std::to_string(id) + ": " + health_text(I.health));
    return PRANDTL_OK;
}

prandtl_status prandtl_batch_time(prandtl_batch *b, int id, double *t) {
    if (!b) return PRANDTL_EINVAL;
    if (!t) return bfail(b, PRANDTL_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(b->mu);
    if (id < 0 || id >= b->cap || !b->solves[id].used) return bfail(b, PRANDTL_EINVAL, "unknown solve id");
    BCK(b, cudaSetDevice(b->device), "cudaSetDevice");
    double v = 0.0;
    BCK(b, cudaMemcpyAsync(&v, reinterpret_cast<char *>(b->d_tab + id) + offsetof(BatchInst, t), sizeof(v),
                           cudaMemcpyDeviceToHost, b->stream),
        "D2H time");
    prandtl_status st = bwait(b);
    if (st == PRANDTL_OK) *t = v;
    return st;
}

prandtl_status prandtl_batch_read(prandtl_batch *b, int id, double *u, int ptr_flags) {
    if (!b) return PRANDTL_EINVAL;
    if (!u) return bfail(b, PRANDTL_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(b->mu);
    if (id < 0 || id >= b->cap || !b->solves[id].used) return bfail(b, PRANDTL_EINVAL, "unknown solve id");
    BCK(b, cudaSetDevice(b->device), "cudaSetDevice");
    const Solve &s = b->solves[id];
    // the LSRK parity and the state-check bits sit next to each other in the record
    static_assert(offsetof(BatchInst, health) == offsetof(BatchInst, cur) + sizeof(int), "record layout");
    int words[2] = {0, 0};
    BCK(b, cudaMemcpyAsync(words, reinterpret_cast<char *>(b->d_tab + id) + offsetof(BatchInst, cur), sizeof(words),
                           cudaMemcpyDeviceToHost, b->stream),
        "D2H parity and state check");
    prandtl_status st = bwait(b);
    if (st != PRANDTL_OK) return st;
    const int cur = b->cfg.scheme == PRANDTL_LSRK45 ? words[0] : 0;
    const char *src = b->arena + s.off + s.L.u[cur & 1];
    const size_t S = (size_t)s.nf * s.Ndof * sizeof(double);
    BCK(b, cudaMemcpyAsync(u, src, S,
                           (ptr_flags & PRANDTL_PTR_DEVICE) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                           b->stream),
        "copy state");
    st = bwait(b);
    if (st == PRANDTL_OK && words[1] != 0)
        return bfail(b, PRANDTL_ENONFINITE, "solve " + std::to_string(id) + ": " + health_text((unsigned)words[1]));
    return st;
}

prandtl_status prandtl_batch_read_many(prandtl_batch *b, int n, const int *ids, double *const *u, int ptr_flags) {
    if (!b) return PRANDTL_EINVAL;
    if (n < 0 || (n > 0 && (!ids || !u))) return bfail(b, PRANDTL_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(b->mu);
    for (int k = 0; k < n; ++k) {
        if (ids[k] < 0 || ids[k] >= b->cap || !b->solves[ids[k]].used)
            return bfail(b, PRANDTL_EINVAL, "unknown solve id " + std::to_string(ids[k]));
        if (!u[k]) return bfail(b, PRANDTL_EINVAL, "null argument");
    }
    if (n == 0) return PRANDTL_OK;
    BCK(b, cudaSetDevice(b->device), "cudaSetDevice");
    // every record's LSRK parity and state-check bits in one copy
    if (!b->h_tab) BCK(b, cudaMallocHost(&b->h_tab, (size_t)b->cap * sizeof(BatchInst)), "pinned solve records");
    BCK(b, cudaMemcpyAsync(b->h_tab, b->d_tab, (size_t)b->cap * sizeof(BatchInst), cudaMemcpyDeviceToHost, b->stream),
        "D2H solve records");
    prandtl_status st = bwait(b);
    if (st != PRANDTL_OK) return st;
    for (int k = 0; k < n; ++k) {
        const Solve &s = b->solves[ids[k]];
        const int cur = b->cfg.scheme == PRANDTL_LSRK45 ? b->h_tab[ids[k]].cur : 0;
        const size_t S = (size_t)s.nf * s.Ndof * sizeof(double);
        BCK(b, cudaMemcpyAsync(u[k], b->arena + s.off + s.L.u[cur & 1], S,
                               (ptr_flags & PRANDTL_PTR_DEVICE) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                               b->stream),
            "copy state");
    }
    if ((st = bwait(b)) != PRANDTL_OK) return st;
    for (int k = 0; k < n; ++k)
        if (b->h_tab[ids[k]].health != 0)
            return bfail(b, PRANDTL_ENONFINITE,
                         "solve " + std::to_string(ids[k]) + ": " + health_text((unsigned)b->h_tab[ids[k]].health));
    return PRANDTL_OK;
}

prandtl_status prandtl_batch_budgets(prandtl_batch *b, int id, double *out) {
    if (!b) return PRANDTL_EINVAL;
    if (!out) return bfail(b, PRANDTL_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(b->mu);
    if (id < 0 || id >= b->cap || !b->solves[id].used) return bfail(b, PRANDTL_EINVAL, "unknown solve id");
    BCK(b, cudaSetDevice(b->device), "cudaSetDevice");
    const Solve &s = b->solves[id];
    int cur = 0;
    if (b->cfg.scheme == PRANDTL_LSRK45) {
        BCK(b, cudaMemcpyAsync(&cur, reinterpret_cast<char *>(b->d_tab + id) + offsetof(BatchInst, cur), sizeof(int),
                               cudaMemcpyDeviceToHost, b->stream),
            "D2H parity");
        prandtl_status st = bwait(b);
        if (st != PRANDTL_OK) return st;
    }
    const char *base = b->arena + s.off;
    const OpTables &T = b->classes.at(s.key).T;
    double *tot = b->d_budget + (size_t)BUDGET_BLOCKS * 12;
    BCK(b, launch_budgets(reinterpret_cast<const double *>(base + s.L.u[cur & 1]), nullptr,
                          reinterpret_cast<const double *>(base + s.L.geo), nullptr, T.w, s.dim, s.order + 1, s.E,
                          s.gamma,
                          b->d_budget, tot, b->stream),
        "budget kernel launch");
    b->launches += 2;
    double buf[12];
    BCK(b, cudaMemcpyAsync(buf, tot, sizeof(buf), cudaMemcpyDeviceToHost, b->stream), "D2H budgets");
    prandtl_status st = bwait(b);
    if (st != PRANDTL_OK) return st;
    for (int f = 0; f < s.nf; ++f) out[f] = buf[f];   // device slots: conserved [0..4], entropy [5]
    out[s.nf] = buf[5];
    return PRANDTL_OK;
}

prandtl_status prandtl_batch_remove(prandtl_batch *b, int id) {
    if (!b) return PRANDTL_EINVAL;
    std::lock_guard<std::mutex> lk(b->mu);
    if (id < 0 || id >= b->cap || !b->solves[id].used) return bfail(b, PRANDTL_EINVAL, "unknown solve id");
    BCK(b, cudaSetDevice(b->device), "cudaSetDevice");
    Solve &s = b->solves[id];
    Class &c = b->classes.at(s.key);
    c.ids.erase(std::find(c.ids.begin(), c.ids.end(), id));
    b->live.erase(std::find(b->live.begin(), b->live.end(), id));
    c.tables_dirty = true;   // uploaded before the next launches
    b->live_dirty = true;
    const int zero = 0;
    prandtl_status st = up_copy(b, b->d_left + id, &zero, sizeof(int));
    // later uploads into this range are ordered after the work already enqueued
    b->alloc.release(s.off, s.L.total);
    s = Solve();
    b->free_ids.push_back(id);
    return st;
}

prandtl_status prandtl_batch_tune_in_steps(prandtl_batch *b) {
    if (!b) return PRANDTL_EINVAL;
    std::lock_guard<std::mutex> lk(b->mu);
    b->err.clear();
    for (auto &kv : b->classes) {
        Class &c = kv.second;
        c.tune_seen = 0;
        c.tune_lift_ms = 0.0;
        c.tune_lift_n = 0;
    }
    b->tune_left = b->nvar;
    return PRANDTL_OK;
}

prandtl_status prandtl_batch_tune(prandtl_batch *b, int reps) {
    if (!b) return PRANDTL_EINVAL;
    if (reps <= 0) return bfail(b, PRANDTL_EINVAL, "reps must be positive");
    std::lock_guard<std::mutex> lk(b->mu);
    b->err.clear();
    b->tune_left = 0;   // replaces tuning inside the steps
    BCK(b, cudaSetDevice(b->device), "cudaSetDevice");
    prandtl_status st = flush_tables(b);
    if (st != PRANDTL_OK) return st;
    st = bwait(b);
    if (st != PRANDTL_OK) return st;
    const bool fp32 = b->cfg.precision == 1;
    // The first stage reads the step-start state and writes only the other RK
    // buffers (LSRK: A_1 = 0), so repeating it leaves the solves unchanged.
    const BatchStage st0 = stage_of(b->cfg.scheme, 0);
    for (auto &kv : b->classes) {
        Class &c = kv.second;
        if (c.ids.empty()) continue;
        if (c.ns) {
            const int lgrid = c.linfo.blocks_per_sm * b->num_sms;
            BCK(b, batch_launch_lift(c.dim, c.order, c.vc, fp32, lgrid, c.dev, st0, c.T, b->stream), "tune lift");
            BCK(b, cudaEventRecord(b->ev0, b->stream), "event");
            for (int r = 0; r < reps; ++r)
                BCK(b, batch_launch_lift(c.dim, c.order, c.vc, fp32, lgrid, c.dev, st0, c.T, b->stream), "tune lift");
            BCK(b, cudaEventRecord(b->ev1, b->stream), "event");
            if ((st = bwait(b)) != PRANDTL_OK) return st;
            float lms = 0.f;
            BCK(b, cudaEventElapsedTime(&lms, b->ev0, b->ev1), "event time");
            c.lift_ms = lms / reps;
            b->launches += reps + 1;
        }
        int best = c.variant;
        double best_ms = 1e300;
        for (int v = 0; v < b->nvar; ++v) {
            c.ms[v] = -1.0;
            if (c.rinfo[v].blocks_per_sm <= 0) continue;
            const int grid = c.rinfo[v].blocks_per_sm * b->num_sms;
            BCK(b, batch_launch_rhs(c.dim, c.order, c.ns, c.vc, fp32, v, grid, c.dev, st0, c.T, b->stream), "tune rhs");
            BCK(b, cudaEventRecord(b->ev0, b->stream), "event");
            for (int r = 0; r < reps; ++r)
                BCK(b, batch_launch_rhs(c.dim, c.order, c.ns, c.vc, fp32, v, grid, c.dev, st0, c.T, b->stream), "tune rhs");
            BCK(b, cudaEventRecord(b->ev1, b->stream), "event");
            if ((st = bwait(b)) != PRANDTL_OK) return st;
            float ms = 0.f;
            BCK(b, cudaEventElapsedTime(&ms, b->ev0, b->ev1), "event time");
            c.ms[v] = ms / reps;
            b->launches += reps + 1;
            if (c.ms[v] < best_ms) { best_ms = c.ms[v]; best = v; }
        }
        if (best != c.variant) b->graph_dirty = true;
        c.variant = best;
    }
    return PRANDTL_OK;
}

prandtl_status prandtl_batch_class_info(prandtl_batch *b, int dim, int order, int parabolic, int *variant,
                                        int *n_variants, double *ms, double *lift_ms) {
    if (!b) return PRANDTL_EINVAL;
    std::lock_guard<std::mutex> lk(b->mu);
    auto it = b->classes.find(class_key(dim, order, parabolic != 0, parabolic != 0));
    if (it == b->classes.end()) it = b->classes.find(class_key(dim, order, parabolic != 0, false));
    if (it == b->classes.end()) return bfail(b, PRANDTL_EINVAL, "no such class in this batch");
    if (variant) *variant = it->second.variant;
    if (n_variants) *n_variants = b->nvar;
    if (ms)
        for (int v = 0; v < b->nvar; ++v) ms[v] = it->second.ms[v];
    if (lift_ms) *lift_ms = it->second.lift_ms;
    return PRANDTL_OK;
}

void *prandtl_batch_stream(const prandtl_batch *b) { return b ? (void *)b->stream : nullptr; }

size_t prandtl_batch_device_bytes(const prandtl_batch *b) { return b ? b->bytes : 0; }
size_t prandtl_batch_arena_bytes(const prandtl_batch *b) { return b ? b->arena_bytes : 0; }
long long prandtl_batch_kernel_launches(const prandtl_batch *b) { return b ? b->launches : 0; }
const char *prandtl_batch_last_error(const prandtl_batch *b) {
    return b ? b->err.c_str() : g_batch_create_error.c_str();
}

}   // extern "C"
