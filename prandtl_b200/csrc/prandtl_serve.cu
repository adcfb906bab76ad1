// prandtl_serve.cu -- request loop over one batch (prandtl_serve_* in the C ABI).
//
// Continuous batching: submit() copies a request into host memory and queues
// it; one worker thread repeats
//   admit queued requests in arrival order while the arena and the solve
//   table have room -> enqueue steps_per_tick steps of every resident solve
//   -> wait -> copy out and retire the solves that finished,
// so requests that arrive while others run join at the next tick and share
// their stage launches.  Requests larger than the whole arena are rejected at
// submit time.  Admission scans the queue in arrival order: a request that
// does not fit yet stays queued and later, smaller requests may be admitted
// past it, but each queued request can be overtaken at most
// kMaxOvertakes times; after that nothing behind it is admitted until it fits
// (so it cannot starve).  A solve that fails its state check (a non-finite
// value, density or pressure <= 0) stops alone: its request completes with
// PRANDTL_ENONFINITE and the others go on.
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/prandtl_b200.h"

namespace prandtl {
namespace host {
bool batch_has_room(prandtl_batch *b, size_t bytes);
}
}   // namespace prandtl

namespace {

using Clock = std::chrono::steady_clock;

// Admissions past one queued request before it must go next.
constexpr int kMaxOvertakes = 64;

struct Request {
    long long ticket = 0;
    prandtl_mesh_desc md{};
    std::vector<double> adj, detj, nor, u0;
    std::vector<int> faces;
    prandtl_config cfg{};
    prandtl_solve_desc solve{};
    double *u_out = nullptr;
    Clock::time_point t_submit, t_done;
    int state = 0;              // 0 queued, 1 resident, 2 done, 3 failed
    prandtl_status status = PRANDTL_OK;   // of a failed request
    int batch_id = -1;
    double dofs = 0;            // nodes * fields
    size_t need = 0;            // arena bytes (prandtl_batch_footprint)
    int overtaken = 0;          // admissions past this request while it waited
    std::string err;
};

}   // namespace

struct prandtl_server {
    prandtl_batch *b = nullptr;
    int steps_per_tick = 1;
    double timeout_s = 120.0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<long long> queue;
    std::unordered_map<long long, std::unique_ptr<Request>> reqs;
    std::unordered_map<int, long long> resident;   // batch id -> ticket
    std::thread worker;
    bool stop = false;
    long long next_ticket = 1;
    prandtl_serve_stats stats{};
    Clock::time_point busy_since;
    bool busy = false;
    std::string err;
};

namespace {

// Admit in arrival order, letting requests that fit pass queued ones that do
// not fit yet, within the overtaking bound.
void admit(prandtl_server *s, std::unique_lock<std::mutex> &lk) {
    std::vector<Request *> waiting;   // skipped so far in this scan
    for (size_t q = 0; q < s->queue.size();) {
        Request *r = s->reqs.at(s->queue[q]).get();
        const bool nothing_resident = s->resident.empty();
        bool try_add = nothing_resident;
        if (!try_add) {
            lk.unlock();
            try_add = prandtl::host::batch_has_room(s->b, r->need);
            lk.lock();
        }
        prandtl_status st = PRANDTL_ENOMEM;
        std::string msg;
        int id = -1;
        if (try_add) {
            lk.unlock();
            st = prandtl_batch_add(s->b, &r->md, &r->cfg, r->u0.data(), PRANDTL_PTR_HOST, &r->solve, &id);
            if (st != PRANDTL_OK) msg = prandtl_batch_last_error(s->b);
            lk.lock();
        }
        if (st == PRANDTL_ENOMEM && !s->resident.empty()) {
            // no room yet: it waits; nothing behind it may pass once it has
            // been overtaken kMaxOvertakes times
            if (r->overtaken >= kMaxOvertakes) return;
            waiting.push_back(r);
            ++q;
            continue;
        }
        s->queue.erase(s->queue.begin() + (long)q);
        if (st != PRANDTL_OK) {
            r->state = 3;
            r->status = st;
            r->err = msg;
            r->t_done = Clock::now();
            s->stats.rejected++;
            s->cv_done.notify_all();
            continue;
        }
        for (Request *w : waiting) w->overtaken++;
        r->state = 1;
        r->batch_id = id;
        std::vector<double>().swap(r->u0);
        s->resident[id] = r->ticket;
    }
}

void worker_loop(prandtl_server *s) {
    std::vector<int> fin(4096);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        s->cv_work.wait_for(lk, std::chrono::milliseconds(20),
                            [&] { return s->stop || !s->queue.empty() || !s->resident.empty(); });
        admit(s, lk);
        if (s->resident.empty()) {
            if (s->busy) {
                s->stats.busy_s += std::chrono::duration<double>(Clock::now() - s->busy_since).count();
                s->busy = false;
            }
            if (s->stop && s->queue.empty()) break;
            continue;
        }
        if (!s->busy) {
            s->busy = true;
            s->busy_since = Clock::now();
        }
        s->stats.resident = (int)s->resident.size();
        lk.unlock();
        prandtl_status st = prandtl_batch_advance(s->b, s->steps_per_tick);
        int nfin = 0;
        if (st == PRANDTL_OK) st = prandtl_batch_finished(s->b, fin.data(), (int)fin.size(), &nfin);
        if (nfin > (int)fin.size()) {
            fin.resize(nfin);
            st = prandtl_batch_finished(s->b, fin.data(), (int)fin.size(), &nfin);
        }
        std::vector<std::pair<int, prandtl_status>> done;
        if (st == PRANDTL_OK) {
            for (int q = 0; q < nfin; ++q) {
                const int id = fin[q];
                Request *r = nullptr;
                {
                    std::lock_guard<std::mutex> g(s->mu);
                    auto it = s->resident.find(id);
                    if (it != s->resident.end()) r = s->reqs.at(it->second).get();
                }
                prandtl_status rs = r ? prandtl_batch_read(s->b, id, r->u_out, PRANDTL_PTR_HOST) : PRANDTL_OK;
                prandtl_batch_remove(s->b, id);
                done.emplace_back(id, rs);
            }
        }
        const std::string berr = st == PRANDTL_OK ? std::string() : prandtl_batch_last_error(s->b);
        lk.lock();
        s->stats.steps += s->steps_per_tick;
        if (st != PRANDTL_OK) {
            // the batch failed: fail every resident and queued request and stop
            s->err = berr;
            for (auto &kv : s->resident) {
                Request *r = s->reqs.at(kv.second).get();
                r->state = 3;
                r->status = st;
                r->err = berr;
                r->t_done = Clock::now();
            }
            s->resident.clear();
            for (long long t : s->queue) {
                Request *r = s->reqs.at(t).get();
                r->state = 3;
                r->status = st;
                r->err = berr;
                r->t_done = Clock::now();
            }
            s->queue.clear();
            s->stop = true;
            s->cv_done.notify_all();
            break;
        }
        const auto now = Clock::now();
        for (auto &d : done) {
            auto it = s->resident.find(d.first);
            if (it == s->resident.end()) continue;
            Request *r = s->reqs.at(it->second).get();
            s->resident.erase(it);
            r->t_done = now;
            if (d.second == PRANDTL_OK) {
                r->state = 2;
                s->stats.completed++;
                s->stats.dof_updates += r->dofs * r->solve.nsteps;
            } else {
                r->state = 3;
                r->status = d.second;
                r->err = d.second == PRANDTL_ENONFINITE ? "the solve failed its state check (stopped early)"
                                                        : "read of the final state failed";
            }
        }
        s->stats.resident = (int)s->resident.size();
        if (!done.empty()) s->cv_done.notify_all();
    }
    if (s->busy) {
        s->stats.busy_s += std::chrono::duration<double>(Clock::now() - s->busy_since).count();
        s->busy = false;
    }
}

}   // namespace

extern "C" {

prandtl_status prandtl_serve_create(const prandtl_batch_config *c, int steps_per_tick, prandtl_server **out) {
    if (!c || !out || steps_per_tick <= 0) return PRANDTL_EINVAL;
    *out = nullptr;
    prandtl_server *s = new prandtl_server();
    prandtl_status st = prandtl_batch_create(c, &s->b);
    if (st != PRANDTL_OK) {
        delete s;
        return st;
    }
    s->steps_per_tick = steps_per_tick;
    s->timeout_s = c->timeout_s > 0 ? c->timeout_s : 120.0;
    s->worker = std::thread(worker_loop, s);
    *out = s;
    return PRANDTL_OK;
}

prandtl_status prandtl_serve_submit(prandtl_server *s, const prandtl_mesh_desc *md, const prandtl_config *cfg,
                                    const double *u0, const prandtl_solve_desc *solve, double *u_out,
                                    long long *ticket) {
    if (!s) return PRANDTL_EINVAL;
    if (!md || !cfg || !u0 || !solve || !u_out || !ticket || md->num_elements <= 0 || md->num_faces < 0 ||
        (md->dim != 2 && md->dim != 3) || md->order < 1 || md->order > 5)
        return PRANDTL_EINVAL;
    size_t need = 0;
    prandtl_status st = prandtl_batch_footprint(s->b, md, cfg, &need);
    if (st != PRANDTL_OK) return st;
    auto r = std::make_unique<Request>();
    const int dim = md->dim, E = md->num_elements, F = md->num_faces;
    long long nd = 1;
    for (int d = 0; d < dim; ++d) nd *= md->order + 1;
    const size_t S = (size_t)(dim + 2) * E * nd;
    r->adj.assign(md->elem_adj, md->elem_adj + (size_t)E * dim * dim);
    r->detj.assign(md->elem_detj, md->elem_detj + E);
    r->faces.assign(md->face_elems, md->face_elems + (size_t)4 * F);
    r->nor.assign(md->face_nor, md->face_nor + (size_t)F * dim);
    r->u0.assign(u0, u0 + S);
    r->md = *md;
    r->md.elem_adj = r->adj.data();
    r->md.elem_detj = r->detj.data();
    r->md.face_elems = r->faces.data();
    r->md.face_nor = r->nor.data();
    r->cfg = *cfg;
    r->solve = *solve;
    r->u_out = u_out;
    r->dofs = (double)S;
    r->need = need;
    r->t_submit = Clock::now();
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return PRANDTL_ECUDA;
    s->stats.submitted++;
    if (need > prandtl_batch_arena_bytes(s->b)) {   // larger than the whole arena
        s->stats.rejected++;
        return PRANDTL_ENOMEM;
    }
    r->ticket = s->next_ticket++;
    *ticket = r->ticket;
    s->queue.push_back(r->ticket);
    s->reqs.emplace(r->ticket, std::move(r));
    s->cv_work.notify_one();
    return PRANDTL_OK;
}

prandtl_status prandtl_serve_poll(prandtl_server *s, long long ticket, int *done, double *seconds) {
    if (!s || !done) return PRANDTL_EINVAL;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return PRANDTL_EINVAL;
    const Request &r = *it->second;
    *done = r.state >= 2 ? 1 : 0;
    if (seconds) *seconds = r.state >= 2 ? std::chrono::duration<double>(r.t_done - r.t_submit).count() : -1.0;
    if (r.state == 3) return r.status != PRANDTL_OK ? r.status : PRANDTL_ECUDA;
    return PRANDTL_OK;
}

prandtl_status prandtl_serve_wait(prandtl_server *s, long long ticket, double timeout_s, double *seconds) {
    if (!s) return PRANDTL_EINVAL;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return PRANDTL_EINVAL;
    Request *r = it->second.get();
    const auto limit = std::chrono::duration<double>(timeout_s > 0 ? timeout_s : s->timeout_s);
    if (!s->cv_done.wait_for(lk, limit, [&] { return r->state >= 2; })) return PRANDTL_ETIMEDOUT;
    if (seconds) *seconds = std::chrono::duration<double>(r->t_done - r->t_submit).count();
    if (r->state == 2) return PRANDTL_OK;
    return r->status != PRANDTL_OK ? r->status : PRANDTL_ECUDA;
}

prandtl_status prandtl_serve_stats_get(prandtl_server *s, prandtl_serve_stats *st) {
    if (!s || !st) return PRANDTL_EINVAL;
    std::lock_guard<std::mutex> lk(s->mu);
    *st = s->stats;
    if (s->busy) st->busy_s += std::chrono::duration<double>(Clock::now() - s->busy_since).count();
    return PRANDTL_OK;
}

prandtl_status prandtl_serve_destroy(prandtl_server *s) {
    if (!s) return PRANDTL_EINVAL;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    if (s->worker.joinable()) s->worker.join();
    prandtl_batch_destroy(s->b);
    delete s;
    return PRANDTL_OK;
}

const char *prandtl_serve_last_error(prandtl_server *s) { return s ? s->err.c_str() : ""; }

}   // extern "C"
