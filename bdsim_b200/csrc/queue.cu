// queue.cu -- the serving queue of the C ABI (bdcu_queue_*): continuous
// batching of ensemble jobs over one slot pool, on top of bdcu_reserve /
// bdcu_update_chains / bdcu_write_arena / bdcu_select / bdcu_run_slice. The
// policy is the Python bdsim_b200.serving.Server's (admission by slots, beads,
// arena and an active-chain cap; time-sliced launches; a snapshot per chunk);
// this file lets a C or C++ host serve without Python.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <list>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "../../include/bdsim_cuda.h"

namespace {

// First-fit allocator of [0, capacity) in integer units (sorted, coalesced
// free list).
class Intervals {
  public:
    explicit Intervals(int64_t capacity = 0) { reset(capacity); }
    void reset(int64_t capacity) {
        free_.clear();
        if (capacity > 0) free_.push_back({0, capacity});
    }
    int64_t alloc(int64_t n) {
        if (n <= 0) return 0;
        for (size_t i = 0; i < free_.size(); ++i) {
            if (free_[i].len >= n) {
                int64_t s = free_[i].start;
                if (free_[i].len == n) {
                    free_.erase(free_.begin() + (long)i);
                } else {
                    free_[i].start += n;
                    free_[i].len -= n;
                }
                return s;
            }
        }
        return -1;
    }
    void release(int64_t start, int64_t n) {
        if (n <= 0) return;
        auto it = std::lower_bound(free_.begin(), free_.end(), start,
                                   [](const Run& r, int64_t s) { return r.start < s; });
        it = free_.insert(it, {start, n});
        size_t i = (size_t)(it - free_.begin());
        if (i + 1 < free_.size() && free_[i].start + free_[i].len == free_[i + 1].start) {
            free_[i].len += free_[i + 1].len;
            free_.erase(free_.begin() + (long)(i + 1));
        }
        if (i > 0 && free_[i - 1].start + free_[i - 1].len == free_[i].start) {
            free_[i - 1].len += free_[i].len;
            free_.erase(free_.begin() + (long)i);
        }
    }

  private:
    struct Run {
        int64_t start, len;
    };
    std::vector<Run> free_;
};

struct Event {
    bdcu_queue_event ev{};
    std::vector<double> positions;  // SNAPSHOT
    std::vector<int32_t> status;    // DONE
};

struct Job {
    int64_t id = 0;
    bdcu_job desc{};  // pointers cleared; the data is held below
    std::vector<double> arena;
    std::vector<double> R0;
    std::vector<int32_t> rng;
    int N = 0;
    int n = 0;
    double t_arrival = 0.0, t_admit = -1.0;
    // running state
    int64_t step = 0;        // steps of the chunks completed
    int64_t chunk_end = -1;  // step count at the end of the chunk in progress (-1: none)
    double t_chunk_end = 0.0;
    int snap = 0;            // snapshots delivered
    int64_t slot0 = -1, bead0 = -1, arena0 = -1, arena_n = 0;
    int64_t work() const { return (int64_t)n * desc.n_steps * (int64_t)N * (int64_t)N; }
};

double elapsed_s(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// Steps of the chunk starting at `step`: the reference loop's count over
// [t0, t0 + (chunk-1)dt] with t0 = time_start + step*dt (the chunking of
// python/bdsim/ensemble.py:119-121).
int chunk_steps(const bdcu_sim& sim, int64_t step, int64_t chunk, int32_t* k) {
    bdcu_sim seg = sim;
    seg.time_start = sim.time_start + (double)step * sim.dt;
    seg.time_end = seg.time_start + (double)(chunk - 1) * sim.dt;
    int64_t kk = 0;
    int rc = bdcu_count_steps(&seg, &kk);
    if (rc) return rc;
    if (kk > 0x7fffffff) return BDCU_E_LIMIT;
    *k = (int32_t)kk;
    return BDCU_OK;
}

}  // namespace

struct bdcu_queue {
    bdcu_queue_config cfg{};
    int device = 0;
    bdcu_ctx* ctx = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    std::chrono::steady_clock::time_point t_created;
    // device state of the pool
    double* R = nullptr;
    double* cache = nullptr;
    int32_t* rng = nullptr;
    int32_t* valid = nullptr;
    int32_t* status = nullptr;
    bdcu_counters* counters = nullptr;
    double* t0 = nullptr;
    int32_t* k = nullptr;
    int32_t* steps_done = nullptr;
    double* t_end = nullptr;
    // pinned host mirrors
    double* t_host = nullptr;
    int32_t* k_host = nullptr;
    int32_t* done_host = nullptr;
    double* tend_host = nullptr;
    int32_t* status_host = nullptr;
    bdcu_counters* cnt_host = nullptr;
    double* snap_host = nullptr;  // staging of delivered positions (grown on demand)
    size_t snap_cap = 0;
    // host view of every slot: steps left in its chunk, time of its next step
    std::vector<int32_t> rem;
    std::vector<double> tnext;
    Intervals slots, beads, arena;
    // scheduler state (touched only by the iterating thread)
    std::list<std::unique_ptr<Job>> queue, running;
    std::vector<int32_t> selected;
    int64_t active_chains = 0;
    // shared with submit / poll / stats (under mu)
    std::mutex mu;
    std::condition_variable cv_work, cv_idle;
    std::deque<std::unique_ptr<Job>> incoming;
    std::deque<Event> events;
    int64_t next_id = 1;
    int64_t n_queued = 0, n_running = 0;
    bdcu_queue_stats st{};
    int failed = 0;  // a failing iteration's code (the queue then stops)
    std::string err;
    // worker
    std::thread worker;
    bool stop = false;
    std::mutex step_mu;  // one iteration at a time
};

namespace {

thread_local std::string g_create_error;  // bdcu_queue_create's failures (no queue to hold them)

int qfail(bdcu_queue* q, int code, const std::string& msg) {
    std::lock_guard<std::mutex> lk(q->mu);
    q->err = msg;
    return code;
}

#define QCK(call)                                                                                        \
    do {                                                                                                 \
        cudaError_t e_ = (call);                                                                         \
        if (e_ != cudaSuccess) return qfail(q, BDCU_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

#define BCK(call)                                                                                        \
    do {                                                                                                 \
        int rc_ = (call);                                                                                \
        if (rc_ != BDCU_OK) return qfail(q, rc_, std::string(#call) + ": " + bdcu_last_error(q->ctx));   \
    } while (0)

void push_event(bdcu_queue* q, Event&& e) {
    std::lock_guard<std::mutex> lk(q->mu);
    q->events.push_back(std::move(e));
}

Event make_event(bdcu_queue* q, const Job& j, int kind) {
    Event e;
    e.ev.kind = kind;
    e.ev.n_traj = j.n;
    e.ev.n_beads = j.N;
    e.ev.job = j.id;
    e.ev.tag = j.desc.tag;
    e.ev.step = j.step;
    e.ev.t_arrival = j.t_arrival;
    e.ev.t_admit = j.t_admit;
    e.ev.t_done = -1.0;
    (void)q;
    return e;
}

void release_all(bdcu_queue* q) {
    if (q->device >= 0) cudaSetDevice(q->device);
    if (q->stream) cudaStreamSynchronize(q->stream);
    if (q->ctx) bdcu_destroy(q->ctx);
    void* dev[] = {q->R, q->cache, q->rng, q->valid, q->status, q->counters, q->t0, q->k, q->steps_done, q->t_end};
    for (void* p : dev)
        if (p) cudaFree(p);
    void* host[] = {q->t_host, q->k_host, q->done_host, q->tend_host, q->status_host, q->cnt_host, q->snap_host};
    for (void* p : host)
        if (p) cudaFreeHost(p);
    if (q->e0) cudaEventDestroy(q->e0);
    if (q->e1) cudaEventDestroy(q->e1);
    if (q->stream) cudaStreamDestroy(q->stream);
    delete q;
}

// Admit queued jobs while the pool has room (Server._admit).
int admit(bdcu_queue* q) {
    if (q->queue.empty()) return BDCU_OK;
    if (q->cfg.policy == BDCU_QUEUE_SJF && q->queue.size() > 1)
        q->queue.sort([](const std::unique_ptr<Job>& a, const std::unique_ptr<Job>& b) {
            if (a->work() != b->work()) return a->work() < b->work();
            return a->t_arrival < b->t_arrival;
        });
    const size_t limit = q->cfg.policy == BDCU_QUEUE_FIFO ? (size_t)q->cfg.lookahead : q->queue.size();
    size_t looked = 0;
    const int max_active = q->cfg.max_active_chains > 0 ? q->cfg.max_active_chains : q->cfg.max_chains;
    for (auto it = q->queue.begin(); it != q->queue.end() && looked < limit;) {
        Job& j = **it;
        const int64_t n = j.n, N = j.N;
        int64_t s0 = -1, b0 = -1, a0 = -1;
        if (q->active_chains + n <= max_active) s0 = q->slots.alloc(n);
        if (s0 >= 0) b0 = q->beads.alloc(n * N);
        if (b0 >= 0) a0 = j.desc.arena_len > 0 ? q->arena.alloc(j.desc.arena_len) : 0;
        if (s0 < 0 || b0 < 0 || a0 < 0) {
            if (b0 >= 0) q->beads.release(b0, n * N);
            if (s0 >= 0) q->slots.release(s0, n);
            ++it;
            ++looked;
            continue;
        }
        cudaStream_t s = q->stream;
        QCK(cudaMemcpyAsync(q->R + 3 * b0, j.R0.data(), sizeof(double) * 3 * n * N, cudaMemcpyHostToDevice, s));
        QCK(cudaMemcpyAsync(q->rng + 3 * s0, j.rng.data(), sizeof(int32_t) * 3 * n, cudaMemcpyHostToDevice, s));
        QCK(cudaMemsetAsync(q->valid + s0, 0, sizeof(int32_t) * n, s));
        QCK(cudaMemsetAsync(q->status + s0, 0, sizeof(int32_t) * n, s));
        QCK(cudaMemsetAsync(q->counters + s0, 0, sizeof(bdcu_counters) * n, s));
        bdcu_phys p = j.desc.phys;
        if (j.desc.arena_len > 0) {
            BCK(bdcu_write_arena(q->ctx, a0, j.arena.data(), j.desc.arena_len));
            if (p.phi_offset >= 0) p.phi_offset += a0;
            if (p.flow_n_times > 0) p.flow_offset += a0;
            if (p.ext_n_entries > 0) p.ext_offset += a0;
        }
        std::vector<bdcu_phys> P((size_t)n, p);
        std::vector<bdcu_sim> S((size_t)n, j.desc.sim);
        std::vector<int32_t> ids((size_t)n);
        std::vector<int64_t> offs((size_t)n);
        for (int64_t t = 0; t < n; ++t) {
            ids[(size_t)t] = (int32_t)(s0 + t);
            offs[(size_t)t] = b0 + t * N;
        }
        BCK(bdcu_update_chains(q->ctx, (int)n, ids.data(), P.data(), S.data(), offs.data()));
        j.slot0 = s0;
        j.bead0 = b0;
        j.arena0 = a0;
        j.arena_n = j.desc.arena_len;
        j.t_admit = elapsed_s(q->t_created);
        j.snap = 1;  // snapshot 0 is the initial state
        if (j.desc.snapshots) {
            Event e = make_event(q, j, BDCU_QEV_SNAPSHOT);
            e.ev.snapshot = 0;
            e.ev.time = j.desc.sim.time_start;
            e.positions = j.R0;
            push_event(q, std::move(e));
        }
        // (pageable uploads return once the source is staged: the copies may go)
        std::vector<double>().swap(j.R0);
        std::vector<int32_t>().swap(j.rng);
        std::vector<double>().swap(j.arena);
        q->active_chains += n;
        q->running.push_back(std::move(*it));
        it = q->queue.erase(it);
        std::lock_guard<std::mutex> lk(q->mu);
        --q->n_queued;
        ++q->n_running;
        q->st.active_chains = q->active_chains;
    }
    return BDCU_OK;
}

// One time-sliced launch over the running jobs' chains, then the snapshots
// and completions it produced (Server._launch_slice and _finish_slice).
int run_slice(bdcu_queue* q) {
    if (q->running.empty()) return BDCU_OK;
    cudaStream_t s = q->stream;
    int64_t hi_slot = 0;
    std::vector<Job*> fresh;
    for (auto& jp : q->running) {
        Job& j = *jp;
        if (j.chunk_end < 0) {  // the job's next chunk: one integrate span
            const int64_t w = j.desc.write_every > 0 ? j.desc.write_every : j.desc.n_steps;
            const int64_t chunk = std::min(w, j.desc.n_steps - j.step);
            int32_t k = 0;
            if (chunk > 0) {
                int rc = chunk_steps(j.desc.sim, j.step, chunk, &k);
                if (rc) return qfail(q, rc, "job " + std::to_string(j.id) + ": bad chunk time span");
            }
            const double t0 = j.desc.sim.time_start + (double)j.step * j.desc.sim.dt;
            for (int64_t c = j.slot0; c < j.slot0 + j.n; ++c) {
                q->rem[(size_t)c] = k;
                q->tnext[(size_t)c] = t0;
            }
            j.chunk_end = j.step + chunk;
            j.t_chunk_end = j.desc.sim.time_start + (double)j.chunk_end * j.desc.sim.dt;
            fresh.push_back(&j);
        }
        hi_slot = std::max(hi_slot, j.slot0 + j.n);
    }
    std::vector<int32_t> sel;
    for (auto& jp : q->running)
        for (int64_t c = jp->slot0; c < jp->slot0 + jp->n; ++c)
            if (q->rem[(size_t)c] > 0) sel.push_back((int32_t)c);
    if (!sel.empty()) {
        for (int64_t c = 0; c < hi_slot; ++c) {
            q->k_host[c] = std::min(q->rem[(size_t)c], q->cfg.slice_steps);
            q->t_host[c] = q->tnext[(size_t)c];
        }
        QCK(cudaMemcpyAsync(q->t0, q->t_host, sizeof(double) * hi_slot, cudaMemcpyHostToDevice, s));
        QCK(cudaMemcpyAsync(q->k, q->k_host, sizeof(int32_t) * hi_slot, cudaMemcpyHostToDevice, s));
        if (q->cfg.cache_mode == BDCU_CACHE_RESET_PER_CALL)  // a new chunk is a new integrate call
            for (Job* j : fresh) QCK(cudaMemsetAsync(q->valid + j->slot0, 0, sizeof(int32_t) * j->n, s));
        if (sel != q->selected) {
            BCK(bdcu_select(q->ctx, (int)sel.size(), sel.data()));
            q->selected = sel;
        }
        QCK(cudaEventRecord(q->e0, s));
        BCK(bdcu_run_slice(q->ctx, q->R, q->rng, q->cache, q->valid, q->t0, q->k, q->status, q->counters,
                           q->cfg.form, BDCU_CACHE_PERSIST, q->cfg.slice_budget_ns, q->steps_done, q->t_end));
        QCK(cudaEventRecord(q->e1, s));
        QCK(cudaMemcpyAsync(q->done_host, q->steps_done, sizeof(int32_t) * hi_slot, cudaMemcpyDeviceToHost, s));
        QCK(cudaMemcpyAsync(q->tend_host, q->t_end, sizeof(double) * hi_slot, cudaMemcpyDeviceToHost, s));
        QCK(cudaMemcpyAsync(q->status_host, q->status, sizeof(int32_t) * hi_slot, cudaMemcpyDeviceToHost, s));
        QCK(cudaStreamSynchronize(s));
        float ms = 0.f;
        QCK(cudaEventElapsedTime(&ms, q->e0, q->e1));
        int64_t moved = 0;
        for (int32_t c : sel) {
            const int32_t d = q->done_host[c];
            q->rem[(size_t)c] -= d;
            if (d > 0) q->tnext[(size_t)c] = q->tend_host[c];
            moved += d;
            if (q->status_host[c] & BDCU_ST_FATAL_MASK) q->rem[(size_t)c] = 0;  // a failed chain stops for good
        }
        std::lock_guard<std::mutex> lk(q->mu);
        q->st.device_ms += ms;
        q->st.slices += 1;
        q->st.selected_chains += (int64_t)sel.size();
        q->st.chain_steps += moved;
    }

    // chunks complete for every chain of a job: deliver them
    std::vector<Job*> done_chunk;
    for (auto& jp : q->running) {
        Job& j = *jp;
        if (j.chunk_end < 0) continue;
        bool pending = false;
        for (int64_t c = j.slot0; c < j.slot0 + j.n && !pending; ++c) pending = q->rem[(size_t)c] > 0;
        if (!pending) done_chunk.push_back(&j);
    }
    if (done_chunk.empty()) return BDCU_OK;
    std::vector<char> last(done_chunk.size(), 0), want(done_chunk.size(), 0);
    std::vector<size_t> at(done_chunk.size(), 0);
    size_t need = 0;
    for (size_t i = 0; i < done_chunk.size(); ++i) {
        Job& j = *done_chunk[i];
        bool all_fatal = true;
        for (int64_t c = j.slot0; c < j.slot0 + j.n && all_fatal; ++c)
            all_fatal = (q->status_host[c] & BDCU_ST_FATAL_MASK) != 0;
        last[i] = (j.chunk_end >= j.desc.n_steps || all_fatal) ? 1 : 0;
        want[i] = (j.desc.snapshots || last[i]) ? 1 : 0;
        at[i] = need;
        if (want[i]) need += (size_t)3 * j.n * j.N;
    }
    if (need > q->snap_cap) {
        const size_t cap = std::max(need, q->snap_cap * 2);
        if (q->snap_host) QCK(cudaFreeHost(q->snap_host));
        q->snap_host = nullptr;
        q->snap_cap = 0;
        QCK(cudaHostAlloc((void**)&q->snap_host, sizeof(double) * cap, cudaHostAllocDefault));
        q->snap_cap = cap;
    }
    for (size_t i = 0; i < done_chunk.size(); ++i) {
        Job& j = *done_chunk[i];
        if (want[i])
            QCK(cudaMemcpyAsync(q->snap_host + at[i], q->R + 3 * j.bead0, sizeof(double) * 3 * j.n * j.N,
                                cudaMemcpyDeviceToHost, s));
        if (last[i]) {
            QCK(cudaMemcpyAsync(q->status_host + j.slot0, q->status + j.slot0, sizeof(int32_t) * j.n,
                                cudaMemcpyDeviceToHost, s));
            QCK(cudaMemcpyAsync(q->cnt_host + j.slot0, q->counters + j.slot0, sizeof(bdcu_counters) * j.n,
                                cudaMemcpyDeviceToHost, s));
        }
    }
    QCK(cudaStreamSynchronize(s));
    const double now = elapsed_s(q->t_created);
    for (size_t i = 0; i < done_chunk.size(); ++i) {
        Job& j = *done_chunk[i];
        j.step = j.chunk_end;
        j.chunk_end = -1;
        const int snap = j.snap++;
        if (want[i]) {
            Event e = make_event(q, j, BDCU_QEV_SNAPSHOT);
            e.ev.snapshot = snap;
            e.ev.time = j.t_chunk_end;
            e.positions.assign(q->snap_host + at[i], q->snap_host + at[i] + (size_t)3 * j.n * j.N);
            push_event(q, std::move(e));
        }
        if (!last[i]) continue;
        Event e = make_event(q, j, BDCU_QEV_DONE);
        e.ev.time = j.t_chunk_end;
        e.ev.t_done = now;
        e.status.assign(q->status_host + j.slot0, q->status_host + j.slot0 + j.n);
        bdcu_counters sum{};
        for (int64_t c = j.slot0; c < j.slot0 + j.n; ++c) {
            const bdcu_counters& r = q->cnt_host[c];
            sum.steps += r.steps;
            sum.dx_products += r.dx_products;
            sum.cheb_terms += r.cheb_terms;
            sum.corrector_iters += r.corrector_iters;
            sum.lanczos_cold += r.lanczos_cold;
            sum.lanczos_warm += r.lanczos_warm;
            sum.cheb_fallbacks += r.cheb_fallbacks;
            sum.nonconverged += r.nonconverged;
        }
        e.ev.counters = sum;
        // retire: the slots, beads and arena go back to the pool
        for (int64_t c = j.slot0; c < j.slot0 + j.n; ++c) q->rem[(size_t)c] = 0;
        q->slots.release(j.slot0, j.n);
        q->beads.release(j.bead0, (int64_t)j.n * j.N);
        if (j.arena_n) q->arena.release(j.arena0, j.arena_n);
        q->active_chains -= j.n;
        j.slot0 = -1;  // retired
        std::lock_guard<std::mutex> lk(q->mu);
        q->events.push_back(std::move(e));
        --q->n_running;
        ++q->st.done;
        q->st.active_chains = q->active_chains;
    }
    q->running.remove_if([](const std::unique_ptr<Job>& jp) { return jp->chunk_end < 0 && jp->slot0 < 0; });
    return BDCU_OK;
}

bool busy_locked(const bdcu_queue* q) { return q->n_queued > 0 || q->n_running > 0; }

// One server iteration: take the submissions, admit, one slice. A failure
// stops the queue (its code is returned by every later call).
int iterate(bdcu_queue* q, int* busy) {
    std::lock_guard<std::mutex> step_lk(q->step_mu);
    {
        std::lock_guard<std::mutex> lk(q->mu);
        if (q->failed) return q->failed;
        while (!q->incoming.empty()) {
            q->queue.push_back(std::move(q->incoming.front()));
            q->incoming.pop_front();
        }
    }
    int rc = BDCU_OK;
    if (cudaSetDevice(q->device) != cudaSuccess) rc = qfail(q, BDCU_E_CUDA, "cudaSetDevice");
    if (!rc) rc = admit(q);
    if (!rc) rc = run_slice(q);
    std::lock_guard<std::mutex> lk(q->mu);
    if (rc) q->failed = rc;
    if (busy) *busy = busy_locked(q) ? 1 : 0;
    if (rc || !busy_locked(q)) q->cv_idle.notify_all();
    return rc;
}

void worker_loop(bdcu_queue* q) {
    cudaSetDevice(q->device);
    for (;;) {
        {
            std::unique_lock<std::mutex> lk(q->mu);
            q->cv_work.wait(lk, [q] { return q->stop || q->failed || busy_locked(q); });
            if (q->stop || q->failed) return;
        }
        if (iterate(q, nullptr)) return;
    }
}

int check_config(const bdcu_queue_config& c, std::string* why) {
    if (c.form != BDCU_FORM_PLAIN_FP64 && c.form != BDCU_FORM_MIXED_FP32) return *why = "unknown form", BDCU_E_ARG;
    if (c.policy != BDCU_QUEUE_FIFO && c.policy != BDCU_QUEUE_SJF) return *why = "unknown policy", BDCU_E_ARG;
    if (c.max_chains < 1 || c.max_active_chains < 0) return *why = "need max_chains >= 1, max_active_chains >= 0", BDCU_E_ARG;
    if (c.bead_capacity < 2 || c.arena_capacity < 0) return *why = "need bead_capacity >= 2, arena_capacity >= 0", BDCU_E_ARG;
    if (c.queue_limit < 0 || c.lookahead < 0) return *why = "negative queue_limit or lookahead", BDCU_E_ARG;
    if (c.slice_steps < 1) return *why = "need slice_steps >= 1", BDCU_E_ARG;
    if (c.cache_mode != BDCU_CACHE_RESET_PER_CALL && c.cache_mode != BDCU_CACHE_PERSIST)
        return *why = "unknown cache mode", BDCU_E_ARG;
    if (c.slice_budget_ns < 0) return *why = "negative slice budget", BDCU_E_ARG;
    if (c.worker != 0 && c.worker != 1) return *why = "worker is 0 or 1", BDCU_E_ARG;
    return BDCU_OK;
}

}  // namespace

extern "C" {

int bdcu_queue_create(int device, const bdcu_queue_config* cfg, bdcu_queue** out) {
    if (!cfg || !out) return g_create_error = "null config or handle", BDCU_E_ARG;
    *out = nullptr;
    std::string why;
    int rc = check_config(*cfg, &why);
    if (rc) return g_create_error = why, rc;
    bdcu_queue* q = new (std::nothrow) bdcu_queue();
    if (!q) return g_create_error = "out of host memory", BDCU_E_NOMEM;
    q->cfg = *cfg;
    if (q->cfg.lookahead == 0) q->cfg.lookahead = 16;
    q->device = device;
    q->t_created = std::chrono::steady_clock::now();
    const int64_t nc = cfg->max_chains, nb = cfg->bead_capacity;
    auto bail = [&](int code, const std::string& msg) {
        g_create_error = msg;
        release_all(q);
        return code;
    };
#define CCK(call)                                                                          \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess) return bail(BDCU_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)
    CCK(cudaSetDevice(device));
    if ((rc = bdcu_create(device, &q->ctx))) return bail(rc, "bdcu_create failed");
    CCK(cudaStreamCreateWithFlags(&q->stream, cudaStreamNonBlocking));
    if ((rc = bdcu_set_stream(q->ctx, q->stream))) return bail(rc, bdcu_last_error(q->ctx));
    if ((rc = bdcu_reserve(q->ctx, (int)nc, nb, cfg->arena_capacity))) return bail(rc, bdcu_last_error(q->ctx));
    CCK(cudaMalloc((void**)&q->R, sizeof(double) * 3 * nb));
    CCK(cudaMalloc((void**)&q->cache, sizeof(double) * 3 * nb));
    CCK(cudaMalloc((void**)&q->rng, sizeof(int32_t) * 3 * nc));
    CCK(cudaMalloc((void**)&q->valid, sizeof(int32_t) * nc));
    CCK(cudaMalloc((void**)&q->status, sizeof(int32_t) * nc));
    CCK(cudaMalloc((void**)&q->counters, sizeof(bdcu_counters) * nc));
    CCK(cudaMalloc((void**)&q->t0, sizeof(double) * nc));
    CCK(cudaMalloc((void**)&q->k, sizeof(int32_t) * nc));
    CCK(cudaMalloc((void**)&q->steps_done, sizeof(int32_t) * nc));
    CCK(cudaMalloc((void**)&q->t_end, sizeof(double) * nc));
    CCK(cudaMemsetAsync(q->R, 0, sizeof(double) * 3 * nb, q->stream));
    CCK(cudaMemsetAsync(q->cache, 0, sizeof(double) * 3 * nb, q->stream));
    CCK(cudaMemsetAsync(q->k, 0, sizeof(int32_t) * nc, q->stream));
    CCK(cudaHostAlloc((void**)&q->t_host, sizeof(double) * nc, cudaHostAllocDefault));
    CCK(cudaHostAlloc((void**)&q->k_host, sizeof(int32_t) * nc, cudaHostAllocDefault));
    CCK(cudaHostAlloc((void**)&q->done_host, sizeof(int32_t) * nc, cudaHostAllocDefault));
    CCK(cudaHostAlloc((void**)&q->tend_host, sizeof(double) * nc, cudaHostAllocDefault));
    CCK(cudaHostAlloc((void**)&q->status_host, sizeof(int32_t) * nc, cudaHostAllocDefault));
    CCK(cudaHostAlloc((void**)&q->cnt_host, sizeof(bdcu_counters) * nc, cudaHostAllocDefault));
    CCK(cudaEventCreate(&q->e0));
    CCK(cudaEventCreate(&q->e1));
    CCK(cudaStreamSynchronize(q->stream));
#undef CCK
    try {
        q->rem.assign((size_t)nc, 0);
        q->tnext.assign((size_t)nc, 0.0);
        q->slots.reset(nc);
        q->beads.reset(nb);
        q->arena.reset(cfg->arena_capacity);
        if (cfg->worker) q->worker = std::thread(worker_loop, q);
    } catch (const std::exception& ex) {
        return bail(BDCU_E_NOMEM, ex.what());
    }
    *out = q;
    return BDCU_OK;
}

int bdcu_queue_destroy(bdcu_queue* q) {
    if (!q) return BDCU_E_ARG;
    {
        std::lock_guard<std::mutex> lk(q->mu);
        q->stop = true;
    }
    q->cv_work.notify_all();
    if (q->worker.joinable()) q->worker.join();
    release_all(q);
    return BDCU_OK;
}

const char* bdcu_queue_last_error(bdcu_queue* q) {
    if (!q) return g_create_error.c_str();
    std::lock_guard<std::mutex> lk(q->mu);
    return q->err.c_str();
}

int bdcu_queue_submit(bdcu_queue* q, const bdcu_job* job, int64_t* job_id, int* accepted) {
    if (!q) return BDCU_E_ARG;
    if (!job || !job_id || !accepted) return qfail(q, BDCU_E_ARG, "null job, job_id or accepted");
    *accepted = 0;
    *job_id = 0;
    const bdcu_job& d = *job;
    if (d.n_traj < 1 || d.n_steps < 0 || d.write_every < 0 || !d.R0 || !d.rng || d.arena_len < 0 ||
        (d.arena_len > 0 && !d.arena) || (d.snapshots != 0 && d.snapshots != 1))
        return qfail(q, BDCU_E_ARG, "bad job: need n_traj >= 1, n_steps >= 0, write_every >= 0, R0, rng, "
                                    "the arena when arena_len > 0, snapshots 0 or 1");
    const int64_t chunk = d.write_every > 0 ? std::min(d.write_every, d.n_steps) : d.n_steps;
    if (chunk > 0x7ffffffe) return qfail(q, BDCU_E_LIMIT, "a chunk of more than 2^31 - 2 steps");
    char msg[256] = {0};
    int rc = bdcu_check_chains(1, &d.phys, &d.sim, d.arena, d.arena_len, msg, (int)sizeof(msg));
    if (rc) return qfail(q, rc, std::string("job record: ") + msg);
    std::unique_ptr<Job> j;
    try {
        j.reset(new Job());
        j->desc = d;
        j->desc.arena = nullptr;
        j->desc.R0 = nullptr;
        j->desc.rng = nullptr;
        j->n = d.n_traj;
        j->N = d.phys.n_beads;
        j->R0.assign(d.R0, d.R0 + (size_t)3 * d.n_traj * d.phys.n_beads);
        j->rng.assign(d.rng, d.rng + (size_t)3 * d.n_traj);
        if (d.arena_len > 0) j->arena.assign(d.arena, d.arena + d.arena_len);
    } catch (const std::exception&) {
        return qfail(q, BDCU_E_NOMEM, "out of host memory copying the job");
    }
    const int max_active = q->cfg.max_active_chains > 0 ? q->cfg.max_active_chains : q->cfg.max_chains;
    std::lock_guard<std::mutex> lk(q->mu);
    if (q->failed) return q->failed;
    j->id = q->next_id++;
    j->t_arrival = elapsed_s(q->t_created);
    *job_id = j->id;
    ++q->st.submitted;
    const bool too_big = j->n > std::min(q->cfg.max_chains, max_active) ||
                         (int64_t)j->n * j->N > q->cfg.bead_capacity || d.arena_len > q->cfg.arena_capacity;
    if (too_big || (q->cfg.queue_limit > 0 && q->n_queued >= q->cfg.queue_limit)) {
        ++q->st.rejected;
        Event e = make_event(q, *j, BDCU_QEV_REJECTED);
        q->events.push_back(std::move(e));
        return BDCU_OK;
    }
    q->incoming.push_back(std::move(j));
    ++q->n_queued;
    *accepted = 1;
    q->cv_work.notify_one();
    return BDCU_OK;
}

int bdcu_queue_step(bdcu_queue* q, int* busy) {
    if (!q) return BDCU_E_ARG;
    if (q->cfg.worker) return qfail(q, BDCU_E_STATE, "bdcu_queue_step on a queue with a worker thread");
    return iterate(q, busy);
}

int bdcu_queue_wait_idle(bdcu_queue* q, int64_t timeout_ms, int* busy) {
    if (!q) return BDCU_E_ARG;
    const auto t0 = std::chrono::steady_clock::now();
    const auto deadline = t0 + std::chrono::milliseconds(timeout_ms < 0 ? 0 : timeout_ms);
    if (q->cfg.worker) {
        std::unique_lock<std::mutex> lk(q->mu);
        auto idle = [q] { return q->failed || !busy_locked(q); };
        if (timeout_ms < 0)
            q->cv_idle.wait(lk, idle);
        else
            q->cv_idle.wait_until(lk, deadline, idle);
        if (busy) *busy = busy_locked(q) ? 1 : 0;
        return q->failed;
    }
    int b = 1;
    while (b) {
        int rc = iterate(q, &b);
        if (rc) return rc;
        if (timeout_ms >= 0 && std::chrono::steady_clock::now() >= deadline) break;
    }
    if (busy) *busy = b;
    return BDCU_OK;
}

int bdcu_queue_poll(bdcu_queue* q, bdcu_queue_event* ev, double* positions, int64_t positions_len, int32_t* status,
                    int32_t status_len, int* got) {
    if (!q) return BDCU_E_ARG;
    if (!ev || !got) return qfail(q, BDCU_E_ARG, "null event or got");
    *got = 0;
    std::lock_guard<std::mutex> lk(q->mu);
    if (q->events.empty()) return BDCU_OK;
    Event& e = q->events.front();
    *ev = e.ev;
    if (positions && !e.positions.empty() && positions_len < (int64_t)e.positions.size()) {
        q->err = "positions buffer smaller than n_traj*n_beads*3";
        return BDCU_E_LIMIT;
    }
    if (status && !e.status.empty() && status_len < (int32_t)e.status.size()) {
        q->err = "status buffer smaller than n_traj";
        return BDCU_E_LIMIT;
    }
    if (positions && !e.positions.empty()) memcpy(positions, e.positions.data(), sizeof(double) * e.positions.size());
    if (status && !e.status.empty()) memcpy(status, e.status.data(), sizeof(int32_t) * e.status.size());
    q->events.pop_front();
    *got = 1;
    return BDCU_OK;
}

int bdcu_queue_get_stats(bdcu_queue* q, bdcu_queue_stats* out) {
    if (!q) return BDCU_E_ARG;
    if (!out) return qfail(q, BDCU_E_ARG, "null stats");
    std::lock_guard<std::mutex> lk(q->mu);
    *out = q->st;
    out->queued = q->n_queued;
    out->running = q->n_running;
    out->pending_events = (int64_t)q->events.size();
    return BDCU_OK;
}

}  // extern "C"
