// Continuous-batching flow server.
//
// A scheduler thread owns the context.  Each tick it (1) admits queued jobs in
// arrival order while the head job's HBM footprint (links ring + RK3
// accumulator + measurement buffers) fits the remaining budget and a slot is
// free, (2) runs steps_per_tick RK3 steps of every resident job as shared
// persistent launches (one group per precision, graph-captured once; the work
// list and its length live in device memory so members join and leave without
// re-capture), (3) measures the jobs that are due, and (4) retires finished
// jobs: results are copied to the caller's arrays, their memory returns to the
// arena and waiters are woken.  A job's arithmetic does not depend on which
// other jobs share its launches, so its results are the same alone and in the
// mix.
//
// Memory: lgf_serve_start reserves the whole budget as one device arena, and
// every job's buffers are one block of it (first fit, neighbouring free blocks
// merged), so admission and retirement make no cudaMalloc / cudaFree (both of
// which would stall the device).  Admission is asynchronous: a job's upload or
// generation runs on a second stream, after the retirements whose memory it
// may reuse (an event), and the job joins the shared launches once its own
// event reports the input in place; resident jobs keep flowing meanwhile.
//
// Snapshots: a job with a snapshot prefix gets, after each measured step, its
// links reordered to file order into a buffer of its own block (on the flow
// stream); a writer thread copies that buffer to the host on a third stream
// once an event says it is complete and writes <prefix>_Flowtime<t>.bin, so
// the flow never waits for the disk (only for a job's previous snapshot,
// should it still be in flight).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <cstdio>
#include <deque>
#include <map>
#include <string>
#include <memory>
#include <mutex>
#include <new>
#include <thread>
#include <vector>

#include "lgf_engine.cuh"

using namespace lgf;

namespace {

struct ServeJob {
    uint64_t id = 0;
    lgf_job job{};
    lgf_job_status st{};
    size_t bytes = 0;
    char* mem = nullptr;             // its block of the arena while admitted
    cudaEvent_t ready = nullptr;     // its input is in place (admission stream)
    double* snap_buf = nullptr;      // file-order snapshot buffer (inside its block), or null
    bool snap_pending = false;       // a snapshot of this job is being written (guarded by snap_mu)
    int snap_err = LGF_OK;           // first failed snapshot write
    LatticeBuf buf;
    int nmeas = 0;
    std::atomic<int> steps_done{0};  // advanced by the worker, read by pollers
    double t = 0.0;
    std::vector<double> tvals;
};

// One device reservation carved into job blocks: first fit over a map of free
// blocks (offset -> length), neighbours merged on release.  Used by the
// scheduler thread only.
class Arena {
public:
    ~Arena() {
        if (base_) cudaFree(base_);
    }
    cudaError_t reserve(size_t bytes) {
        cudaError_t e = cudaMalloc(&base_, bytes);
        if (e != cudaSuccess) {
            base_ = nullptr;
            return e;
        }
        size_ = bytes;
        free_[0] = bytes;
        return cudaSuccess;
    }
    char* alloc(size_t n) {
        n = round(n);
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < n) continue;
            const size_t off = it->first, len = it->second;
            free_.erase(it);
            if (len > n) free_[off + n] = len - n;
            return base_ + off;
        }
        return nullptr;
    }
    void release(char* p, size_t n) {
        n = round(n);
        size_t off = (size_t)(p - base_);
        auto next = free_.lower_bound(off);
        if (next != free_.end() && off + n == next->first) {
            n += next->second;
            free_.erase(next);
        }
        auto prev = free_.lower_bound(off);
        if (prev != free_.begin()) {
            --prev;
            if (prev->first + prev->second == off) {
                off = prev->first;
                n += prev->second;
                free_.erase(prev);
            }
        }
        free_[off] = n;
    }

private:
    static size_t round(size_t n) { return (n + 255) & ~size_t(255); }
    char* base_ = nullptr;
    size_t size_ = 0;
    std::map<size_t, size_t> free_;
};

struct SnapTask {
    ServeJob* job;
    cudaEvent_t ev;  // the snapshot buffer is complete (flow stream)
    std::string path;
    size_t bytes;
};

size_t snapshot_bytes(const int shape[4]) {
    return (size_t)shape[0] * shape[1] * shape[2] * shape[3] * 4 * 18 * sizeof(double);
}

double now_s(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

struct lgf_server {
    lgf_ctx* ctx = nullptr;
    lgf_serve_config cfg{};
    std::chrono::steady_clock::time_point t0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done, cv_idle;
    int waiters = 0;  // threads inside lgf_serve_wait; stop frees the server only when none is left
    std::deque<ServeJob*> queue;
    std::map<uint64_t, std::unique_ptr<ServeJob>> jobs;
    std::vector<ServeJob*> staging;  // admitted, input still arriving
    std::vector<ServeJob*> active;
    size_t used = 0;
    Arena arena;
    cudaStream_t adm = nullptr;        // admission stream: uploads and generation
    cudaEvent_t retired_ev = nullptr;  // recorded on the flow stream at each retirement
    // snapshot writer
    std::thread snap_thread;
    cudaStream_t snap_stream = nullptr;
    std::mutex snap_mu;
    std::condition_variable snap_cv, snap_done_cv;
    std::deque<SnapTask> snap_q;
    bool snap_stop = false;
    uint64_t next_id = 1;
    bool stopping = false;
    std::thread worker;
    std::unique_ptr<GroupBase> group[2];
    std::vector<LatticeBuf*> members[2];  // current member list of each group
    std::vector<int> measured[2];         // current measured subset of each group
    TileShape shape[2];
    long long max_tiles[2] = {0, 0};
    int fatal = LGF_OK;

    // statistics (worker thread; read under mu)
    long long n_ticks = 0, n_steps = 0, n_meas = 0, n_done = 0, n_snap = 0;
    double busy_s = 0.0;
    struct TickEv { cudaEvent_t a, b; };
    std::deque<TickEv> tick_ev;      // ticks whose device time is not counted yet
    std::vector<TickEv> ev_free;     // recycled event pairs
    void collect_ticks(bool wait);

    void run();
    void snap_run();
    int snapshot(ServeJob* j);
    void wait_snapshot(ServeJob* j);
    int tick(std::vector<ServeJob*>& act);
    int admit(ServeJob* j);
    int retire(ServeJob* j);
    void finish(ServeJob* j, int state, int err);
};

// writer thread: one snapshot at a time, in the order they were taken
void lgf_server::snap_run() {
    cudaSetDevice(ctx->device);
    std::vector<double> host;
    for (;;) {
        SnapTask t;
        {
            std::unique_lock<std::mutex> lk(snap_mu);
            snap_cv.wait(lk, [&] { return snap_stop || !snap_q.empty(); });
            if (snap_q.empty()) return;
            t = snap_q.front();
            snap_q.pop_front();
        }
        int rc = LGF_OK;
        host.resize(t.bytes / sizeof(double));
        cudaError_t e = cudaStreamWaitEvent(snap_stream, t.ev, 0);
        if (e == cudaSuccess) e = cudaMemcpyAsync(host.data(), t.job->snap_buf, t.bytes, cudaMemcpyDeviceToHost, snap_stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(snap_stream);
        if (e != cudaSuccess) {
            cudaGetLastError();
            rc = LGF_ECUDA;
        } else {
            FILE* f = std::fopen(t.path.c_str(), "wb");
            const bool ok = f && std::fwrite(host.data(), 1, t.bytes, f) == t.bytes;
            if (f && std::fclose(f) != 0) rc = LGF_EIO;
            if (!ok) rc = LGF_EIO;
        }
        cudaEventDestroy(t.ev);
        std::lock_guard<std::mutex> lk(snap_mu);
        if (rc != LGF_OK && t.job->snap_err == LGF_OK) t.job->snap_err = rc;
        t.job->snap_pending = false;
        snap_done_cv.notify_all();
    }
}

void lgf_server::wait_snapshot(ServeJob* j) {
    std::unique_lock<std::mutex> lk(snap_mu);
    snap_done_cv.wait(lk, [&] { return !j->snap_pending; });
}

// the job's current links (after a measured step) to its snapshot file
int lgf_server::snapshot(ServeJob* j) {
    wait_snapshot(j);  // the buffer holds the previous snapshot until it is written
    int rc = launch_to_file(ctx, j->buf, j->snap_buf);
    if (rc != LGF_OK) return rc;
    SnapTask t;
    t.job = j;
    t.bytes = snapshot_bytes(j->job.shape);
    t.path = std::string(j->job.snapshot_prefix) + "_Flowtime" + std::to_string(j->t) + ".bin";
    LGF_CUDA_TRY(ctx, cudaEventCreateWithFlags(&t.ev, cudaEventDisableTiming));
    cudaError_t e = cudaEventRecord(t.ev, ctx->stream);
    if (e != cudaSuccess) {
        cudaEventDestroy(t.ev);
        return set_error(ctx, LGF_ECUDA, "snapshot event failed: %s", cudaGetErrorString(e));
    }
    {
        std::lock_guard<std::mutex> lk(mu);
        ++n_snap;
    }
    std::lock_guard<std::mutex> lk(snap_mu);
    j->snap_pending = true;
    snap_q.push_back(t);
    snap_cv.notify_one();
    return LGF_OK;
}

void lgf_server::finish(ServeJob* j, int state, int err) {
    wait_snapshot(j);  // its buffer lives in the job's block
    // the flow stream's work on this job's block is enqueued by now; a later
    // admission that reuses the block waits for this point
    if (j->mem) {
        cudaEventRecord(retired_ev, ctx->stream);
        arena.release(j->mem, j->bytes);
        j->mem = nullptr;
    }
    if (j->ready) {
        cudaEventDestroy(j->ready);
        j->ready = nullptr;
    }
    buf_free(j->buf);
    std::lock_guard<std::mutex> lk(mu);
    used -= j->bytes;
    if (state == LGF_JOB_DONE) ++n_done;
    j->st.state = state;
    j->st.error = err;
    j->st.end_s = now_s(t0);
    j->st.steps_done = j->steps_done;
    cv_done.notify_all();
}

// Lay the job out in its arena block and enqueue its input on the admission
// stream, behind the retirements whose memory the block may reuse.
int lgf_server::admit(ServeJob* j) {
    buf_place(j->buf, j->job.shape, j->job.precision, j->nmeas, j->mem);
    if (j->job.snapshot_prefix) j->snap_buf = (double*)(j->mem + placed_bytes(j->job.shape, j->job.precision, j->nmeas));
    LGF_CUDA_TRY(ctx, cudaEventCreateWithFlags(&j->ready, cudaEventDisableTiming));
    LGF_CUDA_TRY(ctx, cudaStreamWaitEvent(adm, retired_ev, 0));
    int rc = j->job.links ? upload_links_on(ctx, j->buf, j->job.links, adm)
                          : launch_generate_on(ctx, j->buf, j->job.seed, j->job.gen_scale, adm);
    if (rc != LGF_OK) return rc;
    j->buf.eps = j->job.flow.eps;
    j->t = j->job.flow.t0;
    LGF_CUDA_TRY(ctx, cudaMemsetAsync(j->buf.slot, 0, sizeof(int), adm));
    LGF_CUDA_TRY(ctx, cudaEventRecord(j->ready, adm));
    return LGF_OK;
}

int lgf_server::retire(ServeJob* j) {
    lgf_job& jb = j->job;
    if (j->nmeas > 0 && jb.meas) {
        const int N0 = j->buf.g.n[0];
        const size_t per = 2 + 2 * (size_t)N0;
        std::vector<double> h(per * j->nmeas);
        LGF_CUDA_TRY(ctx, cudaMemcpyAsync(h.data(), j->buf.meas, h.size() * sizeof(double), cudaMemcpyDeviceToHost,
                                          ctx->stream));
        LGF_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
        for (int m = 0; m < j->nmeas; ++m) {
            jb.meas->t[m] = j->tvals[m];
            jb.meas->E[m] = h[m * per];
            jb.meas->Q[m] = h[m * per + 1];
            if (jb.meas->E_slice) std::memcpy(jb.meas->E_slice + (size_t)m * N0, &h[m * per + 2], N0 * sizeof(double));
            if (jb.meas->Q_slice)
                std::memcpy(jb.meas->Q_slice + (size_t)m * N0, &h[m * per + 2 + N0], N0 * sizeof(double));
        }
        jb.meas->count = j->nmeas;
    } else if (jb.meas) {
        jb.meas->count = 0;
    }
    if (jb.links_out) return download_links(ctx, j->buf, jb.links_out);
    return LGF_OK;
}

// one scheduling tick over the resident jobs
int lgf_server::tick(std::vector<ServeJob*>& act) {
    std::vector<ServeJob*> byprec[2];
    for (auto* j : act) byprec[j->job.precision].push_back(j);
    for (int p = 0; p < 2; ++p) {
        if (byprec[p].empty()) continue;
        if (!group[p]) {
            group[p].reset(make_group(ctx, p, shape[p], std::max(cfg.max_active, 1), max_tiles[p], true, true,
                                          std::min(std::max(cfg.max_active, 1), 32)));
            if (!group[p]) return LGF_ENOMEM;
        }
        std::vector<LatticeBuf*> m;
        for (auto* j : byprec[p]) m.push_back(&j->buf);
        int rc = LGF_OK;
        if (m != members[p]) {
            rc = group[p]->set_members(m);
            if (rc != LGF_OK) return rc;
            members[p] = m;
            measured[p] = {-1};
        }
        auto measure = [&](const std::vector<int>& which) -> int {
            if (which != measured[p]) {
                int e = group[p]->set_measured(which);
                if (e != LGF_OK) return e;
                measured[p] = which;
            }
            {
                std::lock_guard<std::mutex> lk(mu);
                ++n_meas;
            }
            return group[p]->replay_measure();
        };
        // measurements at t0 for newly admitted jobs
        std::vector<int> which;
        for (size_t i = 0; i < byprec[p].size(); ++i) {
            ServeJob* j = byprec[p][i];
            if (j->steps_done == 0 && j->job.flow.measure_at_t0 && j->tvals.empty()) {
                which.push_back((int)i);
                j->tvals.push_back(j->t);
            }
        }
        if (!which.empty()) {
            rc = measure(which);
            if (rc != LGF_OK) return rc;
        }
        const int k = std::max(cfg.steps_per_tick, 1);
        for (int s = 0; s < k; ++s) {
            // members that already reached their step count leave the list
            std::vector<ServeJob*> run;
            for (auto* j : byprec[p])
                if (j->steps_done < j->job.flow.nsteps) run.push_back(j);
            if (run.empty()) break;
            if (run.size() != byprec[p].size()) {
                byprec[p] = run;
                m.clear();
                for (auto* j : run) m.push_back(&j->buf);
                rc = group[p]->set_members(m);
                if (rc != LGF_OK) return rc;
                members[p] = m;
                measured[p] = {-1};
            }
            rc = group[p]->replay_step();
            if (rc != LGF_OK) return rc;
            {
                std::lock_guard<std::mutex> lk(mu);
                ++n_steps;
            }
            which.clear();
            for (size_t i = 0; i < run.size(); ++i) {
                ServeJob* j = run[i];
                j->steps_done++;
                j->t += j->job.flow.eps;  // GradientFlow.cpp:52
                const lgf_flow_opts& o = j->job.flow;
                if (p == LGF_PREC_FP32MIXED && o.reunit_every > 0 && j->steps_done % o.reunit_every == 0) {
                    rc = launch_reunitarize(ctx, j->buf);
                    if (rc != LGF_OK) return rc;
                }
                if (o.meas_every > 0 && j->steps_done % o.meas_every == 0) {
                    which.push_back((int)i);
                    j->tvals.push_back(j->t);
                }
            }
            if (!which.empty()) {
                rc = measure(which);
                if (rc != LGF_OK) return rc;
                for (int i : which)
                    if (run[i]->job.snapshot_prefix) {
                        rc = snapshot(run[i]);
                        if (rc != LGF_OK) return rc;
                    }
            }
        }
    }
    return LGF_OK;
}

// add the device time of completed ticks to busy_s (all of them when wait)
void lgf_server::collect_ticks(bool wait) {
    while (!tick_ev.empty()) {
        TickEv t = tick_ev.front();
        if (wait) cudaEventSynchronize(t.b);
        const cudaError_t q = cudaEventQuery(t.b);
        if (q == cudaErrorNotReady) break;
        if (q != cudaSuccess) cudaGetLastError();
        float ms = 0.f;
        if (q == cudaSuccess && cudaEventElapsedTime(&ms, t.a, t.b) == cudaSuccess) {
            std::lock_guard<std::mutex> lk(mu);
            busy_s += ms * 1e-3;
        }
        tick_ev.pop_front();
        ev_free.push_back(t);
    }
}

void lgf_server::run() {
    cudaSetDevice(ctx->device);
    for (;;) {
        collect_ticks(false);
        std::vector<ServeJob*> admitted;
        {
            std::unique_lock<std::mutex> lk(mu);
            if (active.empty() && staging.empty() && queue.empty() && !stopping)
                cv_work.wait_for(lk, std::chrono::milliseconds(20));
            if (stopping) break;
            // arrival-order admission by HBM footprint, free slots and a free
            // arena block (the head waits for retirements if none fits)
            while (!queue.empty() && (int)(active.size() + staging.size() + admitted.size()) < cfg.max_active &&
                   used + queue.front()->bytes <= cfg.hbm_budget_bytes) {
                ServeJob* j = queue.front();
                j->mem = arena.alloc(j->bytes);
                if (!j->mem) break;
                queue.pop_front();
                used += j->bytes;
                j->st.state = LGF_JOB_RUNNING;
                j->st.start_s = now_s(t0);
                admitted.push_back(j);
            }
        }
        for (auto* j : admitted) {
            int rc = admit(j);
            if (rc != LGF_OK) finish(j, LGF_JOB_FAILED, rc);
            else staging.push_back(j);
        }
        // jobs whose input has arrived join the shared launches; with nothing
        // else to run, wait for the first of them
        if (active.empty() && !staging.empty()) cudaEventSynchronize(staging.front()->ready);
        std::vector<ServeJob*> still;
        for (auto* j : staging) {
            const cudaError_t q = cudaEventQuery(j->ready);
            if (q == cudaSuccess) {
                active.push_back(j);
            } else if (q == cudaErrorNotReady) {
                still.push_back(j);
            } else {
                cudaGetLastError();
                finish(j, LGF_JOB_FAILED, set_error(ctx, LGF_ECUDA, "job input failed: %s", cudaGetErrorString(q)));
            }
        }
        staging.swap(still);
        if (active.empty()) continue;
        TickEv te{nullptr, nullptr};
        if (!ev_free.empty()) {
            te = ev_free.back();
            ev_free.pop_back();
        } else if (cudaEventCreate(&te.a) != cudaSuccess || cudaEventCreate(&te.b) != cudaSuccess) {
            cudaGetLastError();
            te = {nullptr, nullptr};
        }
        if (te.a) cudaEventRecord(te.a, ctx->stream);
        int rc = tick(active);
        if (te.a) {
            cudaEventRecord(te.b, ctx->stream);
            tick_ev.push_back(te);
        }
        {
            std::lock_guard<std::mutex> lk(mu);
            ++n_ticks;
        }
        collect_ticks(false);
        if (rc != LGF_OK) {
            for (auto* j : active) finish(j, LGF_JOB_FAILED, rc);
            active.clear();
            continue;
        }
        std::vector<ServeJob*> keep;
        for (auto* j : active) {
            if (j->steps_done >= j->job.flow.nsteps) {
                int r2 = retire(j);
                wait_snapshot(j);
                if (r2 == LGF_OK) r2 = j->snap_err;  // a snapshot that could not be written fails the job
                finish(j, r2 == LGF_OK ? LGF_JOB_DONE : LGF_JOB_FAILED, r2);
            } else {
                keep.push_back(j);
            }
        }
        active.swap(keep);
    }
    cudaStreamSynchronize(ctx->stream);
    cudaStreamSynchronize(adm);
    collect_ticks(true);
    for (auto& t : ev_free) {
        cudaEventDestroy(t.a);
        cudaEventDestroy(t.b);
    }
    ev_free.clear();
    for (auto* j : staging) finish(j, LGF_JOB_FAILED, LGF_ESHUTDOWN);
    staging.clear();
    for (auto* j : active) finish(j, LGF_JOB_FAILED, LGF_ESHUTDOWN);
    active.clear();
    group[0].reset();
    group[1].reset();
    {
        std::lock_guard<std::mutex> lk(snap_mu);
        snap_stop = true;
        snap_cv.notify_all();
    }
    if (snap_thread.joinable()) snap_thread.join();
}

// Kernel shape (block size, measurement warps per plane) of the shared
// launches of one precision: the defaults.  A shape tuned on one volume
// class is not carried over to every job of a mix: a one-warp-per-plane
// measurement tuned (by under 2%) on 24^3x48 slowed a served mix of four
// volumes by 12%.  Each job's work order is still its own class's tuned
// order (the groups' per-volume lists).
static TileShape serve_shape(const lgf_ctx*, int prec) { return default_shape(prec); }

extern "C" {

int lgf_serve_start(lgf_ctx* ctx, const lgf_serve_config* cfg, lgf_server** out) {
    if (!ctx || !cfg || !out) return LGF_EINVAL;
    *out = nullptr;
    if (cfg->max_active < 1 || cfg->hbm_budget_bytes == 0) return set_error(ctx, LGF_EINVAL, "empty serve budget");
    cudaSetDevice(ctx->device);
    lgf_server* s = new (std::nothrow) lgf_server();
    if (!s) return LGF_ENOMEM;
    s->ctx = ctx;
    s->cfg = *cfg;
    if (s->cfg.steps_per_tick < 1) s->cfg.steps_per_tick = 1;
    s->t0 = std::chrono::steady_clock::now();
    cudaError_t e = s->arena.reserve(cfg->hbm_budget_bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        delete s;
        return set_error(ctx, LGF_ENOMEM, "cannot reserve the %zu-byte serving budget: %s", cfg->hbm_budget_bytes,
                         cudaGetErrorString(e));
    }
    if (cudaStreamCreateWithFlags(&s->adm, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&s->snap_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&s->retired_ev, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        if (s->adm) cudaStreamDestroy(s->adm);
        if (s->snap_stream) cudaStreamDestroy(s->snap_stream);
        delete s;
        return set_error(ctx, LGF_ECUDA, "cannot create the admission streams");
    }
    for (int p = 0; p < 2; ++p) {
        s->shape[p] = serve_shape(ctx, p);  // jobs of every volume share the server's launches
        // the budget bounds the resident sites: every site costs at least its links ring + accumulator
        const size_t per_site = (p == 0 ? 8 : 4) * (3 * 4 * 18 + 4 * 8);
        const long long max_sites = (long long)(cfg->hbm_budget_bytes / per_site) + 1;
        s->max_tiles[p] = (4 * max_sites) / s->shape[p].threads + 2LL * cfg->max_active + 1;
    }
    s->snap_thread = std::thread([s] { s->snap_run(); });
    s->worker = std::thread([s] { s->run(); });
    *out = s;
    return LGF_OK;
}

int lgf_serve_submit(lgf_server* s, const lgf_job* job, uint64_t* id) {
    if (!s || !job || !id) return LGF_EINVAL;
    if (!valid_shape(job->shape) || (job->precision != LGF_PREC_FP64 && job->precision != LGF_PREC_FP32MIXED) ||
        job->flow.nsteps < 0 || job->flow.meas_every < 0 || job->flow.reunit_every < 0 || job->shape[0] > 256)
        return LGF_EINVAL;
    const int nm = count_measurements(job->flow);
    if (nm > 0 && (!job->meas || !job->meas->t || !job->meas->E || !job->meas->Q || job->meas->capacity < nm))
        return LGF_EINVAL;
    auto j = std::make_unique<ServeJob>();
    j->job = *job;
    j->nmeas = nm;
    j->bytes = placed_bytes(job->shape, job->precision, nm);
    if (job->snapshot_prefix) j->bytes += (snapshot_bytes(job->shape) + 255) & ~size_t(255);
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stopping) return LGF_ESHUTDOWN;
    if (j->bytes > s->cfg.hbm_budget_bytes) return LGF_ENOMEM;  // could never be admitted
    j->id = s->next_id++;
    j->st.state = LGF_JOB_QUEUED;
    j->st.submit_s = now_s(s->t0);
    *id = j->id;
    s->queue.push_back(j.get());
    s->jobs[j->id] = std::move(j);
    s->cv_work.notify_all();
    return LGF_OK;
}

int lgf_serve_stats_get(lgf_server* s, lgf_serve_stats* st) {
    if (!s || !st) return LGF_EINVAL;
    std::lock_guard<std::mutex> lk(s->mu);
    st->wall_s = now_s(s->t0);
    st->device_busy_s = s->busy_s;
    st->ticks = s->n_ticks;
    st->steps = s->n_steps;
    st->measurements = s->n_meas;
    st->jobs_done = s->n_done;
    st->snapshots = s->n_snap;
    return LGF_OK;
}

int lgf_serve_poll(lgf_server* s, uint64_t id, lgf_job_status* st) {
    if (!s) return LGF_EINVAL;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->jobs.find(id);
    if (it == s->jobs.end()) return LGF_ENOTFOUND;
    if (st) {
        *st = it->second->st;
        st->steps_done = it->second->steps_done;
    }
    const int state = it->second->st.state;
    return (state == LGF_JOB_DONE || state == LGF_JOB_FAILED) ? LGF_OK : LGF_EBUSY;
}

int lgf_serve_wait(lgf_server* s, uint64_t id, double timeout_s, lgf_job_status* st) {
    if (!s) return LGF_EINVAL;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->jobs.find(id);
    if (it == s->jobs.end()) return LGF_ENOTFOUND;
    ServeJob* j = it->second.get();
    auto done = [&] { return j->st.state == LGF_JOB_DONE || j->st.state == LGF_JOB_FAILED; };
    ++s->waiters;
    const bool ok = s->cv_done.wait_for(lk, std::chrono::duration<double>(std::max(timeout_s, 0.0)), done);
    if (st) {
        *st = j->st;
        st->steps_done = j->steps_done;
    }
    if (--s->waiters == 0) s->cv_idle.notify_all();
    return ok ? LGF_OK : LGF_ETIMEDOUT;
}

int lgf_serve_stop(lgf_server* s) {
    if (!s) return LGF_EINVAL;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stopping = true;
        for (auto* j : s->queue) {
            j->st.state = LGF_JOB_FAILED;
            j->st.error = LGF_ESHUTDOWN;
            j->st.end_s = now_s(s->t0);
        }
        s->queue.clear();
        s->cv_work.notify_all();
    }
    if (s->worker.joinable()) s->worker.join();
    {
        // every job has ended by now; let threads blocked in lgf_serve_wait
        // return before the server is freed
        std::unique_lock<std::mutex> lk(s->mu);
        s->cv_done.notify_all();
        s->cv_idle.wait(lk, [s] { return s->waiters == 0; });
    }
    cudaEventDestroy(s->retired_ev);
    cudaStreamDestroy(s->adm);
    cudaStreamDestroy(s->snap_stream);
    delete s;
    return LGF_OK;
}

}  // extern "C"
