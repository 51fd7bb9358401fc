// Batched flow of many configurations of uneven volumes, and the autotuner.
//
// Jobs of one precision are packed, smallest first, into waves whose working
// set of one RK3 stage (input and output link buffers plus the su(3)
// accumulator) fits in the 126 MB L2 (budget 96 MB).  A wave is one group:
// every RK3 stage of all its jobs is a single persistent launch over the
// wave's shared tile list, one RK3 step (three stage launches) is captured
// once as a CUDA graph and replayed, and jobs that finish early leave the
// work list (the graph reads the list and its length from device memory, so
// it is not re-captured).  Waves run one after another, so a wave's links stay
// in L2 from one stage to the next; a job too large for any wave forms a wave
// of its own (it fills the GPU alone).  Each job's arithmetic is exactly what
// lgf_flow does for it alone.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <new>
#include <vector>

#include "lgf_engine.cuh"

using namespace lgf;

namespace {

struct JobRun {
    lgf_job* job;
    LatticeBuf buf;
    int nmeas = 0;
    std::vector<double> tvals;
    double t = 0.0;
};

int validate_job(lgf_ctx* ctx, const lgf_job& j) {
    if (!valid_shape(j.shape)) return set_error(ctx, LGF_EINVAL, "job lattice extents must be even and >= 4");
    if (j.precision != LGF_PREC_FP64 && j.precision != LGF_PREC_FP32MIXED)
        return set_error(ctx, LGF_EINVAL, "unknown precision %d", j.precision);
    if (j.flow.nsteps < 0 || j.flow.meas_every < 0 || j.flow.reunit_every < 0)
        return set_error(ctx, LGF_EINVAL, "negative step count or interval");
    const int nm = count_measurements(j.flow);
    if (nm > 0 && (!j.meas || !j.meas->t || !j.meas->E || !j.meas->Q || j.meas->capacity < nm))
        return set_error(ctx, LGF_EINVAL, "job result arrays missing or capacity < %d", nm);
    return LGF_OK;
}

// tile shape for a wave whose largest lattice has this shape: tuned once per
// precision and volume class (a small lattice prefers more, smaller blocks)
TileShape shape_for(lgf_ctx* ctx, int prec, const int shape[4]) {
    const long long V = 1LL * shape[0] * shape[1] * shape[2] * shape[3];
    if (has_tuned(ctx, prec, V)) return tuned_shape(ctx, prec, V);
    TileShape best = default_shape(prec);
    if (tune_shape(ctx, prec, shape, &best) != LGF_OK) {
        ctx->err.clear();
        return default_shape(prec);
    }
    return best;
}

int fetch_results(lgf_ctx* ctx, JobRun& r) {
    lgf_job& j = *r.job;
    if (r.nmeas > 0 && j.meas) {
        const int N0 = r.buf.g.n[0];
        const size_t per = 2 + 2 * (size_t)N0;
        std::vector<double> h(per * r.nmeas);
        LGF_CUDA_TRY(ctx, cudaMemcpyAsync(h.data(), r.buf.meas, h.size() * sizeof(double), cudaMemcpyDeviceToHost,
                                          ctx->stream));
        LGF_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
        for (int m = 0; m < r.nmeas; ++m) {
            j.meas->t[m] = r.tvals[m];
            j.meas->E[m] = h[m * per];
            j.meas->Q[m] = h[m * per + 1];
            if (j.meas->E_slice) std::memcpy(j.meas->E_slice + (size_t)m * N0, &h[m * per + 2], N0 * sizeof(double));
            if (j.meas->Q_slice) std::memcpy(j.meas->Q_slice + (size_t)m * N0, &h[m * per + 2 + N0], N0 * sizeof(double));
        }
        j.meas->count = r.nmeas;
    } else if (j.meas) {
        j.meas->count = 0;
    }
    if (j.links_out) return download_links(ctx, r.buf, j.links_out);
    return LGF_OK;
}

// Flow one wave of jobs (same precision) in lockstep on the precision's group
// (dynamic: the wave becomes its member set and the captured graphs stay
// valid); adds the kernel launches issued to *launches.
int run_wave(lgf_ctx* ctx, int prec, std::vector<JobRun*>& runs, GroupBase* grp, int* launches) {
    std::vector<LatticeBuf*> members;
    std::vector<double> eps;
    for (auto* r : runs) {
        members.push_back(&r->buf);
        eps.push_back(r->job->flow.eps);
        r->buf.eps = r->job->flow.eps;
        LGF_CUDA_TRY(ctx, cudaMemsetAsync(r->buf.slot, 0, sizeof(int), ctx->stream));
        r->t = r->job->flow.t0;
    }
    int rc = grp->set_members(members);
    if (rc != LGF_OK) return rc;
    int maxsteps = 0;
    for (auto* r : runs) maxsteps = std::max(maxsteps, r->job->flow.nsteps);

    std::vector<int> last_measured{-1};
    auto measure = [&](const std::vector<int>& which) -> int {
        if (which.empty()) return LGF_OK;
        if (which != last_measured) {
            int e = grp->set_measured(which);
            if (e != LGF_OK) return e;
            last_measured = which;
        }
        *launches += 3;
        return grp->replay_measure();
    };
    // t0 measurements
    {
        std::vector<int> which;
        for (size_t i = 0; i < runs.size(); ++i)
            if (runs[i]->job->flow.measure_at_t0) {
                which.push_back((int)i);
                runs[i]->tvals.push_back(runs[i]->t);
            }
        rc = measure(which);
        if (rc != LGF_OK) return rc;
    }
    std::vector<JobRun*> active = runs;
    for (int s = 1; s <= maxsteps; ++s) {
        // jobs whose step count is reached leave the work list
        std::vector<JobRun*> still;
        for (auto* r : active)
            if (r->job->flow.nsteps >= s) still.push_back(r);
        if (still.size() != active.size()) {
            active = still;
            members.clear();
            for (auto* r : active) members.push_back(&r->buf);
            rc = grp->set_members(members);
            if (rc != LGF_OK) return rc;
            last_measured = {-1};
        }
        if (active.empty()) break;
        rc = grp->replay_step();
        if (rc != LGF_OK) return rc;
        *launches += grp->launches_per_step();
        std::vector<int> which;
        for (size_t i = 0; i < active.size(); ++i) {
            JobRun* r = active[i];
            r->t += r->job->flow.eps;  // GradientFlow.cpp:52
            const lgf_flow_opts& o = r->job->flow;
            if (prec == LGF_PREC_FP32MIXED && o.reunit_every > 0 && s % o.reunit_every == 0) {
                rc = launch_reunitarize(ctx, r->buf);
                if (rc != LGF_OK) return rc;
                *launches += 1;
            }
            if (o.meas_every > 0 && s % o.meas_every == 0) {
                which.push_back((int)i);
                r->tvals.push_back(r->t);
            }
        }
        rc = measure(which);
        if (rc != LGF_OK) return rc;
    }
    return LGF_OK;
}

// L2-sized waves: jobs sorted by volume, packed greedily while the wave's
// per-stage working set fits the budget; order inside a wave is the input order.
#ifndef LGF_BATCH_WAVE_MB
#define LGF_BATCH_WAVE_MB 96  // 0: every job of a precision in one wave
#endif
const size_t L2_WAVE_BYTES = (size_t)LGF_BATCH_WAVE_MB << 20;

std::vector<std::vector<JobRun*>> l2_waves(const std::vector<JobRun*>& jobs, int prec) {
    const size_t rs = prec == LGF_PREC_FP64 ? 8 : 4;
    auto stage_bytes = [&](const JobRun* r) { return (size_t)r->buf.g.V * 4 * (2 * 18 + 8) * rs; };
    std::vector<JobRun*> order = jobs;
    std::stable_sort(order.begin(), order.end(), [](const JobRun* a, const JobRun* b) { return a->buf.g.V < b->buf.g.V; });
    std::vector<std::vector<JobRun*>> waves;
    size_t cur = 0;
    for (JobRun* r : order) {
        const size_t b = stage_bytes(r);
        if (waves.empty() || (L2_WAVE_BYTES > 0 && cur + b > L2_WAVE_BYTES)) {
            waves.emplace_back();
            cur = 0;
        }
        waves.back().push_back(r);
        cur += b;
    }
    return waves;
}

}  // namespace

extern "C" {

int lgf_batch_run(lgf_ctx* ctx, lgf_job* jobs, int njobs, lgf_batch_stats* stats) {
    if (!ctx || (!jobs && njobs > 0) || njobs < 0) return LGF_EINVAL;
    cudaSetDevice(ctx->device);
    for (int i = 0; i < njobs; ++i) {
        int rc = validate_job(ctx, jobs[i]);
        if (rc != LGF_OK) return rc;
    }
    std::vector<std::unique_ptr<JobRun>> runs;
    auto cleanup = [&]() {
        cudaStreamSynchronize(ctx->stream);
        for (auto& r : runs) buf_free(r->buf);
    };
    double site_steps = 0.0;
    for (int i = 0; i < njobs; ++i) {
        auto r = std::make_unique<JobRun>();
        r->job = &jobs[i];
        r->nmeas = count_measurements(jobs[i].flow);
        int rc = buf_alloc(ctx, r->buf, jobs[i].shape, jobs[i].precision, r->nmeas);
        if (rc == LGF_OK)
            rc = jobs[i].links ? upload_links(ctx, r->buf, jobs[i].links)
                               : launch_generate(ctx, r->buf, jobs[i].seed, jobs[i].gen_scale);
        runs.push_back(std::move(r));
        if (rc != LGF_OK) {
            cleanup();
            return rc;
        }
        site_steps += (double)runs.back()->buf.g.V * jobs[i].flow.nsteps;
    }
    // group the jobs by precision and pick each group's block size (autotuned
    // once per context, before the timed region)
    std::vector<JobRun*> groups[2];
    TileShape shapes[2];
    for (int prec = 0; prec < 2; ++prec) {
        int big[4] = {4, 4, 4, 4};
        long long bigV = 0;
        for (auto& r : runs)
            if (r->job->precision == prec) {
                groups[prec].push_back(r.get());
                if ((long long)r->buf.g.V > bigV) {
                    bigV = r->buf.g.V;
                    std::memcpy(big, r->job->shape, sizeof big);
                }
            }
        if (!groups[prec].empty()) shapes[prec] = shape_for(ctx, prec, big);
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int launches = 0, rc = LGF_OK, threads_used = 0;
    cudaEventRecord(e0, ctx->stream);
    for (int prec = 0; prec < 2 && rc == LGF_OK; ++prec) {
        if (groups[prec].empty()) continue;
        threads_used = shapes[prec].threads;
        // one group for every wave of this precision, sized for the largest:
        // a wave replaces the previous one's members without a new group, a
        // new capture or a device synchronisation in between
        const auto waves = l2_waves(groups[prec], prec);
        long long max_tiles = 1;
        int max_members = 1;
        for (const auto& wave : waves) {
            long long t = 0;
            for (auto* r : wave) t += (4LL * r->buf.g.V + shapes[prec].threads - 1) / shapes[prec].threads;
            max_tiles = std::max(max_tiles, t);
            max_members = std::max(max_members, (int)wave.size());
        }
        std::unique_ptr<GroupBase> grp(make_group(ctx, prec, shapes[prec], max_members, max_tiles, true, true,
                                                  std::min(max_members, 32)));
        if (!grp) {
            rc = ctx->err.empty() ? set_error(ctx, LGF_ENOMEM, "group creation failed") : LGF_ECUDA;
            break;
        }
        for (auto wave : waves) {
            rc = run_wave(ctx, prec, wave, grp.get(), &launches);
            if (rc != LGF_OK) break;
        }
    }
    cudaEventRecord(e1, ctx->stream);
    cudaError_t e = cudaEventSynchronize(e1);
    float ms = 0.f;
    if (e == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc == LGF_OK && e != cudaSuccess) rc = set_error(ctx, LGF_ECUDA, "batch failed: %s", cudaGetErrorString(e));
    for (auto& r : runs) {
        if (rc != LGF_OK) break;
        rc = fetch_results(ctx, *r);
    }
    if (stats) {
        stats->seconds = ms * 1e-3;
        stats->site_steps = site_steps;
        stats->launches = launches;
        stats->block_threads = threads_used;
    }
    cleanup();
    return rc;
}

}  // extern "C"
