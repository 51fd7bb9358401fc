// Autotuner of the launch shapes and work orders (TileShape) of the RK3 stage
// and measurement kernels, per precision and lattice volume class.
//
// On a lattice of the job's own shape (generated links; the volume decides
// which orders keep the stencil's neighbours in L1/L2), candidates are timed
// with CUDA events on the context's stream (each over at least ~20 ms of
// launches; a candidate must beat the current shape by 2%), one parameter at
// a time:
//   stage:       block size {128, 256, 384},
//                then the tile order {x1 columns per CTA, row blocks through
//                x0}, then (row blocks) the block budget {2, 8, 32 MB};
//   measurement: warps per plane {2, 1}, then the block budget {2, 8, 64 MB}.
// The winner is recorded in the context and used by every later group whose
// largest lattice falls in the same volume class (within a factor of two).
// No candidate changes a result: only block shapes and tile order differ.
#include <cuda_runtime.h>

#include <algorithm>
#include <memory>
#include <vector>

#include "lgf_engine.cuh"

namespace lgf {

namespace {

struct Timer {
    cudaEvent_t a = nullptr, b = nullptr;
    Timer() {
        cudaEventCreate(&a);
        cudaEventCreate(&b);
    }
    ~Timer() {
        cudaEventDestroy(a);
        cudaEventDestroy(b);
    }
};

// mean ms of `reps` launches of kernel k (0..2: RK3 stage k+1 of a step; the
// three together for k = -1; 3: the measurement kernel) under shape t
int time_shape(lgf_ctx* ctx, int prec, LatticeBuf& b, const TileShape& t, int k, int reps, float* ms) {
    const long long tiles = (4LL * b.g.V + t.threads - 1) / t.threads;
    std::unique_ptr<GroupBase> g(make_group(ctx, prec, t, 1, tiles, false));
    if (!g) return ctx->err.empty() ? set_error(ctx, LGF_ENOMEM, "tuning group creation failed") : LGF_ECUDA;
    std::vector<LatticeBuf*> m{&b};
    int rc = g->set_members(m);
    if (rc == LGF_OK && k == 3) rc = g->set_measured({0});
    auto launch = [&]() { return k < 0 ? g->launch_step() : g->launch_one(k); };
    if (rc == LGF_OK) rc = launch();  // warm-up: module load, first touch
    if (rc != LGF_OK) return rc;
    Timer tm;
    LGF_CUDA_TRY(ctx, cudaEventRecord(tm.a, ctx->stream));
    for (int i = 0; i < reps && rc == LGF_OK; ++i) rc = launch();
    LGF_CUDA_TRY(ctx, cudaEventRecord(tm.b, ctx->stream));
    LGF_CUDA_TRY(ctx, cudaEventSynchronize(tm.b));
    if (rc != LGF_OK) return rc;
    float total = 0.f;
    LGF_CUDA_TRY(ctx, cudaEventElapsedTime(&total, tm.a, tm.b));
    *ms = total / reps;
    return LGF_OK;
}

}  // namespace

int tune_shape(lgf_ctx* ctx, int prec, const int shape[4], TileShape* best) {
    LatticeBuf b;
    int rc = buf_alloc(ctx, b, shape, prec, 1);
    if (rc != LGF_OK) return rc;
    rc = launch_generate(ctx, b, 12345, 0.5);
    b.eps = 0.01;
    TileShape cur = default_shape(prec);
    float cur_ms = 0.f;
    const double MB = double(1 << 20);
    // A candidate replaces the current shape only when it is more than 2%
    // faster, each timed over at least ~20 ms of launches: the clock of a
    // power-capped GPU wanders by about that much, and a shape chosen on
    // noise would follow the volume class everywhere.
    const float KEEP = 0.98f, TARGET_MS = 20.f;
    // ---- RK3 stage: one step (three stage launches) per repetition
    float probe = 0.f;
    if (rc == LGF_OK) rc = time_shape(ctx, prec, b, cur, -1, 1, &probe);
    const int reps = std::max(3, std::min(200, (int)(TARGET_MS / std::max(probe, 1e-3f))));
    if (rc == LGF_OK) rc = time_shape(ctx, prec, b, cur, -1, reps, &cur_ms);
    auto try_stage = [&](TileShape t) {
        if (rc != LGF_OK || t == cur) return;
        float ms = 0.f;
        rc = time_shape(ctx, prec, b, t, -1, reps, &ms);
        if (rc == LGF_OK && ms < KEEP * cur_ms) {
            cur = t;
            cur_ms = ms;
        }
    };
    for (int th : {128, 256, 384}) {
        if (th > stage_max_threads(prec)) continue;
        TileShape t = cur;
        t.threads = th;
        try_stage(t);
    }
    {
        TileShape t = cur;
        t.stage_order = 1 - cur.stage_order;
        try_stage(t);
    }
    if (cur.stage_order == 0)
        for (double mb : {2.0, 8.0, 32.0}) {
            TileShape t = cur;
            t.stage_budget = mb * MB;
            try_stage(t);
        }
    // ---- measurement kernel alone, starting from whole-slice blocks (the
    // fewest DRAM bytes: 1.16x the link bytes against 2.05x for 2 MB blocks
    // on 24^3x48); smaller blocks replace them only when 2% faster (on 48^4
    // whole slices no longer fit L2 and are 45% slower)
    cur.meas_budget = 64.0 * MB;
    float meas_ms = 0.f;
    if (rc == LGF_OK) rc = time_shape(ctx, prec, b, cur, 3, 1, &probe);
    const int mreps = std::max(3, std::min(200, (int)(TARGET_MS / std::max(probe, 1e-3f))));
    if (rc == LGF_OK) rc = time_shape(ctx, prec, b, cur, 3, mreps, &meas_ms);
    auto try_meas = [&](TileShape t) {
        if (rc != LGF_OK || t == cur) return;
        float ms = 0.f;
        rc = time_shape(ctx, prec, b, t, 3, mreps, &ms);
        if (rc == LGF_OK && ms < KEEP * meas_ms) {
            cur = t;
            meas_ms = ms;
        }
    };
    {
        TileShape t = cur;
        t.meas_split = 3 - cur.meas_split;
        try_meas(t);
    }
    for (double mb : {8.0, 2.0}) {
        TileShape t = cur;
        t.meas_budget = mb * MB;
        try_meas(t);
    }
    cudaStreamSynchronize(ctx->stream);
    buf_free(b);
    if (rc != LGF_OK) return rc;
    record_tuned(ctx, prec, 1LL * shape[0] * shape[1] * shape[2] * shape[3], cur);
    if (best) *best = cur;
    return LGF_OK;
}

}  // namespace lgf

using namespace lgf;

static void to_abi(const TileShape& t, lgf_tile_shape* o) {
    o->stage_threads = t.threads;
    o->stage_order = t.stage_order;
    o->stage_budget_kb = (int)(t.stage_budget / 1024.0);
    o->meas_budget_kb = (int)(t.meas_budget / 1024.0);
    o->meas_split = t.meas_split;
}

extern "C" {

int lgf_autotune(lgf_ctx* ctx, int precision, const int shape[4], int* best_threads) {
    lgf_tile_shape t;
    int rc = lgf_autotune_tiles(ctx, precision, shape, &t);
    if (rc == LGF_OK && best_threads) *best_threads = t.stage_threads;
    return rc;
}

int lgf_autotune_tiles(lgf_ctx* ctx, int precision, const int shape[4], lgf_tile_shape* best) {
    if (!ctx) return LGF_EINVAL;
    if (precision != LGF_PREC_FP64 && precision != LGF_PREC_FP32MIXED) return LGF_EINVAL;
    if (!valid_shape(shape)) return set_error(ctx, LGF_EINVAL, "autotune shape must be even and >= 4");
    cudaSetDevice(ctx->device);
    TileShape t;
    int rc = tune_shape(ctx, precision, shape, &t);
    if (rc == LGF_OK && best) to_abi(t, best);
    return rc;
}

int lgf_set_tiles(lgf_ctx* ctx, int precision, const int shape[4], const lgf_tile_shape* tiles) {
    if (!ctx || !tiles) return LGF_EINVAL;
    if (precision != LGF_PREC_FP64 && precision != LGF_PREC_FP32MIXED) return LGF_EINVAL;
    if (!valid_shape(shape)) return set_error(ctx, LGF_EINVAL, "lattice extents must be even and >= 4");
    TileShape t;
    t.threads = tiles->stage_threads;
    t.stage_order = tiles->stage_order;
    t.stage_budget = tiles->stage_budget_kb * 1024.0;
    t.meas_budget = tiles->meas_budget_kb * 1024.0;
    t.meas_split = tiles->meas_split;
    if (t.threads < 128 || t.threads % 128 || t.threads > stage_max_threads(precision) ||
        (t.stage_order != 0 && t.stage_order != 1) ||
        tiles->stage_budget_kb < 1 || tiles->meas_budget_kb < 1 || (t.meas_split != 1 && t.meas_split != 2))
        return set_error(ctx, LGF_EINVAL, "invalid tile shape");
    record_tuned(ctx, precision, 1LL * shape[0] * shape[1] * shape[2] * shape[3], t);
    return LGF_OK;
}

int lgf_get_tiles(lgf_ctx* ctx, int precision, const int shape[4], lgf_tile_shape* tiles) {
    if (!ctx || !tiles || !valid_shape(shape)) return LGF_EINVAL;
    to_abi(tuned_shape(ctx, precision, 1LL * shape[0] * shape[1] * shape[2] * shape[3]), tiles);
    return LGF_OK;
}

}  // extern "C"
