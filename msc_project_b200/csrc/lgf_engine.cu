// Engine core: device buffers of a lattice, groups of resident lattices with
// persistent multi-lattice launches and CUDA-graph capture, and the C ABI for
// contexts, lattices, the flow loop, measurements and diagnostics.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "lgf_engine.cuh"

namespace lgf {

int set_error(lgf_ctx* ctx, int code, const char* fmt, ...) {
    if (ctx) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof buf, fmt, ap);
        va_end(ap);
        ctx->err = buf;
    }
    return code;
}

bool valid_shape(const int shape[4]) {
    if (!shape) return false;
    long long v = 1;
    for (int d = 0; d < 4; ++d) {
        if (shape[d] < 4 || (shape[d] % 2) != 0) return false;  // Lattice.cpp:42-49 (even); >= 4 for the 1x3 loops
        v *= shape[d];
    }
    return v * 4 < (1LL << 31) - 1024;  // link-thread indices are int
}

static size_t real_size(int prec) { return prec == LGF_PREC_FP64 ? sizeof(double) : sizeof(float); }

size_t footprint_bytes(const int shape[4], int precision, int meas_slots) {
    const size_t V = (size_t)shape[0] * shape[1] * shape[2] * shape[3], Vp = padded_sites(V);
    const size_t rs = real_size(precision);
    const size_t nchunk = ((size_t)shape[1] * shape[2] * shape[3] + MEAS_SITES - 1) / MEAS_SITES;
    size_t b = 3 * Vp * 4 * 18 * rs;             // link ring
    b += Vp * 4 * 8 * rs;                         // su(3) accumulator
    b += (size_t)shape[0] * nchunk * sizeof(double2) + (size_t)shape[0] * sizeof(double2);
    b += (size_t)std::max(meas_slots, 1) * (2 + 2 * (size_t)shape[0]) * sizeof(double) + 256;
    return b;
}

// Stage block size until the autotuner has run: FP64 256 threads (64 sites x 4
// directions: one block per SM whose eight warps share their neighbours in
// L1; 9% faster per stage than 128 on 24^3x48, 19% per job on 48^4), FP32 128
// (three blocks per SM; 256 is 20% slower).
int default_threads(int precision) { return precision == LGF_PREC_FP64 ? 256 : 128; }

static const lgf_ctx::Tuned* find_tuned(const lgf_ctx* ctx, int precision, long long volume) {
    for (const auto& t : ctx->tuned)
        if (t.prec == precision && volume <= 2 * t.volume && t.volume <= 2 * volume) return &t;
    return nullptr;
}

int stage_threads(const lgf_ctx* ctx, int precision, long long volume) {
    const lgf_ctx::Tuned* t = find_tuned(ctx, precision, volume);
    return t ? t->threads : default_threads(precision);
}

void record_tuned(lgf_ctx* ctx, int precision, long long volume, int threads) {
    for (auto& t : ctx->tuned)
        if (t.prec == precision && t.volume == volume) {
            t.threads = threads;
            return;
        }
    ctx->tuned.push_back({precision, volume, threads});
}

void buf_free(LatticeBuf& b) {
    if (b.U[0]) cudaFree(b.U[0]);  // U[1], U[2] lie in the same allocation
    if (b.A) cudaFree(b.A);
    if (b.partial) cudaFree(b.partial);
    if (b.slice_sums) cudaFree(b.slice_sums);
    if (b.meas) cudaFree(b.meas);
    if (b.slot) cudaFree(b.slot);
    b = LatticeBuf();
}

int buf_alloc(lgf_ctx* ctx, LatticeBuf& b, const int shape[4], int precision, int meas_slots) {
    b = LatticeBuf();
    b.g = make_geom(shape);
    b.prec = precision;
    const size_t Vp = padded_sites((size_t)b.g.V);  // the layout's whole 32-site blocks
    const size_t rs = real_size(precision);
    b.nchunk = (b.g.Vs + MEAS_SITES - 1) / MEAS_SITES;
    cudaError_t e = cudaSuccess;
    // the link ring as one allocation: U1 (FP64) or U1..U2 (FP32) then spans
    // at least V*4*18 doubles, the upload/download staging area
    const size_t ring = Vp * 4 * 18 * rs;
    e = cudaMalloc(&b.U[0], 3 * ring);
    if (e == cudaSuccess) {
        b.U[1] = (char*)b.U[0] + ring;
        b.U[2] = (char*)b.U[0] + 2 * ring;
    }
    if (e == cudaSuccess) e = cudaMalloc(&b.A, Vp * 4 * 8 * rs);
    if (e == cudaSuccess) e = cudaMalloc(&b.partial, (size_t)b.g.n[0] * b.nchunk * sizeof(double2));
    if (e == cudaSuccess) e = cudaMalloc(&b.slice_sums, (size_t)b.g.n[0] * sizeof(double2));
    if (e == cudaSuccess) e = cudaMalloc(&b.slot, sizeof(int));
    if (e == cudaSuccess) {
        b.meas_cap = std::max(meas_slots, 1);
        e = cudaMalloc(&b.meas, (size_t)b.meas_cap * (2 + 2 * (size_t)b.g.n[0]) * sizeof(double));
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        buf_free(b);
        return set_error(ctx, LGF_ENOMEM, "device allocation of a %dx%dx%dx%d lattice (%zu bytes) failed: %s",
                         shape[0], shape[1], shape[2], shape[3], footprint_bytes(shape, precision, meas_slots),
                         cudaGetErrorString(e));
    }
    return LGF_OK;
}

int buf_grow_meas(lgf_ctx* ctx, LatticeBuf& b, int meas_slots) {
    if (meas_slots <= b.meas_cap) return LGF_OK;
    double* m = nullptr;
    cudaError_t e = cudaMalloc(&m, (size_t)meas_slots * (2 + 2 * (size_t)b.g.n[0]) * sizeof(double));
    if (e != cudaSuccess) {
        cudaGetLastError();
        return set_error(ctx, LGF_ENOMEM, "measurement buffer allocation failed: %s", cudaGetErrorString(e));
    }
    cudaFree(b.meas);
    b.meas = m;
    b.meas_cap = meas_slots;
    return LGF_OK;
}

int count_measurements(const lgf_flow_opts& o) {
    int n = o.measure_at_t0 ? 1 : 0;
    if (o.meas_every > 0) n += o.nsteps / o.meas_every;
    return n;
}

// ------------------------------------------------------------ work order
// The persistent kernels take tiles in list order, so the list order sets the
// L2 reuse distance of the stencil.  In plain site order the x0 +- 1 (and, in
// the measurement, up to +- 3) neighbours of a site are reused one slice of
// work later; once a slice of work exceeds the L2 budget they come from HBM
// again.  Large lattices are therefore ordered in blocks of x1 (and x2) rows,
// each block swept through every x0 slice before the next block starts.  Only
// the order changes: the set of tiles is the same, and no result depends on
// it (no reduction runs in tile order).
// Block budgets, measured on 16^4 .. 48^4 (FP64, 100 steps): 8 MB / 2 MB gave
// +5% on 24^3x48 and +7% on 32^4 over the plain site order; 24/8, 12/4, 4/1
// and smaller were between the two.
#ifndef LGF_STAGE_L2_MB
#define LGF_STAGE_L2_MB 8  // MB of stage work per block and slice
#endif
#ifndef LGF_MEAS_L2_MB
#define LGF_MEAS_L2_MB 2  // MB of links read per block and slice (x0 +- 3: 7 slices live)
#endif
static const double STAGE_L2_BUDGET = LGF_STAGE_L2_MB * double(1 << 20);
static const double MEAS_L2_BUDGET = LGF_MEAS_L2_MB * double(1 << 20);

// A block: x1 in [a1, b1), x2 in [a2, b2), all x3.  One block per slice when
// a slice of work fits the budget; else blocks of whole x1 rows, at least
// MIN_ROWS deep so that most x1 neighbours stay inside; else (lattices whose
// x1 rows are themselves large) square (x1, x2) blocks.
struct SiteBlock { int a1, b1, a2, b2; };
#ifndef LGF_MIN_ROWS
#define LGF_MIN_ROWS 4
#endif
static const int MIN_ROWS = LGF_MIN_ROWS;

static std::vector<SiteBlock> site_blocks(const Geom& g, double budget, double bytes_per_site) {
    std::vector<SiteBlock> out;
    const int N1 = g.n[1], N2 = g.n[2], N3 = g.n[3];
    const double sites = budget / bytes_per_site;  // sites of one block and slice
    if ((double)g.Vs <= sites) {
        out.push_back({0, N1, 0, N2});
    } else if ((double)MIN_ROWS * N2 * N3 <= sites) {
        const int r = std::max(1, (int)(sites / ((double)N2 * N3)));
        for (int a = 0; a < N1; a += r) out.push_back({a, std::min(a + r, N1), 0, N2});
    } else {
        const int side = std::max(1, (int)std::sqrt(sites / N3));
        for (int a = 0; a < N1; a += side)
            for (int c = 0; c < N2; c += side) out.push_back({a, std::min(a + side, N1), c, std::min(c + side, N2)});
    }
    return out;
}

// stage tiles of T consecutive sites (first site a multiple of T) of lattice
// i, each assigned to the block row that holds its first site
static void append_stage_tiles(std::vector<int2>& tiles, int i, const Geom& g, int T, double bytes_per_site) {
    const long long N3 = g.n[3], row = (long long)g.n[2] * N3;
    for (const SiteBlock& b : site_blocks(g, STAGE_L2_BUDGET, bytes_per_site))
        for (long long x0 = 0; x0 < g.n[0]; ++x0)
            for (long long x1 = b.a1; x1 < b.b1; ++x1) {
                const long long base = x0 * g.Vs + x1 * row;
                const long long lo = base + b.a2 * N3, hi = base + b.b2 * N3;
                for (long long s0 = (lo + T - 1) / T * T; s0 < hi; s0 += T) tiles.push_back(make_int2(i, (int)s0));
            }
}

#ifndef LGF_STAGE_ORDER
#define LGF_STAGE_ORDER 1  // stage tile order: 0 blocks of x1 rows swept through x0, 1 x1 columns per CTA
#endif
// Column order: a column is the tiles at one (x0, position in the x1 row) for
// x1 = 0..N1-1.  Columns are taken G at a time (G = the persistent grid) and
// listed row by row, so CTA b walks column b along x1: the x1 - 1 neighbours
// of its tile are the links of the tile it did before.  Needs tiles that lie
// inside one x1 row (N2 N3 a multiple of T) and bands of G columns that span
// at least 8 x0 slices (else most x0 neighbours fall on a band edge: 48^4
// with 64-site tiles spans 4); returns false otherwise.  Measured against the
// blocked order: +3-4% flow-only on 24^3x48 and 32^4.
static bool append_stage_tiles_columns(std::vector<int2>& tiles, int i, const Geom& g, int T, int G) {
    const long long row = (long long)g.n[2] * g.n[3];
    if (row % T || G < 1) return false;
    const long long per_row = row / T, ncol = g.n[0] * per_row;
    if (8 * per_row > G && ncol > G) return false;
    for (long long c0 = 0; c0 < ncol; c0 += G) {
        const long long c1 = std::min(c0 + (long long)G, ncol);
        for (long long x1 = 0; x1 < g.n[1]; ++x1)
            for (long long c = c0; c < c1; ++c)
                tiles.push_back(make_int2(i, (int)((c / per_row) * g.Vs + x1 * row + (c % per_row) * T)));
    }
    return true;
}

// measurement tiles (lattice, slice, 32-site chunk of the slice) of lattice i
static void append_measure_tiles(std::vector<int4>& tiles, int i, const Geom& g, double bytes_per_site) {
    const long long N3 = g.n[3], row = (long long)g.n[2] * N3;
    for (const SiteBlock& b : site_blocks(g, MEAS_L2_BUDGET, bytes_per_site))
        for (int t = 0; t < g.n[0]; ++t)
            for (long long x1 = b.a1; x1 < b.b1; ++x1) {
                const long long lo = x1 * row + b.a2 * N3, hi = x1 * row + b.b2 * N3;
                for (long long c = (lo + MEAS_SITES - 1) / MEAS_SITES; c * MEAS_SITES < hi; ++c)
                    tiles.push_back(make_int4(i, t, (int)c, 0));
            }
}

// ------------------------------------------------------------------ groups
template <typename R> class Group : public GroupBase {
public:
    Group(lgf_ctx* ctx, int threads, int max_members, long long max_tiles, bool dynamic)
        : ctx_(ctx), threads_(threads), max_members_(max_members), max_tiles_(max_tiles), dynamic_(dynamic) {}
    ~Group() override {
        if (step_exec_) cudaGraphExecDestroy(step_exec_);
        if (meas_exec_) cudaGraphExecDestroy(meas_exec_);
        cudaFree(d_desc_);
        cudaFree(d_tiles_);
        cudaFree(d_mtiles_);
        cudaFree(d_rtiles_);
        cudaFree(d_jobs_);
        cudaFree(d_counts_);
    }

    int init() {
        LGF_CUDA_TRY(ctx_, cudaMalloc(&d_desc_, sizeof(LatDesc<R>) * max_members_));
        LGF_CUDA_TRY(ctx_, cudaMalloc(&d_tiles_, sizeof(int2) * max_tiles_));
        LGF_CUDA_TRY(ctx_, cudaMalloc(&d_counts_, sizeof(int) * 4));
        LGF_CUDA_TRY(ctx_, cudaMemsetAsync(d_counts_, 0, sizeof(int) * 4, ctx_->stream));
        int nb = 0;
        LGF_CUDA_TRY(ctx_, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_rk3_stage<R, 1>, threads_, 0));
        stage_grid_max_ = std::max(1, nb) * ctx_->sm_count;
        LGF_CUDA_TRY(ctx_, prepare_measure_kernel<R>());
        LGF_CUDA_TRY(ctx_, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_measure<R>, MEAS_SITES * MEAS_WARPS,
                                                                         measure_smem_bytes<R>()));
        meas_grid_max_ = std::max(1, nb) * ctx_->sm_count;
        if (dynamic_) {
            // members change after capture: size the measurement lists for the
            // largest resident set the tile capacity allows (x0 extents <= 256)
            mtiles_cap_ = max_tiles_ * threads_ / (4 * MEAS_SITES) + 256LL * max_members_;
            rtiles_cap_ = 256LL * max_members_;
            jobs_cap_ = max_members_;
            LGF_CUDA_TRY(ctx_, cudaMalloc(&d_mtiles_, sizeof(int4) * mtiles_cap_));
            LGF_CUDA_TRY(ctx_, cudaMalloc(&d_rtiles_, sizeof(int2) * rtiles_cap_));
            LGF_CUDA_TRY(ctx_, cudaMalloc(&d_jobs_, sizeof(int) * jobs_cap_));
        }
        return LGF_OK;
    }

    int set_members(const std::vector<LatticeBuf*>& members) override {
        if ((int)members.size() > max_members_)
            return set_error(ctx_, LGF_EINVAL, "group holds at most %d lattices", max_members_);
        members_ = members;
        h_desc_.resize(members.size());
        std::vector<int2> tiles;
        long long mt = 0;
        for (size_t i = 0; i < members.size(); ++i) {
            const LatticeBuf& b = *members[i];
            LatDesc<R>& d = h_desc_[i];
            d.g = b.g;
            d.U0 = (cplx<R>*)b.U[0];
            d.U1 = (cplx<R>*)b.U[1];
            d.U2 = (cplx<R>*)b.U[2];
            d.A = (R*)b.A;
            d.partial = b.partial;
            d.slice_sums = b.slice_sums;
            d.meas = b.meas;
            d.slot = b.slot;
            d.nchunk = b.nchunk;
            d.eps = (R)b.eps;
            // a tile is threads_/4 consecutive sites with all four link directions;
            // per site a stage reads and writes 4 links and 4 su(3) accumulators
            if (!(LGF_STAGE_ORDER == 1 && append_stage_tiles_columns(tiles, (int)i, b.g, threads_ / 4, stage_grid_max_)))
                append_stage_tiles(tiles, (int)i, b.g, threads_ / 4, 4.0 * (2 * 18 + 8) * sizeof(R));
            mt += (long long)b.g.n[0] * b.nchunk;
        }
        if ((long long)tiles.size() > max_tiles_)
            return set_error(ctx_, LGF_EINVAL, "work list of %zu tiles exceeds the group capacity %lld", tiles.size(),
                             max_tiles_);
        ntiles_ = (int)tiles.size();
        if (!members.empty())
            LGF_CUDA_TRY(ctx_, cudaMemcpyAsync(d_desc_, h_desc_.data(), sizeof(LatDesc<R>) * members.size(),
                                               cudaMemcpyHostToDevice, ctx_->stream));
        if (ntiles_)
            LGF_CUDA_TRY(ctx_, cudaMemcpyAsync(d_tiles_, tiles.data(), sizeof(int2) * tiles.size(),
                                               cudaMemcpyHostToDevice, ctx_->stream));
        h_counts_[0] = ntiles_;
        LGF_CUDA_TRY(ctx_, cudaMemcpyAsync(d_counts_, &h_counts_[0], sizeof(int), cudaMemcpyHostToDevice, ctx_->stream));
        // measurement lists sized for every member at once
        if (mt > mtiles_cap_) {
            cudaFree(d_mtiles_);
            d_mtiles_ = nullptr;
            if (step_exec_ || meas_exec_) return set_error(ctx_, LGF_EINVAL, "measurement list grew after capture");
            LGF_CUDA_TRY(ctx_, cudaMalloc(&d_mtiles_, sizeof(int4) * std::max(mt, 1LL)));
            mtiles_cap_ = mt;
        }
        long long rt = 0;
        for (auto* b : members) rt += b->g.n[0];
        if (rt > rtiles_cap_ || (long long)members.size() > jobs_cap_) {
            if (step_exec_ || meas_exec_) return set_error(ctx_, LGF_EINVAL, "reduction list grew after capture");
            cudaFree(d_rtiles_);
            cudaFree(d_jobs_);
            rtiles_cap_ = std::max(rt, (long long)max_members_ * 64);
            jobs_cap_ = max_members_;
            LGF_CUDA_TRY(ctx_, cudaMalloc(&d_rtiles_, sizeof(int2) * rtiles_cap_));
            LGF_CUDA_TRY(ctx_, cudaMalloc(&d_jobs_, sizeof(int) * jobs_cap_));
        }
        return LGF_OK;
    }

    int set_eps(const std::vector<double>& eps) override {
        for (size_t i = 0; i < h_desc_.size() && i < eps.size(); ++i) h_desc_[i].eps = (R)eps[i];
        if (!h_desc_.empty())
            LGF_CUDA_TRY(ctx_, cudaMemcpyAsync(d_desc_, h_desc_.data(), sizeof(LatDesc<R>) * h_desc_.size(),
                                               cudaMemcpyHostToDevice, ctx_->stream));
        return LGF_OK;
    }

    int set_measured(const std::vector<int>& which) override {
        h_mtiles_.clear();
        h_rtiles_.clear();
        h_jobs_.clear();
        for (int i : which) {
            const LatticeBuf& b = *members_[i];
            append_measure_tiles(h_mtiles_, i, b.g, 4.0 * 18 * sizeof(R));
            for (int t = 0; t < b.g.n[0]; ++t) h_rtiles_.push_back(make_int2(i, t));
            h_jobs_.push_back(i);
        }
        if ((long long)h_mtiles_.size() > mtiles_cap_ || (long long)h_rtiles_.size() > rtiles_cap_ ||
            (long long)h_jobs_.size() > jobs_cap_)
            return set_error(ctx_, LGF_EINVAL, "measurement list exceeds capacity");
        if (!h_mtiles_.empty()) {
            LGF_CUDA_TRY(ctx_, cudaMemcpyAsync(d_mtiles_, h_mtiles_.data(), sizeof(int4) * h_mtiles_.size(),
                                               cudaMemcpyHostToDevice, ctx_->stream));
            LGF_CUDA_TRY(ctx_, cudaMemcpyAsync(d_rtiles_, h_rtiles_.data(), sizeof(int2) * h_rtiles_.size(),
                                               cudaMemcpyHostToDevice, ctx_->stream));
            LGF_CUDA_TRY(ctx_, cudaMemcpyAsync(d_jobs_, h_jobs_.data(), sizeof(int) * h_jobs_.size(),
                                               cudaMemcpyHostToDevice, ctx_->stream));
        }
        h_counts_[1] = (int)h_mtiles_.size();
        h_counts_[2] = (int)h_rtiles_.size();
        h_counts_[3] = (int)h_jobs_.size();
        LGF_CUDA_TRY(ctx_, cudaMemcpyAsync(d_counts_ + 1, &h_counts_[1], 3 * sizeof(int), cudaMemcpyHostToDevice,
                                           ctx_->stream));
        // the host copy must outlive the async copies: wait for them here
        LGF_CUDA_TRY(ctx_, cudaStreamSynchronize(ctx_->stream));
        return LGF_OK;
    }

    int stage_grid() const { return dynamic_ ? stage_grid_max_ : std::max(1, std::min(ntiles_, stage_grid_max_)); }
    int meas_grid() const {
        return dynamic_ ? meas_grid_max_ : std::max(1, std::min((int)std::max<long long>(mtiles_cap_, 1), meas_grid_max_));
    }

    int launch_step() override {
        if (!dynamic_ && ntiles_ == 0) return LGF_OK;
        const int grid = stage_grid();
        {
            NvtxRange r("lgf.rk3_stage1");
            k_rk3_stage<R, 1><<<grid, threads_, 0, ctx_->stream>>>(d_desc_, d_tiles_, d_counts_);
        }
        {
            NvtxRange r("lgf.rk3_stage2");
            k_rk3_stage<R, 2><<<grid, threads_, 0, ctx_->stream>>>(d_desc_, d_tiles_, d_counts_);
        }
        {
            NvtxRange r("lgf.rk3_stage3");
            k_rk3_stage<R, 3><<<grid, threads_, 0, ctx_->stream>>>(d_desc_, d_tiles_, d_counts_);
        }
        LGF_CUDA_TRY(ctx_, cudaGetLastError());
        return LGF_OK;
    }

    // a single kernel: k = 0..2 stage k+1, k = 3 the measurement kernel alone
    int launch_one(int k) override {
        if (k < 3) {
            const int grid = stage_grid();
            if (k == 0) k_rk3_stage<R, 1><<<grid, threads_, 0, ctx_->stream>>>(d_desc_, d_tiles_, d_counts_);
            if (k == 1) k_rk3_stage<R, 2><<<grid, threads_, 0, ctx_->stream>>>(d_desc_, d_tiles_, d_counts_);
            if (k == 2) k_rk3_stage<R, 3><<<grid, threads_, 0, ctx_->stream>>>(d_desc_, d_tiles_, d_counts_);
        } else {
            k_measure<R><<<meas_grid(), dim3(MEAS_SITES, MEAS_WARPS), measure_smem_bytes<R>(), ctx_->stream>>>(
                d_desc_, d_mtiles_, d_counts_ + 1, MeasOut{});
        }
        LGF_CUDA_TRY(ctx_, cudaGetLastError());
        return LGF_OK;
    }

    int launch_measure() override {
        NvtxRange r("lgf.measure_launch");
        const int mg = meas_grid();
        const int rg = dynamic_ ? ctx_->sm_count : std::max(1, (int)std::min<long long>(rtiles_cap_, 4 * ctx_->sm_count));
        const int jg = dynamic_ ? std::min(jobs_cap_, 4 * ctx_->sm_count) : std::max(1, (int)std::min<long long>(jobs_cap_, 4 * ctx_->sm_count));
        k_measure<R><<<mg, dim3(MEAS_SITES, MEAS_WARPS), measure_smem_bytes<R>(), ctx_->stream>>>(
            d_desc_, d_mtiles_, d_counts_ + 1, MeasOut{});
        k_reduce_slices<R><<<rg, RED_THREADS, 0, ctx_->stream>>>(d_desc_, d_rtiles_, d_counts_ + 2);
        k_reduce_total<R><<<std::max(1, jg), RED_THREADS, 0, ctx_->stream>>>(d_desc_, d_jobs_, d_counts_ + 3);
        LGF_CUDA_TRY(ctx_, cudaGetLastError());
        return LGF_OK;
    }

    int capture() override {
        if (step_exec_) {
            cudaGraphExecDestroy(step_exec_);
            step_exec_ = nullptr;
        }
        if (meas_exec_) {
            cudaGraphExecDestroy(meas_exec_);
            meas_exec_ = nullptr;
        }
        int rc = capture_one(true, &step_exec_);
        if (rc != LGF_OK) return rc;
        return capture_one(false, &meas_exec_);
    }
    int replay_step() override {
        NvtxRange r("lgf.rk3_step");
        if (!step_exec_) {
            int rc = capture();
            if (rc != LGF_OK) return rc;
        }
        LGF_CUDA_TRY(ctx_, cudaGraphLaunch(step_exec_, ctx_->stream));
        return LGF_OK;
    }
    int replay_measure() override {
        NvtxRange r("lgf.measure");
        if (!meas_exec_) {
            int rc = capture();
            if (rc != LGF_OK) return rc;
        }
        LGF_CUDA_TRY(ctx_, cudaGraphLaunch(meas_exec_, ctx_->stream));
        return LGF_OK;
    }
    int launches_per_step() const override { return 3; }
    int threads() const override { return threads_; }

private:
    int capture_one(bool step, cudaGraphExec_t* out) {
        cudaGraph_t graph = nullptr;
        LGF_CUDA_TRY(ctx_, cudaStreamBeginCapture(ctx_->stream, cudaStreamCaptureModeThreadLocal));
        int rc = step ? launch_step() : launch_measure();
        cudaError_t e = cudaStreamEndCapture(ctx_->stream, &graph);
        if (rc != LGF_OK) {
            if (graph) cudaGraphDestroy(graph);
            return rc;
        }
        if (e != cudaSuccess) return set_error(ctx_, LGF_ECUDA, "graph capture failed: %s", cudaGetErrorString(e));
        e = cudaGraphInstantiate(out, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) return set_error(ctx_, LGF_ECUDA, "graph instantiate failed: %s", cudaGetErrorString(e));
        return LGF_OK;
    }

    lgf_ctx* ctx_;
    int threads_;
    int max_members_;
    long long max_tiles_;
    bool dynamic_;
    std::vector<LatticeBuf*> members_;
    std::vector<LatDesc<R>> h_desc_;
    std::vector<int4> h_mtiles_;
    std::vector<int2> h_rtiles_;
    std::vector<int> h_jobs_;
    int h_counts_[4] = {0, 0, 0, 0};
    LatDesc<R>* d_desc_ = nullptr;
    int2* d_tiles_ = nullptr;
    int4* d_mtiles_ = nullptr;
    int2* d_rtiles_ = nullptr;
    int* d_jobs_ = nullptr;
    int* d_counts_ = nullptr;  // ntiles, nmtiles, nrtiles, njobs
    long long mtiles_cap_ = 0, rtiles_cap_ = 0;
    int jobs_cap_ = 0;
    int ntiles_ = 0;
    int stage_grid_max_ = 1, meas_grid_max_ = 1;
    cudaGraphExec_t step_exec_ = nullptr, meas_exec_ = nullptr;
};

GroupBase* make_group(lgf_ctx* ctx, int precision, int threads, int max_members, long long max_tiles, bool dynamic) {
    GroupBase* g = nullptr;
    if (precision == LGF_PREC_FP64) {
        auto* p = new (std::nothrow) Group<double>(ctx, threads, max_members, max_tiles, dynamic);
        if (p && p->init() != LGF_OK) { delete p; p = nullptr; }
        g = p;
    } else {
        auto* p = new (std::nothrow) Group<float>(ctx, threads, max_members, max_tiles, dynamic);
        if (p && p->init() != LGF_OK) { delete p; p = nullptr; }
        g = p;
    }
    return g;
}

// ----------------------------------------------------------- link movement
static inline int blocks_for(long long n, int t) { return (int)((n + t - 1) / t); }

// one block per 32-site layout block (the transpose kernels above)
int launch_to_device(lgf_ctx* ctx, LatticeBuf& b, const double* dev_file) {
    const int V = b.g.V;
    const int nb = blocks_for(V, LAYOUT_BLOCK);
    if (b.prec == LGF_PREC_FP64)
        k_to_device<double><<<nb, CONV_THREADS, 0, ctx->stream>>>((const double2*)dev_file, (cplx<double>*)b.U[0], V);
    else
        k_to_device<float><<<nb, CONV_THREADS, 0, ctx->stream>>>((const double2*)dev_file, (cplx<float>*)b.U[0], V);
    LGF_CUDA_TRY(ctx, cudaGetLastError());
    return LGF_OK;
}

int launch_to_file(lgf_ctx* ctx, const LatticeBuf& b, double* dev_file) {
    const int V = b.g.V;
    const int nb = blocks_for(V, LAYOUT_BLOCK);
    if (b.prec == LGF_PREC_FP64)
        k_to_file<double><<<nb, CONV_THREADS, 0, ctx->stream>>>((const cplx<double>*)b.U[0], (double2*)dev_file, V);
    else
        k_to_file<float><<<nb, CONV_THREADS, 0, ctx->stream>>>((const cplx<float>*)b.U[0], (double2*)dev_file, V);
    LGF_CUDA_TRY(ctx, cudaGetLastError());
    return LGF_OK;
}

int launch_generate(lgf_ctx* ctx, LatticeBuf& b, unsigned long long seed, double scale) {
    const int V = b.g.V;
    if (b.prec == LGF_PREC_FP64)
        k_generate_G<double><<<blocks_for(4LL * V, 128), 128, 0, ctx->stream>>>((cplx<double>*)b.U[0], V, seed, scale);
    else
        k_generate_G<float><<<blocks_for(4LL * V, 128), 128, 0, ctx->stream>>>((cplx<float>*)b.U[0], V, seed, scale);
    LGF_CUDA_TRY(ctx, cudaGetLastError());
    return LGF_OK;
}

int launch_reunitarize(lgf_ctx* ctx, LatticeBuf& b) {
    const int V = b.g.V;
    if (b.prec == LGF_PREC_FP64)
        k_reunitarize<double><<<blocks_for(4LL * V, 256), 256, 0, ctx->stream>>>((cplx<double>*)b.U[0], V);
    else
        k_reunitarize<float><<<blocks_for(4LL * V, 256), 256, 0, ctx->stream>>>((cplx<float>*)b.U[0], V);
    LGF_CUDA_TRY(ctx, cudaGetLastError());
    return LGF_OK;
}

// Links cross the PCIe/C2C link as float64 file order; the reorder to the
// device layout (and the float conversion of the mixed form) runs on the GPU.
// The file-order copy is staged in the lattice's own ring: between flows the
// links live in U0 and U1 (FP64) or U1..U2 (FP32) is scratch of at least the
// file size, so an upload or download allocates no device memory.  A
// page-locked caller buffer is one DMA; pageable memory goes through the
// context's two pinned chunks, the host copy of one chunk overlapping the
// DMA of the other.
static const size_t PIN_CHUNK = 32u << 20;

static double* file_staging(const LatticeBuf& b) { return (double*)b.U[1]; }

static bool is_pinned(const void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

static cudaError_t ensure_pinned_chunks(lgf_ctx* ctx) {
    if (ctx->pin[0]) return cudaSuccess;
    cudaError_t e = cudaSuccess;
    for (int k = 0; k < 2 && e == cudaSuccess; ++k) {
        e = cudaMallocHost(&ctx->pin[k], PIN_CHUNK);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->pin_done[k], cudaEventDisableTiming);
    }
    if (e != cudaSuccess) release_pinned_chunks(ctx);
    return e;
}

void release_pinned_chunks(lgf_ctx* ctx) {
    for (int k = 0; k < 2; ++k) {
        if (ctx->pin_done[k]) cudaEventDestroy(ctx->pin_done[k]);
        if (ctx->pin[k]) cudaFreeHost(ctx->pin[k]);
        ctx->pin_done[k] = nullptr;
        ctx->pin[k] = nullptr;
    }
}

int upload_links(lgf_ctx* ctx, LatticeBuf& b, const double* host) {
    const size_t bytes = (size_t)b.g.V * 4 * 18 * sizeof(double);
    char* stage = (char*)file_staging(b);
    cudaError_t e = cudaSuccess;
    if (is_pinned(host)) {
        e = cudaMemcpyAsync(stage, host, bytes, cudaMemcpyHostToDevice, ctx->stream);
    } else {
        std::lock_guard<std::mutex> lk(ctx->pin_mu);
        e = ensure_pinned_chunks(ctx);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return set_error(ctx, LGF_ENOMEM, "pinned staging allocation failed: %s", cudaGetErrorString(e));
        }
        for (size_t off = 0, i = 0; off < bytes && e == cudaSuccess; off += PIN_CHUNK, ++i) {
            const size_t n = std::min(PIN_CHUNK, bytes - off);
            const int k = (int)(i & 1);
            e = cudaEventSynchronize(ctx->pin_done[k]);  // the DMA that last read chunk k has finished
            if (e != cudaSuccess) break;
            std::memcpy(ctx->pin[k], (const char*)host + off, n);
            e = cudaMemcpyAsync(stage + off, ctx->pin[k], n, cudaMemcpyHostToDevice, ctx->stream);
            if (e == cudaSuccess) e = cudaEventRecord(ctx->pin_done[k], ctx->stream);
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);  // chunks free for the next caller
    }
    if (e != cudaSuccess) return set_error(ctx, LGF_ECUDA, "upload failed: %s", cudaGetErrorString(e));
    int rc = launch_to_device(ctx, b, (const double*)stage);
    e = cudaStreamSynchronize(ctx->stream);
    if (rc == LGF_OK && e != cudaSuccess) rc = set_error(ctx, LGF_ECUDA, "upload failed: %s", cudaGetErrorString(e));
    return rc;
}

int download_links(lgf_ctx* ctx, const LatticeBuf& b, double* host) {
    const size_t bytes = (size_t)b.g.V * 4 * 18 * sizeof(double);
    char* stage = (char*)file_staging(b);
    int rc = launch_to_file(ctx, b, (double*)stage);
    if (rc != LGF_OK) return rc;
    cudaError_t e = cudaSuccess;
    if (is_pinned(host)) {
        e = cudaMemcpyAsync(host, stage, bytes, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    } else {
        std::lock_guard<std::mutex> lk(ctx->pin_mu);
        e = ensure_pinned_chunks(ctx);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return set_error(ctx, LGF_ENOMEM, "pinned staging allocation failed: %s", cudaGetErrorString(e));
        }
        // chunk i+1 is copied to the device-side buffer while the host drains chunk i
        const size_t nchunks = (bytes + PIN_CHUNK - 1) / PIN_CHUNK;
        auto issue = [&](size_t i) {
            const size_t off = i * PIN_CHUNK, n = std::min(PIN_CHUNK, bytes - off);
            cudaError_t r = cudaMemcpyAsync(ctx->pin[i & 1], stage + off, n, cudaMemcpyDeviceToHost, ctx->stream);
            return r == cudaSuccess ? cudaEventRecord(ctx->pin_done[i & 1], ctx->stream) : r;
        };
        e = issue(0);
        for (size_t i = 0; i < nchunks && e == cudaSuccess; ++i) {
            if (i + 1 < nchunks) e = issue(i + 1);
            if (e == cudaSuccess) e = cudaEventSynchronize(ctx->pin_done[i & 1]);
            if (e != cudaSuccess) break;
            const size_t off = i * PIN_CHUNK;
            std::memcpy((char*)host + off, ctx->pin[i & 1], std::min(PIN_CHUNK, bytes - off));
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    }
    if (e != cudaSuccess) return set_error(ctx, LGF_ECUDA, "download failed: %s", cudaGetErrorString(e));
    return LGF_OK;
}

}  // namespace lgf

using namespace lgf;


// One measurement-kernel pass over a single lattice with per-site (and,
// when asked, per (site, plane) F / F^) outputs; no reduction.
template <typename R> static int single_lattice_measure(lgf_ctx* ctx, LatticeBuf& b, const MeasOut& out) {
    std::vector<int4> mt;
    for (int t = 0; t < b.g.n[0]; ++t)
        for (int c = 0; c < b.nchunk; ++c) mt.push_back(make_int4(0, t, c, 0));
    const int n = (int)mt.size();
    LatDesc<R> d{};
    d.g = b.g;
    d.U0 = (cplx<R>*)b.U[0];
    d.partial = b.partial;
    d.nchunk = b.nchunk;
    void* ddesc = nullptr;
    int4* dmt = nullptr;
    int* dn = nullptr;
    cudaError_t e = prepare_measure_kernel<R, true>();
    if (e == cudaSuccess) e = cudaMalloc(&ddesc, sizeof d);
    if (e == cudaSuccess) e = cudaMalloc(&dmt, sizeof(int4) * n);
    if (e == cudaSuccess) e = cudaMalloc(&dn, sizeof(int));
    if (e == cudaSuccess) e = cudaMemcpyAsync(ddesc, &d, sizeof d, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dmt, mt.data(), sizeof(int4) * n, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dn, &n, sizeof(int), cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) {
        k_measure<R, true><<<std::min(n, 4 * ctx->sm_count), dim3(MEAS_SITES, MEAS_WARPS), measure_smem_bytes<R, true>(),
                             ctx->stream>>>((const LatDesc<R>*)ddesc, dmt, dn, out);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cudaFree(ddesc);
    cudaFree(dmt);
    cudaFree(dn);
    if (e != cudaSuccess) return set_error(ctx, LGF_ECUDA, "measurement pass failed: %s", cudaGetErrorString(e));
    return LGF_OK;
}

static int single_measure(lgf_ctx* ctx, LatticeBuf& b, const MeasOut& out) {
    return b.prec == LGF_PREC_FP64 ? single_lattice_measure<double>(ctx, b, out)
                                   : single_lattice_measure<float>(ctx, b, out);
}

// =================================================================== C ABI
extern "C" {

int lgf_version(void) { return 10000; }

int lgf_ctx_create(int device, lgf_ctx** out) {
    if (!out) return LGF_EINVAL;
    *out = nullptr;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        cudaGetLastError();
        return LGF_ECUDA;
    }
    if (device < 0 || device >= n) return LGF_EINVAL;
    if (cudaSetDevice(device) != cudaSuccess) return LGF_ECUDA;
    lgf_ctx* ctx = new (std::nothrow) lgf_ctx();
    if (!ctx) return LGF_ENOMEM;
    ctx->device = device;
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) {
        delete ctx;
        return LGF_ECUDA;
    }
    // place lgf_measure_noalloc's fixed scratch now, before the caller's own
    // allocations (modules load lazily otherwise)
    if (noalloc_preload(device) != LGF_OK) {
        cudaStreamDestroy(ctx->stream);
        delete ctx;
        return LGF_ECUDA;
    }
    *out = ctx;
    return LGF_OK;
}

int lgf_ctx_destroy(lgf_ctx* ctx) {
    if (!ctx) return LGF_EINVAL;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    release_pinned_chunks(ctx);
    cudaStreamDestroy(ctx->stream);
    delete ctx;
    return LGF_OK;
}

const char* lgf_last_error(const lgf_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

size_t lgf_lattice_footprint(const int shape[4], int precision) {
    if (!valid_shape(shape) || (precision != LGF_PREC_FP64 && precision != LGF_PREC_FP32MIXED)) return 0;
    return footprint_bytes(shape, precision, 1);
}

int lgf_lattice_create(lgf_ctx* ctx, const int shape[4], int precision, lgf_lattice** out) {
    if (!ctx || !out) return LGF_EINVAL;
    *out = nullptr;
    if (!valid_shape(shape))
        return set_error(ctx, LGF_EINVAL, "lattice extents must be even and >= 4 (Lattice.cpp:42-49)");
    if (precision != LGF_PREC_FP64 && precision != LGF_PREC_FP32MIXED)
        return set_error(ctx, LGF_EINVAL, "unknown precision %d", precision);
    cudaSetDevice(ctx->device);
    lgf_lattice* lat = new (std::nothrow) lgf_lattice();
    if (!lat) return LGF_ENOMEM;
    lat->ctx = ctx;
    int rc = buf_alloc(ctx, lat->buf, shape, precision, 1);
    if (rc != LGF_OK) {
        delete lat;
        return rc;
    }
    *out = lat;
    return LGF_OK;
}

int lgf_lattice_destroy(lgf_lattice* lat) {
    if (!lat) return LGF_EINVAL;
    cudaSetDevice(lat->ctx->device);
    cudaStreamSynchronize(lat->ctx->stream);
    delete lat->group;
    buf_free(lat->buf);
    delete lat;
    return LGF_OK;
}

int lgf_upload_links(lgf_lattice* lat, const double* links) {
    if (!lat || !links) return LGF_EINVAL;
    cudaSetDevice(lat->ctx->device);
    return upload_links(lat->ctx, lat->buf, links);
}

int lgf_download_links(lgf_lattice* lat, double* links) {
    if (!lat || !links) return LGF_EINVAL;
    cudaSetDevice(lat->ctx->device);
    return download_links(lat->ctx, lat->buf, links);
}

int lgf_generate_links(lgf_lattice* lat, uint64_t seed, double scale) {
    if (!lat) return LGF_EINVAL;
    cudaSetDevice(lat->ctx->device);
    int rc = launch_generate(lat->ctx, lat->buf, seed, scale);
    if (rc != LGF_OK) return rc;
    LGF_CUDA_TRY(lat->ctx, cudaStreamSynchronize(lat->ctx->stream));
    return LGF_OK;
}

static int lattice_group(lgf_lattice* lat, GroupBase** out) {
    lgf_ctx* ctx = lat->ctx;
    const int threads = stage_threads(ctx, lat->buf.prec, lat->buf.g.V);
    if (lat->group && lat->group_threads != threads) {
        cudaStreamSynchronize(ctx->stream);
        delete lat->group;
        lat->group = nullptr;
    }
    if (!lat->group) {
        const long long ntiles = (4LL * lat->buf.g.V + threads - 1) / threads;
        lat->group = make_group(ctx, lat->buf.prec, threads, 1, ntiles, false);
        if (!lat->group) return ctx->err.empty() ? set_error(ctx, LGF_ENOMEM, "group creation failed") : LGF_ECUDA;
        lat->group_threads = threads;
        std::vector<LatticeBuf*> m{&lat->buf};
        int rc = lat->group->set_members(m);
        if (rc != LGF_OK) return rc;
        rc = lat->group->set_measured({0});
        if (rc != LGF_OK) return rc;
    }
    *out = lat->group;
    return LGF_OK;
}

static int fetch_meas(lgf_ctx* ctx, const LatticeBuf& b, int nmeas, std::vector<double>& host) {
    const size_t per = 2 + 2 * (size_t)b.g.n[0];
    host.resize(per * std::max(nmeas, 1));
    if (nmeas > 0)
        LGF_CUDA_TRY(ctx, cudaMemcpyAsync(host.data(), b.meas, per * nmeas * sizeof(double), cudaMemcpyDeviceToHost,
                                          ctx->stream));
    LGF_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return LGF_OK;
}

int lgf_flow(lgf_lattice* lat, const lgf_flow_opts* o, lgf_meas* out) {
    if (!lat || !o) return LGF_EINVAL;
    lgf_ctx* ctx = lat->ctx;
    if (o->nsteps < 0 || o->meas_every < 0 || o->reunit_every < 0)
        return set_error(ctx, LGF_EINVAL, "negative step count or interval");
    const int nmeas = count_measurements(*o);
    if (nmeas > 0) {
        if (!out || !out->t || !out->E || !out->Q)
            return set_error(ctx, LGF_EINVAL, "measurements requested but no result arrays given");
        if (out->capacity < nmeas)
            return set_error(ctx, LGF_EINVAL, "result capacity %d < %d measurements", out->capacity, nmeas);
    }
    cudaSetDevice(ctx->device);
    NvtxRange flow_range("lgf.flow");
    const double* meas_before = lat->buf.meas;
    int rc = buf_grow_meas(ctx, lat->buf, nmeas);
    if (rc != LGF_OK) return rc;
    if (lat->group && lat->buf.meas != meas_before) {
        // the measurement buffer moved: refresh the descriptor
        std::vector<LatticeBuf*> m{&lat->buf};
        rc = lat->group->set_members(m);
        if (rc != LGF_OK) return rc;
    }
    GroupBase* grp = nullptr;
    rc = lattice_group(lat, &grp);
    if (rc != LGF_OK) return rc;
    lat->buf.eps = o->eps;
    rc = grp->set_eps({o->eps});
    if (rc != LGF_OK) return rc;
    LGF_CUDA_TRY(ctx, cudaMemsetAsync(lat->buf.slot, 0, sizeof(int), ctx->stream));
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    LGF_CUDA_TRY(ctx, cudaEventCreate(&ev0));
    LGF_CUDA_TRY(ctx, cudaEventCreate(&ev1));
    struct EvGuard {
        cudaEvent_t a, b;
        ~EvGuard() { cudaEventDestroy(a); cudaEventDestroy(b); }
    } evg{ev0, ev1};
    LGF_CUDA_TRY(ctx, cudaEventRecord(ev0, ctx->stream));
    std::vector<double> tvals;
    double t = o->t0;
    if (o->measure_at_t0) {
        rc = grp->replay_measure();
        if (rc != LGF_OK) return rc;
        tvals.push_back(t);
    }
    const bool reunit = lat->buf.prec == LGF_PREC_FP32MIXED && o->reunit_every > 0;
    for (int s = 1; s <= o->nsteps; ++s) {
        rc = grp->replay_step();
        if (rc != LGF_OK) return rc;
        t += o->eps;  // GradientFlow.cpp:52
        if (reunit && s % o->reunit_every == 0) {
            rc = launch_reunitarize(ctx, lat->buf);
            if (rc != LGF_OK) return rc;
        }
        if (o->meas_every > 0 && s % o->meas_every == 0) {
            rc = grp->replay_measure();
            if (rc != LGF_OK) return rc;
            tvals.push_back(t);
        }
    }
    LGF_CUDA_TRY(ctx, cudaEventRecord(ev1, ctx->stream));
    std::vector<double> host;
    rc = fetch_meas(ctx, lat->buf, nmeas, host);
    if (rc != LGF_OK) return rc;
    float flow_ms = 0.f;
    LGF_CUDA_TRY(ctx, cudaEventElapsedTime(&flow_ms, ev0, ev1));
    lat->last_flow_s = flow_ms * 1e-3;
    if (out) {
        const int N0 = lat->buf.g.n[0];
        const size_t per = 2 + 2 * (size_t)N0;
        for (int m = 0; m < nmeas; ++m) {
            out->t[m] = tvals[m];
            out->E[m] = host[m * per + 0];
            out->Q[m] = host[m * per + 1];
            if (out->E_slice) std::memcpy(out->E_slice + (size_t)m * N0, &host[m * per + 2], N0 * sizeof(double));
            if (out->Q_slice) std::memcpy(out->Q_slice + (size_t)m * N0, &host[m * per + 2 + N0], N0 * sizeof(double));
        }
        out->count = nmeas;
    }
    return LGF_OK;
}

int lgf_measure(lgf_lattice* lat, double* E, double* Q, double* E_slice, double* Q_slice) {
    if (!lat) return LGF_EINVAL;
    lgf_flow_opts o{};
    o.eps = lat->buf.eps;
    o.nsteps = 0;
    o.measure_at_t0 = 1;
    double t, e, q;
    lgf_meas m{};
    m.capacity = 1;
    m.t = &t;
    m.E = &e;
    m.Q = &q;
    m.E_slice = E_slice;
    m.Q_slice = Q_slice;
    int rc = lgf_flow(lat, &o, &m);
    if (rc != LGF_OK) return rc;
    if (E) *E = e;
    if (Q) *Q = q;
    return LGF_OK;
}

int lgf_site_densities(lgf_lattice* lat, double* e_site, double* q_site) {
    if (!lat) return LGF_EINVAL;
    lgf_ctx* ctx = lat->ctx;
    cudaSetDevice(ctx->device);
    LatticeBuf& b = lat->buf;
    const size_t V = (size_t)b.g.V;
    double *de = nullptr, *dq = nullptr;
    LGF_CUDA_TRY(ctx, cudaMalloc(&de, V * sizeof(double)));
    cudaError_t e = cudaMalloc(&dq, V * sizeof(double));
    MeasOut mo{};
    mo.e = de;
    mo.q = dq;
    int rc = e == cudaSuccess ? single_measure(ctx, b, mo)
                              : set_error(ctx, LGF_ENOMEM, "site density buffers: %s", cudaGetErrorString(e));
    if (rc == LGF_OK && e_site) e = cudaMemcpy(e_site, de, V * sizeof(double), cudaMemcpyDeviceToHost);
    if (rc == LGF_OK && e == cudaSuccess && q_site) e = cudaMemcpy(q_site, dq, V * sizeof(double), cudaMemcpyDeviceToHost);
    if (rc == LGF_OK && e != cudaSuccess) rc = set_error(ctx, LGF_ECUDA, "site densities copy: %s", cudaGetErrorString(e));
    cudaFree(de);
    cudaFree(dq);
    return rc;
}

int lgf_measure_flowed(lgf_lattice* lat, double* E_improved, double* Q_clover) {
    if (!lat) return LGF_EINVAL;
    lgf_ctx* ctx = lat->ctx;
    cudaSetDevice(ctx->device);
    LatticeBuf& b = lat->buf;
    const size_t V = (size_t)b.g.V;
    double *de = nullptr, *dq = nullptr;
    LGF_CUDA_TRY(ctx, cudaMalloc(&de, V * sizeof(double)));
    cudaError_t e = cudaMalloc(&dq, V * sizeof(double));
    MeasOut mo{};
    mo.e_imp = de;
    mo.q_clov = dq;
    int rc = e == cudaSuccess ? single_measure(ctx, b, mo)
                              : set_error(ctx, LGF_ENOMEM, "density buffers: %s", cudaGetErrorString(e));
    std::vector<double> he(V), hq(V);
    if (rc == LGF_OK) e = cudaMemcpy(he.data(), de, V * sizeof(double), cudaMemcpyDeviceToHost);
    if (rc == LGF_OK && e == cudaSuccess) e = cudaMemcpy(hq.data(), dq, V * sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(de);
    cudaFree(dq);
    if (rc == LGF_OK && e != cudaSuccess) rc = set_error(ctx, LGF_ECUDA, "density copy: %s", cudaGetErrorString(e));
    if (rc != LGF_OK) return rc;
    // fixed-order sums in global site order (ImprovedEnergyDensity.cpp:26, UnImprovedTopologicalCharge.cpp:21)
    double se = 0.0, sq = 0.0;
    for (size_t i = 0; i < V; ++i) {
        se += he[i];
        sq += hq[i];
    }
    const double PI = 3.14159265358979323846;
    if (E_improved) *E_improved = se * (1.0 / (double)V);
    if (Q_clover) *Q_clover = sq * (1.0 / (4.0 * PI * PI));
    return LGF_OK;
}

int lgf_last_flow_seconds(lgf_lattice* lat, double* seconds) {
    if (!lat || !seconds) return LGF_EINVAL;
    *seconds = lat->last_flow_s;
    return LGF_OK;
}

int lgf_profile_kernels(lgf_lattice* lat, double eps, int nrep, double ms[4]) {
    if (!lat || !ms || nrep < 1) return LGF_EINVAL;
    lgf_ctx* ctx = lat->ctx;
    cudaSetDevice(ctx->device);
    GroupBase* grp = nullptr;
    int rc = lattice_group(lat, &grp);
    if (rc != LGF_OK) return rc;
    lat->buf.eps = eps;
    rc = grp->set_eps({eps});
    if (rc != LGF_OK) return rc;
    LGF_CUDA_TRY(ctx, cudaMemsetAsync(lat->buf.slot, 0, sizeof(int), ctx->stream));
    std::vector<cudaEvent_t> ev(2 * 4 * nrep);
    for (auto& e : ev) LGF_CUDA_TRY(ctx, cudaEventCreate(&e));
    double acc[4] = {0, 0, 0, 0};
    cudaError_t err = cudaSuccess;
    for (int r = 0; r < nrep && rc == LGF_OK; ++r) {
        for (int k = 0; k < 4 && rc == LGF_OK; ++k) {
            cudaEventRecord(ev[(r * 4 + k) * 2], ctx->stream);
            rc = grp->launch_one(k);
            cudaEventRecord(ev[(r * 4 + k) * 2 + 1], ctx->stream);
        }
    }
    if (rc == LGF_OK) err = cudaStreamSynchronize(ctx->stream);
    if (rc == LGF_OK && err == cudaSuccess) {
        for (int r = 0; r < nrep; ++r)
            for (int k = 0; k < 4; ++k) {
                float m = 0.f;
                cudaEventElapsedTime(&m, ev[(r * 4 + k) * 2], ev[(r * 4 + k) * 2 + 1]);
                acc[k] += m;
            }
        for (int k = 0; k < 4; ++k) ms[k] = acc[k] / nrep;
    }
    for (auto& e : ev) cudaEventDestroy(e);
    if (rc != LGF_OK) return rc;
    if (err != cudaSuccess) return set_error(ctx, LGF_ECUDA, "profiling failed: %s", cudaGetErrorString(err));
    return LGF_OK;
}

int lgf_unitarity(lgf_lattice* lat, double* max_unit_err, double* max_det_err) {
    if (!lat) return LGF_EINVAL;
    lgf_ctx* ctx = lat->ctx;
    cudaSetDevice(ctx->device);
    const int V = lat->buf.g.V;
    const int nb = blocks_for(4LL * V, 256);
    double2* dp = nullptr;
    LGF_CUDA_TRY(ctx, cudaMalloc(&dp, sizeof(double2) * nb));
    if (lat->buf.prec == LGF_PREC_FP64)
        k_unitarity<double><<<nb, 256, 0, ctx->stream>>>((const cplx<double>*)lat->buf.U[0], V, dp);
    else
        k_unitarity<float><<<nb, 256, 0, ctx->stream>>>((const cplx<float>*)lat->buf.U[0], V, dp);
    std::vector<double2> h(nb);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), dp, sizeof(double2) * nb, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cudaFree(dp);
    if (e != cudaSuccess) return set_error(ctx, LGF_ECUDA, "unitarity check failed: %s", cudaGetErrorString(e));
    double mu = 0.0, md = 0.0;
    for (const auto& v : h) {
        mu = std::max(mu, v.x);
        md = std::max(md, v.y);
    }
    if (max_unit_err) *max_unit_err = mu;
    if (max_det_err) *max_det_err = md;
    return LGF_OK;
}

int lgf_debug_gradient(lgf_lattice* lat, double* Z) {
    if (!lat || !Z) return LGF_EINVAL;
    lgf_ctx* ctx = lat->ctx;
    cudaSetDevice(ctx->device);
    const LatticeBuf& b = lat->buf;
    const size_t bytes = (size_t)b.g.V * 4 * 18 * sizeof(double);
    double2* d = nullptr;
    LGF_CUDA_TRY(ctx, cudaMalloc(&d, bytes));
    if (b.prec == LGF_PREC_FP64)
        k_debug_gradient<double><<<blocks_for(4LL * b.g.V, 128), 128, 0, ctx->stream>>>((const cplx<double>*)b.U[0], b.g, d);
    else
        k_debug_gradient<float><<<blocks_for(4LL * b.g.V, 128), 128, 0, ctx->stream>>>((const cplx<float>*)b.U[0], b.g, d);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(Z, d, bytes, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cudaFree(d);
    if (e != cudaSuccess) return set_error(ctx, LGF_ECUDA, "debug gradient failed: %s", cudaGetErrorString(e));
    return LGF_OK;
}

int lgf_debug_fields(lgf_lattice* lat, double* clover_F, double* improved_F) {
    if (!lat) return LGF_EINVAL;
    lgf_ctx* ctx = lat->ctx;
    cudaSetDevice(ctx->device);
    LatticeBuf& b = lat->buf;
    const size_t bytes = (size_t)b.g.V * 6 * 18 * sizeof(double);
    double2 *dc = nullptr, *di = nullptr;
    LGF_CUDA_TRY(ctx, cudaMalloc(&dc, bytes));
    cudaError_t e = cudaMalloc(&di, bytes);
    MeasOut mo{};
    mo.dbg_clover = dc;
    mo.dbg_improved = di;
    int rc = e == cudaSuccess ? single_measure(ctx, b, mo)
                              : set_error(ctx, LGF_ENOMEM, "debug field buffers: %s", cudaGetErrorString(e));
    if (rc == LGF_OK && clover_F) e = cudaMemcpy(clover_F, dc, bytes, cudaMemcpyDeviceToHost);
    if (rc == LGF_OK && e == cudaSuccess && improved_F) e = cudaMemcpy(improved_F, di, bytes, cudaMemcpyDeviceToHost);
    if (rc == LGF_OK && e != cudaSuccess) rc = set_error(ctx, LGF_ECUDA, "debug fields copy: %s", cudaGetErrorString(e));
    cudaFree(dc);
    cudaFree(di);
    return rc;
}

int lgf_exp_su3(lgf_ctx* ctx, int precision, const double* iP, double* out, long long n) {
    if (!ctx || !iP || !out || n < 0 || n > (1LL << 28)) return LGF_EINVAL;
    if (precision != LGF_PREC_FP64 && precision != LGF_PREC_FP32MIXED) return LGF_EINVAL;
    if (n == 0) return LGF_OK;
    cudaSetDevice(ctx->device);
    const size_t bytes = (size_t)n * 18 * sizeof(double);
    double2 *di = nullptr, *dout = nullptr;
    LGF_CUDA_TRY(ctx, cudaMalloc(&di, bytes));
    cudaError_t e = cudaMalloc(&dout, bytes);
    if (e == cudaSuccess) e = cudaMemcpyAsync(di, iP, bytes, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) {
        if (precision == LGF_PREC_FP64)
            k_debug_exp<double><<<blocks_for(n, 128), 128, 0, ctx->stream>>>(di, dout, (int)n);
        else
            k_debug_exp<float><<<blocks_for(n, 128), 128, 0, ctx->stream>>>(di, dout, (int)n);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, dout, bytes, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cudaFree(di);
    cudaFree(dout);
    if (e != cudaSuccess) return set_error(ctx, LGF_ECUDA, "exp failed: %s", cudaGetErrorString(e));
    return LGF_OK;
}

}  // extern "C"
