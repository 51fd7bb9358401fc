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
#include <type_traits>
#include <vector>

#include "lgf_engine.cuh"
#include "lgf_tiles.h"

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
#ifndef LGF_FP64_THREADS
#define LGF_FP64_THREADS 384
#endif
#ifndef LGF_FP32_THREADS
#define LGF_FP32_THREADS 128
#endif
int default_threads(int precision) { return precision == LGF_PREC_FP64 ? LGF_FP64_THREADS : LGF_FP32_THREADS; }

int stage_max_threads(int precision) { return precision == LGF_PREC_FP64 ? LGF_STAGE_MAXT_D : LGF_STAGE_MAXT_F; }

TileShape default_shape(int precision) {
    TileShape t;
    t.threads = default_threads(precision);
    return t;
}

static const lgf_ctx::Tuned* find_tuned(const lgf_ctx* ctx, int precision, long long volume) {
    const lgf_ctx::Tuned* best = nullptr;
    for (const auto& t : ctx->tuned)
        if (t.prec == precision && volume <= 2 * t.volume && t.volume <= 2 * volume)
            if (!best || std::llabs(t.volume - volume) < std::llabs(best->volume - volume)) best = &t;
    return best;
}

TileShape tuned_shape(const lgf_ctx* ctx, int precision, long long volume) {
    const lgf_ctx::Tuned* t = find_tuned(ctx, precision, volume);
    return t ? t->shape : default_shape(precision);
}

bool has_tuned(const lgf_ctx* ctx, int precision, long long volume) { return find_tuned(ctx, precision, volume) != nullptr; }

void record_tuned(lgf_ctx* ctx, int precision, long long volume, const TileShape& shape) {
    for (auto& t : ctx->tuned)
        if (t.prec == precision && t.volume == volume) {
            t.shape = shape;
            return;
        }
    ctx->tuned.push_back({precision, volume, shape});
}

void buf_free(LatticeBuf& b) {
    if (b.placed) {  // the memory belongs to the caller (a server's arena)
        b = LatticeBuf();
        return;
    }
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

// The same buffers laid out inside one block of caller memory, each part
// starting on a 256-byte boundary (placed_bytes gives the block's size).
static inline size_t align256(size_t n) { return (n + 255) & ~size_t(255); }

size_t placed_bytes(const int shape[4], int precision, int meas_slots) {
    const size_t V = (size_t)shape[0] * shape[1] * shape[2] * shape[3], Vp = padded_sites(V);
    const size_t rs = real_size(precision);
    const size_t nchunk = ((size_t)shape[1] * shape[2] * shape[3] + MEAS_SITES - 1) / MEAS_SITES;
    return align256(3 * Vp * 4 * 18 * rs) + align256(Vp * 4 * 8 * rs) +
           align256((size_t)shape[0] * nchunk * sizeof(double2)) + align256((size_t)shape[0] * sizeof(double2)) +
           align256(sizeof(int)) + align256((size_t)std::max(meas_slots, 1) * (2 + 2 * (size_t)shape[0]) * sizeof(double));
}

void buf_place(LatticeBuf& b, const int shape[4], int precision, int meas_slots, void* mem) {
    b = LatticeBuf();
    b.g = make_geom(shape);
    b.prec = precision;
    b.placed = true;
    const size_t Vp = padded_sites((size_t)b.g.V), rs = real_size(precision);
    b.nchunk = (b.g.Vs + MEAS_SITES - 1) / MEAS_SITES;
    char* p = (char*)mem;
    const size_t ring = Vp * 4 * 18 * rs;
    b.U[0] = p;
    b.U[1] = p + ring;
    b.U[2] = p + 2 * ring;
    p += align256(3 * ring);
    b.A = p;
    p += align256(Vp * 4 * 8 * rs);
    b.partial = (double2*)p;
    p += align256((size_t)b.g.n[0] * b.nchunk * sizeof(double2));
    b.slice_sums = (double2*)p;
    p += align256((size_t)b.g.n[0] * sizeof(double2));
    b.slot = (int*)p;
    p += align256(sizeof(int));
    b.meas_cap = std::max(meas_slots, 1);
    b.meas = (double*)p;
}

int buf_grow_meas(lgf_ctx* ctx, LatticeBuf& b, int meas_slots) {
    if (meas_slots <= b.meas_cap) return LGF_OK;
    if (b.placed) return set_error(ctx, LGF_EINVAL, "a placed lattice holds %d measurement slots", b.meas_cap);
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

// The measurement lists of a subset of a group's members, assembled on the
// device from the per-member segments of the group's full measurement tile
// list (built once per change of members), so that choosing which members a
// measurement covers is one small copy and this launch, with no host wait.
//   sel = [nsel, total tiles, total slices, 0,
//          the launch segments (first tile, tiles) of the measurement kernel,
//          one pair per launch slot (read by k_measure itself),
//          then per selected member k: member, segment offset, tiles, first
//          output tile, N0, first output slice]
// Outputs: mtiles (the selected segments back to back), rtiles (member, t)
// for t < N0, jobs[k] = member, counts = {tiles, slices, nsel}.  Grid
// (max(nsel, 1), any): block (k, y) copies a share of segment k.
constexpr int SEL_HEADER = 4, SEL_FIELDS = 6;
__global__ void __launch_bounds__(256) k_select_measure(const int* __restrict__ sel, int fields,
                                                        const int4* __restrict__ all, int4* __restrict__ mtiles,
                                                        int2* __restrict__ rtiles, int* __restrict__ jobs,
                                                        int* __restrict__ counts) {
    const int nsel = sel[0];
    if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) {
        counts[0] = sel[1];
        counts[1] = sel[2];
        counts[2] = nsel;
    }
    const int k = blockIdx.x;
    if (k >= nsel) return;
    const int* f = sel + fields + SEL_FIELDS * k;
    const int member = f[0], off = f[1], n = f[2], mstart = f[3], n0 = f[4], rstart = f[5];
    for (int i = blockIdx.y * blockDim.x + threadIdx.x; i < n; i += gridDim.y * blockDim.x)
        mtiles[mstart + i] = all[off + i];
    if (blockIdx.y == 0) {
        for (int t = threadIdx.x; t < n0; t += blockDim.x) rtiles[rstart + t] = make_int2(member, t);
        if (threadIdx.x == 0) jobs[k] = member;
    }
}

static inline size_t align16(size_t n) { return (n + 15) & ~size_t(15); }


// ------------------------------------------------------------------ groups
template <typename R> class Group : public GroupBase {
public:
    Group(lgf_ctx* ctx, const TileShape& shape, int max_members, long long max_tiles, bool dynamic, bool per_volume,
          int slots)
        : ctx_(ctx), shape_(shape), threads_(shape.threads), max_members_(max_members), max_tiles_(max_tiles),
          dynamic_(dynamic), per_volume_(per_volume), slots_(std::max(1, std::min(slots, max_members))),
          step_execs_(slots_ + 1, nullptr), meas_execs_(slots_ + 1, nullptr) {}
    ~Group() override {
        cudaStreamSynchronize(ctx_->stream);  // the lists are in use until then
        drop_graphs();
        cudaFree(d_desc_);
        cudaFree(d_tiles_);
        cudaFree(d_mtiles_);
        cudaFree(d_all_mtiles_);
        cudaFree(d_rtiles_);
        cudaFree(d_jobs_);
        cudaFree(d_counts_);
        cudaFree(d_seg_);
        cudaFree(d_sel_);
    }

    int init() {
        LGF_CUDA_TRY(ctx_, cudaMalloc(&d_desc_, sizeof(LatDesc<R>) * max_members_));
        LGF_CUDA_TRY(ctx_, cudaMalloc(&d_tiles_, sizeof(int2) * max_tiles_));
        LGF_CUDA_TRY(ctx_, cudaMalloc(&d_counts_, sizeof(int) * 4));
        LGF_CUDA_TRY(ctx_, cudaMalloc(&d_seg_, sizeof(int2) * slots_));
        LGF_CUDA_TRY(ctx_, cudaMalloc(&d_sel_, sizeof(int) * sel_ints(max_members_)));
        LGF_CUDA_TRY(ctx_, cudaMemsetAsync(d_counts_, 0, sizeof(int) * 4, ctx_->stream));
        LGF_CUDA_TRY(ctx_, cudaMemsetAsync(d_seg_, 0, sizeof(int2) * slots_, ctx_->stream));
        LGF_CUDA_TRY(ctx_, cudaMemsetAsync(d_sel_, 0, sizeof(int) * sel_ints(max_members_), ctx_->stream));
        int nb = 0;
        LGF_CUDA_TRY(ctx_, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_rk3_stage<R, 1>, threads_, 0));
        stage_grid_max_ = std::max(1, nb) * ctx_->sm_count;
        if (shape_.meas_split == 2) {
            LGF_CUDA_TRY(ctx_, (prepare_measure_kernel<R, false, 2>()));
            LGF_CUDA_TRY(ctx_, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_measure<R, false, 2>,
                                                                             MEAS_SITES * 12, measure_smem_bytes<R>()));
        } else {
            LGF_CUDA_TRY(ctx_, (prepare_measure_kernel<R, false, 1>()));
            LGF_CUDA_TRY(ctx_, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_measure<R, false, 1>,
                                                                             MEAS_SITES * 6, measure_smem_bytes<R>()));
        }
        meas_grid_max_ = std::max(1, nb) * ctx_->sm_count;
        if (dynamic_) {
            // members change after capture: size the measurement lists for the
            // largest resident set the tile capacity allows (x0 extents <= 256)
            mtiles_cap_ = max_tiles_ * threads_ / (4 * MEAS_SITES) + 256LL * max_members_;
            rtiles_cap_ = 256LL * max_members_;
            jobs_cap_ = max_members_;
            LGF_CUDA_TRY(ctx_, cudaMalloc(&d_mtiles_, sizeof(int4) * mtiles_cap_));
            LGF_CUDA_TRY(ctx_, cudaMalloc(&d_all_mtiles_, sizeof(int4) * mtiles_cap_));
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
        std::vector<int4> mtiles;
        seg_off_.assign(members.size(), 0);
        seg_len_.assign(members.size(), 0);
        std::vector<int> stage_len(members.size(), 0);
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
            const TileShape ls = list_shape(b.g.V);
            const size_t t0 = tiles.size();
            if (!(ls.stage_order == 1 && append_stage_tiles_columns(tiles, (int)i, b.g, threads_ / 4, stage_grid_max_)))
                append_stage_tiles(tiles, (int)i, b.g, threads_ / 4, ls.stage_budget, 4.0 * (2 * 18 + 8) * sizeof(R));
            stage_len[i] = (int)(tiles.size() - t0);
            // this member's segment of the measurement list
            seg_off_[i] = (int)mtiles.size();
            append_measure_tiles(mtiles, (int)i, b.g, ls.meas_budget, 4.0 * 18 * sizeof(R));
            seg_len_[i] = (int)mtiles.size() - seg_off_[i];
        }
        if ((long long)tiles.size() > max_tiles_)
            return set_error(ctx_, LGF_EINVAL, "work list of %zu tiles exceeds the group capacity %lld", tiles.size(),
                             max_tiles_);
        const long long mt = (long long)mtiles.size();
        if (mt > mtiles_cap_) {
            if (captured()) return set_error(ctx_, LGF_EINVAL, "measurement list grew after capture");
            LGF_CUDA_TRY(ctx_, cudaStreamSynchronize(ctx_->stream));
            cudaFree(d_mtiles_);
            cudaFree(d_all_mtiles_);
            d_mtiles_ = d_all_mtiles_ = nullptr;
            LGF_CUDA_TRY(ctx_, cudaMalloc(&d_mtiles_, sizeof(int4) * std::max(mt, 1LL)));
            LGF_CUDA_TRY(ctx_, cudaMalloc(&d_all_mtiles_, sizeof(int4) * std::max(mt, 1LL)));
            mtiles_cap_ = mt;
        }
        long long rt = 0;
        for (auto* b : members) rt += b->g.n[0];
        if (rt > rtiles_cap_ || (long long)members.size() > jobs_cap_) {
            if (captured()) return set_error(ctx_, LGF_EINVAL, "reduction list grew after capture");
            LGF_CUDA_TRY(ctx_, cudaStreamSynchronize(ctx_->stream));
            cudaFree(d_rtiles_);
            cudaFree(d_jobs_);
            rtiles_cap_ = std::max(rt, (long long)max_members_ * 64);
            jobs_cap_ = max_members_;
            LGF_CUDA_TRY(ctx_, cudaMalloc(&d_rtiles_, sizeof(int2) * rtiles_cap_));
            LGF_CUDA_TRY(ctx_, cudaMalloc(&d_jobs_, sizeof(int) * jobs_cap_));
        }
        ntiles_ = (int)tiles.size();
        // the stage's launch segments (unused slots empty)
        std::vector<int2> segs = member_runs(stage_len, slots_, 8LL * stage_grid_max_);
        stage_nseg_ = (int)segs.size();
        segs.resize(slots_, make_int2(0, 0));
        // one page-locked area carries the descriptors, both tile lists and the segments
        const size_t bd = align16(sizeof(LatDesc<R>) * members.size()), bt = align16(sizeof(int2) * tiles.size()),
                     bm = align16(sizeof(int4) * mtiles.size()), bs = sizeof(int2) * slots_;
        std::lock_guard<std::mutex> lk(ctx_->list_mu);
        char* h = nullptr;
        LGF_CUDA_TRY(ctx_, ctx_->list_stage.acquire(bd + bt + bm + bs, &h));
        std::memcpy(h, h_desc_.data(), sizeof(LatDesc<R>) * members.size());
        std::memcpy(h + bd, tiles.data(), sizeof(int2) * tiles.size());
        std::memcpy(h + bd + bt, mtiles.data(), sizeof(int4) * mtiles.size());
        std::memcpy(h + bd + bt + bm, segs.data(), bs);
        if (!members.empty())
            LGF_CUDA_TRY(ctx_, cudaMemcpyAsync(d_desc_, h, sizeof(LatDesc<R>) * members.size(), cudaMemcpyHostToDevice,
                                               ctx_->stream));
        if (ntiles_)
            LGF_CUDA_TRY(ctx_, cudaMemcpyAsync(d_tiles_, h + bd, sizeof(int2) * tiles.size(), cudaMemcpyHostToDevice,
                                               ctx_->stream));
        if (mt)
            LGF_CUDA_TRY(ctx_, cudaMemcpyAsync(d_all_mtiles_, h + bd + bt, sizeof(int4) * mtiles.size(),
                                               cudaMemcpyHostToDevice, ctx_->stream));
        LGF_CUDA_TRY(ctx_, cudaMemcpyAsync(d_seg_, h + bd + bt + bm, bs, cudaMemcpyHostToDevice, ctx_->stream));
        LGF_CUDA_TRY(ctx_, ctx_->list_stage.release(ctx_->stream));
        return LGF_OK;
    }

    int set_eps(const std::vector<double>& eps) override {
        for (size_t i = 0; i < h_desc_.size() && i < eps.size(); ++i) h_desc_[i].eps = (R)eps[i];
        if (h_desc_.empty()) return LGF_OK;
        std::lock_guard<std::mutex> lk(ctx_->list_mu);
        char* h = nullptr;
        LGF_CUDA_TRY(ctx_, ctx_->list_stage.acquire(sizeof(LatDesc<R>) * h_desc_.size(), &h));
        std::memcpy(h, h_desc_.data(), sizeof(LatDesc<R>) * h_desc_.size());
        LGF_CUDA_TRY(ctx_, cudaMemcpyAsync(d_desc_, h, sizeof(LatDesc<R>) * h_desc_.size(), cudaMemcpyHostToDevice,
                                           ctx_->stream));
        LGF_CUDA_TRY(ctx_, ctx_->list_stage.release(ctx_->stream));
        return LGF_OK;
    }

    // The selection table goes through a page-locked area and the lists are
    // assembled on the device (k_select_measure): no host wait.
    int set_measured(const std::vector<int>& which) override {
        if ((int)which.size() > max_members_) return set_error(ctx_, LGF_EINVAL, "measurement list exceeds capacity");
        std::vector<int> sel(sel_ints((int)which.size()), 0);
        std::vector<int> lens(which.size());
        long long tm = 0, tr = 0;
        for (size_t k = 0; k < which.size(); ++k) {
            const int i = which[k];
            if (i < 0 || i >= (int)members_.size()) return set_error(ctx_, LGF_EINVAL, "no member %d to measure", i);
            lens[k] = seg_len_[i];
            int* f = &sel[sel_fields() + SEL_FIELDS * k];
            f[0] = i;
            f[1] = seg_off_[i];
            f[2] = seg_len_[i];
            f[3] = (int)tm;
            f[4] = members_[i]->g.n[0];
            f[5] = (int)tr;
            tm += seg_len_[i];
            tr += members_[i]->g.n[0];
        }
        if (tm > mtiles_cap_ || tr > rtiles_cap_ || (long long)which.size() > jobs_cap_)
            return set_error(ctx_, LGF_EINVAL, "measurement list exceeds capacity");
        sel[0] = (int)which.size();
        sel[1] = (int)tm;
        sel[2] = (int)tr;
        // the measurement kernel's launch segments, over the selected members in list order
        const std::vector<int2> segs = member_runs(lens, slots_, 8LL * meas_grid_max_);
        for (size_t k = 0; k < segs.size(); ++k) {
            sel[SEL_HEADER + 2 * k] = segs[k].x;
            sel[SEL_HEADER + 2 * k + 1] = segs[k].y;
        }
        meas_nseg_ = (int)segs.size();
        {
            std::lock_guard<std::mutex> lk(ctx_->list_mu);
            char* h = nullptr;
            LGF_CUDA_TRY(ctx_, ctx_->list_stage.acquire(sizeof(int) * sel.size(), &h));
            std::memcpy(h, sel.data(), sizeof(int) * sel.size());
            LGF_CUDA_TRY(ctx_, cudaMemcpyAsync(d_sel_, h, sizeof(int) * sel.size(), cudaMemcpyHostToDevice, ctx_->stream));
            LGF_CUDA_TRY(ctx_, ctx_->list_stage.release(ctx_->stream));
        }
        k_select_measure<<<dim3(std::max<int>(1, (int)which.size()), 16), 256, 0, ctx_->stream>>>(
            d_sel_, sel_fields(), d_all_mtiles_, d_mtiles_, d_rtiles_, d_jobs_, d_counts_ + 1);
        LGF_CUDA_TRY(ctx_, cudaGetLastError());
        return LGF_OK;
    }

    int launch_step() override { return launch_stages(stage_nseg_); }

    // a single kernel: k = 0..2 stage k+1, k = 3 the measurement kernel alone
    // (every launch segment of it)
    int launch_one(int k) override {
        if (k < 3) {
            for (int j = 0; j < stage_nseg_; ++j) launch_stage(k + 1, j);
        } else {
            launch_measure_kernel(meas_nseg_);
        }
        LGF_CUDA_TRY(ctx_, cudaGetLastError());
        return LGF_OK;
    }

    int launch_measure() override { return launch_measurement(meas_nseg_); }

    // drop the graphs and capture those of the current segment counts
    int capture() override {
        drop_graphs();
        int rc = capture_one(true, stage_nseg_, &step_execs_[stage_nseg_]);
        if (rc != LGF_OK) return rc;
        return capture_one(false, meas_nseg_, &meas_execs_[meas_nseg_]);
    }
    // graph launch; a graph per count of launch segments, captured on first use
    int replay_step() override {
        NvtxRange r("lgf.rk3_step");
        cudaGraphExec_t& g = step_execs_[stage_nseg_];
        if (!g) {
            int rc = capture_one(true, stage_nseg_, &g);
            if (rc != LGF_OK) return rc;
        }
        LGF_CUDA_TRY(ctx_, cudaGraphLaunch(g, ctx_->stream));
        return LGF_OK;
    }
    int replay_measure() override {
        NvtxRange r("lgf.measure");
        cudaGraphExec_t& g = meas_execs_[meas_nseg_];
        if (!g) {
            int rc = capture_one(false, meas_nseg_, &g);
            if (rc != LGF_OK) return rc;
        }
        LGF_CUDA_TRY(ctx_, cudaGraphLaunch(g, ctx_->stream));
        return LGF_OK;
    }
    int launches_per_step() const override { return 3; }
    int threads() const override { return threads_; }
    const TileShape& shape() const override { return shape_; }

private:
    int stage_grid() const { return dynamic_ ? stage_grid_max_ : std::max(1, std::min(ntiles_, stage_grid_max_)); }
    int meas_grid() const {
        return dynamic_ ? meas_grid_max_ : std::max(1, std::min((int)std::max<long long>(mtiles_cap_, 1), meas_grid_max_));
    }
    // ints of a selection table for n members: header, launch segments, member fields
    int sel_fields() const { return SEL_HEADER + 2 * slots_; }
    size_t sel_ints(int n) const { return (size_t)sel_fields() + (size_t)SEL_FIELDS * std::max(n, 1); }
    bool captured() const {
        for (auto g : step_execs_) if (g) return true;
        for (auto g : meas_execs_) if (g) return true;
        return false;
    }
    void drop_graphs() {
        for (auto& g : step_execs_) if (g) { cudaGraphExecDestroy(g); g = nullptr; }
        for (auto& g : meas_execs_) if (g) { cudaGraphExecDestroy(g); g = nullptr; }
    }

    // stage S over launch segment j of the tile list
    void launch_stage(int S, int j) {
        const int grid = stage_grid();
        const int2* seg = d_seg_ + j;
        if (S == 1) k_rk3_stage<R, 1><<<grid, threads_, 0, ctx_->stream>>>(d_desc_, d_tiles_, seg);
        if (S == 2) k_rk3_stage<R, 2><<<grid, threads_, 0, ctx_->stream>>>(d_desc_, d_tiles_, seg);
        if (S == 3) k_rk3_stage<R, 3><<<grid, threads_, 0, ctx_->stream>>>(d_desc_, d_tiles_, seg);
    }
    int launch_stages(int nseg) {
        if (!dynamic_ && ntiles_ == 0) return LGF_OK;
        static const char* names[3] = {"lgf.rk3_stage1", "lgf.rk3_stage2", "lgf.rk3_stage3"};
        for (int S = 1; S <= 3; ++S) {
            NvtxRange r(names[S - 1]);
            for (int j = 0; j < nseg; ++j) launch_stage(S, j);
        }
        LGF_CUDA_TRY(ctx_, cudaGetLastError());
        return LGF_OK;
    }
    int launch_measurement(int nseg) {
        NvtxRange r("lgf.measure_launch");
        const int rg = dynamic_ ? ctx_->sm_count : std::max(1, (int)std::min<long long>(rtiles_cap_, 4 * ctx_->sm_count));
        const int jg = dynamic_ ? std::min(jobs_cap_, 4 * ctx_->sm_count) : std::max(1, (int)std::min<long long>(jobs_cap_, 4 * ctx_->sm_count));
        launch_measure_kernel(nseg);
        k_reduce_slices<R><<<rg, RED_THREADS, 0, ctx_->stream>>>(d_desc_, d_rtiles_, d_counts_ + 2);
        k_reduce_total<R><<<std::max(1, jg), RED_THREADS, 0, ctx_->stream>>>(d_desc_, d_jobs_, d_counts_ + 3);
        LGF_CUDA_TRY(ctx_, cudaGetLastError());
        return LGF_OK;
    }
    // the measurement kernel over launch segments 0..nseg-1 (read from the selection table)
    void launch_measure_kernel(int nseg) {
        const int grid = meas_grid();
        const int2* segs = reinterpret_cast<const int2*>(d_sel_ + SEL_HEADER);
        for (int j = 0; j < nseg; ++j) {
            if (shape_.meas_split == 2)
                k_measure<R, false, 2><<<grid, dim3(MEAS_SITES, 12), measure_smem_bytes<R>(), ctx_->stream>>>(
                    d_desc_, d_mtiles_, segs + j, MeasOut{});
            else
                k_measure<R, false, 1><<<grid, dim3(MEAS_SITES, 6), measure_smem_bytes<R>(), ctx_->stream>>>(
                    d_desc_, d_mtiles_, segs + j, MeasOut{});
        }
    }

    int capture_one(bool step, int nseg, cudaGraphExec_t* out) {
        cudaGraph_t graph = nullptr;
        LGF_CUDA_TRY(ctx_, cudaStreamBeginCapture(ctx_->stream, cudaStreamCaptureModeThreadLocal));
        int rc = step ? launch_stages(nseg) : launch_measurement(nseg);
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

    // The work order (tile order and block budgets) of one member's lists.
    // The group's shape fixes the kernels (block size, measurement split);
    // in a group of uneven volumes (per_volume_: batches, serving) each
    // member is ordered as tuned for its own volume class, else by the
    // defaults -- an order tuned on 24^3x48 (whole-slice measurement blocks)
    // costs a 48^4 member 40% in the measurement.
    TileShape list_shape(long long V) const {
        if (!per_volume_) return shape_;
        const int prec = std::is_same<R, double>::value ? LGF_PREC_FP64 : LGF_PREC_FP32MIXED;
        return has_tuned(ctx_, prec, V) ? tuned_shape(ctx_, prec, V) : default_shape(prec);
    }

    lgf_ctx* ctx_;
    TileShape shape_;
    int threads_;
    int max_members_;
    long long max_tiles_;
    bool dynamic_;
    bool per_volume_;
    std::vector<LatticeBuf*> members_;
    std::vector<LatDesc<R>> h_desc_;
    std::vector<int> seg_off_, seg_len_;  // each member's segment of d_all_mtiles_
    LatDesc<R>* d_desc_ = nullptr;
    int2* d_tiles_ = nullptr;
    int4* d_mtiles_ = nullptr;      // the measured members' tiles (k_select_measure)
    int4* d_all_mtiles_ = nullptr;  // every member's measurement tiles
    int* d_sel_ = nullptr;          // selection table of the next measurement
    int2* d_rtiles_ = nullptr;
    int* d_jobs_ = nullptr;
    int* d_counts_ = nullptr;  // (unused), nmtiles, nrtiles, njobs
    long long mtiles_cap_ = 0, rtiles_cap_ = 0;
    int jobs_cap_ = 0;
    int ntiles_ = 0;
    int stage_grid_max_ = 1, meas_grid_max_ = 1;
    int slots_;                                   // launch slots per kernel (member_runs)
    int stage_nseg_ = 1, meas_nseg_ = 1;           // launch segments in use
    int2* d_seg_ = nullptr;                        // the stage's launch segments
    std::vector<cudaGraphExec_t> step_execs_, meas_execs_;  // by segment count
};

GroupBase* make_group(lgf_ctx* ctx, int precision, const TileShape& shape, int max_members, long long max_tiles,
                      bool dynamic, bool per_volume, int launch_slots) {
    if (shape.threads < 128 || shape.threads % 128 || shape.threads > stage_max_threads(precision) ||
        (shape.meas_split != 1 && shape.meas_split != 2) || shape.stage_budget <= 0 || shape.meas_budget <= 0) {
        set_error(ctx, LGF_EINVAL, "invalid tile shape (threads %d, measurement split %d)", shape.threads,
                  shape.meas_split);
        return nullptr;
    }
    GroupBase* g = nullptr;
    if (precision == LGF_PREC_FP64) {
        auto* p = new (std::nothrow) Group<double>(ctx, shape, max_members, max_tiles, dynamic, per_volume, launch_slots);
        if (p && p->init() != LGF_OK) { delete p; p = nullptr; }
        g = p;
    } else {
        auto* p = new (std::nothrow) Group<float>(ctx, shape, max_members, max_tiles, dynamic, per_volume, launch_slots);
        if (p && p->init() != LGF_OK) { delete p; p = nullptr; }
        g = p;
    }
    return g;
}

// ----------------------------------------------------------- link movement
static inline int blocks_for(long long n, int t) { return (int)((n + t - 1) / t); }

// one block per 32-site layout block (the transpose kernels above)
static int launch_to_device_on(lgf_ctx* ctx, LatticeBuf& b, const double* dev_file, cudaStream_t st) {
    const int V = b.g.V;
    const int nb = blocks_for(V, LAYOUT_BLOCK);
    if (b.prec == LGF_PREC_FP64)
        k_to_device<double><<<nb, CONV_THREADS, 0, st>>>((const double2*)dev_file, (cplx<double>*)b.U[0], V);
    else
        k_to_device<float><<<nb, CONV_THREADS, 0, st>>>((const double2*)dev_file, (cplx<float>*)b.U[0], V);
    LGF_CUDA_TRY(ctx, cudaGetLastError());
    return LGF_OK;
}

int launch_to_device(lgf_ctx* ctx, LatticeBuf& b, const double* dev_file) {
    return launch_to_device_on(ctx, b, dev_file, ctx->stream);
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

int launch_generate_on(lgf_ctx* ctx, LatticeBuf& b, unsigned long long seed, double scale, cudaStream_t st) {
    const int V = b.g.V;
    if (b.prec == LGF_PREC_FP64)
        k_generate_G<double><<<blocks_for(4LL * V, 128), 128, 0, st>>>((cplx<double>*)b.U[0], V, seed, scale);
    else
        k_generate_G<float><<<blocks_for(4LL * V, 128), 128, 0, st>>>((cplx<float>*)b.U[0], V, seed, scale);
    LGF_CUDA_TRY(ctx, cudaGetLastError());
    return LGF_OK;
}

int launch_generate(lgf_ctx* ctx, LatticeBuf& b, unsigned long long seed, double scale) {
    return launch_generate_on(ctx, b, seed, scale, ctx->stream);
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

int upload_links_on(lgf_ctx* ctx, LatticeBuf& b, const double* host, cudaStream_t st) {
    const size_t bytes = (size_t)b.g.V * 4 * 18 * sizeof(double);
    char* stage = (char*)file_staging(b);
    cudaError_t e = cudaSuccess;
    if (is_pinned(host)) {
        e = cudaMemcpyAsync(stage, host, bytes, cudaMemcpyHostToDevice, st);
    } else {
        std::lock_guard<std::mutex> lk(ctx->pin_mu);
        e = ensure_pinned_chunks(ctx);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return set_error(ctx, LGF_ENOMEM, "pinned staging allocation failed: %s", cudaGetErrorString(e));
        }
        // a chunk is refilled only after the DMA that last read it (on
        // whichever stream) has finished: its event
        for (size_t off = 0, i = 0; off < bytes && e == cudaSuccess; off += PIN_CHUNK, ++i) {
            const size_t n = std::min(PIN_CHUNK, bytes - off);
            const int k = (int)(i & 1);
            e = cudaEventSynchronize(ctx->pin_done[k]);
            if (e != cudaSuccess) break;
            std::memcpy(ctx->pin[k], (const char*)host + off, n);
            e = cudaMemcpyAsync(stage + off, ctx->pin[k], n, cudaMemcpyHostToDevice, st);
            if (e == cudaSuccess) e = cudaEventRecord(ctx->pin_done[k], st);
        }
    }
    if (e != cudaSuccess) return set_error(ctx, LGF_ECUDA, "upload failed: %s", cudaGetErrorString(e));
    return launch_to_device_on(ctx, b, (const double*)stage, st);
}

int upload_links(lgf_ctx* ctx, LatticeBuf& b, const double* host) {
    int rc = upload_links_on(ctx, b, host, ctx->stream);
    const cudaError_t e = cudaStreamSynchronize(ctx->stream);
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
    int2* dn = nullptr;
    const int2 seg = make_int2(0, n);
    cudaError_t e = prepare_measure_kernel<R, true>();
    if (e == cudaSuccess) e = cudaMalloc(&ddesc, sizeof d);
    if (e == cudaSuccess) e = cudaMalloc(&dmt, sizeof(int4) * n);
    if (e == cudaSuccess) e = cudaMalloc(&dn, sizeof(int2));
    if (e == cudaSuccess) e = cudaMemcpyAsync(ddesc, &d, sizeof d, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dmt, mt.data(), sizeof(int4) * n, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dn, &seg, sizeof(int2), cudaMemcpyHostToDevice, ctx->stream);
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
    const TileShape shape = tuned_shape(ctx, lat->buf.prec, lat->buf.g.V);
    if (lat->group && lat->group_shape != shape) {
        cudaStreamSynchronize(ctx->stream);
        delete lat->group;
        lat->group = nullptr;
    }
    if (!lat->group) {
        const long long ntiles = (4LL * lat->buf.g.V + shape.threads - 1) / shape.threads;
        lat->group = make_group(ctx, lat->buf.prec, shape, 1, ntiles, false);
        if (!lat->group) return ctx->err.empty() ? set_error(ctx, LGF_ENOMEM, "group creation failed") : LGF_ECUDA;
        lat->group_shape = shape;
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
