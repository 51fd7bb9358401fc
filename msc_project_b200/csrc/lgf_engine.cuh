// Internal engine API shared by the C ABI (lgf_capi.cu), the batch runner and
// the continuous-batching server.  Not installed; no C++ type crosses the
// public boundary (include/lgf_b200.h).
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/lgf_b200.h"
#include "lgf_kernels.cuh"

// NVTX ranges around the host-side launch points (RK3 steps, stages,
// measurements), visible on an Nsight timeline; header-only NVTX is a no-op
// unless a tool is attached.  -DLGF_NO_NVTX compiles them out.
#ifndef LGF_NO_NVTX
#include <nvtx3/nvToolsExt.h>
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};
#else
struct NvtxRange {
    explicit NvtxRange(const char*) {}
};
#endif

namespace lgf {
// Launch shapes and work orders of a group's kernels, chosen per (precision,
// volume class) by the autotuner.  Every choice gives the same results bit
// for bit: only the block shapes and the order of the tiles change (no
// reduction runs in tile order).
struct TileShape {
    int threads = 256;            // stage block size: a multiple of 128, at most stage_max_threads()
    int stage_order = 1;          // 0: blocks of x1 rows swept through x0; 1: x1 columns per CTA
    double stage_budget = 8.0 * (1 << 20);  // blocked order: stage bytes per row block and slice
    double meas_budget = 2.0 * (1 << 20);   // measurement: link bytes per row block and slice
    int meas_split = 2;           // measurement warps per plane (1: 6-warp blocks, 2: 12-warp blocks)
    bool operator==(const TileShape& o) const {
        return threads == o.threads && stage_order == o.stage_order && stage_budget == o.stage_budget &&
               meas_budget == o.meas_budget && meas_split == o.meas_split;
    }
    bool operator!=(const TileShape& o) const { return !(*this == o); }
};
}  // namespace lgf

namespace lgf {
// Page-locked areas for the host->device copies of the groups' lists.  A copy
// from pageable memory may make the driver wait for the stream; from these
// areas it never does.  Two areas are used in turn, and one is rewritten only
// after the copies that last read it have completed (its event) -- normally
// long before, since the other area was used in between.
class PinnedStage {
public:
    ~PinnedStage() {
        for (int k = 0; k < 2; ++k) {
            if (ev_[k]) cudaEventSynchronize(ev_[k]);
            if (ev_[k]) cudaEventDestroy(ev_[k]);
            if (buf_[k]) cudaFreeHost(buf_[k]);
        }
    }
    // an area of at least n bytes for the next copies
    cudaError_t acquire(size_t n, char** out) {
        cur_ ^= 1;
        cudaError_t e = cudaSuccess;
        if (!ev_[cur_]) e = cudaEventCreateWithFlags(&ev_[cur_], cudaEventDisableTiming);
        else e = cudaEventSynchronize(ev_[cur_]);
        if (e != cudaSuccess) return e;
        if (cap_[cur_] < n) {
            if (buf_[cur_]) cudaFreeHost(buf_[cur_]);
            buf_[cur_] = nullptr;
            cap_[cur_] = 0;
            const size_t c = std::max<size_t>(n + n / 2, 4096);
            e = cudaMallocHost(&buf_[cur_], c);
            if (e != cudaSuccess) return e;
            cap_[cur_] = c;
        }
        *out = buf_[cur_];
        return cudaSuccess;
    }
    // the copies from the current area have been issued on stream s
    cudaError_t release(cudaStream_t s) { return cudaEventRecord(ev_[cur_], s); }

private:
    char* buf_[2] = {nullptr, nullptr};
    size_t cap_[2] = {0, 0};
    cudaEvent_t ev_[2] = {nullptr, nullptr};
    int cur_ = 1;
};

}  // namespace lgf

struct lgf_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    int sm_count = 0;
    std::string err;
    // autotuned tile shapes: (precision, lattice volume, shape); a result
    // applies to volumes within a factor of two of the tuned one
    struct Tuned { int prec; long long volume; lgf::TileShape shape; };
    std::vector<Tuned> tuned;
    // two pinned host chunks for uploads/downloads from pageable memory
    // (allocated on first use; a server's worker shares them, hence the lock)
    void* pin[2] = {nullptr, nullptr};
    cudaEvent_t pin_done[2] = {nullptr, nullptr};
    std::mutex pin_mu;
    // page-locked staging of the groups' list copies (shared by every group
    // of the context, allocated on first use and kept: freeing page-locked
    // memory would stall the device each time a group ends)
    lgf::PinnedStage list_stage;
    std::mutex list_mu;
};

namespace lgf {

int set_error(lgf_ctx* ctx, int code, const char* fmt, ...);
#define LGF_CUDA_TRY(ctx, call)                                                                          \
    do {                                                                                                 \
        cudaError_t e_ = (call);                                                                         \
        if (e_ != cudaSuccess)                                                                           \
            return ::lgf::set_error((ctx), LGF_ECUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                                    __FILE__, __LINE__);                                                 \
    } while (0)

bool valid_shape(const int shape[4]);
size_t footprint_bytes(const int shape[4], int precision, int meas_slots);
int default_threads(int precision);
int stage_max_threads(int precision);  // the stage kernel's launch bound for this precision
TileShape default_shape(int precision);
// the tuned shape for a lattice of this precision and volume, else the default
TileShape tuned_shape(const lgf_ctx* ctx, int precision, long long volume);
bool has_tuned(const lgf_ctx* ctx, int precision, long long volume);
void record_tuned(lgf_ctx* ctx, int precision, long long volume, const TileShape& shape);
// times the candidate shapes on a lattice of this shape; the fastest is recorded and returned
int tune_shape(lgf_ctx* ctx, int precision, const int shape[4], TileShape* best);

// Device resources of one lattice (precision-erased).
struct LatticeBuf {
    Geom g{};
    int prec = LGF_PREC_FP64;
    void* U[3] = {nullptr, nullptr, nullptr};
    void* A = nullptr;
    double2* partial = nullptr;
    double2* slice_sums = nullptr;
    double* meas = nullptr;
    int meas_cap = 0;
    int* slot = nullptr;
    int nchunk = 0;
    double eps = 0.0;
    bool placed = false;  // laid out in caller memory (buf_place): buf_free does not free it
};

int buf_alloc(lgf_ctx* ctx, LatticeBuf& b, const int shape[4], int precision, int meas_slots);
// bytes of one block holding a lattice's buffers, and their layout inside such a block
size_t placed_bytes(const int shape[4], int precision, int meas_slots);
void buf_place(LatticeBuf& b, const int shape[4], int precision, int meas_slots, void* mem);
int buf_grow_meas(lgf_ctx* ctx, LatticeBuf& b, int meas_slots);
void buf_free(LatticeBuf& b);

// A set of resident lattices of one precision flowed by shared launches.
// Launch arguments live in device memory (descriptor table, tile lists and
// their counts), so a captured CUDA graph stays valid while members change.
class GroupBase {
public:
    virtual ~GroupBase() {}
    // (re)define the members; order = descriptor index
    virtual int set_members(const std::vector<LatticeBuf*>& members) = 0;
    // refresh the eps of the member descriptors (device table)
    virtual int set_eps(const std::vector<double>& eps) = 0;
    // the subset of members measured by the next measurement launch
    virtual int set_measured(const std::vector<int>& which) = 0;
    virtual int launch_step() = 0;       // one RK3 step of every member (3 stage launches)
    virtual int launch_measure() = 0;    // measurement of the measured subset (3 launches)
    virtual int launch_one(int k) = 0;   // one kernel alone: stage k+1 (k<3) or the measurement kernel
    virtual int capture() = 0;           // capture step and measurement graphs
    virtual int replay_step() = 0;       // graph launch (captures on first use)
    virtual int replay_measure() = 0;
    virtual int launches_per_step() const = 0;
    virtual int threads() const = 0;
    virtual const TileShape& shape() const = 0;
};

// dynamic: members change after the graphs are captured; per_volume: each
// member's lists follow the work order tuned for its own volume class;
// launch_slots: each kernel runs as up to this many launches, one per run of
// whole members (member_runs: large lattices get launches of their own)
GroupBase* make_group(lgf_ctx* ctx, int precision, const TileShape& shape, int max_members, long long max_tiles,
                      bool dynamic, bool per_volume = false, int launch_slots = 1);

int launch_reunitarize(lgf_ctx* ctx, LatticeBuf& b);
int launch_to_device(lgf_ctx* ctx, LatticeBuf& b, const double* dev_file_order);
int launch_to_file(lgf_ctx* ctx, const LatticeBuf& b, double* dev_file_order);
int launch_generate(lgf_ctx* ctx, LatticeBuf& b, unsigned long long seed, double scale);
int launch_generate_on(lgf_ctx* ctx, LatticeBuf& b, unsigned long long seed, double scale, cudaStream_t st);

// host<->device copies of file-order links, staged in the lattice's ring
int upload_links(lgf_ctx* ctx, LatticeBuf& b, const double* host);
// the same, enqueued on stream st without waiting for it: page-locked host
// memory is read by the DMA later (keep it valid until st gets there);
// pageable memory has been copied to the context's pinned chunks on return
int upload_links_on(lgf_ctx* ctx, LatticeBuf& b, const double* host, cudaStream_t st);
int download_links(lgf_ctx* ctx, const LatticeBuf& b, double* host);
void release_pinned_chunks(lgf_ctx* ctx);

// measurement schedule of FlowSavedGaugeConfigurations for one job
int count_measurements(const lgf_flow_opts& o);

// loads lgf_measure_noalloc's module (and scratch array) on device dev, which
// must be current (lgf_noalloc.cu)
int noalloc_preload(int dev);

}  // namespace lgf

struct lgf_lattice {
    lgf_ctx* ctx = nullptr;
    lgf::LatticeBuf buf;
    lgf::GroupBase* group = nullptr;  // single-member group, created on first flow
    lgf::TileShape group_shape;
    double last_flow_s = 0.0;
    unsigned long long hb_epoch = 0;  // heatbath random-number stream position
};
