/*
 * lgf_b200.h — C ABI of the B200 Wilson-flow engine (liblgf_b200.so).
 *
 * The engine replaces the compute of the LGF reference's
 * FlowSavedGaugeConfigurations workflow (LGF/LGF.cpp:163-196): the Luscher RK3
 * gradient flow and the E(t)/Q(t) measurements.  Host code (C++, see
 * lgf_dropin.h, or any FFI) keeps the reference's parameters, file layout and
 * outputs and calls these functions with plain pointers and sizes.
 *
 * Conventions
 *   - every function returns an int status: LGF_OK (0) or a negative LGF_E*;
 *     lgf_last_error(ctx) gives a message for the last failure on that context.
 *   - host buffers are owned by the caller; device memory is owned by the
 *     library.  No exceptions and no C++ types cross this boundary.
 *   - link arrays on the host are float64 in the reference's saved-configuration
 *     order (LGF/Field/SU3_field.cpp:329-332): for global site
 *     g = ((x0*N1 + x1)*N2 + x2)*N3 + x3 (x0 slowest, LGF/Lattice/Lattice.cpp:423-436)
 *     and direction mu = 0..3, the link is 9 complex numbers, row-major,
 *     (re, im) interleaved, at double offset (g*4 + mu)*18.
 *   - a context and everything created from it must be used from one host
 *     thread at a time.  A server (lgf_serve_*) is safe from any threads.
 */
#ifndef LGF_B200_H
#define LGF_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LGF_OK 0
#define LGF_EINVAL (-1)     /* bad argument (shape, precision, null pointer, size) */
#define LGF_ENOMEM (-2)     /* device allocation failed or admission impossible */
#define LGF_ECUDA (-3)      /* a CUDA runtime call failed */
#define LGF_EIO (-4)        /* file could not be read/written */
#define LGF_ETIMEDOUT (-5)  /* a bounded wait expired */
#define LGF_ENOTFOUND (-6)  /* unknown job id */
#define LGF_EBUSY (-7)      /* result not ready yet */
#define LGF_ESHUTDOWN (-8)  /* server stopped */
#define LGF_ETOOBIG (-9)    /* size beyond the fixed maximum of lgf_measure_noalloc */

#define LGF_PREC_FP64 0       /* the plain form: links and arithmetic in float64 */
#define LGF_PREC_FP32MIXED 1  /* float32 links/RK3; float64 CH coefficients, reductions */

typedef struct lgf_ctx lgf_ctx;
typedef struct lgf_lattice lgf_lattice;

int lgf_version(void);

/* One context per GPU.  Replaces mpiWrapper::begin_parallelSession
 * (LGF/mpiWrapper.cpp:7-16): one process drives one GPU, no halo exchange. */
int lgf_ctx_create(int device, lgf_ctx** out);
int lgf_ctx_destroy(lgf_ctx* ctx);
const char* lgf_last_error(const lgf_ctx* ctx);

/* A device-resident periodic lattice ("torus", LGF/Lattice/Lattice.cpp:447-459).
 * Every extent must be even (LGF/Lattice/Lattice.cpp:42-49) and >= 4.
 * Replaces Lattice(params, true) + SU3_field U(lattice, 4) (LGF/LGF.cpp:166,171). */
int lgf_lattice_create(lgf_ctx* ctx, const int shape[4], int precision, lgf_lattice** out);
int lgf_lattice_destroy(lgf_lattice* lat);
/* device bytes a lattice of this shape/precision holds, RK3 scratch included */
size_t lgf_lattice_footprint(const int shape[4], int precision);

/* Replace SU3_field::loadSU3FromFile / saveSU3ToFile's data movement
 * (LGF/Field/SU3_field.cpp:260-352, 89-172): V*4*18 doubles, file order. */
int lgf_upload_links(lgf_lattice* lat, const double* links);
int lgf_download_links(lgf_lattice* lat, double* links);
/* Synthetic input: U = exp(i*scale*sum_a h_a lambda_a/2), h_a ~ N(0,1) from a
 * counter hash of (seed, link, a).  No reference counterpart (input generator). */
int lgf_generate_links(lgf_lattice* lat, uint64_t seed, double scale);

/* Measurement results, host arrays owned by the caller. */
typedef struct lgf_meas {
    int capacity;     /* in: number of slots in t, E, Q (and per-slice arrays) */
    int count;        /* out: measurements written */
    double* t;        /* [capacity] flow time of each measurement */
    double* E;        /* [capacity] energy density, EnergyDensity::calculate */
    double* Q;        /* [capacity] topological charge, TopologicalCharge::calculate */
    double* E_slice;  /* [capacity*N0] or NULL: mean e(x) over each x0 slice */
    double* Q_slice;  /* [capacity*N0] or NULL: each x0 slice's share of Q */
} lgf_meas;

typedef struct lgf_flow_opts {
    double eps;          /* flow step epsilon (FlowParameters::getepsilon) */
    int nsteps;          /* RK3 steps (FlowParameters::getflowSteps) */
    int meas_every;      /* measure after every k-th step; 0 = never (FlowParameters::getMeasuringInterval) */
    double t0;           /* flow time at entry (GradientFlow::SetFlowTime, GradientFlow.cpp:64-66) */
    int measure_at_t0;   /* 1: measure once before the first step (LGF/LGF.cpp:180,184) */
    int reunit_every;    /* FP32-mixed only: reunitarise every k steps (0 = never) */
} lgf_flow_opts;

/* The flow loop of FlowSavedGaugeConfigurations (LGF/LGF.cpp:175-188) on the
 * lattice's current links: GradientFlow::flow (GradientFlow.cpp:22-60) nsteps
 * times, measuring Q then E (GradientFlow.cpp:77-84) at t0 when asked and after
 * every meas_every-th step.  t accumulates as t += eps (GradientFlow.cpp:52).
 * out may be NULL when nothing is measured; otherwise out->capacity must hold
 * every measurement. */
int lgf_flow(lgf_lattice* lat, const lgf_flow_opts* opts, lgf_meas* out);

/* One measurement of E and Q now (TopologicalCharge::calculate,
 * EnergyDensity::calculate).  E_slice/Q_slice may be NULL ([N0] otherwise). */
int lgf_measure(lgf_lattice* lat, double* E, double* Q, double* E_slice, double* Q_slice);
/* per-site e(x) = sum_{mu<nu} ReTr(F F) (clover F) and q(x) (improved F,
 * before the 1/(4 pi^2)), [V] each in global site order; either may be NULL */
int lgf_site_densities(lgf_lattice* lat, double* e_site, double* q_site);
/* The observables of MeasureFlowedGaugeConfigurations (LGF/LGF.cpp:228-255):
 * E with the improved F (ImprovedEnergyDensity::calculate,
 * LGF/Observables/ImprovedEnergyDensity.cpp:9-34) and Q with the clover F
 * (UnImprovedTopologicalCharge::calculate, UnImprovedTopologicalCharge.cpp:8-29). */
int lgf_measure_flowed(lgf_lattice* lat, double* E_improved, double* Q_clover);
/* max over links of ||U^dag U - 1||_F and |det U - 1| */
int lgf_unitarity(lgf_lattice* lat, double* max_unit_err, double* max_det_err);

/* Diagnostic per-function outputs for parity tests (file-order layouts):
 *   gradient: Z(x,mu) of Wilson::calculate_FlowGradient (Wilson.cpp:55-71), V*4*18
 *   fields:   clover F (SU3_field.cpp:533-587) and improved F (:588-597) for
 *             planes (01,02,03,12,13,23), V*6*18 each (either may be NULL)
 *   exp:      HermTrLessExp (LGF/Math/SU3_mat.cpp:216-289) of n anti-Hermitian
 *             traceless matrices, n*18 doubles in and out */
int lgf_debug_gradient(lgf_lattice* lat, double* Z);
int lgf_debug_fields(lgf_lattice* lat, double* clover_F, double* improved_F);
int lgf_exp_su3(lgf_ctx* ctx, int precision, const double* iP, double* out, long long n);

/* Kernel timing for roofline reports (no reference counterpart): launches each
 * RK3 stage kernel and the measurement kernel nrep times on the lattice's
 * current links (the links are advanced by the stage launches) and returns
 * the mean device time per launch in milliseconds, measured with CUDA events
 * on the engine's stream: ms[0..2] = stages 1..3, ms[3] = measurement. */
int lgf_profile_kernels(lgf_lattice* lat, double eps, int nrep, double ms[4]);
/* Device seconds (CUDA events on the engine's stream) of the step and
 * measurement launches of the last lgf_flow call on this lattice. */
int lgf_last_flow_seconds(lgf_lattice* lat, double* seconds);

/* E and Q of a configuration that is already in device memory, without
 * allocating any device memory.  No counterpart in the reference.
 *
 * For callers that cannot call cudaMalloc: code whose GPU memory is owned by
 * another allocator (a framework's caching pool, a server that reserves all
 * memory at start-up) or a loop that must never enter the driver's allocator.
 *   links   device pointer, 16-byte aligned, float64 in file order (V*4*18)
 *   out     device pointer, 2 + 2*N0 doubles: [E, Q, E_slice[N0], Q_slice[N0]]
 *   stream  the cudaStream_t to launch on (NULL = legacy default stream)
 * The launches are asynchronous on that stream; out is valid once it completes.
 * Scratch is a fixed device array inside the library (4 MiB + 4 KiB per GPU,
 * held until exit): N0 <= 256 and N0 * ceil(N1*N2*N3/32) <= 262144 (48^4 fits,
 * 64^4 does not); larger lattices return LGF_ETOOBIG.  CUDA loads a module
 * (and with it this array) lazily by default: the array's device address is
 * looked up -- which loads it -- by lgf_ctx_create on that device, or else by
 * the first lgf_measure_noalloc call there.  Make one of the two before
 * reserving the rest of the GPU's memory and before any stream capture.
 * An error left pending by earlier work on the calling thread is not
 * cleared: the call then returns LGF_ECUDA without launching.  Calls share
 * the array: calls that may overlap on one GPU (other streams, other host
 * threads) race and must be ordered by the caller. */
int lgf_measure_noalloc(const double* links, const int shape[4], double* out, void* stream);

/* ------------------------------------------------------- configurations */
/* Input generation on the GPU (SU3_field::InitializeHotStart / ColdStart,
 * LGF/Field/SU3_field.cpp:440-466; SU3_Heatbath::update,
 * LGF/SU3_Heatbath/SU3_Heatbath.cpp:16-224).  lgf_heatbath runs n_iter x (one
 * Cabibbo-Marinari heatbath sweep + or_per_hb overrelaxation sweeps) at beta,
 * drawing from a counter-based generator keyed by seed; successive calls on
 * the same lattice continue the stream.  *rejected (may be NULL) counts SU(2)
 * subgroup updates whose bounded rejection loop found no sample (left unchanged). */
int lgf_hot_start(lgf_lattice* lat, uint64_t seed);
int lgf_cold_start(lgf_lattice* lat);
int lgf_heatbath(lgf_lattice* lat, double beta, int n_iter, int or_per_hb, uint64_t seed, uint64_t* rejected);
/* n_sweeps overrelaxation sweeps alone (SU3_Heatbath::OverRelaxation, SU3_Heatbath.cpp:58-111):
 * microcanonical, the Wilson action is unchanged up to rounding */
int lgf_overrelax(lgf_lattice* lat, int n_sweeps);
/* SU3_field::Avg_Plaquette (SU3_field.cpp:485-499): sum ReTr P / (3 * 6 * V) */
int lgf_plaquette(lgf_lattice* lat, double* avg);

/* ------------------------------------------------------------------ batch */
/* A flow job: one configuration, its flow schedule and its result arrays. */
typedef struct lgf_job {
    int shape[4];
    int precision;          /* LGF_PREC_* */
    const double* links;    /* host links in file order, or NULL to generate */
    uint64_t seed;          /* generator seed when links == NULL */
    double gen_scale;       /* generator scale when links == NULL (0.5 in the configs) */
    lgf_flow_opts flow;     /* eps, nsteps, meas_every, t0, measure_at_t0, reunit_every */
    lgf_meas* meas;         /* results (may be NULL) */
    double* links_out;      /* optional: final links, file order */
    /* serving only (ignored by lgf_batch_run): when not NULL, the links after
     * each measured RK3 step are written to <snapshot_prefix>_Flowtime<t>.bin,
     * t formatted like the reference's saved flowed configurations
     * (std::to_string, LGF/LGF.cpp:194) in the same file layout, so a job can
     * be resumed from its last snapshot (links = file, flow.t0 = t) */
    const char* snapshot_prefix;
} lgf_job;

typedef struct lgf_batch_stats {
    double seconds;         /* device time of the whole batch (CUDA events) */
    double site_steps;      /* sum over jobs of V * nsteps */
    int launches;           /* kernel launches (graph nodes) issued */
    int block_threads;      /* thread-block size chosen for the RK3 stage kernel */
} lgf_batch_stats;

/* Flow many configurations of uneven volumes together: every RK3 stage of all
 * jobs is ONE persistent launch over a shared work list of (job, site block)
 * tiles, each RK3 step of the batch is captured once as a CUDA graph and
 * replayed, and the stage kernel's block shape is chosen by the autotuner.
 * Results are identical to flowing each job alone with lgf_flow.  stats may be NULL. */
int lgf_batch_run(lgf_ctx* ctx, lgf_job* jobs, int njobs, lgf_batch_stats* stats);

/* Launch shapes and work orders of the RK3 stage and measurement kernels
 * (no reference counterpart: the reference has no launch configuration).
 * Every choice gives bit-identical results; only speed differs. */
typedef struct lgf_tile_shape {
    int stage_threads;    /* RK3 stage block size: 128, 256 or 384 (4 link directions x threads/4 sites) */
    int stage_order;      /* 0: blocks of x1 rows swept through x0; 1: x1 columns walked per block */
    int stage_budget_kb;  /* order 0: stage working set per row block and x0 slice */
    int meas_budget_kb;   /* measurement: link bytes per row block and x0 slice (7 slices live) */
    int meas_split;       /* measurement warps per plane: 1 (6-warp blocks) or 2 (12-warp blocks) */
} lgf_tile_shape;

/* Autotuner: time the candidate tile shapes for one precision on a lattice
 * of this shape (generated links) with CUDA events, one parameter at a time,
 * and remember the fastest in this context for lattices of this volume class
 * (within a factor of two); lgf_flow, lgf_batch_run and the server use it.
 * lgf_autotune returns only the stage block size.  best may be NULL. */
int lgf_autotune_tiles(lgf_ctx* ctx, int precision, const int shape[4], lgf_tile_shape* best);
int lgf_autotune(lgf_ctx* ctx, int precision, const int shape[4], int* best_threads);
/* Set / read the shape used for this precision and volume class. */
int lgf_set_tiles(lgf_ctx* ctx, int precision, const int shape[4], const lgf_tile_shape* tiles);
int lgf_get_tiles(lgf_ctx* ctx, int precision, const int shape[4], lgf_tile_shape* tiles);

/* ---------------------------------------------------------------- serving */
typedef struct lgf_server lgf_server;

typedef struct lgf_serve_config {
    size_t hbm_budget_bytes;   /* admission budget for resident jobs (links + RK3 scratch) */
    int max_active;            /* maximum concurrently flowing jobs (slots; up to 32 of them get launches of their own) */
    int steps_per_tick;        /* RK3 steps per scheduling tick */
} lgf_serve_config;

#define LGF_JOB_QUEUED 0
#define LGF_JOB_RUNNING 1
#define LGF_JOB_DONE 2
#define LGF_JOB_FAILED 3

typedef struct lgf_job_status {
    int state;                 /* LGF_JOB_* */
    int error;                 /* LGF_* status when FAILED */
    double submit_s;           /* times on the server's monotonic clock, seconds */
    double start_s;
    double end_s;
    int steps_done;
} lgf_job_status;

/* A continuous-batching flow server on one context: jobs are admitted by their
 * HBM footprint as memory and slots free up, flow together in shared launches
 * with other resident jobs, and leave when done.  The job's arrays (links,
 * meas, links_out) must stay valid until the job is DONE or FAILED. */
int lgf_serve_start(lgf_ctx* ctx, const lgf_serve_config* cfg, lgf_server** out);
int lgf_serve_submit(lgf_server* srv, const lgf_job* job, uint64_t* id);
int lgf_serve_poll(lgf_server* srv, uint64_t id, lgf_job_status* st);
int lgf_serve_wait(lgf_server* srv, uint64_t id, double timeout_s, lgf_job_status* st);
int lgf_serve_stop(lgf_server* srv);

/* Counters of a running server (no reference counterpart).  device_busy_s is
 * the device time of the scheduling ticks, summed from CUDA events around each
 * tick's launches (ticks whose events have not completed yet are left out);
 * against the wall time since the start it shows how much of the stream the
 * kernels themselves take. */
typedef struct lgf_serve_stats {
    double wall_s;             /* since lgf_serve_start */
    double device_busy_s;      /* device time of completed ticks */
    long long ticks;
    long long steps;           /* RK3 steps launched (shared launches count once) */
    long long measurements;    /* measurement launches (each covers the jobs due) */
    long long jobs_done;
    long long snapshots;
} lgf_serve_stats;
int lgf_serve_stats_get(lgf_server* srv, lgf_serve_stats* st);

#ifdef __cplusplus
}
#endif
#endif
