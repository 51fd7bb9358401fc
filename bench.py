"""Benchmark of the Wilson-flow hot path (FlowSavedGaugeConfigurations).

Workload (the plain FP64 throughput configuration): a 24^3 x 48 lattice
(shape {48,24,24,24}, x0 = time), generator-G links (seed 7, scale 0.5),
flowed with eps = 0.01 to t = 3.0 (300 RK3 steps) measuring E and Q at t = 0
and every 10 steps.  One bench step = one such flow job.  The links
(382 MB in float64) are larger than the 126 MB L2, so no flush is needed.

metric: site-RK3-steps/s = V * RK3 steps / time (whole job, measurements
included).  `value`: device time of the flow launches with the links resident
in HBM (CUDA events on the engine's stream), summed over the K timed jobs,
max over ranks.  `e2e`: the same jobs through the public C ABI from pinned
host memory -- upload of the configuration, the flow, and the read-back of
E(t), Q(t) -- timed on the host around the synchronous calls.  `flow_only`:
the same 300 steps without measurements.  Forms (rank 0 at N=1): FP64 rate
against volume (16^4 to 48^4), FP32-mixed on 32^4, the batched 64-configuration ensemble, a served Poisson stream at a
sweep of arrival rates, and heatbath generation.

--impl reference runs the LGF reference itself (oracle/_ref/lgf_ref, the
unmodified sources) on the host cores: one single-rank process per core,
each flowing a 16^4 sample of the generator input (per-site cost as on
24^3x48: both exceed the host caches), RK3 steps and one E/Q measurement
timed apart; value = processes * V * 300 / (300 step times + 31 measurement
times), the bench job's schedule.

--gpus N (under torchrun) runs N independent replicas, one per GPU ("replicas
only": the flow of one lattice does not shard); value sums all ranks' work
over the slowest rank's time.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

SHAPE = (48, 24, 24, 24)
EPS = 0.01
NSTEPS = 300
MEAS = 10
SEED = 7
WORKLOAD = "24^3x48 (shape 48,24,24,24) FP64 Wilson flow, eps 0.01 to t=3.0, E/Q at t=0 and every 10 steps"
# Algorithmic bytes and flops (canonical counts of the scope table):
#   per site per RK3 step: FP64 4480 B (3 x (read+write 4 links) + su(3)
#   accumulator), FP32-mixed 2240 B; 42,888 flops.  A stage launch is 1/3.
BYTES_PER_SITE_STAGE = {0: 4480.0 / 3, 1: 2240.0 / 3}
FLOPS_PER_SITE_STAGE = 42888.0 / 3
# DRAM traffic of one stage launch from ncu (dram__bytes_read.sum +
# dram__bytes_write.sum), scaled to this workload; see profiles/.
NCU_STAGE_TRAFFIC_BYTES = {0: 1111.5e6, 1: 534.9e6}  # stage-2 launch; profiles/k_rk3_stage_*_24x24x24x48.md
FP64_FMA_PER_SM_PER_CLK = 64  # B200: 64 FP64 FMA lanes per SM (nominal)
FP32_FMA_PER_SM_PER_CLK = 128  # B200: 128 FP32 FMA lanes per SM (nominal)
N_SM = 148


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        mhz, maxmhz, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                mhz.append(float(f[1]))
                maxmhz = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(mhz) if mhz else None, "sm_max_mhz": maxmhz,
                "reasons": sorted(reasons), "samples": len(mhz)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    return world, rank, local, dist


def reduce_max(dist, x: float) -> float:
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(dist):
    if dist is not None:
        import torch
        dist.barrier()
        torch.cuda.synchronize()


# --------------------------------------------------------------- reference
# The reference's per-site cost on lattices that exceed the host's caches is
# volume-independent (16^4 and 24^3x48 both stream their fields from DRAM),
# so each host core flows a 16^4 sample of the bench's generator input; the
# full 24^3x48 lattice costs ~45 s per RK3 step on one core (REF_SAMPLE_SHAPE
# can be set to it with --ref-shape).
REF_SAMPLE_SHAPE = (16, 16, 16, 16)


def run_reference_sample(nproc: int, steps: int, warm: int, shape=REF_SAMPLE_SHAPE):
    """nproc single-rank reference processes in parallel (oracle/_ref/lgf_ref
    cpusplit: the unmodified GradientFlow/observable code), each flowing the
    generator-G (seed 7) configuration of `shape` for `steps` RK3 steps timed
    one by one, then one E/Q measurement.  The rate applies the bench job's
    schedule (NSTEPS steps, a measurement at t=0 and every MEAS steps) to the
    slowest process's median step and measurement times."""
    import tempfile

    from oracle import oracle as O
    if not O.reference_available():
        return None, "oracle/_ref/lgf_ref not built"
    V = int(shape[0] * shape[1] * shape[2] * shape[3])
    with tempfile.TemporaryDirectory() as tmp:
        inp = Path(tmp) / "g7.bin"
        O.generate_G(shape, SEED, 0.5).tofile(inp)

        def one(_):
            out = O.run_reference(["cpusplit", inp, *shape, steps], timeout=3600)
            line = [ln for ln in out.stdout.splitlines() if ln.startswith("{")][-1]
            return json.loads(line)

        with ThreadPoolExecutor(max_workers=nproc) as ex:
            res = list(ex.map(one, range(nproc)))
    per_step = [max(r["step_s"][i] for r in res) for i in range(warm, steps)]
    meas_s = max(r["measure_s"] for r in res)
    t_step = statistics.median(per_step)
    nmeas = 1 + NSTEPS // MEAS
    job_s = NSTEPS * t_step + nmeas * meas_s  # one process's job on the sample lattice
    value = nproc * V * NSTEPS / job_s
    return {"value": value, "per_step_s": per_step, "measure_s": meas_s, "cores": nproc, "host_cpu": host_cpu(),
            "host_threads": os.cpu_count(),
            "flow_only": nproc * V / t_step,
            "lattice_setup_s": max(r["setup_s"] for r in res),
            "sample": f"{nproc} parallel single-rank reference processes (no MPI on the host), each the "
                      f"{'x'.join(map(str, shape))} generator-G seed-7 configuration: {steps} RK3 steps timed one by "
                      f"one (first {warm} untimed) and one E/Q measurement; rate = the bench job's schedule "
                      f"({NSTEPS} steps + {nmeas} measurements) at the slowest process's median step and "
                      f"measurement times; the Lattice/field setup and input read (lattice_setup_s) is excluded"}, None


def host_cpu() -> str:
    """The host CPU's model name (Linux /proc/cpuinfo), for the baseline record."""
    try:
        for ln in Path("/proc/cpuinfo").read_text().splitlines():
            if ln.startswith("model name"):
                return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def _ref_shape(args):
    return tuple(int(x) for x in args.ref_shape.split(",")) if args.ref_shape else REF_SAMPLE_SHAPE


def reference_arm(args):
    world, rank, local, dist = int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), 0, None
    if rank != 0:
        return
    nproc = args.ref_procs or os.cpu_count() or 1
    shape = _ref_shape(args)
    res, err = run_reference_sample(nproc, args.warmup + args.steps, args.warmup, shape)
    if res is None:
        print(json.dumps({"impl": "reference", "unavailable": err}))
        return
    line = {
        "impl": "reference",
        "metric": "site-RK3-steps/s", "value": res["value"], "unit": "site-RK3-steps/s",
        "n_gpus": 0, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * statistics.median(res["per_step_s"]),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "reference_sample": f"{'x'.join(map(str, shape))} per process",
                   "step": "one RK3 step of every process (wall, slowest process); one E/Q measurement after them"},
        "cpu_baseline": {"value": res["value"], "unit": "site-RK3-steps/s", "cores": res["cores"],
                         "kind": "reference", "sample": res["sample"], "measure_s": res["measure_s"],
                         "flow_only": res["flow_only"], "lattice_setup_s": res["lattice_setup_s"],
                         "host_cpu": res["host_cpu"], "host_threads": res["host_threads"]},
        "e2e": {"value": res["value"], "unit": "site-RK3-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


# ------------------------------------------------------------------- forms
def _flow_timed(ctx, lat, eps, nsteps, meas, reunit=0):
    r = lat.flow(eps, nsteps, meas, 0.0, True, reunit)
    secs = ctypes.c_double()
    ctx.check(ctx.lib.lgf_last_flow_seconds(lat.h, ctypes.byref(secs)))
    return r, secs.value


def form_fp32mixed(ctx):
    """FP32-mixed against plain FP64 on the 32^4 configuration: generator G
    seed 11, eps 0.01 to t=5.0 (500 steps), E/Q every 10 steps, FP32 links
    reunitarised every 10 steps."""
    import numpy as np
    from msc_project_b200 import FP32MIXED, FP64
    shape, steps, meas = (32, 32, 32, 32), 500, 10
    V = int(np.prod(shape))
    res = {}
    for name, prec, reunit in (("fp64", FP64, 0), ("fp32mixed", FP32MIXED, 10)):
        with ctx.lattice(shape, prec) as lat:
            lat.generate(11, 0.5)
            _flow_timed(ctx, lat, 0.01, 20, 10, reunit)  # warm-up: module load, graph capture
            lat.generate(11, 0.5)
            r, sec = _flow_timed(ctx, lat, 0.01, steps, meas, reunit)
            u, d = lat.unitarity()
        res[name] = (r, sec, u, d)
    r64, s64, _, _ = res["fp64"]
    r32, s32, u32, d32 = res["fp32mixed"]
    return {"config": "32^4 G seed 11, eps 0.01, 500 steps, E/Q every 10, reunitarise every 10",
            "fp64_site_steps_per_s": V * steps / s64, "fp32mixed_site_steps_per_s": V * steps / s32,
            "speedup": s64 / s32,
            "max_rel_dE": float(np.max(np.abs(r32.E - r64.E) / np.abs(r64.E))),
            "max_abs_dQ": float(np.max(np.abs(r32.Q - r64.Q))),
            "max_unit_err": u32, "max_det_err": d32,
            "gates": {"dQ<1e-3": bool(np.max(np.abs(r32.Q - r64.Q)) < 1e-3),
                      "dE/E<1e-5": bool(np.max(np.abs(r32.E - r64.E) / np.abs(r64.E)) < 1e-5)}}


def form_volumes(ctx):
    """FP64 throughput against volume: 16^4, 24^3x48, 32^4 and 48^4 (generator
    G seed 7), eps 0.01, 100 RK3 steps, E/Q at t=0 and every 10 steps, and the
    same 100 steps without measurements."""
    import numpy as np
    from msc_project_b200 import FP64
    out = []
    secs = ctypes.c_double()
    for shape in ((16, 16, 16, 16), (48, 24, 24, 24), (32, 32, 32, 32), (48, 48, 48, 48)):
        V = int(np.prod(shape))
        with ctx.lattice(shape, FP64) as lat:
            lat.generate(7, 0.5)
            _flow_timed(ctx, lat, 0.01, 10, 10)  # warm-up: graph capture for this lattice
            _, sec = _flow_timed(ctx, lat, 0.01, 100, 10)
            lat.flow(0.01, 100, 0, 0.0, False, 0)
            ctx.check(ctx.lib.lgf_last_flow_seconds(lat.h, ctypes.byref(secs)))
        out.append({"shape": list(shape), "sites": V, "site_steps_per_s": V * 100 / sec,
                    "flow_only_site_steps_per_s": V * 100 / secs.value})
    return out


ENSEMBLE = [((8, 8, 8, 8), 16), ((12, 12, 12, 12), 16), ((16, 16, 16, 16), 16), ((32, 16, 16, 16), 8),
            ((48, 24, 24, 24), 8)]


def form_batched(ctx):
    """The 64-configuration ensemble of uneven volumes (seeds 100-163), eps 0.01
    to t=2.0 (200 steps), E/Q every 10 steps: one batched run per precision
    against the same jobs flowed one after another with lgf_flow."""
    import numpy as np
    from msc_project_b200 import FP32MIXED, FP64, Job
    out = {}
    results = {}
    for name, prec, reunit in (("fp64", FP64, 0), ("fp32mixed", FP32MIXED, 10)):
        def jobs():
            js, seed = [], 100
            for shape, n in ENSEMBLE:
                for _ in range(n):
                    js.append(Job(shape, prec, seed=seed, nsteps=200, meas_every=10, reunit_every=reunit))
                    seed += 1
            return js
        ctx.batch_run([Job((8, 8, 8, 8), prec, seed=1, nsteps=10, meas_every=10, reunit_every=reunit)])  # warm-up
        js = jobs()
        st = ctx.batch_run(js)
        seq = 0.0
        for j in jobs():
            with ctx.lattice(j.shape, prec) as lat:
                lat.generate(j.seed, 0.5)
                _, sec = _flow_timed(ctx, lat, 0.01, 200, 10, reunit)
                seq += sec
        out[name] = {"site_steps_per_s": st.site_steps / st.seconds, "seconds": st.seconds,
                     "sequential_seconds": seq, "batching_speedup": seq / st.seconds,
                     "launches": st.launches, "block_threads": st.block_threads,
                     "tiles": ctx.get_tiles(prec, ENSEMBLE[-1][0])}
        results[name] = js
    dq = max(float(np.max(np.abs(a.result.Q - b.result.Q))) for a, b in zip(results["fp32mixed"], results["fp64"]))
    de = max(float(np.max(np.abs(a.result.E - b.result.E) / np.abs(b.result.E)))
             for a, b in zip(results["fp32mixed"], results["fp64"]))
    out["configs"] = 64
    out["sites"] = int(sum(np.prod(s) * n for s, n in ENSEMBLE))
    # the regime batching exists for: many small lattices, each too small to fill the GPU
    small = [Job((8, 8, 8, 8), FP32MIXED, seed=200 + i, nsteps=200, meas_every=10, reunit_every=10) for i in range(64)]
    st = ctx.batch_run(small)
    seq = 0.0
    for j in small[:16]:
        with ctx.lattice(j.shape, FP32MIXED) as lat:
            lat.generate(j.seed, 0.5)
            _, sec = _flow_timed(ctx, lat, 0.01, 200, 10, 10)
            seq += sec
    seq *= 4.0  # 16 of the 64 timed one by one; all have the same shape and schedule
    out["small_lattices_fp32mixed"] = {"configs": "64 x 8^4, 200 steps, E/Q every 10",
                                       "site_steps_per_s": st.site_steps / st.seconds,
                                       "sequential_site_steps_per_s": st.site_steps / seq,
                                       "batching_speedup": seq / st.seconds}
    out["fp32mixed_vs_fp64"] = {"max_abs_dQ": dq, "max_rel_dE": de,
                                "speedup": out["fp32mixed"]["site_steps_per_s"] / out["fp64"]["site_steps_per_s"]}
    return out


def form_served(ctx, njobs: int, rate: float, seed: int = 5):
    """A served stream: Poisson arrivals (rate jobs/s) of FP32-mixed jobs with
    volume uniform over {16^4, 24^3x48, 32^4, 48^4}, t_max ~ U[1,8], eps 0.01,
    E/Q every 5 steps, per-job seed; admission by HBM footprint."""
    import numpy as np
    from msc_project_b200 import FP32MIXED, Job, Server
    rng = np.random.default_rng(seed)
    vols = [(16, 16, 16, 16), (48, 24, 24, 24), (32, 32, 32, 32), (48, 48, 48, 48)]
    specs = []
    for i in range(njobs):
        shape = vols[int(rng.integers(0, 4))]
        tmax = float(rng.uniform(1.0, 8.0))
        specs.append((shape, 1000 + i, int(round(tmax / 0.01))))

    def make_jobs():
        return [Job(shape, FP32MIXED, seed=sd, nsteps=n, meas_every=5, reunit_every=10) for shape, sd, n in specs]
    jobs = make_jobs()
    # rate = inf: every job arrives at t = 0 (the saturated server)
    gaps = np.zeros(njobs) if not np.isfinite(rate) else rng.exponential(1.0 / rate, size=njobs)
    try:
        import torch
        free, _ = torch.cuda.mem_get_info()
    except Exception:
        free = 120 << 30
    budget = int(free * 0.6)
    with Server(ctx, budget, max_active=16, steps_per_tick=5) as srv:
        srv.submit(Job((16, 16, 16, 16), FP32MIXED, seed=1, nsteps=5, meas_every=5, reunit_every=10))  # warm-up
        ids = []
        t0 = time.perf_counter()
        for j, g in zip(jobs, gaps):
            if g > 0:
                time.sleep(float(g))
            ids.append(srv.submit(j))
        sts = [srv.wait(i, 3600.0) for i in ids]
        makespan = time.perf_counter() - t0
        time.sleep(0.1)  # the scheduler counts the last ticks' device time
        stats = srv.stats()
    lat = np.array([s.end_s - s.submit_s for s in sts])
    work = sum(int(np.prod(j.shape)) * j.nsteps for j in jobs)
    out = {"jobs": njobs, "rate_per_s": rate if np.isfinite(rate) else "all at t=0", "jobs_per_s": njobs / makespan,
           "p50_latency_s": float(np.percentile(lat, 50)), "p99_latency_s": float(np.percentile(lat, 99)),
           "site_steps_per_s": work / makespan, "hbm_budget_bytes": budget,
           "device_busy_frac": stats["device_busy_s"] / stats["wall_s"], "server_stats": stats,
           "all_done": all(s.state == 2 for s in sts)}
    if not np.isfinite(rate):
        # the same jobs as one offline batch (lgf_batch_run): what continuous
        # batching costs against knowing every job up front
        st = ctx.batch_run(make_jobs())
        out["batched_same_jobs_site_steps_per_s"] = st.site_steps / st.seconds
        out["vs_batched_same_jobs"] = out["site_steps_per_s"] / out["batched_same_jobs_site_steps_per_s"]
    return out


def form_heatbath(ctx):
    """Input generation: hot start and 20 x (Cabibbo-Marinari heatbath + 5
    overrelaxation sweeps) at beta = 6.0 on 24^3x48, FP64.  Rate in
    site-sweeps/s (one sweep = every link updated once, HB or OR)."""
    import numpy as np
    from msc_project_b200 import FP64
    V = int(np.prod(SHAPE))
    with ctx.lattice(SHAPE, FP64) as lat:
        lat.hot_start(1)
        lat.heatbath(6.0, 1, 5, seed=1)  # warm-up
        t0 = time.perf_counter()
        rej = lat.heatbath(6.0, 20, 5, seed=2)
        sec = time.perf_counter() - t0
        plaq = lat.plaquette()
    return {"config": "24^3x48, beta 6.0, 20 x (CM heatbath + 5 OR)", "site_sweeps_per_s": V * 20 * 6 / sec,
            "seconds": sec, "plaquette": plaq, "rejected_subgroup_updates": rej}


# ------------------------------------------------------------------ engine
def engine_arm(args):
    import numpy as np
    world, rank, local, dist = dist_setup()
    from msc_project_b200 import FP32MIXED, FP64, Context
    from msc_project_b200 import _capi as C
    prec = FP64 if args.precision == "fp64" else FP32MIXED
    V = int(np.prod(SHAPE))
    ctx = Context(local)
    # tile shapes for this volume class, chosen once before any timing (the
    # autotuner times its candidates on a lattice of this shape)
    tiles = ctx.autotune_tiles(prec, SHAPE) if not args.no_autotune else ctx.get_tiles(prec, SHAPE)
    lat = ctx.lattice(SHAPE, prec)
    lat.generate(SEED, 0.5)
    reunit = 10 if prec == FP32MIXED else 0
    nmeas = 1 + NSTEPS // MEAS

    def job():
        return lat.flow(EPS, NSTEPS, MEAS, 0.0, True, reunit)

    for _ in range(args.warmup):
        job()
    secs = ctypes.c_double()
    barrier(dist)
    dev_s = 0.0
    with ClockSampler(local) as clk:
        t0 = time.perf_counter()
        for _ in range(args.steps):
            job()
            ctx.check(ctx.lib.lgf_last_flow_seconds(lat.h, ctypes.byref(secs)))
            dev_s += secs.value
        wall = time.perf_counter() - t0
    barrier(dist)
    dev_s = reduce_max(dist, dev_s)
    value = world * V * NSTEPS * args.steps / dev_s

    # ---- the flow alone (no measurements), device-timed like the job
    lat.flow(EPS, 30, 0, 0.0, False, reunit)
    secs_fo = 0.0
    for _ in range(2):
        lat.flow(EPS, NSTEPS, 0, 0.0, False, reunit)
        ctx.check(ctx.lib.lgf_last_flow_seconds(lat.h, ctypes.byref(secs)))
        secs_fo += secs.value
    flow_only = world * V * NSTEPS * 2 / reduce_max(dist, secs_fo)

    # ---- end to end through the public ABI from pinned host memory
    import torch
    host = torch.empty(V * 72, dtype=torch.float64, pin_memory=True)
    links_np = host.numpy()
    links_np[:] = lat.download()
    lat2 = ctx.lattice(SHAPE, prec)
    ptr = ctypes.cast(host.data_ptr(), ctypes.POINTER(ctypes.c_double))

    def e2e_job():
        ctx.check(ctx.lib.lgf_upload_links(lat2.h, ptr))
        return lat2.flow(EPS, NSTEPS, MEAS, 0.0, True, reunit)

    e2e_job()
    barrier(dist)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_job()
    e2e_s = reduce_max(dist, time.perf_counter() - t0)
    e2e_value = world * V * NSTEPS * args.steps / e2e_s
    lat2.close()

    # ---- dominant kernel: the RK3 stage launch (CUDA events on the engine stream)
    ms = (ctypes.c_double * 4)()
    ctx.check(ctx.lib.lgf_profile_kernels(lat.h, EPS, 5, ms))
    stage_ms = (ms[0] + ms[1] + ms[2]) / 3.0
    hbm_peak, peak_kind = measured_peaks()
    stage_bytes = V * BYTES_PER_SITE_STAGE[prec]
    achieved = stage_bytes / (stage_ms * 1e-3) / 1e9
    clocks = clk.summary()
    mhz = clocks["sm_mhz"] or 1965.0
    pipe_name = "fp64" if prec == FP64 else "fp32"
    fma_lanes = FP64_FMA_PER_SM_PER_CLK if prec == FP64 else FP32_FMA_PER_SM_PER_CLK
    fma_peak = N_SM * fma_lanes * 2 * mhz * 1e6 / 1e12
    stage_tflops = V * FLOPS_PER_SITE_STAGE / (stage_ms * 1e-3) / 1e12

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        res, err = run_reference_sample(args.ref_procs or os.cpu_count() or 1, 3, 1, _ref_shape(args))
        if res:
            cpu = {"value": res["value"], "unit": "site-RK3-steps/s", "cores": res["cores"], "kind": "reference",
                   "sample": res["sample"], "measure_s": res["measure_s"], "flow_only": res["flow_only"],
                   "lattice_setup_s": res["lattice_setup_s"], "host_cpu": res["host_cpu"],
                   "host_threads": res["host_threads"]}
        else:
            cpu = {"value": None, "unavailable": err}

    forms = None
    if rank == 0 and world == 1 and not args.no_forms:
        rates = [float(r) for r in args.serve_rates.split(",") if r]
        makers = {"volumes_fp64": lambda: form_volumes(ctx), "fp32mixed": lambda: form_fp32mixed(ctx),
                  "batched": lambda: form_batched(ctx),
                  "served": lambda: [form_served(ctx, args.serve_jobs, r) for r in rates],
                  "heatbath": lambda: form_heatbath(ctx)}
        wanted = list(makers) if args.forms == "all" else args.forms.split(",")
        forms = {k: makers[k]() for k in wanted}
        if "served" in forms and "batched" in forms:
            sat = [f for f in forms["served"] if f["rate_per_s"] == "all at t=0"]
            if sat:
                forms["served_saturated_vs_batched_fp32mixed"] = (
                    sat[0]["site_steps_per_s"] / forms["batched"]["fp32mixed"]["site_steps_per_s"])

    launches_per_job = 3 * NSTEPS + 3 * nmeas + (NSTEPS // 10 if reunit else 0)
    line = {
        "metric": "site-RK3-steps/s", "value": value, "unit": "site-RK3-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dev_s / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if prec == FP64 else "f32+f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "precision": args.precision, "sites": V, "rk3_steps_per_step": NSTEPS,
                   "tiles": tiles,
                   "measurements_per_step": nmeas, "l2": "inputs larger than L2 (382 MB links)",
                   "parallelism": f"replicas x{world}"},
        "e2e": {"value": e2e_value, "unit": "site-RK3-steps/s", "h2d_bytes_per_step": V * 72 * 8,
                "d2h_bytes_per_step": nmeas * 3 * 8},
        "flow_only": {"value": flow_only, "unit": "site-RK3-steps/s",
                      "note": "the same 300 steps without E/Q measurements (device time)"},
        "roofline": {"bound": pipe_name, "kernel": "k_rk3_stage (mean of the 3 stages)",
                     "achieved": stage_tflops, "peak": fma_peak, "unit": "TFLOP/s", "frac": stage_tflops / fma_peak,
                     "peak_kind": f"nominal: {N_SM} SM x {fma_lanes} {pipe_name.upper()} FMA lanes x 2 flops x the run's "
                                  f"median SM clock (no measured {pipe_name.upper()} peak exists for this pool)",
                     "binding": f"{pipe_name} FMA pipe: one stage is "
                                f"{V * FLOPS_PER_SITE_STAGE / (fma_peak * 1e12) * 1e3:.3f} ms of FMA work at the nominal "
                                f"peak and {stage_bytes / (hbm_peak * 1e9) * 1e3:.3f} ms of HBM traffic at the measured "
                                f"copy rate",
                     "flops_per_launch": V * FLOPS_PER_SITE_STAGE,
                     "traffic": NCU_STAGE_TRAFFIC_BYTES[prec],
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one stage-2 launch on this "
                                       "workload (profiles/k_rk3_stage_*), a constant carried from that capture, not "
                                       "re-measured by this run",
                     "algorithmic_bytes": stage_bytes,
                     "hbm": {"achieved": achieved, "peak": hbm_peak, "unit": "GB/s", "frac": achieved / hbm_peak,
                             "peak_kind": peak_kind},
                     "stage_ms": stage_ms, "measure_ms": ms[3]},
        "cpu_baseline": cpu,
        "forms": forms,
        "clocks": clocks,
        "gpu_launches": launches_per_job * args.steps,
        "wall_s": wall,
    }
    if rank == 0:
        print(json.dumps(line))
    lat.close()
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()


def profile_case(args):
    """One launch of each RK3 stage kernel and of the measurement kernel on the
    bench lattice (the case the ncu captures under profiles/ use)."""
    import numpy as np
    from msc_project_b200 import FP32MIXED, FP64, Context
    prec = FP64 if args.precision == "fp64" else FP32MIXED
    with Context(0) as ctx:
        if args.tiles:
            ctx.set_tiles(prec, SHAPE, **json.loads(args.tiles))
        lat = ctx.lattice(SHAPE, prec)
        lat.generate(SEED, 0.5)
        ms = (ctypes.c_double * 4)()
        ctx.check(ctx.lib.lgf_profile_kernels(lat.h, EPS, 1, ms))  # first launches load the modules
        ctx.check(ctx.lib.lgf_profile_kernels(lat.h, EPS, args.profile_reps, ms))
        print(json.dumps({"profile_case": list(SHAPE), "precision": args.precision,
                          "tiles": ctx.get_tiles(prec, SHAPE), "stage_ms": [ms[0], ms[1], ms[2]],
                          "measure_ms": ms[3]}))
        lat.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["engine", "reference"], default="engine")
    ap.add_argument("--precision", choices=["fp64", "fp32mixed"], default="fp64")
    ap.add_argument("--ref-procs", type=int, default=0)
    ap.add_argument("--ref-shape", default="", help="lattice of the reference's per-process sample, e.g. 48,24,24,24 "
                                                    "(default 16,16,16,16)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-forms", action="store_true", help="skip the forms (volumes, FP32-mixed, batched, served, heatbath)")
    ap.add_argument("--forms", default="all", help="comma list of forms to run (default all)")
    ap.add_argument("--serve-jobs", type=int, default=30, help="jobs per arrival rate of the served form")
    ap.add_argument("--serve-rates", default="0.5,1.0,inf",
                    help="Poisson arrival rates (jobs/s) swept by the served form; inf = all jobs at t = 0")
    ap.add_argument("--profile", action="store_true", help="one launch of each kernel (for ncu captures)")
    ap.add_argument("--profile-reps", type=int, default=1)
    ap.add_argument("--tiles", default="", help='--profile: tile shape fields as JSON, e.g. {"meas_budget_kb": 65536}')
    ap.add_argument("--no-autotune", action="store_true", help="use the default tile shapes instead of tuning them")
    args = ap.parse_args()
    if args.profile:
        profile_case(args)
    elif args.impl == "reference":
        reference_arm(args)
    else:
        engine_arm(args)


if __name__ == "__main__":
    main()
