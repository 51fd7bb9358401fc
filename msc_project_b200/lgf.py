"""Python mirror of the reference's flow interface over the C ABI.

The names follow the LGF reference so tests read like its own workflow:
``SimulationParameters`` / ``FlowParameters`` (LGF/SimulationParameters.h),
``FlowSavedGaugeConfigurations`` (LGF/LGF.cpp:163-196),
``ResumeFlowedConfiguration`` (LGF/LGF.cpp:197-226),
``MeasureQdensityDistribution`` (LGF/LGF.cpp:114-124),
``MeasureFlowedGaugeConfigurations`` (LGF/LGF.cpp:228-255) -- these four call the
C++ drop-in inside liblgf_b200.so -- plus ``Context`` / ``Lattice`` for direct
use of the engine (upload, flow, measure, batch, serve).

Link arrays are float64 in the reference's file order (V*4*18).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _capi as C

FP64 = C.LGF_PREC_FP64
FP32MIXED = C.LGF_PREC_FP32MIXED


class LGFError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"LGF status {code}: {msg}")
        self.code = code


def _dp(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _shape(shape) -> ctypes.Array:
    s = [int(x) for x in shape]
    if len(s) != 4:
        raise ValueError("shape must have 4 extents (NrDims = 4)")
    return (ctypes.c_int * 4)(*s)


def volume(shape) -> int:
    return int(np.prod([int(s) for s in shape]))


def precision_code(p) -> int:
    if p in (FP64, "fp64", "FP64"):
        return FP64
    if p in (FP32MIXED, "fp32mixed", "fp32", "FP32MIXED"):
        return FP32MIXED
    raise ValueError(f"unknown precision {p!r}")


@dataclass
class FlowResult:
    t: np.ndarray
    E: np.ndarray
    Q: np.ndarray
    E_slice: np.ndarray | None = None
    Q_slice: np.ndarray | None = None


class Context:
    """One GPU (lgf_ctx)."""

    def __init__(self, device: int = 0):
        self.lib = C.load()
        h = ctypes.c_void_p()
        rc = self.lib.lgf_ctx_create(device, ctypes.byref(h))
        if rc != C.LGF_OK:
            raise LGFError(rc, f"cannot create a context on CUDA device {device}")
        self.h = h
        self.device = device

    def error(self) -> str:
        return self.lib.lgf_last_error(self.h).decode()

    def check(self, rc: int):
        if rc != C.LGF_OK:
            raise LGFError(rc, self.error())

    def close(self):
        if self.h:
            self.lib.lgf_ctx_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def lattice(self, shape, precision=FP64) -> "Lattice":
        return Lattice(self, shape, precision)

    def exp_su3(self, iP: np.ndarray, precision=FP64) -> np.ndarray:
        a = np.ascontiguousarray(iP, dtype=np.float64).reshape(-1)
        out = np.empty_like(a)
        self.check(self.lib.lgf_exp_su3(self.h, precision_code(precision), _dp(a), _dp(out), a.size // 18))
        return out

    def autotune(self, precision, shape) -> int:
        best = ctypes.c_int()
        self.check(self.lib.lgf_autotune(self.h, precision_code(precision), _shape(shape), ctypes.byref(best)))
        return best.value

    def autotune_tiles(self, precision, shape) -> dict:
        """Tune the stage and measurement tile shapes for this volume class; returns the choice."""
        t = C.lgf_tile_shape()
        self.check(self.lib.lgf_autotune_tiles(self.h, precision_code(precision), _shape(shape), ctypes.byref(t)))
        return {f: getattr(t, f) for f, _ in C.lgf_tile_shape._fields_}

    def set_tiles(self, precision, shape, **tiles):
        """Fix the tile shape of this precision and volume class (fields of lgf_tile_shape)."""
        t = C.lgf_tile_shape()
        cur = self.get_tiles(precision, shape)
        cur.update(tiles)
        for f, _ in C.lgf_tile_shape._fields_:
            setattr(t, f, int(cur[f]))
        self.check(self.lib.lgf_set_tiles(self.h, precision_code(precision), _shape(shape), ctypes.byref(t)))

    def get_tiles(self, precision, shape) -> dict:
        t = C.lgf_tile_shape()
        self.check(self.lib.lgf_get_tiles(self.h, precision_code(precision), _shape(shape), ctypes.byref(t)))
        return {f: getattr(t, f) for f, _ in C.lgf_tile_shape._fields_}

    def batch_run(self, jobs: list["Job"]) -> C.lgf_batch_stats:
        arr = (C.lgf_job * len(jobs))()
        for i, j in enumerate(jobs):
            arr[i] = j._struct()
        st = C.lgf_batch_stats()
        self.check(self.lib.lgf_batch_run(self.h, arr, len(jobs), ctypes.byref(st)))
        for j in jobs:
            j._collect()
        return st


class Lattice:
    """A device-resident lattice (lgf_lattice)."""

    def __init__(self, ctx: Context, shape, precision=FP64):
        self.ctx = ctx
        self.lib = ctx.lib
        self.shape = tuple(int(s) for s in shape)
        self.precision = precision_code(precision)
        h = ctypes.c_void_p()
        ctx.check(self.lib.lgf_lattice_create(ctx.h, _shape(self.shape), self.precision, ctypes.byref(h)))
        self.h = h

    @property
    def V(self) -> int:
        return volume(self.shape)

    def close(self):
        if self.h:
            self.lib.lgf_lattice_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def upload(self, links: np.ndarray):
        a = np.ascontiguousarray(links, dtype=np.float64).reshape(-1)
        if a.size != self.V * 72:
            raise ValueError(f"expected {self.V * 72} doubles, got {a.size}")
        self.ctx.check(self.lib.lgf_upload_links(self.h, _dp(a)))

    def download(self) -> np.ndarray:
        out = np.empty(self.V * 72)
        self.ctx.check(self.lib.lgf_download_links(self.h, _dp(out)))
        return out

    def generate(self, seed: int, scale: float = 0.5):
        self.ctx.check(self.lib.lgf_generate_links(self.h, ctypes.c_uint64(seed), scale))

    def flow(self, eps: float, nsteps: int, meas_every: int, t0: float = 0.0, measure_at_t0: bool = True,
             reunit_every: int = 0, slices: bool = False) -> FlowResult:
        o = C.lgf_flow_opts(eps, nsteps, meas_every, t0, 1 if measure_at_t0 else 0, reunit_every)
        n = (1 if measure_at_t0 else 0) + (nsteps // meas_every if meas_every > 0 else 0)
        res = FlowResult(np.zeros(n), np.zeros(n), np.zeros(n))
        if slices:
            res.E_slice = np.zeros((n, self.shape[0]))
            res.Q_slice = np.zeros((n, self.shape[0]))
        m = C.lgf_meas(n, 0, _dp(res.t), _dp(res.E), _dp(res.Q), _dp(res.E_slice), _dp(res.Q_slice))
        self.ctx.check(self.lib.lgf_flow(self.h, ctypes.byref(o), ctypes.byref(m)))
        return res

    def measure(self, slices: bool = False):
        E = ctypes.c_double()
        Q = ctypes.c_double()
        es = np.zeros(self.shape[0]) if slices else None
        qs = np.zeros(self.shape[0]) if slices else None
        self.ctx.check(self.lib.lgf_measure(self.h, ctypes.byref(E), ctypes.byref(Q), _dp(es), _dp(qs)))
        return (E.value, Q.value, es, qs) if slices else (E.value, Q.value)

    def site_densities(self):
        e = np.empty(self.V)
        q = np.empty(self.V)
        self.ctx.check(self.lib.lgf_site_densities(self.h, _dp(e), _dp(q)))
        return e, q

    def hot_start(self, seed: int):
        self.ctx.check(self.lib.lgf_hot_start(self.h, ctypes.c_uint64(seed)))

    def cold_start(self):
        self.ctx.check(self.lib.lgf_cold_start(self.h))

    def heatbath(self, beta: float, n_iter: int, or_per_hb: int, seed: int) -> int:
        """n_iter x (heatbath sweep + or_per_hb overrelaxation sweeps); returns rejected subgroup updates."""
        rej = ctypes.c_uint64()
        self.ctx.check(self.lib.lgf_heatbath(self.h, beta, n_iter, or_per_hb, ctypes.c_uint64(seed),
                                             ctypes.byref(rej)))
        return rej.value

    def overrelax(self, n_sweeps: int):
        self.ctx.check(self.lib.lgf_overrelax(self.h, n_sweeps))

    def plaquette(self) -> float:
        p = ctypes.c_double()
        self.ctx.check(self.lib.lgf_plaquette(self.h, ctypes.byref(p)))
        return p.value

    def measure_flowed(self):
        """(E with the improved F, Q with the clover F): MeasureFlowedGaugeConfigurations' observables."""
        a = ctypes.c_double()
        b = ctypes.c_double()
        self.ctx.check(self.lib.lgf_measure_flowed(self.h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def unitarity(self):
        a = ctypes.c_double()
        b = ctypes.c_double()
        self.ctx.check(self.lib.lgf_unitarity(self.h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def debug_gradient(self) -> np.ndarray:
        out = np.empty(self.V * 72)
        self.ctx.check(self.lib.lgf_debug_gradient(self.h, _dp(out)))
        return out

    def debug_fields(self):
        c = np.empty(self.V * 108)
        i = np.empty(self.V * 108)
        self.ctx.check(self.lib.lgf_debug_fields(self.h, _dp(c), _dp(i)))
        return c, i


@dataclass
class Job:
    """One flow job (lgf_job) for lgf_batch_run / the server."""
    shape: tuple
    precision: int = FP64
    links: np.ndarray | None = None
    seed: int = 0
    gen_scale: float = 0.5
    eps: float = 0.01
    nsteps: int = 0
    meas_every: int = 0
    t0: float = 0.0
    measure_at_t0: bool = True
    reunit_every: int = 0
    want_links: bool = False
    slices: bool = False
    snapshot_prefix: str | None = None  # serving: links at each measurement -> <prefix>_Flowtime<t>.bin
    result: FlowResult | None = None
    links_out: np.ndarray | None = None
    _keep: list = field(default_factory=list, repr=False)

    def nmeas(self) -> int:
        return (1 if self.measure_at_t0 else 0) + (self.nsteps // self.meas_every if self.meas_every > 0 else 0)

    def _struct(self) -> C.lgf_job:
        n = self.nmeas()
        self.result = FlowResult(np.zeros(n), np.zeros(n), np.zeros(n))
        if self.slices:
            self.result.E_slice = np.zeros((n, int(self.shape[0])))
            self.result.Q_slice = np.zeros((n, int(self.shape[0])))
        m = C.lgf_meas(n, 0, _dp(self.result.t), _dp(self.result.E), _dp(self.result.Q),
                       _dp(self.result.E_slice), _dp(self.result.Q_slice))
        lk = None
        if self.links is not None:
            lk = np.ascontiguousarray(self.links, dtype=np.float64).reshape(-1)
        if self.want_links:
            self.links_out = np.empty(volume(self.shape) * 72)
        self._keep = [m, lk]
        j = C.lgf_job()
        j.shape = _shape(self.shape)
        j.precision = precision_code(self.precision)
        j.links = _dp(lk)
        j.seed = self.seed
        j.gen_scale = self.gen_scale
        j.flow = C.lgf_flow_opts(self.eps, self.nsteps, self.meas_every, self.t0, 1 if self.measure_at_t0 else 0,
                                 self.reunit_every)
        j.meas = ctypes.pointer(m)
        j.links_out = _dp(self.links_out)
        if self.snapshot_prefix is not None:
            pref = str(self.snapshot_prefix).encode()
            self._keep.append(pref)
            j.snapshot_prefix = pref
        return j

    def _collect(self):
        pass


class Server:
    """Continuous-batching flow server (lgf_server)."""

    def __init__(self, ctx: Context, hbm_budget_bytes: int, max_active: int = 64, steps_per_tick: int = 1):
        self.ctx = ctx
        self.lib = ctx.lib
        cfg = C.lgf_serve_config(int(hbm_budget_bytes), int(max_active), int(steps_per_tick))
        h = ctypes.c_void_p()
        ctx.check(self.lib.lgf_serve_start(ctx.h, ctypes.byref(cfg), ctypes.byref(h)))
        self.h = h
        self._jobs = {}

    def submit(self, job: Job) -> int:
        s = job._struct()
        job._keep.append(s)
        jid = ctypes.c_uint64()
        rc = self.lib.lgf_serve_submit(self.h, ctypes.byref(s), ctypes.byref(jid))
        if rc != C.LGF_OK:
            raise LGFError(rc, "submit rejected")
        self._jobs[jid.value] = job
        return jid.value

    def stats(self) -> dict:
        """Counters of the running server (lgf_serve_stats_get)."""
        st = C.lgf_serve_stats()
        self.ctx.check(self.lib.lgf_serve_stats_get(self.h, ctypes.byref(st)))
        return {f: getattr(st, f) for f, _ in C.lgf_serve_stats._fields_}

    def poll(self, jid: int):
        st = C.lgf_job_status()
        rc = self.lib.lgf_serve_poll(self.h, ctypes.c_uint64(jid), ctypes.byref(st))
        return rc, st

    def wait(self, jid: int, timeout: float = 600.0) -> C.lgf_job_status:
        st = C.lgf_job_status()
        rc = self.lib.lgf_serve_wait(self.h, ctypes.c_uint64(jid), timeout, ctypes.byref(st))
        if rc != C.LGF_OK:
            raise LGFError(rc, f"wait for job {jid}")
        return st

    def stop(self):
        if self.h:
            self.lib.lgf_serve_stop(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.stop()


# ------------------------------------------------------ reference workflows
class SimulationParameters:
    """LGF/SimulationParameters.h:3-47 (same constructor arguments)."""

    def __init__(self, NrDims, extdofs, shape, beta, cuts, LatticeType="torus"):
        if LatticeType not in ("torus", "torus_OpenT"):
            raise SystemExit("Lattice type was not recognised!\nTry <torus> or <torus_OpenT>")
        self.NrDims, self.extdofs, self.shape, self.beta, self.cuts = NrDims, extdofs, list(shape), beta, list(cuts)
        self.LatticeType = LatticeType


class FlowParameters:
    """LGF/SimulationParameters.h:49-86 (same constructor arguments)."""

    def __init__(self, ConfigurationStart, ConfigurationStop, flowSteps, epsilon, measure_every_nth_step, dataFolder):
        self.start, self.stop, self.flowSteps = ConfigurationStart, ConfigurationStop, flowSteps
        self.epsilon, self.measureEvery, self.dataFolder = epsilon, measure_every_nth_step, dataFolder


def configure(precision=FP64, reunit_every: int = 10, device: int = 0, batch: int = 1):
    """Engine options of the drop-in workflows; batch > 1 flows that many saved
    configurations together in FlowSavedGaugeConfigurations."""
    lib = C.load()
    rc = lib.lgf_dropin_configure(precision_code(precision), reunit_every, device)
    if rc == C.LGF_OK:
        rc = lib.lgf_dropin_set_batch(batch)
    if rc != C.LGF_OK:
        raise LGFError(rc, "bad drop-in configuration")


def FlowSavedGaugeConfigurations(params: SimulationParameters, flowParams: FlowParameters) -> int:
    lib = C.load()
    return lib.lgf_dropin_flow_saved(_shape(params.shape), params.beta, flowParams.start, flowParams.stop,
                                     flowParams.flowSteps, flowParams.epsilon, flowParams.measureEvery,
                                     flowParams.dataFolder.encode())


def ResumeFlowedConfiguration(params, flowParams, flowTime_pickup: float) -> int:
    lib = C.load()
    return lib.lgf_dropin_resume_flowed(_shape(params.shape), params.beta, flowParams.start, flowParams.stop,
                                        flowParams.flowSteps, flowParams.epsilon, flowParams.measureEvery,
                                        flowParams.dataFolder.encode(), flowTime_pickup)


class HBParameters:
    """LGF/SimulationParameters.h:88-124 (same constructor arguments)."""

    def __init__(self, ConfigurationStart, ConfigurationStop, ThermSteps, OR_per_HB, configSep, dataFolder):
        self.start, self.stop, self.ThermSteps = ConfigurationStart, ConfigurationStop, ThermSteps
        self.OR_per_HB, self.configSep, self.dataFolder = OR_per_HB, configSep, dataFolder


def GenerateHeatBathGaugeConfigurations(params, HBparams, seed: int = 1) -> int:
    lib = C.load()
    return lib.lgf_dropin_generate_heatbath(_shape(params.shape), params.beta, HBparams.start, HBparams.stop,
                                            HBparams.ThermSteps, HBparams.OR_per_HB, HBparams.configSep,
                                            HBparams.dataFolder.encode(), ctypes.c_uint64(seed))


def MeasureFlowedGaugeConfigurations(params, flowParams) -> int:
    lib = C.load()
    return lib.lgf_dropin_measure_flowed(_shape(params.shape), params.beta, flowParams.start, flowParams.stop,
                                         flowParams.flowSteps, flowParams.epsilon, flowParams.measureEvery,
                                         flowParams.dataFolder.encode())


def MeasureQdensityDistribution(params, flowParams) -> int:
    lib = C.load()
    return lib.lgf_dropin_measure_qdensity(_shape(params.shape), params.beta, flowParams.start, flowParams.stop,
                                           flowParams.flowSteps, flowParams.epsilon, flowParams.measureEvery,
                                           flowParams.dataFolder.encode())
