"""ctypes bindings to liblgf_b200.so (declarations mirror include/lgf_b200.h
and include/lgf_dropin.h).  Loading fails loudly when the library is missing:
there is no CPU fallback."""
from __future__ import annotations

import ctypes
from pathlib import Path

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "liblgf_b200.so"

LGF_OK = 0
LGF_EINVAL = -1
LGF_ENOMEM = -2
LGF_ECUDA = -3
LGF_EIO = -4
LGF_ETIMEDOUT = -5
LGF_ENOTFOUND = -6
LGF_EBUSY = -7
LGF_ESHUTDOWN = -8
LGF_ETOOBIG = -9

LGF_PREC_FP64 = 0
LGF_PREC_FP32MIXED = 1

LGF_JOB_QUEUED, LGF_JOB_RUNNING, LGF_JOB_DONE, LGF_JOB_FAILED = 0, 1, 2, 3

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_vp = ctypes.c_void_p


class lgf_meas(ctypes.Structure):
    _fields_ = [("capacity", ctypes.c_int), ("count", ctypes.c_int), ("t", _dp), ("E", _dp), ("Q", _dp),
                ("E_slice", _dp), ("Q_slice", _dp)]


class lgf_flow_opts(ctypes.Structure):
    _fields_ = [("eps", ctypes.c_double), ("nsteps", ctypes.c_int), ("meas_every", ctypes.c_int),
                ("t0", ctypes.c_double), ("measure_at_t0", ctypes.c_int), ("reunit_every", ctypes.c_int)]


class lgf_job(ctypes.Structure):
    _fields_ = [("shape", ctypes.c_int * 4), ("precision", ctypes.c_int), ("links", _dp), ("seed", ctypes.c_uint64),
                ("gen_scale", ctypes.c_double), ("flow", lgf_flow_opts), ("meas", ctypes.POINTER(lgf_meas)),
                ("links_out", _dp), ("snapshot_prefix", ctypes.c_char_p)]


class lgf_batch_stats(ctypes.Structure):
    _fields_ = [("seconds", ctypes.c_double), ("site_steps", ctypes.c_double), ("launches", ctypes.c_int),
                ("block_threads", ctypes.c_int)]


class lgf_tile_shape(ctypes.Structure):
    _fields_ = [("stage_threads", ctypes.c_int), ("stage_order", ctypes.c_int), ("stage_budget_kb", ctypes.c_int),
                ("meas_budget_kb", ctypes.c_int), ("meas_split", ctypes.c_int)]


class lgf_serve_config(ctypes.Structure):
    _fields_ = [("hbm_budget_bytes", ctypes.c_size_t), ("max_active", ctypes.c_int), ("steps_per_tick", ctypes.c_int)]


class lgf_serve_stats(ctypes.Structure):
    _fields_ = [("wall_s", ctypes.c_double), ("device_busy_s", ctypes.c_double), ("ticks", ctypes.c_longlong),
                ("steps", ctypes.c_longlong), ("measurements", ctypes.c_longlong), ("jobs_done", ctypes.c_longlong),
                ("snapshots", ctypes.c_longlong)]


class lgf_job_status(ctypes.Structure):
    _fields_ = [("state", ctypes.c_int), ("error", ctypes.c_int), ("submit_s", ctypes.c_double),
                ("start_s", ctypes.c_double), ("end_s", ctypes.c_double), ("steps_done", ctypes.c_int)]


# name -> (restype, argtypes); every symbol include/*.h declares
SIGNATURES = {
    "lgf_version": (ctypes.c_int, []),
    "lgf_ctx_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(_vp)]),
    "lgf_ctx_destroy": (ctypes.c_int, [_vp]),
    "lgf_last_error": (ctypes.c_char_p, [_vp]),
    "lgf_lattice_create": (ctypes.c_int, [_vp, _ip, ctypes.c_int, ctypes.POINTER(_vp)]),
    "lgf_lattice_destroy": (ctypes.c_int, [_vp]),
    "lgf_lattice_footprint": (ctypes.c_size_t, [_ip, ctypes.c_int]),
    "lgf_upload_links": (ctypes.c_int, [_vp, _dp]),
    "lgf_download_links": (ctypes.c_int, [_vp, _dp]),
    "lgf_generate_links": (ctypes.c_int, [_vp, ctypes.c_uint64, ctypes.c_double]),
    "lgf_flow": (ctypes.c_int, [_vp, ctypes.POINTER(lgf_flow_opts), ctypes.POINTER(lgf_meas)]),
    "lgf_measure": (ctypes.c_int, [_vp, _dp, _dp, _dp, _dp]),
    "lgf_site_densities": (ctypes.c_int, [_vp, _dp, _dp]),
    "lgf_unitarity": (ctypes.c_int, [_vp, _dp, _dp]),
    "lgf_measure_flowed": (ctypes.c_int, [_vp, _dp, _dp]),
    "lgf_debug_gradient": (ctypes.c_int, [_vp, _dp]),
    "lgf_debug_fields": (ctypes.c_int, [_vp, _dp, _dp]),
    "lgf_exp_su3": (ctypes.c_int, [_vp, ctypes.c_int, _dp, _dp, ctypes.c_longlong]),
    "lgf_profile_kernels": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_int, _dp]),
    "lgf_last_flow_seconds": (ctypes.c_int, [_vp, _dp]),
    "lgf_measure_noalloc": (ctypes.c_int, [_dp, _ip, _dp, _vp]),
    "lgf_hot_start": (ctypes.c_int, [_vp, ctypes.c_uint64]),
    "lgf_cold_start": (ctypes.c_int, [_vp]),
    "lgf_heatbath": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_uint64,
                                    ctypes.POINTER(ctypes.c_uint64)]),
    "lgf_plaquette": (ctypes.c_int, [_vp, _dp]),
    "lgf_overrelax": (ctypes.c_int, [_vp, ctypes.c_int]),
    "lgf_batch_run": (ctypes.c_int, [_vp, ctypes.POINTER(lgf_job), ctypes.c_int, ctypes.POINTER(lgf_batch_stats)]),
    "lgf_autotune": (ctypes.c_int, [_vp, ctypes.c_int, _ip, _ip]),
    "lgf_autotune_tiles": (ctypes.c_int, [_vp, ctypes.c_int, _ip, ctypes.POINTER(lgf_tile_shape)]),
    "lgf_set_tiles": (ctypes.c_int, [_vp, ctypes.c_int, _ip, ctypes.POINTER(lgf_tile_shape)]),
    "lgf_get_tiles": (ctypes.c_int, [_vp, ctypes.c_int, _ip, ctypes.POINTER(lgf_tile_shape)]),
    "lgf_serve_start": (ctypes.c_int, [_vp, ctypes.POINTER(lgf_serve_config), ctypes.POINTER(_vp)]),
    "lgf_serve_submit": (ctypes.c_int, [_vp, ctypes.POINTER(lgf_job), ctypes.POINTER(ctypes.c_uint64)]),
    "lgf_serve_poll": (ctypes.c_int, [_vp, ctypes.c_uint64, ctypes.POINTER(lgf_job_status)]),
    "lgf_serve_wait": (ctypes.c_int, [_vp, ctypes.c_uint64, ctypes.c_double, ctypes.POINTER(lgf_job_status)]),
    "lgf_serve_stop": (ctypes.c_int, [_vp]),
    "lgf_serve_stats_get": (ctypes.c_int, [_vp, ctypes.POINTER(lgf_serve_stats)]),
    "lgf_dropin_configure": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "lgf_dropin_set_batch": (ctypes.c_int, [ctypes.c_int]),
    "lgf_dropin_flow_saved": (ctypes.c_int, [_ip, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_double, ctypes.c_int, ctypes.c_char_p]),
    "lgf_dropin_resume_flowed": (ctypes.c_int, [_ip, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                ctypes.c_double, ctypes.c_int, ctypes.c_char_p, ctypes.c_double]),
    "lgf_dropin_measure_flowed": (ctypes.c_int, [_ip, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                 ctypes.c_double, ctypes.c_int, ctypes.c_char_p]),
    "lgf_dropin_generate_heatbath": (ctypes.c_int, [_ip, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                    ctypes.c_int, ctypes.c_int, ctypes.c_char_p, ctypes.c_uint64]),
    "lgf_dropin_measure_qdensity": (ctypes.c_int, [_ip, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                   ctypes.c_double, ctypes.c_int, ctypes.c_char_p]),
}

_lib = None


def load(path: Path | None = None) -> ctypes.CDLL:
    """Load liblgf_b200.so (built in-tree by msc_project_b200.build, or the
    file named by $LGF_LIB).  Raises if it is missing or lacks a declared
    symbol."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    import os
    p = Path(path) if path else Path(os.environ.get("LGF_LIB", LIB_PATH))
    if not p.exists():
        raise RuntimeError(f"{p} is missing: build it with `python -m msc_project_b200.build` "
                           "(the engine has no CPU fallback)")
    lib = ctypes.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)  # AttributeError if the symbol is not exported
        f.restype = res
        f.argtypes = args
    if path is None:
        _lib = lib
    return lib
