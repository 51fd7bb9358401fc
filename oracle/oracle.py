"""CPU ORACLE loader — test infrastructure, not the product.

ctypes bindings to ``oracle/liblgf_oracle.so`` (the plain-C restatement of the
LGF reference's Wilson-flow path, ``oracle/lgf_oracle.c``) and a runner for
``oracle/_ref/lgf_ref`` (the unmodified reference sources built by
``oracle/Makefile``).  Only ``tests/``, ``__graft_entry__.smoke()`` and
``bench.py``'s CPU-baseline leg import this module, and only as the checker.

All link arrays are float64 in the reference's file order: shape
``(V, 4, 3, 3)`` complex128 or ``(V*4*18,)`` float64, global site index with
x0 slowest (LGF/Lattice/Lattice.cpp:423-436).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liblgf_oracle.so"
REF_BIN = HERE / "_ref" / "lgf_ref"

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def build(ref_dir: str | os.PathLike | None = None) -> None:
    """Compile the oracle restatement with oracle/Makefile, and the reference
    harness too when ``ref_dir`` (or the environment variable LGF_REFERENCE)
    names the reference's ``LGF/`` source directory."""
    ref = ref_dir if ref_dir is not None else os.environ.get("LGF_REFERENCE")
    cmd = ["make", "-s", "-C", str(HERE)]
    if ref and (Path(ref) / "LGF.cpp").exists():
        cmd.append(f"REF={Path(ref).resolve()}")
    subprocess.run(cmd, check=True)


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = ctypes.CDLL(str(LIB_PATH))
        L.lgfo_volume.restype = ctypes.c_longlong
        L.lgfo_volume.argtypes = [_ip]
        for name in ("lgfo_staple", "lgfo_flow_gradient"):
            f = getattr(L, name)
            f.restype = None
            f.argtypes = [_dp, _ip, ctypes.c_longlong, ctypes.c_int, _dp]
        for name in ("lgfo_clover_F", "lgfo_improved_F"):
            f = getattr(L, name)
            f.restype = None
            f.argtypes = [_dp, _ip, ctypes.c_longlong, ctypes.c_int, ctypes.c_int, _dp]
        L.lgfo_exp_iP_many.restype = None
        L.lgfo_exp_iP_many.argtypes = [_dp, _dp, ctypes.c_longlong]
        L.lgfo_rk3_step.restype = None
        L.lgfo_rk3_step.argtypes = [_dp, _ip, ctypes.c_double, _dp]
        for name in ("lgfo_energy_density", "lgfo_topological_charge"):
            f = getattr(L, name)
            f.restype = ctypes.c_double
            f.argtypes = [_dp, _ip, _dp]
        L.lgfo_site_densities.restype = None
        L.lgfo_site_densities.argtypes = [_dp, _ip, _dp, _dp]
        L.lgfo_flow.restype = ctypes.c_int
        L.lgfo_flow.argtypes = [_dp, _ip, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                _dp, _dp, _dp]
        L.lgfo_generate_G.restype = None
        L.lgfo_generate_G.argtypes = [_ip, ctypes.c_ulonglong, ctypes.c_double, _dp]
        L.lgfo_unitarity.restype = None
        L.lgfo_unitarity.argtypes = [_dp, ctypes.c_longlong, _dp, _dp]
        _lib = L
    return _lib


def _d(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def _shape(shape) -> ctypes.Array:
    return (ctypes.c_int * 4)(*[int(s) for s in shape])


def volume(shape) -> int:
    return int(np.prod([int(s) for s in shape]))


def as_links(U: np.ndarray) -> np.ndarray:
    """Any view of a link field -> contiguous float64 (V*4*18,)."""
    if np.iscomplexobj(U):
        U = np.ascontiguousarray(U, dtype=np.complex128).view(np.float64)
    return np.ascontiguousarray(U, dtype=np.float64).reshape(-1)


def generate_G(shape, seed: int, scale: float = 0.5) -> np.ndarray:
    """Generator G: U = exp(i*scale*sum_a h_a T^a) per link (file order)."""
    out = np.empty(volume(shape) * 4 * 18, dtype=np.float64)
    lib().lgfo_generate_G(_shape(shape), ctypes.c_ulonglong(seed), scale, _d(out))
    return out


def staple(U, shape, site: int, mu: int) -> np.ndarray:
    out = np.empty(18)
    lib().lgfo_staple(_d(as_links(U)), _shape(shape), site, mu, _d(out))
    return out


def flow_gradient(U, shape, site: int, mu: int) -> np.ndarray:
    out = np.empty(18)
    lib().lgfo_flow_gradient(_d(as_links(U)), _shape(shape), site, mu, _d(out))
    return out


def clover_F(U, shape, site: int, mu: int, nu: int) -> np.ndarray:
    out = np.empty(18)
    lib().lgfo_clover_F(_d(as_links(U)), _shape(shape), site, mu, nu, _d(out))
    return out


def improved_F(U, shape, site: int, mu: int, nu: int) -> np.ndarray:
    out = np.empty(18)
    lib().lgfo_improved_F(_d(as_links(U)), _shape(shape), site, mu, nu, _d(out))
    return out


def exp_iP(iP: np.ndarray) -> np.ndarray:
    a = as_links(iP)
    out = np.empty_like(a)
    lib().lgfo_exp_iP_many(_d(a), _d(out), a.size // 18)
    return out


def rk3_step(U: np.ndarray, shape, eps: float) -> np.ndarray:
    a = as_links(U).copy()
    scratch = np.empty(3 * a.size)
    lib().lgfo_rk3_step(_d(a), _shape(shape), eps, _d(scratch))
    return a


def energy_density(U, shape, per_slice: bool = False):
    a = as_links(U)
    sl = np.empty(int(shape[0]))
    E = lib().lgfo_energy_density(_d(a), _shape(shape), _d(sl))
    return (E, sl) if per_slice else E


def topological_charge(U, shape, per_slice: bool = False):
    a = as_links(U)
    sl = np.empty(int(shape[0]))
    Q = lib().lgfo_topological_charge(_d(a), _shape(shape), _d(sl))
    return (Q, sl) if per_slice else Q


def site_densities(U, shape):
    a = as_links(U)
    V = volume(shape)
    e = np.empty(V)
    q = np.empty(V)
    lib().lgfo_site_densities(_d(a), _shape(shape), _d(e), _d(q))
    return e, q


def flow(U, shape, eps: float, nsteps: int, meas_every: int, t0: float = 0.0):
    """FlowSavedGaugeConfigurations' sequence on one configuration.
    Returns (t, E, Q, U_final)."""
    a = as_links(U).copy()
    nmax = 1 + (nsteps // meas_every if meas_every > 0 else 0)
    t = np.empty(nmax)
    E = np.empty(nmax)
    Q = np.empty(nmax)
    m = lib().lgfo_flow(_d(a), _shape(shape), eps, nsteps, meas_every, t0, _d(t), _d(E), _d(Q))
    if m < 0:
        raise MemoryError("oracle flow scratch allocation failed")
    return t[:m], E[:m], Q[:m], a


def unitarity(U) -> tuple[float, float]:
    a = as_links(U)
    mu = ctypes.c_double()
    md = ctypes.c_double()
    lib().lgfo_unitarity(_d(a), a.size // 18, ctypes.byref(mu), ctypes.byref(md))
    return mu.value, md.value


def reference_available() -> bool:
    return REF_BIN.exists() and os.access(REF_BIN, os.X_OK)


def run_reference(args, env=None, cwd=None, timeout=None) -> subprocess.CompletedProcess:
    """Run the unmodified-reference harness (oracle/_ref/lgf_ref)."""
    if not reference_available():
        raise FileNotFoundError(f"{REF_BIN} not built (make -C oracle)")
    e = dict(os.environ)
    if env:
        e.update(env)
    return subprocess.run([str(REF_BIN), *map(str, args)], capture_output=True, text=True, env=e, cwd=cwd,
                          timeout=timeout, check=True)
