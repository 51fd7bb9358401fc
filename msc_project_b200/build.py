"""Build the engine in-tree for sm_100a.

    python -m msc_project_b200.build        (or build() from Python)

produces
    msc_project_b200/liblgf_b200.so   CUDA kernels + C ABI (include/lgf_b200.h)
                                      + C++ drop-in host (include/lgf_dropin.h)
    msc_project_b200/lgf_flow         command-line driver with the reference's arguments

with nvcc -gencode arch=compute_100a,code=sm_100a.  Objects go to
msc_project_b200/_build/ and are rebuilt only when a source or header changed.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
HOST = PKG / "host"
BUILD = PKG / "_build"
LIB = PKG / "liblgf_b200.so"
CLI = PKG / "lgf_flow"

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr", *ARCH]
CXXFLAGS = ["-O2", "-std=c++17", "-fPIC", "-Wall"]

CU_SOURCES = ["lgf_engine.cu", "lgf_batch.cu", "lgf_serve.cu", "lgf_tune.cu", "lgf_noalloc.cu", "lgf_heatbath.cu"]
CPP_SOURCES = ["lgf_dropin.cpp"]


def _headers():
    return list(CSRC.glob("*.cuh")) + list((ROOT / "include").glob("*.h"))


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(map(str, cmd)), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {' '.join(map(str, cmd[:3]))} ...")
    return r


def build(verbose: bool = False, ptxas_info: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    hdrs = _headers()
    jobs = []
    objs = []
    for src in CU_SOURCES:
        s = CSRC / src
        if not s.exists():
            continue
        o = BUILD / (s.stem + ".o")
        objs.append(o)
        if _stale(o, [s, *hdrs]) or ptxas_info:
            extra = ["-Xptxas", "-v"] if ptxas_info else []
            jobs.append([NVCC, *NVFLAGS, *extra, "-c", str(s), "-o", str(o)])
    for src in CPP_SOURCES:
        s = HOST / src
        o = BUILD / (s.stem + ".o")
        objs.append(o)
        if _stale(o, [s, *hdrs]):
            jobs.append(["g++", *CXXFLAGS, "-c", str(s), "-o", str(o)])
    with ThreadPoolExecutor(max_workers=4) as ex:
        results = list(ex.map(lambda c: _run(c, verbose), jobs))
    if ptxas_info:
        for r in results:
            sys.stdout.write(r.stderr)
    if _stale(LIB, objs):
        _run([NVCC, "-shared", *ARCH, "-o", str(LIB), *map(str, objs), "--cudart", "static"], verbose)
    main_src = HOST / "lgf_main.cpp"
    if _stale(CLI, [main_src, LIB, *hdrs]):
        _run(["g++", *CXXFLAGS[:-1], "-o", str(CLI), str(main_src), f"-L{PKG}", "-llgf_b200",
              "-Wl,-rpath,$ORIGIN"], verbose)
    return LIB


if __name__ == "__main__":
    build(verbose=True, ptxas_info="--ptxas" in sys.argv)
    print("built", LIB, CLI)
