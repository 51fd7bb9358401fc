"""C-ABI boundary checks that need no GPU: the library loads, exports every
function include/*.h declares, and rejects bad input before touching a device."""
import ctypes
import re
import subprocess

import pytest
from conftest import ROOT

from msc_project_b200 import _capi as C


def declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        for m in re.finditer(r"\b(lgf_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    lib = C.load()
    declared = declared_functions()
    assert len(declared) >= 25
    missing = [n for n in sorted(declared) if not hasattr(lib, n)]
    assert not missing, missing
    # the ctypes table covers the same set
    assert declared == set(C.SIGNATURES)
    out = subprocess.run(["nm", "-D", "--defined-only", str(C.LIB_PATH)], capture_output=True, text=True).stdout
    for n in declared:
        assert re.search(rf"\bT {n}$", out, flags=re.M), n


def test_footprint_and_validation_without_gpu():
    lib = C.load()
    s = (ctypes.c_int * 4)(8, 8, 8, 8)
    b64 = lib.lgf_lattice_footprint(s, C.LGF_PREC_FP64)
    b32 = lib.lgf_lattice_footprint(s, C.LGF_PREC_FP32MIXED)
    V = 8 ** 4
    assert b64 >= V * (3 * 576 + 256) and b32 >= V * (3 * 288 + 128) and b32 < b64
    assert lib.lgf_lattice_footprint((ctypes.c_int * 4)(8, 8, 7, 8), C.LGF_PREC_FP64) == 0  # odd extent
    assert lib.lgf_lattice_footprint((ctypes.c_int * 4)(8, 8, 8, 2), C.LGF_PREC_FP64) == 0  # < 4
    assert lib.lgf_lattice_footprint(s, 7) == 0
    assert lib.lgf_ctx_create(0, None) == C.LGF_EINVAL
    assert lib.lgf_version() >= 10000


def test_dropin_missing_input_reports_io_error(tmp_path):
    lib = C.load()
    s = (ctypes.c_int * 4)(8, 8, 8, 8)
    folder = str(tmp_path) + "/"
    rc = lib.lgf_dropin_flow_saved(s, 6.0, 0, 1, 10, 0.01, 1, folder.encode())
    assert rc == C.LGF_EIO
    # like the reference, the input directory is created on load (SU3_field.cpp:278)
    assert (tmp_path / "ensembles/su3/beta6_000000/8X8X8X8/LHMC_3_of_0_330000").is_dir()


def test_cli_rejects_missing_arguments():
    cli = ROOT / "msc_project_b200" / "lgf_flow"
    r = subprocess.run([str(cli), "4", "4"], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr
