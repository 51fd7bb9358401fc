"""The engine's index arithmetic and work lists, checked on the CPU.

msc_project_b200/csrc/lgf_check_index.cu is compiled here with -DLGF_CHECKED,
which makes every host-side use of the lattice index helpers assert that
coordinates, directions and site indices stay in range, and run on small
lattices (distinct extents, ragged slices, tails shorter than a layout
block).  It compares the neighbours of the staple and the measurement's loop
walks with plain coordinate arithmetic, checks that the device layout is a
bijection into the padded buffers, and that every tile list covers each tile
once.  Host code only: no GPU is used."""
import os
import shutil
import subprocess

import pytest
from conftest import ROOT

NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"


@pytest.mark.skipif(not os.path.exists(NVCC), reason="nvcc not available")
def test_index_arithmetic_checked_build(tmp_path):
    exe = tmp_path / "lgf_check_index"
    src = ROOT / "msc_project_b200" / "csrc" / "lgf_check_index.cu"
    subprocess.run([NVCC, "-std=c++17", "-O1", "-DLGF_CHECKED", "--expt-relaxed-constexpr",
                    "-gencode", "arch=compute_100a,code=sm_100a", "-o", str(exe), str(src)], check=True,
                   capture_output=True, text=True, timeout=600)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "index check ok" in r.stdout
