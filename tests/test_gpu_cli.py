"""The C++ command-line driver (msc_project_b200/lgf_flow): LGF's positional
arguments (LGF/LGF.cpp:30-31, ParseCLargs :308-373) into the C++ drop-in."""
import subprocess

import numpy as np
import pytest
from conftest import GOLDEN, ROOT, golden_json

pytestmark = pytest.mark.gpu

CLI = ROOT / "msc_project_b200" / "lgf_flow"


def place_hb8_input(tmp_path):
    d = tmp_path / "ensembles/su3/beta6_000000/8X8X8X8/LHMC_3_of_0_330000"
    d.mkdir(parents=True)
    (d / "torus_extdof4_0.bin").write_bytes((GOLDEN / "hb8_seed1.bin").read_bytes())


def test_cli_flow_matches_reference_csv(tmp_path):
    place_hb8_input(tmp_path)
    g = golden_json("flow8_hb_seed1.json")
    r = subprocess.run([str(CLI), "4", "4", "6.0", "8", "8", "8", "8", "0", "0", "0", "0", "0", "0", "100", "0.01",
                        "1", str(tmp_path) + "/"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    obs = tmp_path / "Observables"
    assert (obs / "EnergyDensity/beta6_000000/8X8X8X8/GF/torus_extdof4_0.csv").read_text() == g["csv_energy"]
    assert (obs / "Topological_Charge/beta6_000000/8X8X8X8/GF/torus_extdof4_0.csv").read_text() == g["csv_topcharge"]
    # the reference's stdout lines: Q before E at every measurement
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith(("Topological Charge =", "Energy Density"))]
    assert len(lines) == 2 * 101 and lines[0].startswith("Topological Charge") and lines[1].startswith("Energy Density")
    assert (tmp_path / "ensembles/su3/beta6_000000/8X8X8X8/GF" / g["flowed_file"]).exists()


def test_cli_fp32mixed(tmp_path):
    place_hb8_input(tmp_path)
    r = subprocess.run([str(CLI), "4", "4", "6.0", "8", "8", "8", "8", "0", "0", "0", "0", "0", "0", "100", "0.01",
                        "10", str(tmp_path) + "/", "--precision", "fp32mixed"], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    rows = (tmp_path / "Observables/EnergyDensity/beta6_000000/8X8X8X8/GF/torus_extdof4_0.csv").read_text().split()
    E = np.array([float(x.split(",")[1]) for x in rows])
    Eg = np.array(golden_json("flow8_hb_seed1.json")["E"])[::10]
    assert len(E) == 11 and np.max(np.abs(E - Eg) / Eg) < 2e-5  # 6 printed digits + FP32-mixed error


def test_cli_integer_epsilon_selects_heatbath(tmp_path):
    # ParseCLargs: an integer in the epsilon position is OR_per_HB (heatbath workflow)
    r = subprocess.run([str(CLI), "4", "4", "6.0", "4", "4", "4", "8", "0", "0", "0", "0", "0", "1", "10", "2",
                        "3", str(tmp_path) + "/"], capture_output=True, text=True, timeout=300,
                       env={"LGF_SEED": "5", "PATH": "/usr/bin:/bin"})
    assert r.returncode == 0, r.stderr
    d = tmp_path / "ensembles/su3/beta6_000000/4X4X4X8/Heatbath_2_ORperHB"
    assert sorted(f.name for f in d.glob("*.bin")) == ["torus_extdof4_0.bin", "torus_extdof4_1.bin"]
    assert r.stdout.count("step: ") == 10 + 3
