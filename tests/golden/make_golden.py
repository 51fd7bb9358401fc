"""Generate the golden fixtures under tests/golden/ from the LGF reference itself.

Runs oracle/_ref/lgf_ref (the unmodified reference sources compiled by
oracle/Makefile with the single-rank MPI stub and the seed shim) and writes:

  hb8_seed1.bin            8^4 input: reference heatbath, beta=6.0, seed 1,
                           8^4, 200 x (Cabibbo-Marinari + 5 OR) sweeps, saved
                           configuration #0 (reference file layout, 2.36 MB)
  flow8_hb_seed1.json      FlowSavedGaugeConfigurations on it: eps=0.01, 100
                           steps, E(t), Q(t) every step at 17 digits (stdout),
                           the reference's two CSV files verbatim, and the
                           SHA-256 + a sample of the flowed configuration
  g4466_seed7.bin          generator-G input (4x4x6x6, seed 7, scale 0.5)
  kernels_g4466.npz        per-function reference outputs on it (staple, flow
                           gradient, clover F, improved F, e(x), q(x), one RK3
                           step) for every 5th site
  flow_g4466.json          FlowSavedGaugeConfigurations on it: 20 steps, meas every 5
  exp_cases.npz            HermTrLessExp on 512 matrices spanning both branches
  flow16_g7.json           16^4 generator-G seed 7: 10 steps, measure every 5
  flow16_g7_t3.json        16^4 generator-G seed 7 as the throughput
                           configuration runs it: eps=0.01 to t=3.0 (300 steps),
                           E/Q at t=0 and every 10 steps, CSVs, and the flowed
                           links' SHA-256 plus 32 sampled sites
  flow24x48_g7.json        24^3x48 generator-G seed 7 (the bench lattice, x0 = 48):
                           3 steps measuring every 3 (t=0 and t=0.03), flowed
                           links' SHA-256 plus 32 sampled sites

Usage:  python tests/golden/make_golden.py [--reference DIR] [--skip-heatbath] [--skip-16]
                                          [--only small|t3|bench]
The heatbath takes ~3 min and the 8^4 flow ~1.5 min on one core; flow16_g7_t3
about 40 min and flow24x48_g7 about 10 min (--only t3 / --only bench make
just those).
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import re
import shutil
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))
from oracle import oracle as O  # noqa: E402

BETA_DIR = "beta6_000000"
# The reference checkout this script reads (override with --reference or LGF_REFERENCE).
REFERENCE_LGF = os.environ.get("LGF_REFERENCE", "/root/reference/LGF")
N_SAMPLE_SITES = 32


def shape_dir(shape):
    return "X".join(str(s) for s in shape)


def run_ref(args, **kw):
    return O.run_reference(args, **kw)


def parse_stdout(text):
    Q = [float(m) for m in re.findall(r"Topological Charge = (\S+)", text)]
    E = [float(m) for m in re.findall(r"Energy Density\s*= (\S+)", text)]
    return E, Q


def reference_flow(work: Path, links: np.ndarray, shape, steps, eps, meas):
    """Place links under the reference's hard-coded input tag and run
    FlowSavedGaugeConfigurations (LGF/LGF.cpp:163-196) for configuration 0."""
    d = work / "ensembles" / "su3" / BETA_DIR / shape_dir(shape) / "LHMC_3_of_0_330000"
    d.mkdir(parents=True, exist_ok=True)
    links.astype(np.float64).tofile(d / "torus_extdof4_0.bin")
    out = run_ref(["flow", str(work) + "/", "6.0", *shape, 0, 0, steps, eps, meas])
    E, Q = parse_stdout(out.stdout)
    obs = work / "Observables"
    csv_q = (obs / "Topological_Charge" / BETA_DIR / shape_dir(shape) / "GF" / "torus_extdof4_0.csv").read_text()
    csv_e = (obs / "EnergyDensity" / BETA_DIR / shape_dir(shape) / "GF" / "torus_extdof4_0.csv").read_text()
    flowed_dir = work / "ensembles" / "su3" / BETA_DIR / shape_dir(shape) / "GF"
    files = sorted(flowed_dir.glob("*.bin"))
    flowed = np.fromfile(files[0]) if files else None
    return E, Q, csv_e, csv_q, files[0].name if files else None, flowed


def reference_resume(work: Path, out: Path):
    """ResumeFlowedConfiguration (LGF/LGF.cpp:197-226) on the flow above: pick
    up the saved t = 1.0 configuration, 50 more steps measuring every 5; the
    reference appends to the same CSV files and saves the t = 1.5 links."""
    shape = (8, 8, 8, 8)
    r = run_ref(["resume", str(work) + "/", "6.0", *shape, 0, 0, 50, 0.01, 5, "1.0"])
    E, Q = parse_stdout(r.stdout)
    obs = work / "Observables"
    csv_q = (obs / "Topological_Charge" / BETA_DIR / shape_dir(shape) / "GF" / "torus_extdof4_0.csv").read_text()
    csv_e = (obs / "EnergyDensity" / BETA_DIR / shape_dir(shape) / "GF" / "torus_extdof4_0.csv").read_text()
    f = work / "ensembles" / "su3" / BETA_DIR / shape_dir(shape) / "GF" / "torus_extdof4_0_Flowtime1.500000.bin"
    flowed = np.fromfile(f)
    t, tv = 1.0, []
    for s in range(1, 51):
        t += 0.01
        if s % 5 == 0:
            tv.append(t)
    rec = {"shape": list(shape), "beta": 6.0, "eps": 0.01, "steps": 50, "meas_every": 5, "t_pickup": 1.0,
           "input": "the t = 1.0 links of flow8_hb_seed1.json", "t": tv, "E": E, "Q": Q,
           "csv_energy": csv_e, "csv_topcharge": csv_q, "flowed_file": f.name,
           "flowed_sha256": hashlib.sha256(flowed.tobytes()).hexdigest(),
           "flowed_sample": flowed[: 4 * 18 * 2].tolist(),
           "generator": "oracle/_ref/lgf_ref (unmodified LGF sources) via tests/golden/make_golden.py"}
    out.write_text(json.dumps(rec, indent=1))


def reference_measure_workflows(tmp: Path, out_json: Path, out_q: Path):
    """The reference's MeasureQdensityDistribution and
    MeasureFlowedGaugeConfigurations (LGF/LGF.cpp:113-123, :228-255) on the
    8^4 heatbath flow's saved t = 1.0 links (FlowParameters(0, 0, 100, 0.01, 1)),
    each in a fresh folder holding only that file."""
    shape = (8, 8, 8, 8)
    rel = Path("ensembles") / "su3" / BETA_DIR / shape_dir(shape) / "GF"
    src = tmp / "f8" / rel / "torus_extdof4_0_Flowtime1.000000.bin"
    res = {}
    for cmd in ("qdensity", "measureflowed"):
        d = tmp / cmd
        (d / rel).mkdir(parents=True)
        shutil.copy(src, d / rel / src.name)
        res[cmd] = run_ref([cmd, str(d) + "/", "6.0", *shape, 0, 0, 100, 0.01, 1])
    q = np.fromfile(tmp / "qdensity" / "Observables" / "Qdensity" / BETA_DIR / shape_dir(shape) / "GF" /
                    "torus_extdof1_0_Flowtime1.000000.bin")
    q.tofile(out_q)
    E, Q = parse_stdout(res["measureflowed"].stdout)
    obs = tmp / "measureflowed" / "Observables"
    rec = {"shape": list(shape), "beta": 6.0, "flow_time": 1.0, "input": "the t = 1.0 links of flow8_hb_seed1.json",
           "E_improved": E, "Q_clover": Q,
           "csv_energy": (obs / "ImprovedEnergyDensity" / BETA_DIR / shape_dir(shape) / "GF" /
                          "torus_extdof4_0.csv").read_text(),
           "csv_topcharge": (obs / "UnImprovedTopological_Charge" / BETA_DIR / shape_dir(shape) / "GF" /
                             "torus_extdof4_0.csv").read_text(),
           "qdensity_file": out_q.name, "qdensity_sha256": hashlib.sha256(q.tobytes()).hexdigest(),
           "generator": "oracle/_ref/lgf_ref (unmodified LGF sources) via tests/golden/make_golden.py"}
    out_json.write_text(json.dumps(rec, indent=1))


def times(n_meas, eps, meas):
    t, out = 0.0, [0.0]
    for s in range(1, (n_meas - 1) * meas + 1):
        t += eps
        if s % meas == 0:
            out.append(t)
    return out


def write_flow_json(path, shape, steps, eps, meas, input_name, E, Q, csv_e, csv_q, fname, flowed):
    rec = {
        "shape": list(shape), "beta": 6.0, "eps": eps, "steps": steps, "meas_every": meas,
        "input": input_name,
        "t": times(len(E), eps, meas), "E": E, "Q": Q,
        "csv_energy": csv_e, "csv_topcharge": csv_q,
        "flowed_file": fname,
        "flowed_sha256": hashlib.sha256(flowed.tobytes()).hexdigest() if flowed is not None else None,
        "flowed_sample": flowed[: 4 * 18 * 2].tolist() if flowed is not None else None,
        "generator": "oracle/_ref/lgf_ref (unmodified LGF sources) via tests/golden/make_golden.py",
    }
    path.write_text(json.dumps(rec, indent=1))


def sample_sites(V, n=N_SAMPLE_SITES):
    """n sites spread over the lattice (first, last and a prime stride between)."""
    return sorted({0, V - 1, *[(k * 7919 * 97) % V for k in range(1, n - 1)]})[:n]


def write_long_flow_json(path, shape, steps, eps, meas, input_name, E, Q, csv_e, csv_q, fname, flowed):
    """Like write_flow_json, plus the flowed links of a spread of sites (the
    first 72 doubles alone would only cover site 0)."""
    write_flow_json(path, shape, steps, eps, meas, input_name, E, Q, csv_e, csv_q, fname, flowed)
    rec = json.loads(path.read_text())
    V = O.volume(shape)
    sites = sample_sites(V)
    rec["sample_sites"] = sites
    rec["flowed_sites"] = flowed.reshape(V, 4 * 18)[sites].tolist()
    path.write_text(json.dumps(rec, indent=1))


def make_long(tmp: Path, which: str):
    """The throughput configurations at their configured lengths and sizes."""
    if which == "t3":
        shape = (16, 16, 16, 16)
        g = O.generate_G(shape, 7, 0.5)
        res = reference_flow(tmp / "f16t3", g, shape, 300, 0.01, 10)
        write_long_flow_json(HERE / "flow16_g7_t3.json", shape, 300, 0.01, 10,
                             "generator G seed 7 scale 0.5", *res)
    elif which == "bench":
        shape = (48, 24, 24, 24)
        g = O.generate_G(shape, 7, 0.5)
        res = reference_flow(tmp / "f2448", g, shape, 3, 0.01, 3)
        write_long_flow_json(HERE / "flow24x48_g7.json", shape, 3, 0.01, 3,
                             "generator G seed 7 scale 0.5", *res)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=REFERENCE_LGF, help="the reference's LGF/ source directory")
    ap.add_argument("--skip-heatbath", action="store_true")
    ap.add_argument("--skip-16", action="store_true")
    ap.add_argument("--only", choices=("small", "t3", "bench"), default=None,
                    help="make only the small fixtures, or only one of the long flows")
    args = ap.parse_args()
    O.build(args.reference)
    if not O.reference_available():
        sys.exit("reference harness not built: the reference tree is needed to make fixtures")
    if args.only in ("t3", "bench"):
        with tempfile.TemporaryDirectory() as tmp:
            make_long(Path(tmp), args.only)
        print("golden fixtures written to", HERE)
        return
    with tempfile.TemporaryDirectory() as tmp:
        tmp = Path(tmp)
        # ---- 8^4 heatbath input + its flow
        hb = HERE / "hb8_seed1.bin"
        if not args.skip_heatbath or not hb.exists():
            run_ref(["heatbath", str(tmp / "hb") + "/", "6.0", 8, 8, 8, 8, 200, 5], env={"LGF_REF_SEED": "1"})
            src = tmp / "hb" / "ensembles" / "su3" / BETA_DIR / "8X8X8X8" / "Heatbath_5_ORperHB" / "torus_extdof4_0.bin"
            shutil.copy(src, hb)
        links = np.fromfile(hb)
        res = reference_flow(tmp / "f8", links, (8, 8, 8, 8), 100, 0.01, 1)
        write_flow_json(HERE / "flow8_hb_seed1.json", (8, 8, 8, 8), 100, 0.01, 1, hb.name, *res)
        reference_resume(tmp / "f8", HERE / "resume8_hb_seed1.json")
        reference_measure_workflows(tmp, HERE / "measure8_t1.json", HERE / "qdensity8_t1.bin")

        # ---- small generator-G lattice: per-function outputs and a short flow
        shape = (4, 4, 6, 6)
        g = O.generate_G(shape, 7, 0.5)
        g.tofile(HERE / "g4466_seed7.bin")
        run_ref(["kernels", HERE / "g4466_seed7.bin", *shape, str(tmp / "k_")])
        V = O.volume(shape)
        sites = np.arange(0, V, 5)
        fields = {}
        for name, per in (("staple", 4), ("grad", 4), ("clover", 6), ("improved", 6), ("rk3step", 4)):
            a = np.fromfile(tmp / f"k_{name}.bin").reshape(V, per, 18)
            fields[name] = a[sites]
        for name in ("edens", "qdens"):
            fields[name] = np.fromfile(tmp / f"k_{name}.bin")[sites]
        np.savez(HERE / "kernels_g4466.npz", sites=sites, shape=np.array(shape), **fields)
        res = reference_flow(tmp / "fg", g, shape, 20, 0.01, 5)
        write_flow_json(HERE / "flow_g4466.json", shape, 20, 0.01, 5, "g4466_seed7.bin", *res)

        # ---- four different extents (every axis distinguishable), generator G seed 9
        shape = (4, 6, 8, 10)
        g4 = O.generate_G(shape, 9, 0.5)
        g4.tofile(tmp / "g46810.bin")
        res = reference_flow(tmp / "f46810", g4, shape, 20, 0.01, 4)
        write_flow_json(HERE / "flow_g46810.json", shape, 20, 0.01, 4, "generator G seed 9 scale 0.5", *res)

        # ---- exponential on both Cayley-Hamilton branches
        rng = np.random.default_rng(2024)
        n = 512
        H = rng.normal(size=(n, 3, 3)) + 1j * rng.normal(size=(n, 3, 3))
        H = (H + np.conj(np.transpose(H, (0, 2, 1)))) / 2
        H -= np.trace(H, axis1=1, axis2=2)[:, None, None] / 3 * np.eye(3)
        scale = np.exp(rng.uniform(np.log(1e-4), np.log(3.0), size=n))[:, None, None]
        iP = np.ascontiguousarray(1j * H * scale)
        iP.view(np.float64).tofile(tmp / "iP.bin")
        run_ref(["exp", tmp / "iP.bin", tmp / "eo.bin"])
        np.savez(HERE / "exp_cases.npz", iP=iP.view(np.float64).reshape(n, 18),
                 exp=np.fromfile(tmp / "eo.bin").reshape(n, 18))

        # ---- 16^4 generator G, seed 7 (throughput-config lattice), short flow
        if not args.skip_16:
            shape = (16, 16, 16, 16)
            g16 = O.generate_G(shape, 7, 0.5)
            res = reference_flow(tmp / "f16", g16, shape, 10, 0.01, 5)
            write_flow_json(HERE / "flow16_g7.json", shape, 10, 0.01, 5, "generator G seed 7 scale 0.5", *res)
        if args.only is None:
            make_long(tmp, "bench")
            make_long(tmp, "t3")
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
