"""GPU parity: the CUDA engine through the C ABI against the reference's golden
vectors and the CPU oracle, plus size-independent properties.

Tolerances (FP64 plain form): E relative 1e-12; Q as |dQ| <= 1e-12 max(1,|Q|);
links 1e-12 absolute.  The kernels use fused multiply-adds and another
summation order than the reference, so agreement is to rounding, not bitwise.
FP32-mixed form: |dQ| < 1e-3, |dE|/E < 1e-5 against FP64.
"""
import hashlib
import os
import tempfile
from pathlib import Path

import numpy as np
import pytest
from conftest import GOLDEN, golden_json, golden_links, q_err, random_gauge, rel_err

from msc_project_b200 import FP32MIXED, FP64, Job
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-12


def as_mats(a, per):
    return np.asarray(a).reshape(-1, per, 18)


# ------------------------------------------------------------ per function
def test_exp_against_reference(ctx):
    z = np.load(GOLDEN / "exp_cases.npz")
    out = ctx.exp_su3(z["iP"], FP64).reshape(-1, 18)
    assert np.max(np.abs(out - z["exp"])) < 1e-13
    out32 = ctx.exp_su3(z["iP"], FP32MIXED).reshape(-1, 18)
    assert np.max(np.abs(out32 - z["exp"])) < 5e-6


def test_exp_against_expm_over_all_scales(ctx):
    """The series (c1 < 0.25) and closed-form (c1 >= 0.25) coefficient paths
    both agree with a dense matrix exponential to rounding."""
    import scipy.linalg as sl
    rng = np.random.default_rng(11)
    n = 400
    H = rng.normal(size=(n, 3, 3)) + 1j * rng.normal(size=(n, 3, 3))
    H = (H + np.conj(np.transpose(H, (0, 2, 1)))) / 2
    H -= np.trace(H, axis1=1, axis2=2)[:, None, None] / 3 * np.eye(3)
    H /= np.linalg.norm(H, axis=(1, 2))[:, None, None]
    scale = np.exp(rng.uniform(np.log(1e-5), np.log(2.0), size=n))[:, None, None]
    iP = np.ascontiguousarray(1j * H * scale)
    c1 = 0.5 * np.sum(np.abs(H * scale) ** 2, axis=(1, 2))
    assert (c1 < 1e-4).any() and ((c1 > 1e-4) & (c1 < 0.25)).any() and (c1 > 0.25).any()
    ref = np.array([sl.expm(m) for m in iP])
    out = ctx.exp_su3(iP.view(np.float64).reshape(n, 18), FP64).reshape(n, 9, 2)
    got = (out[..., 0] + 1j * out[..., 1]).reshape(n, 3, 3)
    assert np.max(np.abs(got - ref)) < 5e-15


def test_exp_zero_is_identity(ctx):
    out = ctx.exp_su3(np.zeros((3, 18)), FP64).reshape(-1, 9, 2)
    assert np.array_equal(out[:, :, 0], np.tile(np.eye(3).reshape(9), (3, 1)))
    assert not out[:, :, 1].any()


def test_kernels_against_reference(ctx):
    k = np.load(GOLDEN / "kernels_g4466.npz")
    shape = tuple(int(s) for s in k["shape"])
    sites = k["sites"]
    with ctx.lattice(shape, FP64) as lat:
        lat.upload(golden_links("g4466_seed7.bin"))
        grad = as_mats(lat.debug_gradient(), 4)
        assert np.max(np.abs(grad[sites] - k["grad"])) < 1e-13
        clov, impr = lat.debug_fields()
        assert np.max(np.abs(as_mats(clov, 6)[sites] - k["clover"])) < 1e-13
        assert np.max(np.abs(as_mats(impr, 6)[sites] - k["improved"])) < 1e-13
        e, q = lat.site_densities()
        assert np.max(np.abs(e[sites] - k["edens"])) < 1e-12
        assert np.max(np.abs(q[sites] - k["qdens"])) < 1e-12
        lat.flow(0.01, 1, 0, measure_at_t0=False)
        after = as_mats(lat.download(), 4)
        assert np.max(np.abs(after[sites] - k["rk3step"])) < 1e-13


def test_generator_matches_oracle(ctx):
    shape = (4, 4, 6, 6)
    with ctx.lattice(shape, FP64) as lat:
        lat.generate(7, 0.5)
        g = lat.download()
    assert np.max(np.abs(g - golden_links("g4466_seed7.bin"))) < 1e-13


def test_upload_download_roundtrip(ctx):
    U = golden_links("hb8_seed1.bin")
    with ctx.lattice((8, 8, 8, 8), FP64) as lat:
        lat.upload(U)
        assert np.array_equal(lat.download(), U)


# ------------------------------------------------------------- end to end
@pytest.mark.parametrize("name,inp", [("flow_g4466.json", "g4466_seed7.bin"),
                                      ("flow8_hb_seed1.json", "hb8_seed1.bin")])
def test_flow_against_reference(ctx, name, inp):
    g = golden_json(name)
    with ctx.lattice(g["shape"], FP64) as lat:
        lat.upload(golden_links(inp))
        r = lat.flow(g["eps"], g["steps"], g["meas_every"])
        Uf = lat.download()
    assert np.allclose(r.t, g["t"], rtol=0, atol=1e-12)
    assert rel_err(r.E, g["E"]) < TOL
    assert q_err(r.Q, g["Q"]) < TOL
    assert np.max(np.abs(Uf[: len(g["flowed_sample"])] - np.array(g["flowed_sample"]))) < TOL


def test_flow8_links_against_oracle(ctx):
    U = golden_links("hb8_seed1.bin")
    shape = (8, 8, 8, 8)
    _, _, _, Uo = O.flow(U, shape, 0.01, 100, 0)
    with ctx.lattice(shape, FP64) as lat:
        lat.upload(U)
        lat.flow(0.01, 100, 0, measure_at_t0=False)
        Ug = lat.download()
    assert np.max(np.abs(Ug - Uo)) < TOL


def test_flow16_against_reference(ctx):
    g = golden_json("flow16_g7.json")
    with ctx.lattice(g["shape"], FP64) as lat:
        lat.generate(7, 0.5)
        r = lat.flow(g["eps"], g["steps"], g["meas_every"])
    # device-generated inputs differ from the host file by rounding only
    assert rel_err(r.E, g["E"]) < 1e-11
    assert q_err(r.Q, g["Q"]) < 1e-11


def test_dropin_flow_saved_matches_reference_outputs(ctx, tmp_path):
    """FlowSavedGaugeConfigurations end to end: same input tree, same CSV bytes,
    same flowed-file name, links within tolerance of the reference's."""
    from msc_project_b200 import FlowParameters, FlowSavedGaugeConfigurations, SimulationParameters, configure
    g = golden_json("flow8_hb_seed1.json")
    folder = str(tmp_path) + "/"
    d = tmp_path / "ensembles/su3/beta6_000000/8X8X8X8/LHMC_3_of_0_330000"
    d.mkdir(parents=True)
    (d / "torus_extdof4_0.bin").write_bytes((GOLDEN / "hb8_seed1.bin").read_bytes())
    configure(FP64)
    rc = FlowSavedGaugeConfigurations(SimulationParameters(4, 4, [8, 8, 8, 8], 6.0, [0, 0, 0, 0]),
                                      FlowParameters(0, 0, 100, 0.01, 1, folder))
    assert rc == 0
    obs = tmp_path / "Observables"
    csv_q = (obs / "Topological_Charge/beta6_000000/8X8X8X8/GF/torus_extdof4_0.csv").read_text()
    csv_e = (obs / "EnergyDensity/beta6_000000/8X8X8X8/GF/torus_extdof4_0.csv").read_text()
    assert csv_q == g["csv_topcharge"]
    assert csv_e == g["csv_energy"]
    import pandas as pd
    df = pd.read_csv(obs / "EnergyDensity/beta6_000000/8X8X8X8/GF/torus_extdof4_0.csv", index_col="t",
                     names=["t", "E0"], sep=",", header=None)
    assert len(df) == 101 and df.index[0] == 0.0 and abs(df.index[-1] - 1.0) < 1e-12
    flowed = tmp_path / "ensembles/su3/beta6_000000/8X8X8X8/GF" / g["flowed_file"]
    Uf = np.fromfile(flowed)
    assert np.max(np.abs(Uf[: len(g["flowed_sample"])] - np.array(g["flowed_sample"]))) < TOL


def test_resume_continues_the_flow(ctx, tmp_path):
    """Flowing 50 + resume 50 equals flowing 100 (ResumeFlowedConfiguration)."""
    from msc_project_b200 import (FlowParameters, FlowSavedGaugeConfigurations, ResumeFlowedConfiguration,
                                  SimulationParameters, configure)
    configure(FP64)
    folder = str(tmp_path) + "/"
    d = tmp_path / "ensembles/su3/beta6_000000/8X8X8X8/LHMC_3_of_0_330000"
    d.mkdir(parents=True)
    (d / "torus_extdof4_0.bin").write_bytes((GOLDEN / "hb8_seed1.bin").read_bytes())
    p = SimulationParameters(4, 4, [8, 8, 8, 8], 6.0, [0, 0, 0, 0])
    assert FlowSavedGaugeConfigurations(p, FlowParameters(0, 0, 50, 0.01, 10, folder)) == 0
    gf = tmp_path / "ensembles/su3/beta6_000000/8X8X8X8/GF"
    assert (gf / "torus_extdof4_0_Flowtime0.500000.bin").exists()
    assert ResumeFlowedConfiguration(p, FlowParameters(0, 0, 50, 0.01, 10, folder), 0.5) == 0
    g = golden_json("flow8_hb_seed1.json")
    Uf = np.fromfile(gf / "torus_extdof4_0_Flowtime1.000000.bin")
    assert np.max(np.abs(Uf[: len(g["flowed_sample"])] - np.array(g["flowed_sample"]))) < 1e-11
    rows = (tmp_path / "Observables/EnergyDensity/beta6_000000/8X8X8X8/GF/torus_extdof4_0.csv").read_text().split()
    assert len(rows) == 6 + 5  # t=0 and every 10th of 50, then 5 more after the resume


def test_qdensity_output(ctx, tmp_path):
    from msc_project_b200 import FlowParameters, MeasureQdensityDistribution, SimulationParameters, configure
    configure(FP64)
    folder = str(tmp_path) + "/"
    gf = tmp_path / "ensembles/su3/beta6_000000/8X8X8X8/GF"
    gf.mkdir(parents=True)
    U = golden_links("hb8_seed1.bin")
    U.tofile(gf / "torus_extdof4_0_Flowtime1.000000.bin")
    assert MeasureQdensityDistribution(SimulationParameters(4, 4, [8, 8, 8, 8], 6.0, [0, 0, 0, 0]),
                                       FlowParameters(0, 0, 100, 0.01, 1, folder)) == 0
    q = np.fromfile(tmp_path / "Observables/Qdensity/beta6_000000/8X8X8X8/GF/torus_extdof1_0_Flowtime1.000000.bin")
    _, qo = O.site_densities(U, (8, 8, 8, 8))
    assert q.shape == (8 ** 4,)
    assert np.reshape(q[: 8 * 8], (8, 8)).shape == (8, 8)  # the analysis slices x-y planes of this array
    assert np.max(np.abs(q - (np.pi ** 2 / 4) * qo)) < 1e-11  # the reference's pi^2/4 prefactor


def _retr(a, b):
    A = (a[0::2] + 1j * a[1::2]).reshape(3, 3)
    B = (b[0::2] + 1j * b[1::2]).reshape(3, 3)
    return float(np.trace(A @ B).real)


def test_measure_flowed_observables_against_oracle(ctx):
    """ImprovedEnergyDensity (improved F) and UnImprovedTopologicalCharge (clover F)."""
    shape = (4, 4, 6, 6)
    U = golden_links("g4466_seed7.bin")
    with ctx.lattice(shape, FP64) as lat:
        lat.upload(U)
        Ei, Qc = lat.measure_flowed()
    planes = [(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)]
    V = O.volume(shape)
    se = sq = 0.0
    for x in range(V):
        Fh = [O.improved_F(U, shape, x, a, b) for a, b in planes]
        Fc = [O.clover_F(U, shape, x, a, b) for a, b in planes]
        se += sum(_retr(f, f) for f in Fh)
        sq += -_retr(Fc[5], Fc[0]) + _retr(Fc[4], Fc[1]) - _retr(Fc[2], Fc[3])
    assert abs(Ei - se / V) < 1e-12 * abs(se / V)
    assert abs(Qc - sq / (4 * np.pi ** 2)) < 1e-12


def test_dropin_measure_flowed_outputs_read_like_the_analysis(ctx, tmp_path):
    import pandas as pd
    from msc_project_b200 import FlowParameters, MeasureFlowedGaugeConfigurations, SimulationParameters, configure
    configure(FP64)
    shape = [4, 4, 6, 6]
    gf = tmp_path / "ensembles/su3/beta6_000000/4X4X6X6/GF"
    gf.mkdir(parents=True)
    U = golden_links("g4466_seed7.bin")
    U.tofile(gf / "torus_extdof4_0_Flowtime1.000000.bin")
    rc = MeasureFlowedGaugeConfigurations(SimulationParameters(4, 4, shape, 6.0, [0, 0, 0, 0]),
                                          FlowParameters(0, 0, 100, 0.01, 1, str(tmp_path) + "/"))
    assert rc == 0
    with ctx.lattice(shape, FP64) as lat:
        lat.upload(U)
        Ei, Qc = lat.measure_flowed()
    obs = tmp_path / "Observables"
    # read the way the offline analysis reads its CSVs (t as the index, one column per configuration)
    q = pd.read_csv(obs / "UnImprovedTopological_Charge/beta6_000000/4X4X6X6/GF/torus_extdof4_0.csv",
                    index_col="t", names=["t", "Q0"], sep=",", header=None)
    e = pd.read_csv(obs / "ImprovedEnergyDensity/beta6_000000/4X4X6X6/GF/torus_extdof4_0.csv",
                    index_col="t", names=["t", "E0"], sep=",", header=None)
    assert list(q.index) == [1.0] and list(e.index) == [1.0]
    assert abs(q["Q0"].iloc[0] - Qc) <= 5e-6 * max(1.0, abs(Qc))
    assert abs(e["E0"].iloc[0] - Ei) <= 5e-6 * abs(Ei)


# ------------------------------------------------------------- properties
def test_gauge_invariance_and_parity(ctx):
    shape = (8, 8, 8, 8)
    U = golden_links("hb8_seed1.bin")
    Ug = random_gauge(U, shape, 99)
    with ctx.lattice(shape, FP64) as lat:
        lat.upload(U)
        r1 = lat.flow(0.01, 20, 10)
        lat.upload(Ug)
        r2 = lat.flow(0.01, 20, 10)
    assert rel_err(r2.E, r1.E) < 1e-11
    assert q_err(r2.Q, r1.Q) < 1e-11


def test_cold_start_stays_trivial(ctx):
    shape = (4, 4, 4, 8)
    V = O.volume(shape)
    U = np.zeros((V, 4, 9, 2))
    U[:, :, [0, 4, 8], 0] = 1.0
    with ctx.lattice(shape, FP64) as lat:
        lat.upload(U.reshape(-1))
        r = lat.flow(0.01, 5, 1)
        assert np.max(np.abs(lat.download() - U.reshape(-1))) < 1e-15
    assert np.max(np.abs(r.E)) < 1e-28 and np.max(np.abs(r.Q)) < 1e-28


def test_timeslices_sum_to_totals(ctx):
    shape = (8, 8, 8, 8)
    with ctx.lattice(shape, FP64) as lat:
        lat.upload(golden_links("hb8_seed1.bin"))
        r = lat.flow(0.01, 10, 5, slices=True)
    assert np.allclose(r.E_slice.mean(axis=1), r.E, rtol=1e-13)
    assert np.allclose(r.Q_slice.sum(axis=1), r.Q, rtol=0, atol=1e-12)


def test_unitarity_after_flow(ctx):
    with ctx.lattice((8, 8, 8, 8), FP64) as lat:
        lat.upload(golden_links("hb8_seed1.bin"))
        lat.flow(0.01, 100, 0, measure_at_t0=False)
        u, d = lat.unitarity()
    assert u < 1e-13 and d < 1e-13


def test_runs_are_deterministic(ctx):
    outs = []
    for _ in range(2):
        with ctx.lattice((8, 8, 8, 8), FP64) as lat:
            lat.upload(golden_links("hb8_seed1.bin"))
            r = lat.flow(0.01, 10, 5)
            outs.append((r.E.copy(), r.Q.copy(), lat.download()))
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])
    assert np.array_equal(outs[0][2], outs[1][2])


# ----------------------------------------------------------- FP32-mixed
def test_fp32_mixed_accuracy(ctx):
    shape = (8, 8, 8, 8)
    U = golden_links("hb8_seed1.bin")
    g = golden_json("flow8_hb_seed1.json")
    with ctx.lattice(shape, FP32MIXED) as lat:
        lat.upload(U)
        r = lat.flow(0.01, 100, 1, reunit_every=10)
        u, d = lat.unitarity()
    assert q_err(r.Q, g["Q"]) < 1e-3
    assert rel_err(r.E, g["E"]) < 1e-5
    assert u < 1e-5 and d < 1e-5


# ----------------------------------------------------- errors at the ABI
def test_invalid_arguments(ctx):
    from msc_project_b200 import LGFError
    with pytest.raises(LGFError):
        ctx.lattice((8, 8, 7, 8))
    import ctypes
    from msc_project_b200 import _capi as C
    h = ctypes.c_void_p()
    assert ctx.lib.lgf_lattice_create(ctx.h, (ctypes.c_int * 4)(8, 8, 8, 8), 5, ctypes.byref(h)) == C.LGF_EINVAL
    assert "precision" in ctx.error()
    with ctx.lattice((4, 4, 4, 4), FP64) as lat:
        with pytest.raises(ValueError):
            lat.upload(np.zeros(10))


def test_unaligned_volume_against_oracle(ctx):
    """V = 6^4 = 1296 sites is not a whole number of the device layout's
    32-site blocks: the padded tail must never leak into links, E or Q."""
    shape = (6, 6, 6, 6)
    U = O.generate_G(shape, 21, 0.5)
    t, E, Q, Uo = O.flow(U, shape, 0.01, 6, 2)
    with ctx.lattice(shape, FP64) as lat:
        lat.upload(U)
        assert np.array_equal(lat.download(), U)
        r = lat.flow(0.01, 6, 2, slices=True)
        Ug = lat.download()
        e, q = lat.site_densities()
        u, d = lat.unitarity()
    assert rel_err(r.E, E) < 1e-12 and q_err(r.Q, Q) < 1e-12
    assert np.max(np.abs(Ug - Uo)) < TOL
    assert np.allclose(r.E_slice.mean(axis=1), r.E, rtol=1e-13)
    eo, qo = O.site_densities(Uo, shape)
    assert np.max(np.abs(e - eo)) < 1e-12 and np.max(np.abs(q - qo)) < 1e-12
    assert u < 1e-13 and d < 1e-13
    with ctx.lattice(shape, FP64) as lat:
        lat.hot_start(4)
        lat.heatbath(6.0, 2, 1, seed=5)
        p1 = lat.plaquette()
        lat.overrelax(3)
        assert abs(lat.plaquette() - p1) < 1e-13


def test_resume_against_reference(ctx, tmp_path):
    """The reference's own ResumeFlowedConfiguration (LGF.cpp:197-226) run on
    its 8^4 heatbath flow: pick up t = 1.0, 50 steps measuring every 5.  The
    drop-in's appended CSV files are byte-identical, E(t)/Q(t) agree to 1e-12
    and the saved t = 1.5 links to 1e-11."""
    from msc_project_b200 import (FlowParameters, FlowSavedGaugeConfigurations, ResumeFlowedConfiguration,
                                  SimulationParameters, configure)
    g = golden_json("resume8_hb_seed1.json")
    configure(FP64)
    folder = str(tmp_path) + "/"
    d = tmp_path / "ensembles/su3/beta6_000000/8X8X8X8/LHMC_3_of_0_330000"
    d.mkdir(parents=True)
    (d / "torus_extdof4_0.bin").write_bytes((GOLDEN / "hb8_seed1.bin").read_bytes())
    p = SimulationParameters(4, 4, [8, 8, 8, 8], 6.0, [0, 0, 0, 0])
    assert FlowSavedGaugeConfigurations(p, FlowParameters(0, 0, 100, 0.01, 1, folder)) == 0
    gf = tmp_path / "ensembles/su3/beta6_000000/8X8X8X8/GF"
    U1 = np.fromfile(gf / "torus_extdof4_0_Flowtime1.000000.bin")
    assert ResumeFlowedConfiguration(p, FlowParameters(0, 0, 50, 0.01, 5, folder), 1.0) == 0
    obs = tmp_path / "Observables"
    assert (obs / "EnergyDensity/beta6_000000/8X8X8X8/GF/torus_extdof4_0.csv").read_text() == g["csv_energy"]
    assert (obs / "Topological_Charge/beta6_000000/8X8X8X8/GF/torus_extdof4_0.csv").read_text() == g["csv_topcharge"]
    Uf = np.fromfile(gf / g["flowed_file"])
    assert np.max(np.abs(Uf[: len(g["flowed_sample"])] - np.array(g["flowed_sample"]))) < 1e-11
    with ctx.lattice((8, 8, 8, 8), FP64) as lat:
        lat.upload(U1)
        r = lat.flow(0.01, 50, 5, t0=1.0, measure_at_t0=False)
    assert np.array_equal(r.t, np.array(g["t"]))
    assert rel_err(r.E, g["E"]) < 1e-12
    assert q_err(r.Q, g["Q"]) < 1e-12


def test_measure_workflows_against_reference(ctx, tmp_path):
    """The reference's own MeasureFlowedGaugeConfigurations and
    MeasureQdensityDistribution (LGF.cpp:228-255, :113-123) on its 8^4 heatbath
    t = 1.0 links: improved E and clover Q to 1e-12 with byte-identical CSV
    files, and the q-density file (with its pi^2/4 prefactor) to 1e-12."""
    from msc_project_b200 import (FlowParameters, FlowSavedGaugeConfigurations, MeasureFlowedGaugeConfigurations,
                                  MeasureQdensityDistribution, SimulationParameters, configure)
    g = golden_json("measure8_t1.json")
    qref = np.fromfile(GOLDEN / g["qdensity_file"])
    configure(FP64)
    p = SimulationParameters(4, 4, [8, 8, 8, 8], 6.0, [0, 0, 0, 0])
    rel = "ensembles/su3/beta6_000000/8X8X8X8"
    src = tmp_path / "flow"
    (src / rel / "LHMC_3_of_0_330000").mkdir(parents=True)
    (src / rel / "LHMC_3_of_0_330000/torus_extdof4_0.bin").write_bytes((GOLDEN / "hb8_seed1.bin").read_bytes())
    assert FlowSavedGaugeConfigurations(p, FlowParameters(0, 0, 100, 0.01, 1, str(src) + "/")) == 0
    U1 = (src / rel / "GF/torus_extdof4_0_Flowtime1.000000.bin").read_bytes()
    for name in ("measure", "qdensity"):
        (tmp_path / name / rel / "GF").mkdir(parents=True)
        (tmp_path / name / rel / "GF/torus_extdof4_0_Flowtime1.000000.bin").write_bytes(U1)
    fp = lambda name: FlowParameters(0, 0, 100, 0.01, 1, str(tmp_path / name) + "/")  # noqa: E731
    assert MeasureFlowedGaugeConfigurations(p, fp("measure")) == 0
    assert MeasureQdensityDistribution(p, fp("qdensity")) == 0
    obs = tmp_path / "measure/Observables"
    assert (obs / "ImprovedEnergyDensity/beta6_000000/8X8X8X8/GF/torus_extdof4_0.csv").read_text() == g["csv_energy"]
    assert (obs / "UnImprovedTopological_Charge/beta6_000000/8X8X8X8/GF/torus_extdof4_0.csv").read_text() == \
        g["csv_topcharge"]
    q = np.fromfile(tmp_path / "qdensity/Observables/Qdensity/beta6_000000/8X8X8X8/GF/"
                    "torus_extdof1_0_Flowtime1.000000.bin")
    assert q.shape == qref.shape and np.max(np.abs(q - qref)) < 1e-12
    with ctx.lattice((8, 8, 8, 8), FP64) as lat:
        lat.upload(np.frombuffer(U1, dtype=np.float64))
        Ei, Qc = lat.measure_flowed()
    assert abs(Ei - g["E_improved"][0]) < 1e-12 * abs(g["E_improved"][0])
    assert abs(Qc - g["Q_clover"][0]) < 1e-12 * max(1.0, abs(g["Q_clover"][0]))


@pytest.mark.parametrize("prec", [FP64, FP32MIXED])
def test_flow_four_extents_against_reference(ctx, prec):
    """Every axis of a different length (4, 6, 8, 10), generator G seed 9:
    the reference's E(t), Q(t) and flowed links (FP64 to 1e-12; the FP32-mixed
    form within its accuracy gates)."""
    g = golden_json("flow_g46810.json")
    U = O.generate_G(g["shape"], 9, 0.5)
    with ctx.lattice(g["shape"], prec) as lat:
        lat.upload(U)
        r = lat.flow(g["eps"], g["steps"], g["meas_every"], reunit_every=10 if prec == FP32MIXED else 0)
        Uf = lat.download()
    tol = TOL if prec == FP64 else 1e-5
    assert np.allclose(r.t, g["t"], rtol=0, atol=1e-12)
    assert rel_err(r.E, g["E"]) < tol
    assert q_err(r.Q, g["Q"]) < (TOL if prec == FP64 else 1e-3)
    assert np.max(np.abs(Uf[: len(g["flowed_sample"])] - np.array(g["flowed_sample"]))) < (TOL if prec == FP64 else 1e-5)


def test_long_flow_against_oracle(ctx):
    """500 RK3 steps (t = 5) of the 8^4 heatbath input: the flow is contracting,
    so the GPU and the oracle stay together to rounding over a long flow
    (E, Q every 100 steps and the final links)."""
    shape = (8, 8, 8, 8)
    U = golden_links("hb8_seed1.bin")
    t, E, Q, Uo = O.flow(U, shape, 0.01, 500, 100)
    with ctx.lattice(shape, FP64) as lat:
        lat.upload(U)
        r = lat.flow(0.01, 500, 100)
        Ug = lat.download()
        u, d = lat.unitarity()
    assert np.array_equal(r.t, t)
    assert rel_err(r.E, E) < 1e-12 and q_err(r.Q, Q) < 1e-12
    assert np.max(np.abs(Ug - Uo)) < 1e-12
    assert u < 1e-13 and d < 1e-13


def test_dropin_batched_equals_one_by_one(ctx, tmp_path):
    """FlowSavedGaugeConfigurations with its configurations flowed together
    (lgf_dropin_set_batch) writes the same CSV bytes and the same flowed files,
    bit for bit, as flowing them one by one; a missing configuration is
    skipped and reported in both modes."""
    from msc_project_b200 import FlowParameters, FlowSavedGaugeConfigurations, SimulationParameters, configure
    shape = [8, 8, 8, 8]
    outs = {}
    for batch in (1, 3):
        root = tmp_path / f"b{batch}"
        d = root / "ensembles/su3/beta6_000000/8X8X8X8/LHMC_3_of_0_330000"
        d.mkdir(parents=True)
        (d / "torus_extdof4_0.bin").write_bytes((GOLDEN / "hb8_seed1.bin").read_bytes())
        O.generate_G(tuple(shape), 3, 0.5).tofile(d / "torus_extdof4_1.bin")
        O.generate_G(tuple(shape), 4, 0.5).tofile(d / "torus_extdof4_3.bin")  # configuration 2 is missing
        configure(FP64, batch=batch)
        rc = FlowSavedGaugeConfigurations(SimulationParameters(4, 4, shape, 6.0, [0, 0, 0, 0]),
                                          FlowParameters(0, 3, 20, 0.01, 5, str(root) + "/"))
        files = {p.relative_to(root).as_posix(): p.read_bytes() for p in root.rglob("*")
                 if p.is_file() and "LHMC" not in p.as_posix()}
        outs[batch] = (rc, files)
    configure(FP64)
    assert outs[1][0] == outs[3][0] != 0  # the missing configuration is reported
    assert set(outs[1][1]) == set(outs[3][1]) and len(outs[1][1]) == 3 * 3
    for k, v in outs[1][1].items():
        assert outs[3][1][k] == v, k
