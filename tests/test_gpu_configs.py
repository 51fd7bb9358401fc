"""The throughput configurations at their configured sizes and lengths.

- 16^4 (generator G, seed 7): eps 0.01 to t = 3.0 (300 RK3 steps), E/Q at t = 0
  and every 10 steps, against the LGF reference's own run of the same input
  (tests/golden/flow16_g7_t3.json): E to 1e-12 relative, Q to 1e-12 max(1,|Q|)
  at all 31 measurements, the flowed links of 32 spread sites to 1e-12, and
  through the drop-in FlowSavedGaugeConfigurations the reference's CSV bytes.
- 24^3 x 48 (the bench lattice, x0 = 48; generator G seed 7): 3 RK3 steps
  with E/Q at t = 0 and t = 0.03 against the reference's run
  (tests/golden/flow24x48_g7.json), and the flowed links of 32 spread sites.
- 32^4 FP32-mixed (generator G, seed 11): eps 0.01 to t = 5.0 (500 steps),
  E/Q every 10 steps, FP32 links reunitarised every 10 steps, against the
  FP64 flow of the same configuration: |dQ| < 1e-3 and |dE|/E < 1e-5 at every
  measurement, max ||U^dag U - 1|| < 1e-6 at the end.
- The 64-configuration ensemble of uneven volumes (seeds 100-163), eps 0.01
  to t = 2.0 (200 steps), E/Q every 10 steps, batched, FP32-mixed against
  FP64 under the same gates for every configuration and measurement.

The reference inputs are the host generator's links (oracle.generate_G), so
the GPU and the reference start from the same bits.
"""
import numpy as np
import pytest
from conftest import GOLDEN, golden_json, q_err, rel_err

from msc_project_b200 import FP32MIXED, FP64, Job
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-12
GATE_DQ = 1e-3
GATE_DE = 1e-5
GATE_UNIT = 1e-6


def _sites_of(U, shape, sites):
    V = O.volume(shape)
    return np.asarray(U).reshape(V, 72)[sites]


@pytest.mark.parametrize("name", ["flow16_g7_t3.json", "flow24x48_g7.json"])
def test_configured_flow_against_reference(ctx, name):
    if not (GOLDEN / name).exists():
        pytest.fail(f"golden {name} missing: tests/golden/make_golden.py makes it")
    g = golden_json(name)
    shape = tuple(g["shape"])
    U = O.generate_G(shape, 7, 0.5)
    with ctx.lattice(shape, FP64) as lat:
        lat.upload(U)
        r = lat.flow(g["eps"], g["steps"], g["meas_every"])
        Uf = lat.download()
    assert len(r.E) == len(g["E"])
    assert np.allclose(r.t, g["t"], rtol=0, atol=1e-12)
    assert rel_err(r.E, g["E"]) < TOL
    assert q_err(r.Q, g["Q"]) < TOL
    sites = g["sample_sites"]
    assert np.max(np.abs(_sites_of(Uf, shape, sites) - np.array(g["flowed_sites"]))) < TOL


def test_dropin_16_4_t3_csv_bytes_match_reference(ctx, tmp_path):
    """FlowSavedGaugeConfigurations at t = 3.0 on 16^4 writes the reference's
    CSV text byte for byte and the reference's flowed-file name."""
    from msc_project_b200 import FlowParameters, FlowSavedGaugeConfigurations, SimulationParameters, configure
    g = golden_json("flow16_g7_t3.json")
    shape = tuple(g["shape"])
    folder = str(tmp_path) + "/"
    d = tmp_path / "ensembles/su3/beta6_000000/16X16X16X16/LHMC_3_of_0_330000"
    d.mkdir(parents=True)
    O.generate_G(shape, 7, 0.5).tofile(d / "torus_extdof4_0.bin")
    configure(FP64)
    rc = FlowSavedGaugeConfigurations(SimulationParameters(4, 4, list(shape), 6.0, [0, 0, 0, 0]),
                                      FlowParameters(0, 0, g["steps"], g["eps"], g["meas_every"], folder))
    assert rc == 0
    obs = tmp_path / "Observables"
    assert (obs / "Topological_Charge/beta6_000000/16X16X16X16/GF/torus_extdof4_0.csv").read_text() == \
        g["csv_topcharge"]
    assert (obs / "EnergyDensity/beta6_000000/16X16X16X16/GF/torus_extdof4_0.csv").read_text() == g["csv_energy"]
    flowed = tmp_path / "ensembles/su3/beta6_000000/16X16X16X16/GF" / g["flowed_file"]
    assert np.max(np.abs(_sites_of(np.fromfile(flowed), shape, g["sample_sites"]) -
                         np.array(g["flowed_sites"]))) < TOL


def test_fp32mixed_gates_32_4_t5(ctx):
    shape, steps, meas = (32, 32, 32, 32), 500, 10
    res = {}
    for prec, reunit in ((FP64, 0), (FP32MIXED, 10)):
        with ctx.lattice(shape, prec) as lat:
            lat.generate(11, 0.5)
            r = lat.flow(0.01, steps, meas, reunit_every=reunit)
            u, d = lat.unitarity()
        res[prec] = (r, u, d)
    r64, u64, _ = res[FP64]
    r32, u32, d32 = res[FP32MIXED]
    assert len(r32.E) == len(r64.E) == 1 + steps // meas
    assert np.all(np.abs(r32.Q - r64.Q) < GATE_DQ)
    assert np.all(np.abs(r32.E - r64.E) / np.abs(r64.E) < GATE_DE)
    assert u32 < GATE_UNIT and d32 < GATE_UNIT
    assert u64 < 1e-13


ENSEMBLE = [((8, 8, 8, 8), 16), ((12, 12, 12, 12), 16), ((16, 16, 16, 16), 16), ((32, 16, 16, 16), 8),
            ((48, 24, 24, 24), 8)]


def test_ensemble_of_64_fp32mixed_gates(ctx):
    runs = {}
    for prec, reunit in ((FP64, 0), (FP32MIXED, 10)):
        jobs, seed = [], 100
        for shape, n in ENSEMBLE:
            for _ in range(n):
                jobs.append(Job(shape, prec, seed=seed, nsteps=200, meas_every=10, reunit_every=reunit))
                seed += 1
        st = ctx.batch_run(jobs)
        assert st.site_steps == sum(int(np.prod(s)) * n for s, n in ENSEMBLE) * 200
        runs[prec] = jobs
    assert len(runs[FP64]) == 64
    for a, b in zip(runs[FP32MIXED], runs[FP64]):
        assert len(a.result.E) == len(b.result.E) == 21
        assert np.all(np.abs(a.result.Q - b.result.Q) < GATE_DQ)
        assert np.all(np.abs(a.result.E - b.result.E) / np.abs(b.result.E) < GATE_DE)
