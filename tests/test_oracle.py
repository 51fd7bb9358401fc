"""The CPU oracle (oracle/lgf_oracle.c) against the golden vectors made by the
LGF reference itself (tests/golden/make_golden.py)."""
import hashlib

import numpy as np
import pytest
from conftest import GOLDEN, golden_json, golden_links, q_err, rel_err

from oracle import oracle as O


@pytest.fixture(scope="module")
def kern():
    return np.load(GOLDEN / "kernels_g4466.npz")


def test_generator_matches_fixture():
    g = O.generate_G((4, 4, 6, 6), 7, 0.5)
    assert np.array_equal(g, golden_links("g4466_seed7.bin"))


def test_per_function_against_reference(kern):
    shape = tuple(int(s) for s in kern["shape"])
    U = golden_links("g4466_seed7.bin")
    planes = [(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)]
    for k, s in enumerate(kern["sites"]):
        s = int(s)
        for mu in range(4):
            assert np.array_equal(O.staple(U, shape, s, mu), kern["staple"][k, mu])
            assert np.array_equal(O.flow_gradient(U, shape, s, mu), kern["grad"][k, mu])
        for p, (a, b) in enumerate(planes):
            assert np.max(np.abs(O.clover_F(U, shape, s, a, b) - kern["clover"][k, p])) < 1e-14
            assert np.max(np.abs(O.improved_F(U, shape, s, a, b) - kern["improved"][k, p])) < 1e-14
    e, q = O.site_densities(U, shape)
    sites = kern["sites"]
    assert np.max(np.abs(e[sites] - kern["edens"])) < 1e-13
    assert np.max(np.abs(q[sites] - kern["qdens"])) < 1e-13
    # one RK3 step is bit-identical to GradientFlow::flow
    r = O.rk3_step(U, shape, 0.01).reshape(-1, 4, 18)
    assert np.array_equal(r[sites], kern["rk3step"])


def test_exp_both_branches_bit_exact():
    z = np.load(GOLDEN / "exp_cases.npz")
    out = O.exp_iP(z["iP"]).reshape(-1, 18)
    assert np.array_equal(out, z["exp"])
    # both Cayley-Hamilton branches are exercised (c1 <= 1e-4 and > 1e-4)
    iP = z["iP"].reshape(-1, 9, 2)
    c1 = 0.5 * np.sum(iP ** 2, axis=(1, 2))
    assert (c1 <= 1e-4).any() and (c1 > 1e-4).any()


@pytest.mark.parametrize("name,inp", [("flow_g4466.json", "g4466_seed7.bin"), ("flow8_hb_seed1.json", "hb8_seed1.bin")])
def test_oracle_flow_against_reference(name, inp):
    g = golden_json(name)
    t, E, Q, Uf = O.flow(golden_links(inp), g["shape"], g["eps"], g["steps"], g["meas_every"])
    assert np.allclose(t, g["t"], rtol=0, atol=1e-12)
    assert rel_err(E, g["E"]) < 1e-12
    assert q_err(Q, g["Q"]) < 1e-12
    # the flowed configuration is byte-identical to the reference's saved file
    assert hashlib.sha256(Uf.tobytes()).hexdigest() == g["flowed_sha256"]


def test_oracle_flow_16():
    g = golden_json("flow16_g7.json")
    U = O.generate_G(g["shape"], 7, 0.5)
    t, E, Q, Uf = O.flow(U, g["shape"], g["eps"], g["steps"], g["meas_every"])
    assert rel_err(E, g["E"]) < 1e-12
    assert q_err(Q, g["Q"]) < 1e-12
    assert hashlib.sha256(Uf.tobytes()).hexdigest() == g["flowed_sha256"]


def test_oracle_resume_against_reference():
    """Continuing the oracle's t = 1.0 links (byte-identical to the reference's)
    for 50 steps reproduces the reference's ResumeFlowedConfiguration: E/Q at
    every measurement and the saved t = 1.5 file byte for byte."""
    g8 = golden_json("flow8_hb_seed1.json")
    g = golden_json("resume8_hb_seed1.json")
    U = golden_links("hb8_seed1.bin")
    _, _, _, U1 = O.flow(U, (8, 8, 8, 8), 0.01, 100, 0)
    assert hashlib.sha256(U1.tobytes()).hexdigest() == g8["flowed_sha256"]
    t, E, Q, U2 = O.flow(U1, (8, 8, 8, 8), 0.01, 50, 5, 1.0)
    assert np.array_equal(t[1:], np.array(g["t"]))  # the reference does not measure at the pickup time
    assert rel_err(E[1:], g["E"]) < 1e-12
    assert q_err(Q[1:], g["Q"]) < 1e-12
    assert hashlib.sha256(U2.tobytes()).hexdigest() == g["flowed_sha256"]


def test_oracle_qdensity_against_reference():
    """The oracle's per-site q(x) on its t = 1.0 links (byte-identical to the
    reference's) times the reference's pi^2/4 prefactor equals the q-density
    file the reference's MeasureQdensityDistribution wrote."""
    g = golden_json("measure8_t1.json")
    qref = np.fromfile(GOLDEN / g["qdensity_file"])
    _, _, _, U1 = O.flow(golden_links("hb8_seed1.bin"), (8, 8, 8, 8), 0.01, 100, 0)
    _, q = O.site_densities(U1, (8, 8, 8, 8))
    assert np.max(np.abs((np.pi ** 2 / 4) * q - qref)) < 1e-13


def test_oracle_flow_four_extents():
    """Every axis of a different length (4, 6, 8, 10): E/Q and the flowed file
    match the reference's, so no two directions are mixed up."""
    g = golden_json("flow_g46810.json")
    U = O.generate_G(g["shape"], 9, 0.5)
    t, E, Q, Uf = O.flow(U, g["shape"], g["eps"], g["steps"], g["meas_every"])
    assert rel_err(E, g["E"]) < 1e-12 and q_err(Q, g["Q"]) < 1e-12
    assert hashlib.sha256(Uf.tobytes()).hexdigest() == g["flowed_sha256"]
