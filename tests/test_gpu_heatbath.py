"""GPU configuration generation: hot/cold start, Cabibbo-Marinari heatbath and
overrelaxation.  The reference seeds from std::random_device, so the heatbath
is compared statistically with the reference's own heatbath configuration (the
8^4 input, beta = 6.0, 200 x (CM + 5 OR)); overrelaxation has an exact
invariant (the Wilson action)."""
import numpy as np
import pytest
from conftest import GOLDEN, golden_links

from msc_project_b200 import FP32MIXED, FP64

pytestmark = pytest.mark.gpu


def numpy_plaquette(U, shape):
    V = int(np.prod(shape))
    M = (U.reshape(V, 4, 18)[:, :, 0::2] + 1j * U.reshape(V, 4, 18)[:, :, 1::2]).reshape(V, 4, 3, 3)
    idx = np.arange(V).reshape(shape)
    tot = 0.0
    for mu in range(4):
        for nu in range(mu + 1, 4):
            xpm = np.roll(idx, -1, axis=mu).reshape(-1)
            xpn = np.roll(idx, -1, axis=nu).reshape(-1)
            P = M[:, mu] @ M[xpm, nu] @ np.conj(np.transpose(M[xpn, mu], (0, 2, 1))) @ np.conj(
                np.transpose(M[:, nu], (0, 2, 1)))
            tot += np.trace(P, axis1=1, axis2=2).real.sum()
    return tot / (3 * 6 * V)


def test_plaquette_matches_numpy(ctx):
    U = golden_links("hb8_seed1.bin")
    with ctx.lattice((8, 8, 8, 8), FP64) as lat:
        lat.upload(U)
        p = lat.plaquette()
    assert abs(p - numpy_plaquette(U, (8, 8, 8, 8))) < 1e-13


def test_starts(ctx):
    with ctx.lattice((4, 4, 4, 8), FP64) as lat:
        lat.cold_start()
        assert lat.plaquette() == 1.0
        lat.hot_start(3)
        u, d = lat.unitarity()
        assert u < 1e-14 and d < 1e-14
        assert abs(lat.plaquette()) < 0.05  # random links: plaquette ~ 0


def test_overrelaxation_keeps_the_action(ctx):
    for prec, tol in ((FP64, 1e-13), (FP32MIXED, 2e-6)):
        with ctx.lattice((8, 8, 8, 8), prec) as lat:
            lat.hot_start(5)
            lat.heatbath(6.0, 5, 0, seed=9)
            p1 = lat.plaquette()
            lat.overrelax(4)
            p2 = lat.plaquette()
            assert abs(p2 - p1) < tol, (prec, p1, p2)
            lat.heatbath(6.0, 1, 0, seed=10)
            assert abs(lat.plaquette() - p1) > 1e-6  # the heatbath does change it


def test_heatbath_reproducible_by_seed(ctx):
    out = []
    for seed in (7, 7, 8):
        with ctx.lattice((4, 4, 4, 4), FP64) as lat:
            lat.hot_start(1)
            lat.heatbath(6.0, 3, 2, seed=seed)
            out.append(lat.download())
    assert np.array_equal(out[0], out[1])
    assert not np.array_equal(out[0], out[2])


def test_heatbath_thermalises_like_the_reference(ctx):
    """Average plaquette after 200 x (CM + 5 OR) at beta = 6.0 on 8^4: four
    GPU chains against the reference's own configuration (seed 1) and the
    large-volume value 0.5937; single 8^4 configurations fluctuate by ~0.002."""
    p_ref = numpy_plaquette(golden_links("hb8_seed1.bin"), (8, 8, 8, 8))
    ps = []
    for seed in (1, 2, 3, 4):
        with ctx.lattice((8, 8, 8, 8), FP64) as lat:
            lat.hot_start(seed)
            rej = lat.heatbath(6.0, 200, 5, seed=100 + seed)
            assert rej <= 10  # of 9.8 million subgroup updates, the bounded rejection loop may give up on a few
            u, d = lat.unitarity()
            assert u < 1e-12 and d < 1e-12
            ps.append(lat.plaquette())
    ps = np.array(ps)
    assert np.all(np.abs(ps - 0.5937) < 0.01), ps
    assert abs(ps.mean() - p_ref) < 0.006, (ps, p_ref)


def test_dropin_generate_heatbath_files(ctx, tmp_path):
    from msc_project_b200 import GenerateHeatBathGaugeConfigurations, HBParameters, SimulationParameters, configure
    configure(FP64)
    p = SimulationParameters(4, 4, [4, 4, 4, 8], 6.0, [0, 0, 0, 0])
    folder = str(tmp_path) + "/"
    assert GenerateHeatBathGaugeConfigurations(p, HBParameters(0, 2, 20, 2, 5, folder), seed=3) == 0
    d = tmp_path / "ensembles/su3/beta6_000000/4X4X4X8/Heatbath_2_ORperHB"
    files = sorted(f.name for f in d.glob("*.bin"))
    assert files == ["torus_extdof4_0.bin", "torus_extdof4_1.bin", "torus_extdof4_2.bin"]
    for f in files:
        U = np.fromfile(d / f)
        assert U.size == 4 * 4 * 4 * 8 * 72
        assert 0.3 < numpy_plaquette(U, (4, 4, 4, 8)) < 0.8
    # continuing an ensemble loads configuration `start` (LGF.cpp:146-148)
    assert GenerateHeatBathGaugeConfigurations(p, HBParameters(2, 3, 0, 2, 5, folder), seed=4) == 0
    assert (d / "torus_extdof4_3.bin").exists()


def test_heatbath_ensemble_matches_the_reference(ctx):
    """Statistical parity with the reference's own heatbath ensemble (nine
    configurations, seeds 1..9, 200 x (CM + 5 OR) at beta 6.0 on 8^4): twelve
    GPU chains give the same mean plaquette and mean E, |Q| after flowing to
    t = 1.0, within three standard errors of the difference.  The GPU chains
    are reproducible by seed, so the check is deterministic."""
    from conftest import golden_json
    g = golden_json("hb8_ensemble.json")
    ref = {k: np.array([c[k] for c in g["configs"]]) for k in ("plaquette", "E_t1", "Q_t1")}
    gpu = {k: [] for k in ref}
    for i in range(12):
        with ctx.lattice((8, 8, 8, 8), FP64) as lat:
            lat.hot_start(200 + i)
            assert lat.heatbath(6.0, 200, 5, seed=300 + i) <= 10
            gpu["plaquette"].append(lat.plaquette())
            r = lat.flow(0.01, 100, 100)
            gpu["E_t1"].append(r.E[-1])
            gpu["Q_t1"].append(r.Q[-1])
    for k, f in (("plaquette", lambda x: x), ("E_t1", lambda x: x), ("Q_t1", np.abs)):
        a, b = f(np.array(gpu[k])), f(ref[k])
        se = np.sqrt(a.var(ddof=1) / len(a) + b.var(ddof=1) / len(b))
        assert abs(a.mean() - b.mean()) < 3 * se, (k, a.mean(), b.mean(), se)
