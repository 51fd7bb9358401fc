"""Properties at the configured sizes, where the CPU reference is too slow to
produce golden values: 24^3 x 48 (the plain FP64 throughput lattice) and 48^4
(the largest served volume); plus edge cases of the ABI."""
import numpy as np
import pytest
from conftest import q_err, random_gauge, rel_err

from msc_project_b200 import FP32MIXED, FP64
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def test_24x24x24x48_gauge_invariance_slices_and_precision_gates(ctx):
    shape = (48, 24, 24, 24)
    with ctx.lattice(shape, FP64) as lat:
        lat.generate(7, 0.5)
        U = lat.download()
        r64 = lat.flow(0.01, 20, 10, slices=True)
        u, d = lat.unitarity()
    assert u < 1e-13 and d < 1e-13
    assert np.allclose(r64.E_slice.mean(axis=1), r64.E, rtol=1e-13)
    assert np.allclose(r64.Q_slice.sum(axis=1), r64.Q, rtol=0, atol=1e-10)
    with ctx.lattice(shape, FP64) as lat:
        lat.upload(random_gauge(U, shape, 123))
        rg = lat.flow(0.01, 20, 10)
    assert rel_err(rg.E, r64.E) < 1e-11
    assert q_err(rg.Q, r64.Q) < 1e-10
    with ctx.lattice(shape, FP32MIXED) as lat:
        lat.upload(U)
        r32 = lat.flow(0.01, 20, 10, reunit_every=10)
    assert rel_err(r32.E, r64.E) < 1e-5 and np.max(np.abs(r32.Q - r64.Q)) < 1e-3


@pytest.mark.parametrize("prec", [FP64, FP32MIXED])
def test_48_4_largest_volume(ctx, prec):
    shape = (48, 48, 48, 48)
    with ctx.lattice(shape, prec) as lat:
        lat.generate(3, 0.5)
        r = lat.flow(0.01, 2, 1, reunit_every=1 if prec == FP32MIXED else 0, slices=True)
        u, _ = lat.unitarity()
    assert np.all(np.isfinite(r.E)) and np.all(np.isfinite(r.Q))
    assert r.E[2] < r.E[1] < r.E[0]  # the flow smooths: E decreases
    assert np.allclose(r.E_slice.mean(axis=1), r.E, rtol=1e-6 if prec == FP32MIXED else 1e-13)
    assert u < (1e-5 if prec == FP32MIXED else 1e-13)


def test_edge_cases(ctx):
    # no steps: only the t0 measurement; no measurement at all; empty batch
    with ctx.lattice((4, 4, 4, 4), FP64) as lat:
        lat.generate(1, 0.5)
        r = lat.flow(0.01, 0, 5)
        assert len(r.E) == 1 and r.t[0] == 0.0
        r = lat.flow(0.01, 3, 0, measure_at_t0=False)
        assert len(r.E) == 0
    st = ctx.batch_run([])
    assert st.site_steps == 0
    # a ragged slice (V/N0 = 6*6*10 = 360, not a multiple of 32) measures like the oracle
    shape = (4, 6, 6, 10)
    U = O.generate_G(shape, 2, 0.5)
    with ctx.lattice(shape, FP64) as lat:
        lat.upload(U)
        E, Q = lat.measure()
    assert abs(E - O.energy_density(U, shape)) < 1e-12 * E
    assert abs(Q - O.topological_charge(U, shape)) < 1e-12


def test_blocked_work_order_matches_oracle(ctx):
    """A lattice whose x0 slice exceeds the L2 block budgets of both kernels
    (stage 8 MB, measurement 2 MB), so both tile lists run in x1-row blocks:
    E, Q and the flowed links agree with the oracle as in plain site order."""
    shape = (4, 20, 18, 18)  # 6480 sites per slice: 9.1 MB of stage work, 3.7 MB of links
    U = O.generate_G(shape, 5, 0.5)
    t, E, Q, Uo = O.flow(U, shape, 0.01, 4, 2)
    with ctx.lattice(shape, FP64) as lat:
        lat.upload(U)
        r = lat.flow(0.01, 4, 2)
        Ug = lat.download()
    assert np.allclose(r.t, t, rtol=0, atol=1e-15)
    assert rel_err(r.E, E) < 1e-12
    assert q_err(r.Q, Q) < 1e-12
    assert np.max(np.abs(Ug - Uo)) < 1e-12
