"""Tile shapes: every launch shape and work order the autotuner can choose
gives bit-identical results (only block shapes and tile order change, and no
reduction runs in tile order), and the autotuner's choice is one of them."""
import itertools

import numpy as np
import pytest

from msc_project_b200 import FP32MIXED, FP64
from oracle import oracle as O

pytestmark = pytest.mark.gpu

# 6480 sites per x0 slice: with the small budgets below both kernels cut the
# slices into (x1, x2) blocks; with the large ones they take whole slices
SHAPE = (4, 20, 18, 18)


def _flow(ctx, prec, U):
    with ctx.lattice(SHAPE, prec) as lat:
        lat.upload(U)
        r = lat.flow(0.01, 4, 2, reunit_every=2 if prec == FP32MIXED else 0, slices=True)
        return r, lat.download()


@pytest.mark.parametrize("prec", [FP64, FP32MIXED])
def test_every_tile_shape_gives_identical_results(ctx, prec):
    U = O.generate_G(SHAPE, 21, 0.5)
    combos = list(itertools.product([128, 256], [0, 1], [256, 8192], [1, 2], [64, 4096]))
    rng = np.random.default_rng(0)
    picks = [combos[i] for i in rng.choice(len(combos), size=10, replace=False)]
    ref = None
    for threads, order, sb, ms, mb in picks:
        ctx.set_tiles(prec, SHAPE, stage_threads=threads, stage_order=order, stage_budget_kb=sb, meas_split=ms,
                      meas_budget_kb=mb)
        assert ctx.get_tiles(prec, SHAPE)["stage_threads"] == threads
        r, Uf = _flow(ctx, prec, U)
        if ref is None:
            ref = (r, Uf)
            continue
        assert np.array_equal(r.E, ref[0].E) and np.array_equal(r.Q, ref[0].Q)
        assert np.array_equal(r.E_slice, ref[0].E_slice) and np.array_equal(r.Q_slice, ref[0].Q_slice)
        assert np.array_equal(Uf, ref[1])


def test_autotuner_choice_is_valid_and_used(ctx):
    U = O.generate_G(SHAPE, 22, 0.5)
    before, _ = _flow(ctx, FP64, U)
    t = ctx.autotune_tiles(FP64, SHAPE)
    assert t["stage_threads"] in (128, 256, 384) and t["stage_order"] in (0, 1) and t["meas_split"] in (1, 2)
    assert t["stage_budget_kb"] > 0 and t["meas_budget_kb"] > 0
    assert ctx.get_tiles(FP64, SHAPE) == t
    after, _ = _flow(ctx, FP64, U)
    assert np.array_equal(before.E, after.E) and np.array_equal(before.Q, after.Q)


def test_invalid_tile_shapes_are_rejected(ctx):
    from msc_project_b200.lgf import LGFError
    for bad in ({"stage_threads": 100}, {"stage_threads": 1024}, {"meas_split": 3}, {"stage_order": 2},
                {"meas_budget_kb": 0}):
        with pytest.raises(LGFError):
            ctx.set_tiles(FP64, (8, 8, 8, 8), **bad)
