"""lgf_measure_noalloc: the measurement for callers that cannot allocate
device memory (their GPU memory belongs to another allocator, or their loop
must not call into the driver's allocator).  It must give what lgf_measure
gives and what the LGF reference measured on the same links, call after call,
although its scratch array is shared and keeps the previous call's contents,
and it must leave the GPU's free memory unchanged.  This file is collected
last on purpose."""
import ctypes

import numpy as np
import pytest
from conftest import golden_json, golden_links, q_err, rel_err

from msc_project_b200 import FP64
from msc_project_b200 import _capi as C

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _device_args(links_np, shape):
    import torch
    dev_links = torch.from_numpy(np.ascontiguousarray(links_np)).to("cuda:0")
    out = torch.full((2 + 2 * shape[0],), float("nan"), dtype=torch.float64, device="cuda:0")
    return dev_links, out


def _call(ctx, dev_links, out, shape):
    import torch
    stream = torch.cuda.current_stream()
    rc = ctx.lib.lgf_measure_noalloc(ctypes.cast(dev_links.data_ptr(), ctypes.POINTER(ctypes.c_double)),
                                     (ctypes.c_int * 4)(*shape),
                                     ctypes.cast(out.data_ptr(), ctypes.POINTER(ctypes.c_double)),
                                     ctypes.c_void_p(stream.cuda_stream))
    assert rc == C.LGF_OK
    stream.synchronize()
    return out.cpu().numpy()


def noalloc(ctx, links_np, shape):
    dev_links, out = _device_args(links_np, shape)
    return _call(ctx, dev_links, out, shape)


def engine(ctx, links_np, shape):
    with ctx.lattice(shape, FP64) as lat:
        lat.upload(links_np)
        E, Q, es, qs = lat.measure(slices=True)
    return E, Q, es, qs


def _cases():
    from oracle import oracle as O
    # larger lattice first, then smaller ones over its leftovers; 4x6x8x10 has
    # four different extents, so a swapped direction or stride cannot pass
    return [(golden_links("hb8_seed1.bin"), (8, 8, 8, 8), golden_json("flow8_hb_seed1.json")),
            (O.generate_G((4, 6, 8, 10), 9, 0.5), (4, 6, 8, 10), golden_json("flow_g46810.json")),
            (golden_links("g4466_seed7.bin"), (4, 4, 6, 6), golden_json("flow_g4466.json"))]


def test_noalloc_matches_measure_and_reference_two_calls_in_a_row(ctx):
    for links, shape, gold in _cases():
        E, Q, es, qs = engine(ctx, links, shape)
        N0 = shape[0]
        for _ in range(2):
            got = noalloc(ctx, links, shape)
            assert rel_err(got[0], E) < TOL
            assert q_err(got[1], Q) < TOL
            assert np.max(np.abs(got[2:2 + N0] - es) / np.abs(es)) < TOL
            assert np.max(np.abs(got[2 + N0:] - qs)) < TOL
            # the reference's own E(t=0), Q(t=0) on the same links
            assert rel_err(got[0], gold["E"][0]) < TOL
            assert q_err(got[1], gold["Q"][0]) < TOL


def test_noalloc_leaves_free_memory_unchanged(ctx):
    import torch
    links, shape, _ = _cases()[1]
    dev_links, out = _device_args(links, shape)
    first = _call(ctx, dev_links, out, shape)  # warm-up: module and scratch already placed
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    again = _call(ctx, dev_links, out, shape)
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after == free_before
    assert np.array_equal(first, again)


def test_noalloc_rejects_lattices_beyond_its_scratch(ctx):
    dummy = (ctypes.c_double * 2)()
    rc = ctx.lib.lgf_measure_noalloc(dummy, (ctypes.c_int * 4)(64, 64, 64, 64), dummy, None)
    assert rc == C.LGF_ETOOBIG
    rc = ctx.lib.lgf_measure_noalloc(dummy, (ctypes.c_int * 4)(8, 8, 7, 8), dummy, None)
    assert rc == C.LGF_EINVAL
