"""lgf_measure_noalloc: the measurement for callers that cannot allocate
device memory (their GPU memory belongs to another allocator, or their loop
must not call into the driver's allocator).  It must give what lgf_measure
gives, call after call, although its scratch array is shared and keeps the
previous call's contents.  This file is collected last on purpose."""
import ctypes

import numpy as np
import pytest
from conftest import golden_links, q_err, rel_err

from msc_project_b200 import FP64
from msc_project_b200 import _capi as C

pytestmark = pytest.mark.gpu

TOL = 1e-12


def noalloc(ctx, links_np, shape):
    import torch
    dev_links = torch.from_numpy(np.ascontiguousarray(links_np)).to("cuda:0")
    out = torch.full((2 + 2 * shape[0],), float("nan"), dtype=torch.float64, device="cuda:0")
    stream = torch.cuda.current_stream()
    rc = ctx.lib.lgf_measure_noalloc(ctypes.cast(dev_links.data_ptr(), ctypes.POINTER(ctypes.c_double)),
                                     (ctypes.c_int * 4)(*shape),
                                     ctypes.cast(out.data_ptr(), ctypes.POINTER(ctypes.c_double)),
                                     ctypes.c_void_p(stream.cuda_stream))
    assert rc == C.LGF_OK
    stream.synchronize()
    return out.cpu().numpy()


def engine(ctx, links_np, shape):
    with ctx.lattice(shape, FP64) as lat:
        lat.upload(links_np)
        E, Q, es, qs = lat.measure(slices=True)
    return E, Q, es, qs


def test_noalloc_matches_measure_two_calls_in_a_row(ctx):
    cases = [(golden_links("hb8_seed1.bin"), (8, 8, 8, 8)),      # larger lattice first
             (golden_links("g4466_seed7.bin"), (4, 4, 6, 6))]    # then a smaller one over its leftovers
    for links, shape in cases:
        got = noalloc(ctx, links, shape)
        E, Q, es, qs = engine(ctx, links, shape)
        N0 = shape[0]
        assert rel_err(got[0], E) < TOL
        assert q_err(got[1], Q) < TOL
        assert np.max(np.abs(got[2:2 + N0] - es) / np.abs(es)) < TOL
        assert np.max(np.abs(got[2 + N0:] - qs)) < TOL


def test_noalloc_rejects_lattices_beyond_its_scratch(ctx):
    dummy = (ctypes.c_double * 2)()
    rc = ctx.lib.lgf_measure_noalloc(dummy, (ctypes.c_int * 4)(64, 64, 64, 64), dummy, None)
    assert rc == C.LGF_ETOOBIG
    rc = ctx.lib.lgf_measure_noalloc(dummy, (ctypes.c_int * 4)(8, 8, 7, 8), dummy, None)
    assert rc == C.LGF_EINVAL
