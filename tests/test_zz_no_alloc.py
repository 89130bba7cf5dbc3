"""The allocation-free edge-cut entry point, checked against the regular one.

gp_edge_cut_device_noalloc serves callers that cannot allocate device memory
(stream capture in progress, allocator callbacks, allocation-free loops, fully
reserved devices): its scratch is a fixed device array shared by every call.
This file is collected last so that a run stopping at the first failure has
run every other test first; it passes alone and after the rest of the suite.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from thegraphpartitioning_b200 import graphs
from helpers import to_np, weighted

pytestmark = pytest.mark.gpu


def _bind(gp):
    lib = gp.lib()
    f = lib.gp_edge_cut_device_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p,
                  C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    return lib, f


def _noalloc(f, rp, ci, ew, vw, part, k):
    cut = C.c_int64(-1)
    pw = np.full(k, -1, dtype=np.int64)
    ptr = lambda t: None if t is None else C.c_void_p(t.data_ptr())
    stream = torch.cuda.current_stream().cuda_stream
    rc = f(rp.numel() - 1, ptr(rp), ptr(ci), ptr(ew), ptr(vw), ptr(part), k, C.c_void_p(stream), C.byref(cut),
           pw.ctypes.data_as(C.POINTER(C.c_int64)))
    return rc, int(cut.value), pw


def test_noalloc_matches_regular_entry_point_twice(gp, cuda):
    lib, f = _bind(gp)
    rp, ci = to_np(*graphs.chung_lu(40000, 150000, seed=7))
    ew, vw = weighted(rp, ci, seed=3)
    d = lambda a: torch.from_numpy(a).to(cuda)
    drp, dci, dew, dvw = d(rp), d(ci), d(ew), d(vw)
    n = len(rp) - 1
    # two calls in a row with different partitions and k: the second must not
    # see the first call's accumulators
    for k, mult in ((13, 7919), (64, 104729)):
        part = d((np.arange(n) * mult % k).astype(np.int32))
        rc, cut, pw = _noalloc(f, drp, dci, dew, dvw, part, k)
        assert rc == 0, lib.gp_last_error().decode()
        cut_ref, pw_ref = gp.edge_cut(drp, dci, part, k, ewgt=dew, vwgt=dvw)
        assert cut == cut_ref
        assert np.array_equal(pw, pw_ref)


def test_noalloc_unit_weights_and_limits(gp, cuda):
    lib, f = _bind(gp)
    rp, ci = graphs.grid2d(200, 300)
    rp, ci = rp.to(cuda), ci.to(cuda)
    part = (torch.arange(rp.numel() - 1, device=cuda) % 4).to(torch.int32)
    rc, cut, pw = _noalloc(f, rp, ci, None, None, part, 4)
    assert rc == 0
    assert (cut, list(pw)) == (lambda r: (r[0], list(r[1])))(gp.edge_cut(rp, ci, part, 4))
    rc, _, _ = _noalloc(f, rp, ci, None, None, part, 1025)   # beyond the scratch
    assert rc == -1 and "GP_NOALLOC_MAX_K" in lib.gp_last_error().decode()
    bad = part.clone()
    bad[17] = 9
    rc, _, _ = _noalloc(f, rp, ci, None, None, bad, 4)       # part id out of range
    assert rc == -1
