"""The allocation-free edge-cut entry point, checked against the regular one
and against the oracle.

gp_edge_cut_device_noalloc serves callers that cannot allocate device memory:
code inside an allocator or memory-pool callback (an allocation would
re-enter the allocator), allocation-free serving loops (an allocation can
block or fail mid-loop) and devices whose memory another framework has
reserved.  Its scratch is a fixed device array shared by every call.  This
file is collected last so that a run stopping at the first failure has run
every other test first; it passes alone and after the rest of the suite.
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


def _device_free_bytes():
    torch.cuda.synchronize()
    return torch.cuda.mem_get_info()[0]


def test_noalloc_matches_regular_entry_point_twice(gp, cuda, oracle_mod):
    lib, f = _bind(gp)
    rp, ci = to_np(*graphs.chung_lu(40000, 150000, seed=7))
    ew, vw = weighted(rp, ci, seed=3)
    d = lambda a: torch.from_numpy(a).to(cuda)
    drp, dci, dew, dvw = d(rp), d(ci), d(ew), d(vw)
    n = len(rp) - 1
    # two partitions with different k: the second call must not see the first
    # call's accumulators
    cases = []
    for k, mult in ((13, 7919), (64, 104729)):
        hpart = (np.arange(n) * mult % k).astype(np.int32)
        cut_ref, pw_ref = gp.edge_cut(drp, dci, d(hpart), k, ewgt=dew, vwgt=dvw)
        cut_or, pw_or = oracle_mod.edge_cut(rp, ci, hpart, k, ewgt=ew, vwgt=vw)
        assert cut_ref == cut_or and np.array_equal(pw_ref, pw_or)
        cases.append((k, d(hpart), cut_or, pw_or))
    # first call on this device: looks up the scratch array's address and
    # loads the kernels
    assert _noalloc(f, drp, dci, dew, dvw, cases[0][1], cases[0][0])[0] == 0, lib.gp_last_error().decode()
    # without the library's cached workspace, two calls in a row take no
    # device memory
    gp.release_workspace()
    free0 = _device_free_bytes()
    for k, part, cut_or, pw_or in cases:
        rc, cut, pw = _noalloc(f, drp, dci, dew, dvw, part, k)
        assert rc == 0, lib.gp_last_error().decode()
        assert cut == cut_or
        assert np.array_equal(pw, pw_or)
    free1 = _device_free_bytes()
    assert free1 >= free0 - (1 << 20), (free0, free1)


def test_noalloc_unit_weights_and_limits(gp, cuda, oracle_mod):
    lib, f = _bind(gp)
    rp, ci = graphs.grid2d(200, 300)
    hpart = (np.arange(rp.numel() - 1) % 4).astype(np.int32)
    cut_or, pw_or = oracle_mod.edge_cut(rp.numpy(), ci.numpy(), hpart, 4)
    rp, ci = rp.to(cuda), ci.to(cuda)
    part = torch.from_numpy(hpart).to(cuda)
    rc, cut, pw = _noalloc(f, rp, ci, None, None, part, 4)
    assert rc == 0
    assert cut == cut_or and np.array_equal(pw, pw_or)
    assert (cut, list(pw)) == (lambda r: (r[0], list(r[1])))(gp.edge_cut(rp, ci, part, 4))
    rc, _, _ = _noalloc(f, rp, ci, None, None, part, 1025)   # beyond the scratch
    assert rc == -1 and "GP_NOALLOC_MAX_K" in lib.gp_last_error().decode()
    bad = part.clone()
    bad[17] = 9
    rc, _, _ = _noalloc(f, rp, ci, None, None, bad, 4)       # part id out of range
    assert rc == -1
