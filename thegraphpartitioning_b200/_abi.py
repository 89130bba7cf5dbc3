"""ctypes mirror of include/gp_partition.h (structures, constants, trace decoding).

Shared by the product binding (thegraphpartitioning_b200.partition) and by the
test-side oracle binding, so both read the same option/stat/trace layouts.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

GP_OK = 0
GP_EINVAL = -1
GP_ENOMEM = -2
GP_ECUDA = -3
GP_ETIMEOUT = -4
GP_EINTERNAL = -5
GP_MAX_K = 1024
GP_OPTIONS_VERSION = 1

GP_TR_MATCH = 1
GP_TR_CONTRACT = 2
GP_TR_INITPART = 3
GP_TR_REFINE_ITER = 4
GP_TR_LEVEL_DONE = 5
GP_TR_PRIO = 6
GP_TR_MOVE_PRIO = 7

ERROR_NAMES = {
    GP_EINVAL: "GP_EINVAL",
    GP_ENOMEM: "GP_ENOMEM",
    GP_ECUDA: "GP_ECUDA",
    GP_ETIMEOUT: "GP_ETIMEOUT",
    GP_EINTERNAL: "GP_EINTERNAL",
}


class GpOptions(C.Structure):
    _fields_ = [
        ("version", C.c_int32),
        ("coarsen_to", C.c_int32),
        ("match_rounds", C.c_int32),
        ("two_hop", C.c_int32),
        ("init_trials", C.c_int32),
        ("refine_max_iters", C.c_int32),
        ("refine_patience", C.c_int32),
        ("lp_filter_den", C.c_int32),
        ("strong_after", C.c_int32),
        ("check_input", C.c_int32),
        ("verbose", C.c_int32),
        ("profile", C.c_int32),
        ("small_level_n", C.c_int32),
        ("ctas_per_sm", C.c_int32),
        ("heavy_deg", C.c_int32),
        ("item_len", C.c_int32),
    ]


class GpStats(C.Structure):
    _fields_ = [
        ("cut", C.c_int64),
        ("max_part_weight", C.c_int64),
        ("total_weight", C.c_int64),
        ("max_allowed", C.c_int64),
        ("imbalance", C.c_double),
        ("levels", C.c_int32),
        ("coarsest_n", C.c_int32),
        ("best_trial", C.c_int32),
        ("refine_iters", C.c_int32),
        ("algo_bytes", C.c_int64),
        ("kernel_launches", C.c_int64),
        ("ms_coarsen", C.c_double),
        ("ms_initial", C.c_double),
        ("ms_refine", C.c_double),
        ("ms_project", C.c_double),
        ("ms_total", C.c_double),
        ("ms_h2d", C.c_double),
        ("ms_d2h", C.c_double),
        ("ms_conn", C.c_double),
        ("conn_launches", C.c_int64),
        ("conn_bytes", C.c_int64),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class GpTraceEvent(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("level", C.c_int32),
        ("iter", C.c_int32),
        ("mode", C.c_int32),
        ("n", C.c_int64),
        ("m", C.c_int64),
        ("cut", C.c_int64),
        ("maxpw", C.c_int64),
        ("count", C.c_int64),
        ("a0", C.POINTER(C.c_int32)),
        ("a1", C.POINTER(C.c_int32)),
        ("a2", C.POINTER(C.c_int32)),
        ("rowptr", C.POINTER(C.c_int64)),
        ("colidx", C.POINTER(C.c_int32)),
        ("ewgt", C.POINTER(C.c_int32)),
        ("vwgt", C.POINTER(C.c_int32)),
    ]


class GpLearnedReport(C.Structure):
    _fields_ = [
        ("cut_learned", C.c_int64),
        ("cut_plain", C.c_int64),
        ("max_part_weight_learned", C.c_int64),
        ("max_part_weight_plain", C.c_int64),
        ("ms_learned", C.c_double),
        ("ms_plain", C.c_double),
        ("ms_gnn", C.c_double),
        ("kept_learned", C.c_int32),
        ("reserved", C.c_int32),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_ if name != "reserved"}


TRACE_FN = C.CFUNCTYPE(None, C.c_void_p, C.POINTER(GpTraceEvent))
# learned matching priorities handed to the oracle: (user, level, m) -> int32[m]
PRIO_FN = C.CFUNCTYPE(C.c_void_p, C.c_void_p, C.c_int32, C.c_int64)


def make_options(**kw) -> GpOptions:
    o = GpOptions()
    o.version = GP_OPTIONS_VERSION
    for key, val in kw.items():
        if not hasattr(o, key):
            raise KeyError(f"unknown option {key!r}")
        setattr(o, key, int(val))
    return o


def _arr(ptr, count, dtype):
    if not ptr or count <= 0:
        return np.zeros(0, dtype=dtype)
    ctype = C.c_int64 if dtype == np.int64 else C.c_int32
    buf = C.cast(ptr, C.POINTER(ctype * count)).contents
    return np.frombuffer(buf, dtype=dtype).copy()


def decode_event(ev: GpTraceEvent) -> dict:
    """Copy one trace event (valid only during the callback) into numpy."""
    d = {
        "kind": ev.kind, "level": ev.level, "iter": ev.iter, "mode": ev.mode,
        "n": ev.n, "m": ev.m, "cut": ev.cut, "maxpw": ev.maxpw, "count": ev.count,
    }
    n = int(ev.n)
    if ev.kind == GP_TR_CONTRACT:
        # a0 is the fine->coarse map of the finer level; its length is the
        # finer level's n, which the caller knows; it is stored by the binding.
        d["rowptr"] = _arr(ev.rowptr, n + 1, np.int64)
        m = int(d["rowptr"][-1]) if n >= 0 else 0
        d["colidx"] = _arr(ev.colidx, m, np.int32)
        d["ewgt"] = _arr(ev.ewgt, m, np.int32)
        d["vwgt"] = _arr(ev.vwgt, n, np.int32)
    elif ev.kind == GP_TR_PRIO:
        d["a0"] = _arr(ev.a0, int(ev.m), np.int32)
    elif ev.kind == GP_TR_MOVE_PRIO:
        d["a0"] = _arr(ev.a0, n, np.int32)
    else:
        for name in ("a0", "a1", "a2"):
            d[name] = _arr(getattr(ev, name), n, np.int32)
    return d


class TraceCollector:
    """Callback object that stores decoded events; tracks the finer level's n
    so that the cmap of a CONTRACT event can be copied with the right length."""

    def __init__(self, kinds=None):
        self.events: list[dict] = []
        self._last_fine_n = 0
        self.kinds = None if kinds is None else frozenset(int(x) for x in kinds)
        self.cfunc = TRACE_FN(self._cb)

    def _cb(self, _user, evp):
        ev = evp.contents
        if ev.kind == GP_TR_MATCH:
            self._last_fine_n = int(ev.n)
        if self.kinds is not None and int(ev.kind) not in self.kinds:
            return
        d = decode_event(ev)
        if ev.kind == GP_TR_CONTRACT:
            d["a0"] = _arr(ev.a0, self._last_fine_n, np.int32)
        self.events.append(d)


def i64p(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_int64)) if a is not None else None


def i32p(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_int32)) if a is not None else None
