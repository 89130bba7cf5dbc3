"""Python binding of the CPU oracle and the METIS baseline harness.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py.  The product package never imports this module.

`partition` runs oracle/oracle.cpp, a sequential restatement of the
deterministic V-cycle the CUDA library implements; `metis` runs METIS 5 from
the CUDA toolkit's libmetis_static.a (the library behind the reference's
`gpmetis` call, src/gpu_part.cu:857).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from thegraphpartitioning_b200._abi import (
    GpOptions, GpStats, TraceCollector, make_options, i32p, i64p, PRIO_FN,
)

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
_lib = None
_metis = None


def build(force: bool = False) -> None:
    """Compile the oracle and the METIS harness (make, g++/gcc)."""
    targets = [os.path.join(BUILD, "libgp_oracle.so"), os.path.join(BUILD, "libgp_metis.so")]
    if force or not all(os.path.exists(t) for t in targets):
        subprocess.run(["make", "-C", HERE, "-s"], check=True)


def _load():
    global _lib
    if _lib is None:
        path = os.path.join(BUILD, "libgp_oracle.so")
        if not os.path.exists(path):
            build()
        lib = C.CDLL(path)
        lib.gpo_partition.restype = C.c_int
        lib.gpo_partition.argtypes = [
            C.c_int64, C.POINTER(C.c_int64), C.POINTER(C.c_int32), C.POINTER(C.c_int32),
            C.POINTER(C.c_int32), C.c_int32, C.c_float, C.c_uint64, C.POINTER(C.c_int32),
            C.POINTER(GpOptions), C.POINTER(GpStats), C.c_void_p, C.c_void_p]
        lib.gpo_partition_prio.restype = C.c_int
        lib.gpo_partition_prio.argtypes = lib.gpo_partition.argtypes + [C.c_void_p, C.c_void_p]
        lib.gpo_partition_prio2.restype = C.c_int
        lib.gpo_partition_prio2.argtypes = lib.gpo_partition.argtypes + [C.c_void_p, C.c_void_p, C.c_void_p,
                                                                          C.c_void_p]
        lib.gpo_edge_cut.restype = C.c_int
        lib.gpo_edge_cut.argtypes = [
            C.c_int64, C.POINTER(C.c_int64), C.POINTER(C.c_int32), C.POINTER(C.c_int32),
            C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.c_int32,
            C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
        lib.gpo_last_error.restype = C.c_char_p
        lib.gpo_compute_lmax.restype = C.c_int64
        lib.gpo_compute_lmax.argtypes = [C.c_int64, C.c_int32, C.c_float]
        lib.gpo_mix64.restype = C.c_uint64
        lib.gpo_mix64.argtypes = [C.c_uint64]
        lib.gpo_edge_hash.restype = C.c_uint32
        lib.gpo_edge_hash.argtypes = [C.c_uint64, C.c_int32, C.c_int32, C.c_int32]
        lib.gpo_loss_bucket.restype = C.c_uint32
        lib.gpo_loss_bucket.argtypes = [C.c_int32]
        _lib = lib
    return _lib


class OracleError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"oracle error {code}: {msg}")
        self.code = code


def _as(a, dtype):
    return None if a is None else np.ascontiguousarray(np.asarray(a), dtype=dtype)


MPRIO_FN = C.CFUNCTYPE(C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_int64)


def partition(rowptr, colidx, k, imbalance=0.03, seed=0, vwgt=None, ewgt=None,
              options=None, trace=False, prio_levels=None, move_prio=None):
    """Full V-cycle on the CPU.  Returns (part, stats_dict, events).

    prio_levels: {level: int32[m_level]} matching priorities replacing the edge
    weights (the learned mode) at the levels listed; other levels use the edge
    weights.  Fails when a listed level's entry count differs.
    move_prio: {(level, iter): int32[n_level]} move priorities replacing the
    (gain, id) order of those label-propagation steps (learned move order)."""
    lib = _load()
    rp = _as(rowptr, np.int64)
    ci = _as(colidx, np.int32)
    vw = _as(vwgt, np.int32)
    ew = _as(ewgt, np.int32)
    n = len(rp) - 1
    part = np.zeros(max(n, 1), dtype=np.int32)
    st = GpStats()
    opt = options if isinstance(options, GpOptions) else make_options(**(options or {}))
    col = TraceCollector() if trace else None
    tfn = C.cast(col.cfunc, C.c_void_p) if col else None
    if move_prio is not None:
        mheld = {(int(l), int(i)): np.ascontiguousarray(a, dtype=np.int32) for (l, i), a in move_prio.items()}
        held = {int(l): np.ascontiguousarray(a, dtype=np.int32) for l, a in (prio_levels or {}).items()}
        bad = []

        def pcb(_user, level, m):
            a = held.get(int(level))
            if a is None or len(a) != int(m):
                return None
            return a.ctypes.data

        def mcb(_user, level, it, n):
            a = mheld.get((int(level), int(it)))
            if a is None:
                return None
            if len(a) != int(n):
                bad.append((int(level), int(it)))
                return None
            return a.ctypes.data

        pfn, mfn = PRIO_FN(pcb), MPRIO_FN(mcb)
        rc = lib.gpo_partition_prio2(n, i64p(rp), i32p(ci), i32p(vw), i32p(ew), int(k), float(imbalance),
                                     int(seed) & 0xFFFFFFFFFFFFFFFF, i32p(part), C.byref(opt), C.byref(st), tfn, None,
                                     C.cast(pfn, C.c_void_p), None, C.cast(mfn, C.c_void_p), None)
        if bad:
            raise OracleError(-1, f"move priorities of the wrong length for (level, iter) = {bad}")
    elif prio_levels is None:
        rc = lib.gpo_partition(n, i64p(rp), i32p(ci), i32p(vw), i32p(ew), int(k), float(imbalance),
                               int(seed) & 0xFFFFFFFFFFFFFFFF, i32p(part), C.byref(opt), C.byref(st), tfn, None)
    else:
        held = {int(l): np.ascontiguousarray(a, dtype=np.int32) for l, a in prio_levels.items()}
        missing = []

        def cb(_user, level, m):
            a = held.get(int(level))
            if a is None:
                return None
            if len(a) != int(m):
                missing.append((int(level), int(m)))
                return None
            return a.ctypes.data

        pfn = PRIO_FN(cb)
        rc = lib.gpo_partition_prio(n, i64p(rp), i32p(ci), i32p(vw), i32p(ew), int(k), float(imbalance),
                                    int(seed) & 0xFFFFFFFFFFFFFFFF, i32p(part), C.byref(opt), C.byref(st), tfn, None,
                                    C.cast(pfn, C.c_void_p), None)
        if missing:
            raise OracleError(-1, f"priorities of the wrong length for (level, m) = {missing}")
    if rc != 0:
        raise OracleError(rc, lib.gpo_last_error().decode())
    return part[:n], st.as_dict(), (col.events if col else [])


def edge_cut(rowptr, colidx, part, k, ewgt=None, vwgt=None):
    """Exact (cut, part_weights) of a partition."""
    lib = _load()
    rp = _as(rowptr, np.int64)
    ci = _as(colidx, np.int32)
    pt = _as(part, np.int32)
    ew = _as(ewgt, np.int32)
    vw = _as(vwgt, np.int32)
    cut = C.c_int64(0)
    pw = np.zeros(int(k), dtype=np.int64)
    rc = lib.gpo_edge_cut(len(rp) - 1, i64p(rp), i32p(ci), i32p(ew), i32p(vw), i32p(pt), int(k),
                          C.byref(cut), i64p(pw))
    if rc != 0:
        raise OracleError(rc, lib.gpo_last_error().decode())
    return int(cut.value), pw


def lmax(total_weight, k, imbalance):
    return int(_load().gpo_compute_lmax(int(total_weight), int(k), float(imbalance)))


def mix64(x):
    return int(_load().gpo_mix64(int(x) & 0xFFFFFFFFFFFFFFFF))


def edge_hash(seed, level, a, b):
    return int(_load().gpo_edge_hash(int(seed) & 0xFFFFFFFFFFFFFFFF, int(level), int(a), int(b)))


def loss_bucket(loss):
    return int(_load().gpo_loss_bucket(int(loss)))


def _load_metis():
    global _metis
    if _metis is None:
        path = os.path.join(BUILD, "libgp_metis.so")
        if not os.path.exists(path):
            build()
        lib = C.CDLL(path)
        lib.gpm_partition.restype = C.c_int
        lib.gpm_partition.argtypes = [
            C.c_int64, C.POINTER(C.c_int64), C.POINTER(C.c_int32), C.POINTER(C.c_int32),
            C.POINTER(C.c_int32), C.c_int32, C.c_int64, C.c_int, C.POINTER(C.c_int32),
            C.POINTER(C.c_int64), C.POINTER(C.c_double)]
        _metis = lib
    return _metis


def metis(rowptr, colidx, k, seed=0, vwgt=None, ewgt=None, recursive=False):
    """METIS 5 PartGraphKway (or Recursive).  Returns (part, cut, seconds)."""
    lib = _load_metis()
    rp = _as(rowptr, np.int64)
    ci = _as(colidx, np.int32)
    vw = _as(vwgt, np.int32)
    ew = _as(ewgt, np.int32)
    n = len(rp) - 1
    part = np.zeros(max(n, 1), dtype=np.int32)
    cut = C.c_int64(0)
    secs = C.c_double(0)
    rc = lib.gpm_partition(n, i64p(rp), i32p(ci), i32p(vw), i32p(ew), int(k), int(seed),
                           1 if recursive else 0, i32p(part), C.byref(cut), C.byref(secs))
    if rc != 1:
        raise RuntimeError(f"METIS returned {rc}")
    return part[:n], int(cut.value), float(secs.value)
