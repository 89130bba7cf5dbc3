"""B200-native multilevel k-way graph partitioner.

Python binding of the C ABI in include/gp_partition.h (libgp_b200.so, built
in-tree by `make -C thegraphpartitioning_b200/csrc`).  There is no CPU
fallback: if the library is missing, every call raises.

    part, stats, _ = partition(rowptr, colidx, k)            # host arrays
    part, stats, _ = partition(d_rowptr, d_colidx, k)        # torch CUDA tensors

The reference (iamrupamroyy/TheGraphPartitioning) exposes the same operation
only as the `gpu_part` executable (src/gpu_part.cu:878); that CLI is rebuilt
as bin/gpu_part on top of this library.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from ._abi import (
    GpOptions, GpStats, GpLearnedReport, TraceCollector, make_options, i32p, i64p, ERROR_NAMES,
)

HERE = os.path.dirname(os.path.abspath(__file__))
# THEGRAPHPARTITIONING_CHECKED=1 selects the bounds-checked build of the same
# sources (device-side index checks; gp_checked_violations reports them)
CHECKED = os.environ.get("THEGRAPHPARTITIONING_CHECKED", "") == "1"
LIB_PATH = os.path.join(HERE, "libgp_b200_checked.so" if CHECKED else "libgp_b200.so")
CLI_PATH = os.path.join(HERE, "bin", "gpu_part")
_lib = None


class GPError(RuntimeError):
    """A GP_E* status returned by the library."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERROR_NAMES.get(code, code)}: {msg}")
        self.code = code


def build() -> None:
    import subprocess
    subprocess.run(["make", "-C", os.path.join(HERE, "csrc"), "-s", "-j8"], check=True)


def lib():
    """Load libgp_b200.so (raises when it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C {os.path.join(HERE, 'csrc')}` "
                           "(there is no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    P64, P32 = C.POINTER(C.c_int64), C.POINTER(C.c_int32)
    L.gp_partition.restype = C.c_int
    L.gp_partition.argtypes = [C.c_int64, P64, P32, P32, P32, C.c_int32, C.c_float, C.c_uint64, P32]
    L.gp_partition_ex.restype = C.c_int
    L.gp_partition_ex.argtypes = [C.c_int64, P64, P32, P32, P32, C.c_int32, C.c_float, C.c_uint64, P32,
                                  C.POINTER(GpOptions), C.POINTER(GpStats), C.c_void_p, C.c_void_p]
    L.gp_partition_device.restype = C.c_int
    L.gp_partition_device.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32,
                                      C.c_float, C.c_uint64, C.c_void_p, C.c_void_p, C.POINTER(GpOptions),
                                      C.POINTER(GpStats), C.c_void_p, C.c_void_p]
    L.gp_edge_cut_device.restype = C.c_int
    L.gp_edge_cut_device.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_int32, C.c_void_p, P64, P64]
    PP64, PP32 = C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)
    L.gp_partition_batch_device.restype = C.c_int
    L.gp_partition_batch_device.argtypes = [C.c_int32, P64, P64, PP64, PP32, PP32, PP32, P32, C.POINTER(C.c_float),
                                            C.POINTER(C.c_uint64), PP32, C.c_void_p, C.c_int32,
                                            C.POINTER(GpOptions), C.POINTER(GpStats)]
    VP = C.c_void_p
    L.gp_gnn_num_params.restype = C.c_int
    L.gp_gnn_create.restype = C.c_int
    L.gp_gnn_create.argtypes = [C.POINTER(VP)]
    L.gp_gnn_destroy.restype = C.c_int
    L.gp_gnn_destroy.argtypes = [VP]
    L.gp_gnn_set_params.restype = C.c_int
    L.gp_gnn_set_params.argtypes = [VP, C.POINTER(C.c_float), C.c_int32]
    L.gp_gnn_set_prio_bits.restype = C.c_int
    L.gp_gnn_set_prio_bits.argtypes = [VP, C.c_int32]
    L.gp_gnn_get_prio_bits.restype = C.c_int
    L.gp_gnn_get_prio_bits.argtypes = [VP]
    L.gp_gnn_set_max_level.restype = C.c_int
    L.gp_gnn_set_max_level.argtypes = [VP, C.c_int32]
    L.gp_gnn_get_max_level.restype = C.c_int
    L.gp_gnn_get_max_level.argtypes = [VP]
    L.gp_gnn_get_params.restype = C.c_int
    L.gp_gnn_get_params.argtypes = [VP, C.POINTER(C.c_float), C.c_int32]
    L.gp_gnn_forward_device.restype = C.c_int
    L.gp_gnn_forward_device.argtypes = [VP, C.c_int64, VP, VP, VP, VP, C.c_int32, VP, VP, VP]
    L.gp_gnn_grad_device.restype = C.c_int
    L.gp_gnn_grad_device.argtypes = [VP, C.c_int64, VP, VP, VP, VP, C.c_int32, VP, VP, C.POINTER(C.c_float),
                                     C.POINTER(C.c_float)]
    L.gp_gnn_train_step_device.restype = C.c_int
    L.gp_gnn_train_step_device.argtypes = [VP, C.c_int32, P64, PP64, PP32, PP32, PP32, P32, C.POINTER(VP),
                                           C.c_float, VP, C.POINTER(C.c_float)]
    L.gp_gnn_move_num_params.restype = C.c_int
    L.gp_gnn_set_move_params.restype = C.c_int
    L.gp_gnn_set_move_params.argtypes = [VP, C.POINTER(C.c_float), C.c_int32]
    L.gp_gnn_get_move_params.restype = C.c_int
    L.gp_gnn_get_move_params.argtypes = [VP, C.POINTER(C.c_float), C.c_int32]
    L.gp_gnn_move_features_device.restype = C.c_int
    L.gp_gnn_move_features_device.argtypes = [C.c_int64, VP, VP, VP, VP, C.c_int32, VP, VP]
    L.gp_gnn_move_scores_device.restype = C.c_int
    L.gp_gnn_move_scores_device.argtypes = [VP, C.c_int64, VP, VP, VP, VP]
    L.gp_gnn_move_grad_device.restype = C.c_int
    L.gp_gnn_move_grad_device.argtypes = [VP, C.c_int64, VP, VP, VP, C.POINTER(C.c_float), C.POINTER(C.c_float)]
    L.gp_gnn_move_train_step_device.restype = C.c_int
    L.gp_gnn_move_train_step_device.argtypes = [VP, C.c_int64, VP, VP, C.c_float, VP, C.POINTER(C.c_float)]
    L.gp_partition_learned_device.restype = C.c_int
    L.gp_partition_learned_device.argtypes = [C.c_int64, VP, VP, VP, VP, C.c_int32, C.c_float, C.c_uint64, VP, VP,
                                              C.POINTER(GpOptions), C.POINTER(GpStats), VP, C.c_int32,
                                              C.POINTER(GpLearnedReport), VP, VP]
    L.gp_default_options.restype = C.c_int
    L.gp_default_options.argtypes = [C.POINTER(GpOptions)]
    L.gp_checked_violations.restype = C.c_int
    L.gp_checked_violations.argtypes = [C.POINTER(C.c_int64), C.POINTER(C.c_int32), C.c_int32]
    L.gp_release_workspace.restype = C.c_int
    L.gp_last_error.restype = C.c_char_p
    L.gp_version.restype = C.c_char_p
    _lib = L
    return L


def _check(rc: int):
    if rc != 0:
        raise GPError(rc, lib().gp_last_error().decode())


def _opts(options):
    if options is None:
        return make_options()
    if isinstance(options, GpOptions):
        return options
    return make_options(**options)


def _is_cuda(x) -> bool:
    return hasattr(x, "is_cuda") and bool(x.is_cuda)


def _ptr(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def _collector(trace):
    if not trace:
        return None
    return TraceCollector(kinds=None if trace is True else trace)


def partition(rowptr, colidx, k: int, imbalance: float = 0.03, seed: int = 0, vwgt=None, ewgt=None,
              options=None, trace: bool = False, out=None, stream=None):
    """Partition a CSR graph into k parts.

    Host inputs (numpy / lists / CPU tensors) go through gp_partition_ex (the
    library copies them to the current device).  torch CUDA tensors go through
    gp_partition_device on `stream` (default: torch's current stream); the
    result is then a CUDA int32 tensor (written into `out` when given).
    trace: True records every event; a collection of GP_TR_* kinds records
    only those.  Returns (part, stats: dict, trace_events: list)."""
    L = lib()
    opt = _opts(options)
    st = GpStats()
    col = _collector(trace)
    tfn = C.cast(col.cfunc, C.c_void_p) if col else None
    seed = int(seed) & 0xFFFFFFFFFFFFFFFF
    if _is_cuda(rowptr):
        import torch
        n = rowptr.numel() - 1
        assert rowptr.dtype == torch.int64 and colidx.dtype == torch.int32
        for t in (rowptr, colidx, vwgt, ewgt):
            if t is not None:
                assert t.is_cuda and t.is_contiguous()
        part = out if out is not None else torch.empty(max(n, 0), dtype=torch.int32, device=rowptr.device)
        if stream is None:
            stream = torch.cuda.current_stream(rowptr.device).cuda_stream
        rc = L.gp_partition_device(n, _ptr(rowptr), _ptr(colidx), _ptr(vwgt), _ptr(ewgt), int(k), float(imbalance),
                                   seed, _ptr(part), C.c_void_p(stream), C.byref(opt), C.byref(st), tfn, None)
        _check(rc)
        return part, st.as_dict(), (col.events if col else [])
    rp = np.ascontiguousarray(np.asarray(rowptr), dtype=np.int64)
    ci = np.ascontiguousarray(np.asarray(colidx), dtype=np.int32)
    vw = None if vwgt is None else np.ascontiguousarray(np.asarray(vwgt), dtype=np.int32)
    ew = None if ewgt is None else np.ascontiguousarray(np.asarray(ewgt), dtype=np.int32)
    n = len(rp) - 1
    part = np.zeros(max(n, 1), dtype=np.int32)
    rc = L.gp_partition_ex(n, i64p(rp), i32p(ci), i32p(vw), i32p(ew), int(k), float(imbalance), seed, i32p(part),
                           C.byref(opt), C.byref(st), tfn, None)
    _check(rc)
    return part[:n], st.as_dict(), (col.events if col else [])


def edge_cut(rowptr, colidx, part, k: int, ewgt=None, vwgt=None, stream=None):
    """Exact (cut, part_weights) of a partition held in torch CUDA tensors."""
    import torch
    L = lib()
    n = rowptr.numel() - 1
    cut = C.c_int64(0)
    pw = np.zeros(int(k), dtype=np.int64)
    if stream is None:
        stream = torch.cuda.current_stream(rowptr.device).cuda_stream
    rc = L.gp_edge_cut_device(n, _ptr(rowptr), _ptr(colidx), _ptr(ewgt), _ptr(vwgt), _ptr(part), int(k),
                              C.c_void_p(stream), C.byref(cut), i64p(pw))
    _check(rc)
    return int(cut.value), pw


def partition_batch(graphs, ks, imbalances=0.03, seeds=0, options=None, workers=0, stream=None, outs=None):
    """Partition many independent graphs (torch CUDA tensors) in one call.

    graphs: list of (rowptr int64, colidx int32[, vwgt, ewgt]) on one device.
    ks / imbalances / seeds: per graph, or one value for all.  Returns
    (parts: list of int32 CUDA tensors, stats: list of dicts).  Each result is
    exactly what partition() returns for that graph alone."""
    import torch
    L = lib()
    G = len(graphs)
    if G == 0:
        return [], []
    per = lambda x, t: list(x) if isinstance(x, (list, tuple)) else [x] * G
    ks, imbs, sds = per(ks, int), per(imbalances, float), per(seeds, int)
    dev = graphs[0][0].device
    ns = np.array([g[0].numel() - 1 for g in graphs], dtype=np.int64)
    ms = np.array([g[1].numel() for g in graphs], dtype=np.int64)
    parts = outs if outs is not None else [torch.empty(int(n), dtype=torch.int32, device=dev) for n in ns]
    vp = lambda ts: (C.c_void_p * G)(*[t.data_ptr() if t is not None else None for t in ts])
    rps = vp([g[0] for g in graphs])
    cis = vp([g[1] for g in graphs])
    vws = vp([g[2] if len(g) > 2 else None for g in graphs])
    ews = vp([g[3] if len(g) > 3 else None for g in graphs])
    pos = vp(parts)
    karr = np.ascontiguousarray(ks, dtype=np.int32)
    iarr = np.ascontiguousarray(imbs, dtype=np.float32)
    sarr = np.ascontiguousarray([s & 0xFFFFFFFFFFFFFFFF for s in sds], dtype=np.uint64)
    st = (GpStats * G)()
    opt = _opts(options)
    if stream is None:
        stream = torch.cuda.current_stream(dev).cuda_stream
    rc = L.gp_partition_batch_device(G, i64p(ns), i64p(ms), rps, cis, vws, ews, i32p(karr),
                                     iarr.ctypes.data_as(C.POINTER(C.c_float)),
                                     sarr.ctypes.data_as(C.POINTER(C.c_uint64)), pos, C.c_void_p(stream),
                                     int(workers), C.byref(opt), st)
    _check(rc)
    return parts, [st[i].as_dict() for i in range(G)]


def shard_graphs(costs, world: int):
    """Deterministic longest-processing-time assignment of graphs to ranks:
    graphs in decreasing cost (ties: lower index) go to the least loaded rank
    (ties: lower rank).  Returns one index list per rank, each in that order."""
    order = sorted(range(len(costs)), key=lambda i: (-int(costs[i]), i))
    load = [0] * world
    shards = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda j: (load[j], j))
        shards[r].append(i)
        load[r] += int(costs[i])
    return shards


class GNN:
    """Learned edge scorer (gp_gnn handle): two message-passing layers,
    hidden 64, BF16 weights used by every kernel, FP32 master copy and
    accumulation.  Its only use in partitioning is the matching priority of
    gp_partition_learned_device.  Parameters are a flat float32 array of
    num_params() values in the layout oracle/gnn_ref.py documents."""

    def __init__(self, params=None, prio_bits: int = 16, max_level: int = -1):
        self._h = C.c_void_p()
        _check(lib().gp_gnn_create(C.byref(self._h)))
        if params is not None:
            self.set_params(params)
        self.prio_bits = prio_bits
        self.max_level = max_level

    @property
    def max_level(self) -> int:
        """Learned priorities at levels 0..max_level, edge weights above (-1: all)."""
        return int(lib().gp_gnn_get_max_level(self._h))

    @max_level.setter
    def max_level(self, level: int) -> None:
        _check(lib().gp_gnn_set_max_level(self._h, int(level)))

    @property
    def prio_bits(self) -> int:
        """Resolution of the matching priority: rint(logit * 2^bits) + 2^30."""
        return int(lib().gp_gnn_get_prio_bits(self._h))

    @prio_bits.setter
    def prio_bits(self, bits: int) -> None:
        _check(lib().gp_gnn_set_prio_bits(self._h, int(bits)))

    @staticmethod
    def num_params() -> int:
        return int(lib().gp_gnn_num_params())

    def set_params(self, params) -> None:
        p = np.ascontiguousarray(np.asarray(params), dtype=np.float32)
        _check(lib().gp_gnn_set_params(self._h, p.ctypes.data_as(C.POINTER(C.c_float)), len(p)))

    def get_params(self) -> np.ndarray:
        p = np.zeros(self.num_params(), dtype=np.float32)
        _check(lib().gp_gnn_get_params(self._h, p.ctypes.data_as(C.POINTER(C.c_float)), len(p)))
        return p

    # ---- move-order head (learned order of the label-propagation afterburner)
    @staticmethod
    def move_num_params() -> int:
        return int(lib().gp_gnn_move_num_params())

    def set_move_params(self, params) -> None:
        """Install the move-order head (None removes it)."""
        if params is None:
            _check(lib().gp_gnn_set_move_params(self._h, None, 0))
            return
        p = np.ascontiguousarray(np.asarray(params), dtype=np.float32)
        _check(lib().gp_gnn_set_move_params(self._h, p.ctypes.data_as(C.POINTER(C.c_float)), len(p)))

    def get_move_params(self):
        """The head's parameters, or None when the model has none."""
        p = np.zeros(self.move_num_params(), dtype=np.float32)
        rc = lib().gp_gnn_get_move_params(self._h, p.ctypes.data_as(C.POINTER(C.c_float)), len(p))
        return p if rc == 0 else None

    @staticmethod
    def move_features(rowptr, dest, gain, vwgt=None, level: int = 0, stream=None):
        """float32[n, 4] CUDA tensor: the head's features of every candidate (dest >= 0)."""
        import torch
        n = rowptr.numel() - 1
        feat = torch.empty((max(n, 0), 4), dtype=torch.float32, device=rowptr.device)
        if stream is None:
            stream = torch.cuda.current_stream(rowptr.device).cuda_stream
        _check(lib().gp_gnn_move_features_device(n, _ptr(rowptr), _ptr(vwgt), _ptr(dest), _ptr(gain), int(level),
                                                 C.c_void_p(stream), _ptr(feat)))
        return feat

    def move_scores(self, feat, stream=None):
        """(score float32, move priority int32) CUDA tensors of feature rows."""
        import torch
        ns = feat.shape[0]
        score = torch.empty(ns, dtype=torch.float32, device=feat.device)
        prio = torch.empty(ns, dtype=torch.int32, device=feat.device)
        if stream is None:
            stream = torch.cuda.current_stream(feat.device).cuda_stream
        _check(lib().gp_gnn_move_scores_device(self._h, ns, _ptr(feat), C.c_void_p(stream), _ptr(score), _ptr(prio)))
        return score, prio

    def move_grad(self, feat, label, stream=None):
        """(mean BCE, gradient float32[move_num_params]) of labelled feature rows."""
        import torch
        loss = C.c_float(0)
        g = np.zeros(self.move_num_params(), dtype=np.float32)
        if stream is None:
            stream = torch.cuda.current_stream(feat.device).cuda_stream
        _check(lib().gp_gnn_move_grad_device(self._h, feat.shape[0], _ptr(feat), _ptr(label), C.c_void_p(stream),
                                             C.byref(loss), g.ctypes.data_as(C.POINTER(C.c_float))))
        return float(loss.value), g

    def move_train_step(self, feat, label, lr: float = 1e-2, stream=None) -> float:
        """One Adam step of the head; returns the loss before it."""
        import torch
        loss = C.c_float(0)
        if stream is None:
            stream = torch.cuda.current_stream(feat.device).cuda_stream
        _check(lib().gp_gnn_move_train_step_device(self._h, feat.shape[0], _ptr(feat), _ptr(label), float(lr),
                                                   C.c_void_p(stream), C.byref(loss)))
        return float(loss.value)

    def save(self, path: str) -> None:
        """params (float32), prio_bits, max_level and the move-order head (when
        present) in one .npz file."""
        extra = {}
        mp = self.get_move_params()
        if mp is not None:
            extra["move_params"] = mp
        with open(path, "wb") as f:
            np.savez(f, params=self.get_params(), prio_bits=np.int32(self.prio_bits),
                     max_level=np.int32(self.max_level), **extra)

    @classmethod
    def load(cls, path: str) -> "GNN":
        z = np.load(path)
        if isinstance(z, np.ndarray):        # bare parameter array
            return cls(cls._fit(z))
        m = cls(cls._fit(z["params"]), int(z["prio_bits"]), int(z["max_level"]) if "max_level" in z.files else -1)
        if "move_params" in z.files:
            m.set_move_params(z["move_params"])
        return m

    @classmethod
    def _fit(cls, p):
        """Parameters saved before the common-neighbour coefficient (the last
        one) existed get it as 0, which reproduces their scores."""
        p = np.asarray(p, dtype=np.float32)
        if len(p) == cls.num_params() - 1:
            p = np.concatenate([p, np.zeros(1, np.float32)])
        return p

    def forward(self, rowptr, colidx, vwgt=None, ewgt=None, level: int = 0, stream=None):
        """(priority int32[m], logit float32[m]) CUDA tensors of one graph."""
        import torch
        n = rowptr.numel() - 1
        m = colidx.numel()
        prio = torch.empty(m, dtype=torch.int32, device=rowptr.device)
        logit = torch.empty(m, dtype=torch.float32, device=rowptr.device)
        if stream is None:
            stream = torch.cuda.current_stream(rowptr.device).cuda_stream
        _check(lib().gp_gnn_forward_device(self._h, n, _ptr(rowptr), _ptr(colidx), _ptr(vwgt), _ptr(ewgt), int(level),
                                           C.c_void_p(stream), _ptr(prio), _ptr(logit)))
        return prio, logit

    def grad(self, rowptr, colidx, label, vwgt=None, ewgt=None, level: int = 0, stream=None):
        """(mean BCE loss, gradient float32[num_params]) of one labelled graph."""
        import torch
        n = rowptr.numel() - 1
        assert label.dtype == torch.uint8 and label.numel() == colidx.numel()
        loss = C.c_float(0)
        g = np.zeros(self.num_params(), dtype=np.float32)
        if stream is None:
            stream = torch.cuda.current_stream(rowptr.device).cuda_stream
        _check(lib().gp_gnn_grad_device(self._h, n, _ptr(rowptr), _ptr(colidx), _ptr(vwgt), _ptr(ewgt), int(level),
                                        _ptr(label), C.c_void_p(stream), C.byref(loss),
                                        g.ctypes.data_as(C.POINTER(C.c_float))))
        return float(loss.value), g

    def train_step(self, samples, lr: float = 1e-3, stream=None) -> float:
        """One Adam step over samples = [(rowptr, colidx, vwgt, ewgt, level, label)];
        returns the mean loss before the step."""
        import torch
        G = len(samples)
        ns = np.array([s[0].numel() - 1 for s in samples], dtype=np.int64)
        vp = lambda ts: (C.c_void_p * G)(*[t.data_ptr() if t is not None else None for t in ts])
        lv = np.array([int(s[4]) for s in samples], dtype=np.int32)
        loss = C.c_float(0)
        dev = samples[0][0].device
        if stream is None:
            stream = torch.cuda.current_stream(dev).cuda_stream
        _check(lib().gp_gnn_train_step_device(self._h, G, i64p(ns), vp([s[0] for s in samples]),
                                              vp([s[1] for s in samples]), vp([s[2] for s in samples]),
                                              vp([s[3] for s in samples]), i32p(lv), vp([s[5] for s in samples]),
                                              float(lr), C.c_void_p(stream), C.byref(loss)))
        return float(loss.value)

    def close(self) -> None:
        if self._h:
            lib().gp_gnn_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


WEIGHTS_PATH = os.path.join(HERE, "gnn_weights.npz")


def default_gnn() -> GNN:
    """The scorer trained by thegraphpartitioning_b200.learned on plain-partitioner
    labels (gnn_weights.npz beside this file)."""
    if not os.path.exists(WEIGHTS_PATH):
        raise RuntimeError(f"{WEIGHTS_PATH} is missing: train it with `python -m thegraphpartitioning_b200.learned train`")
    return GNN.load(WEIGHTS_PATH)


def partition_learned(rowptr, colidx, k: int, model: GNN, imbalance: float = 0.03, seed: int = 0, vwgt=None,
                      ewgt=None, options=None, fallback: bool = True, trace: bool = False, out=None, stream=None):
    """V-cycle with the model's scores as matching priorities (torch CUDA
    tensors).  fallback=True also runs the plain V-cycle and keeps the learned
    partition only when its exact cut <= the plain cut (balance permitting).
    Returns (part, stats, report, trace_events)."""
    import torch
    L = lib()
    opt = _opts(options)
    st = GpStats()
    rep = GpLearnedReport()
    col = _collector(trace)
    tfn = C.cast(col.cfunc, C.c_void_p) if col else None
    n = rowptr.numel() - 1
    assert rowptr.is_cuda and rowptr.dtype == torch.int64 and colidx.dtype == torch.int32
    part = out if out is not None else torch.empty(max(n, 0), dtype=torch.int32, device=rowptr.device)
    if stream is None:
        stream = torch.cuda.current_stream(rowptr.device).cuda_stream
    rc = L.gp_partition_learned_device(n, _ptr(rowptr), _ptr(colidx), _ptr(vwgt), _ptr(ewgt), int(k),
                                       float(imbalance), int(seed) & 0xFFFFFFFFFFFFFFFF, _ptr(part), C.c_void_p(stream),
                                       C.byref(opt), C.byref(st), model._h, 1 if fallback else 0, C.byref(rep), tfn, None)
    _check(rc)
    return part, st.as_dict(), rep.as_dict(), (col.events if col else [])


def default_options() -> GpOptions:
    o = GpOptions()
    _check(lib().gp_default_options(C.byref(o)))
    return o


def checked_violations(clear: bool = True):
    """Bounds-checked build only: (violations counted, first failing site as
    translation unit * 100000 + line, or -1) since the last clear."""
    cnt, site = C.c_int64(0), C.c_int32(0)
    _check(lib().gp_checked_violations(C.byref(cnt), C.byref(site), 1 if clear else 0))
    return int(cnt.value), int(site.value)


def release_workspace() -> None:
    _check(lib().gp_release_workspace())


def version() -> str:
    return lib().gp_version().decode()
