"""Python view of the partitioner's C ABI (include/sbp.h), through ctypes.

This mirrors GSAP's host interface for the SBP path: a ``Graph`` with both
CSR directions and weighted node degrees (GSAP/graph.hpp:32-45), a loader
with GSAP's TSV semantics (GSAP/load.hpp:6-133) and ``partition(g)``
(GSAP/partition.hpp:852-954), which fills ``g.partitions``.  Every call goes
to the CUDA library ``libsbp.so`` built in-tree; there is no fallback, and a
missing library is an ImportError.
"""
from __future__ import annotations

import ctypes as C
import types
import os
import struct
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libsbp.so")

if not os.path.exists(_LIB_PATH):
    raise ImportError(
        f"{_LIB_PATH} is missing: build it with `python -m gsap_b200.build` "
        "(the partitioner has no CPU fallback)")

_lib = C.CDLL(_LIB_PATH)

_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


class _GraphCSR(C.Structure):
    _fields_ = [("N", C.c_int32), ("E", C.c_int32),
                ("out_ptr", C.c_void_p), ("out_idx", C.c_void_p), ("out_w", C.c_void_p),
                ("in_ptr", C.c_void_p), ("in_idx", C.c_void_p), ("in_w", C.c_void_p),
                ("deg_out", C.c_void_p), ("deg_in", C.c_void_p)]


class Options(C.Structure):
    """sbp_options; defaults are GSAP's hyper-parameters (partition.hpp:855-861).

    exact = 1 scores moves and merges by the exact change of the MDL, mh = 1
    accepts nodal moves by Metropolis-Hastings at inverse temperature beta
    (per bit); the defaults (0, 0) reproduce GSAP."""
    _fields_ = [("seed", C.c_uint64), ("num_proposals", C.c_int32),
                ("reduction_rate", C.c_float), ("max_nodal_itr", C.c_int32),
                ("num_batches", C.c_int32), ("threshold1", C.c_float),
                ("threshold2", C.c_float), ("window", C.c_int32), ("max_outer", C.c_int32),
                ("device", C.c_int32), ("use_graphs", C.c_int32), ("verbose", C.c_int32),
                ("dense_max", C.c_int32), ("exact", C.c_int32), ("mh", C.c_int32),
                ("beta", C.c_double), ("ref_grid", C.c_int32), ("phase_timing", C.c_int32)]


class Report(C.Structure):
    _fields_ = [("B", C.c_int32), ("S", C.c_double), ("outer_steps", C.c_int32),
                ("nodal_itrs", C.c_int32), ("nodal_proposals", C.c_int64),
                ("accepted_moves", C.c_int64), ("ms_total", C.c_double),
                ("ms_merge", C.c_double), ("ms_nodal", C.c_double),
                ("ms_rebuild", C.c_double), ("ms_h2d", C.c_double),
                ("bytes_nodal", C.c_double), ("bytes_rebuild", C.c_double),
                ("bytes_merge", C.c_double), ("status", C.c_int32),
                ("ms_device", C.c_double), ("ms_nodal_kernel", C.c_double),
                ("nodal_launches", C.c_int64), ("kernel_launches", C.c_int64),
                ("graph_captures", C.c_int64), ("graph_replays", C.c_int64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class BatchReport(C.Structure):
    _fields_ = [("count", C.c_int32), ("max_active", C.c_int32), ("ticks", C.c_int64),
                ("kernel_launches", C.c_int64), ("ms_total", C.c_double),
                ("ms_device", C.c_double), ("peak_bytes", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class ServerOptions(C.Structure):
    _fields_ = [("partition", Options), ("hbm_budget", C.c_uint64), ("max_active", C.c_int32),
                ("max_queued", C.c_int32), ("lanes", C.c_int32), ("lane_split", C.c_int32)]


class JobTimes(C.Structure):
    _fields_ = [("ms_queue", C.c_double), ("ms_run", C.c_double), ("ms_latency", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_int64), ("completed", C.c_int64), ("failed", C.c_int64),
                ("active", C.c_int32), ("queued", C.c_int32), ("max_active_seen", C.c_int32),
                ("ticks", C.c_int64), ("bytes_active", C.c_double), ("peak_bytes", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class _DcsbmParams(C.Structure):
    _fields_ = [("N", C.c_int32), ("B", C.c_int32), ("alpha", C.c_double),
                ("p_in", C.c_double), ("deg_min", C.c_int32), ("deg_max", C.c_int32),
                ("exponent", C.c_double), ("seed", C.c_uint64)]


def _sig(name, res, *args):
    f = getattr(_lib, name)
    f.restype = res
    f.argtypes = list(args)
    return f


_vp = C.c_void_p
_sig("sbp_default_options", None, C.POINTER(Options))
_sig("sbp_last_error", C.c_char_p)
_sig("sbp_status_string", C.c_char_p, C.c_int)
_sig("sbp_partition", C.c_int, C.POINTER(_GraphCSR), C.POINTER(Options), _vp, C.POINTER(Report))
_sig("sbp_graph_upload", C.c_int, C.POINTER(_GraphCSR), C.c_int32, C.POINTER(_vp))
_sig("sbp_graph_release", C.c_int, _vp)
_sig("sbp_partition_resident", C.c_int, _vp, C.POINTER(Options), _vp, C.POINTER(Report))
_sig("sbp_build_blockmodel", C.c_int, C.POINTER(_GraphCSR), _vp, C.c_int32, _vp, _vp, _vp, _vp,
     _vp, _vp, _vp, _vp, C.POINTER(C.c_int64))
_sig("sbp_delta_mdl_nodal", C.c_int, C.POINTER(_GraphCSR), _vp, C.c_int32, C.c_int32, _vp, _vp,
     _vp)
_sig("sbp_delta_mdl_merge", C.c_int, C.POINTER(_GraphCSR), _vp, C.c_int32, C.c_int32, _vp, _vp,
     _vp, _vp)
_sig("sbp_delta_mdl_nodal_mode", C.c_int, C.POINTER(_GraphCSR), _vp, C.c_int32, C.c_int32, _vp,
     _vp, C.c_int32, _vp, _vp)
_sig("sbp_delta_mdl_merge_mode", C.c_int, C.POINTER(_GraphCSR), _vp, C.c_int32, C.c_int32, _vp,
     C.c_int32, _vp, _vp, _vp)
_sig("sbp_nodal_batch_mode", C.c_int, C.POINTER(_GraphCSR), _vp, C.c_int32, C.c_uint64,
     C.c_uint32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_double, _vp, _vp,
     C.POINTER(C.c_double))
_sig("sbp_apply_merges", C.c_int, C.c_int32, C.c_int32, _vp, _vp, _vp, C.POINTER(C.c_int32))
_sig("sbp_apply_merges_device", C.c_int, C.c_int32, C.c_int32, _vp, _vp, C.c_int32, _vp,
     C.POINTER(C.c_int32))
_sig("sbp_merge_proposals", C.c_int, C.POINTER(_GraphCSR), _vp, C.c_int32, C.c_int32, C.c_uint64,
     C.c_uint32, _vp)
_sig("sbp_nodal_batch", C.c_int, C.POINTER(_GraphCSR), _vp, C.c_int32, C.c_uint64, C.c_uint32,
     C.c_int32, C.c_int32, _vp, _vp, C.POINTER(C.c_double))
_sig("sbp_nodal_sweeps", C.c_int, C.POINTER(_GraphCSR), _vp, C.c_int32, C.c_uint64, C.c_uint32,
     C.c_int32, C.c_int32, C.c_int32, _vp)
_sig("sbp_merge_step", C.c_int, C.POINTER(_GraphCSR), _vp, C.c_int32, C.c_int32, C.c_int32,
     C.c_uint64, C.c_uint32, _vp, _vp, C.POINTER(C.c_int32))
_sig("sbp_merge_step_mode", C.c_int, C.POINTER(_GraphCSR), _vp, C.c_int32, C.c_int32, C.c_int32,
     C.c_uint64, C.c_uint32, C.c_int32, _vp, _vp, C.POINTER(C.c_int32))
_sig("sbp_mdl", C.c_int, C.POINTER(_GraphCSR), _vp, C.c_int32, C.POINTER(C.c_double),
     C.POINTER(C.c_double))
_sig("sbp_mdl_mode", C.c_int, C.POINTER(_GraphCSR), _vp, C.c_int32, C.c_int32,
     C.POINTER(C.c_double), C.POINTER(C.c_double))
_sig("sbp_mdl_device_static", C.c_int, C.c_int32, C.c_int32, C.c_int32, _vp, _vp, _vp, _vp, _vp,
     _vp, _vp, _vp)
_sig("sbp_partition_batch", C.c_int, _vp, C.c_int32, C.POINTER(Options), _vp, C.c_uint64, _vp,
     _vp, C.POINTER(BatchReport))
_sig("sbp_job_bytes", C.c_uint64, C.c_int32, C.c_int32, C.POINTER(Options))
_sig("sbp_server_default_options", None, C.POINTER(ServerOptions))
_sig("sbp_server_create", C.c_int, C.POINTER(ServerOptions), C.POINTER(_vp))
_sig("sbp_server_submit", C.c_int, _vp, C.POINTER(_GraphCSR), C.c_uint64, C.POINTER(C.c_int64))
_sig("sbp_server_poll", C.c_int, _vp, C.c_int64, C.c_int32, _vp, C.POINTER(Report),
     C.POINTER(JobTimes))
_sig("sbp_server_stats_get", C.c_int, _vp, C.POINTER(ServerStats))
_sig("sbp_server_destroy", C.c_int, _vp)
_sig("sbp_dcsbm_generate", C.c_int, C.POINTER(_DcsbmParams), C.POINTER(_vp))
_sig("sbp_edges_size", C.c_int, _vp, C.POINTER(C.c_int32), C.POINTER(C.c_int32))
_sig("sbp_edges_copy", C.c_int, _vp, _vp, _vp, _vp, _vp)
_sig("sbp_edges_free", None, _vp)
_sig("sbp_csr_from_edges", C.c_int, C.c_int32, C.c_int32, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
     _vp, _vp, _vp)
_sig("sbp_load_tsv", C.c_int, C.c_char_p, C.c_char_p, C.POINTER(_vp))
_sig("sbp_evaluate", C.c_int, C.c_int32, _vp, _vp, C.POINTER(C.c_double),
     C.POINTER(C.c_double), C.POINTER(C.c_double))
_sig("sbp_graph_from_device_edges", C.c_int, C.c_int32, C.c_int32, _vp, _vp, _vp, C.c_int32,
     C.POINTER(_vp))
_sig("sbp_dcsbm_generate_device", C.c_int, C.POINTER(_DcsbmParams), C.c_int32, _vp,
     C.POINTER(_vp))
_sig("sbp_graph_shape", C.c_int, _vp, C.POINTER(C.c_int32), C.POINTER(C.c_int32))
_sig("sbp_graph_download", C.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp)

LIB_PATH = _LIB_PATH
EXPORTED = [
    "sbp_default_options", "sbp_status_string", "sbp_last_error", "sbp_partition",
    "sbp_graph_upload", "sbp_graph_release", "sbp_partition_resident", "sbp_build_blockmodel",
    "sbp_delta_mdl_nodal", "sbp_delta_mdl_merge", "sbp_merge_proposals", "sbp_nodal_batch",
    "sbp_merge_step", "sbp_nodal_sweeps", "sbp_mdl", "sbp_dcsbm_generate", "sbp_edges_size", "sbp_edges_copy",
    "sbp_edges_free", "sbp_csr_from_edges", "sbp_load_tsv", "sbp_evaluate",
    "sbp_mdl_device_static", "sbp_job_bytes", "sbp_partition_batch", "sbp_server_default_options",
    "sbp_server_create", "sbp_server_submit", "sbp_server_poll", "sbp_server_stats_get",
    "sbp_server_destroy", "sbp_delta_mdl_nodal_mode", "sbp_delta_mdl_merge_mode",
    "sbp_nodal_batch_mode", "sbp_mdl_mode", "sbp_apply_merges", "sbp_apply_merges_device",
    "sbp_merge_step_mode", "sbp_graph_from_device_edges", "sbp_dcsbm_generate_device",
    "sbp_graph_shape", "sbp_graph_download",
]


class SbpError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{_lib.sbp_status_string(status).decode()}: {msg}")
        self.status = status


def _check(st):
    if st != 0:
        raise SbpError(st, _lib.sbp_last_error().decode())


def _p(a):
    return a.ctypes.data_as(_vp) if a is not None else None


def default_options(**kw) -> Options:
    o = Options()
    _lib.sbp_default_options(C.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise TypeError(f"unknown option {k}")
        setattr(o, k, v)
    return o


@dataclass
class Graph:
    """A directed graph in both CSR directions (GSAP/graph.hpp:32-45, with
    an N+1 row pointer).  ``partitions`` is filled by :func:`partition` and
    ``true_partitions`` holds planted labels when known (-1 otherwise)."""
    N: int
    E: int
    out_ptr: np.ndarray
    out_idx: np.ndarray
    out_w: np.ndarray
    in_ptr: np.ndarray
    in_idx: np.ndarray
    in_w: np.ndarray
    deg_out: np.ndarray
    deg_in: np.ndarray
    true_partitions: Optional[np.ndarray] = None
    partitions: Optional[np.ndarray] = None
    _keep: list = field(default_factory=list, repr=False)

    def csr(self) -> _GraphCSR:
        s = _GraphCSR()
        s.N, s.E = self.N, self.E
        s.out_ptr, s.out_idx, s.out_w = _p(self.out_ptr), _p(self.out_idx), _p(self.out_w)
        s.in_ptr, s.in_idx, s.in_w = _p(self.in_ptr), _p(self.in_idx), _p(self.in_w)
        s.deg_out, s.deg_in = _p(self.deg_out), _p(self.deg_in)
        return s

    @staticmethod
    def from_edges(N, src, dst, w=None, truth=None) -> "Graph":
        src = np.ascontiguousarray(src, dtype=np.int32)
        dst = np.ascontiguousarray(dst, dtype=np.int32)
        E = int(src.size)
        w = np.ones(E, np.uint32) if w is None else np.ascontiguousarray(w, dtype=np.uint32)
        arrs = dict(out_ptr=np.zeros(N + 1, np.int32), out_idx=np.zeros(max(E, 1), np.int32),
                    out_w=np.zeros(max(E, 1), np.uint32), in_ptr=np.zeros(N + 1, np.int32),
                    in_idx=np.zeros(max(E, 1), np.int32), in_w=np.zeros(max(E, 1), np.uint32),
                    deg_out=np.zeros(N, np.uint32), deg_in=np.zeros(N, np.uint32))
        _check(_lib.sbp_csr_from_edges(N, E, _p(src), _p(dst), _p(w), *[_p(arrs[k]) for k in (
            "out_ptr", "out_idx", "out_w", "in_ptr", "in_idx", "in_w", "deg_out", "deg_in")]))
        for k in ("out_idx", "out_w", "in_idx", "in_w"):
            arrs[k] = arrs[k][:E].copy()
        t = None if truth is None else np.ascontiguousarray(truth, dtype=np.int32)
        return Graph(N=N, E=E, true_partitions=t, **arrs)

    def edges(self):
        """(src, dst, w) in out-CSR order."""
        src = np.repeat(np.arange(self.N, dtype=np.int32), np.diff(self.out_ptr))
        return src, self.out_idx.copy(), self.out_w.copy()


def _edges_to_graph(h) -> Graph:
    N, E = C.c_int32(), C.c_int32()
    _check(_lib.sbp_edges_size(h, C.byref(N), C.byref(E)))
    src = np.empty(max(E.value, 1), np.int32)
    dst = np.empty(max(E.value, 1), np.int32)
    w = np.empty(max(E.value, 1), np.uint32)
    truth = np.empty(N.value, np.int32)
    _check(_lib.sbp_edges_copy(h, _p(src), _p(dst), _p(w), _p(truth)))
    _lib.sbp_edges_free(h)
    E = E.value
    return Graph.from_edges(N.value, src[:E], dst[:E], w[:E], truth)


def dcsbm(N, B, alpha, p_in, seed=0, deg_min=5, deg_max=50, exponent=2.5) -> Graph:
    """Seeded directed DCSBM graph with planted labels (sbp_dcsbm_generate)."""
    p = _DcsbmParams(N=N, B=B, alpha=float(alpha), p_in=float(p_in), deg_min=deg_min,
                     deg_max=deg_max, exponent=float(exponent), seed=seed)
    h = _vp()
    _check(_lib.sbp_dcsbm_generate(C.byref(p), C.byref(h)))
    return _edges_to_graph(h)


# The GraphChallenge-style variants: (p_in, Dirichlet alpha)
VARIANTS = {"LL": (0.8, 20.0), "LH": (0.8, 1.0), "HL": (0.5, 20.0), "HH": (0.5, 1.0)}


def dcsbm_variant(variant, N, B, seed=0) -> Graph:
    p_in, alpha = VARIANTS[variant]
    return dcsbm(N, B, alpha, p_in, seed=seed)


def load_tsv(path, truth_path=None) -> Graph:
    """A GraphChallenge TSV read with GSAP/load.hpp's semantics."""
    h = _vp()
    _check(_lib.sbp_load_tsv(path.encode(), truth_path.encode() if truth_path else None,
                             C.byref(h)))
    return _edges_to_graph(h)


def read_file(cat, size, root):
    """readFile(cat, size) of GSAP/load.hpp:6-49, with the dataset root given."""
    sub = {"LL": "lowOverlap_lowBlockSizeVar", "LH": "lowOverlap_highBlockSizeVar",
           "HL": "highOverlap_lowBlockSizeVar", "HH": "highOverlap_highBlockSizeVar"}[cat]
    n = {"1k": "1000", "5k": "5000", "20k": "20000", "50k": "50000", "200k": "200000",
         "1m": "1000000"}[size]
    base = os.path.join(root, sub, size, f"{n}_nodes")
    return load_tsv(base + ".tsv", base + "_truePartition.tsv")


def partition(g: Graph, options: Optional[Options] = None, **kw):
    """partition(g) of GSAP/partition.hpp:852-954: fills g.partitions and
    returns the run report."""
    o = options or default_options(**kw)
    lab = np.empty(g.N, np.int32)
    rep = Report()
    st = _lib.sbp_partition(C.byref(g.csr()), C.byref(o), _p(lab), C.byref(rep))
    _check(st)
    g.partitions = lab
    return rep.as_dict()


def job_bytes(N, E, options: Optional[Options] = None, **kw):
    """Device arena bytes of one job (the batch / server admission unit)."""
    o = options or default_options(**kw)
    return int(_lib.sbp_job_bytes(N, E, C.byref(o)))


def partition_batch(graphs, options: Optional[Options] = None, seeds=None, hbm_budget=0, **kw):
    """sbp_partition_batch: partitions the graphs together; returns
    (labels per graph, report per graph, batch report)."""
    o = options or default_options(**kw)
    n = len(graphs)
    csrs = (_GraphCSR * max(n, 1))()
    for i, g in enumerate(graphs):
        csrs[i] = g.csr()
    labs = [np.empty(g.N, np.int32) for g in graphs]
    ptrs = (C.c_void_p * max(n, 1))(*[lab.ctypes.data for lab in labs])
    reps = (Report * max(n, 1))()
    seed_arr = None
    if seeds is not None:
        seed_arr = np.ascontiguousarray(seeds, dtype=np.uint64)
        assert seed_arr.size == n
    br = BatchReport()
    st = _lib.sbp_partition_batch(C.cast(csrs, _vp), n, C.byref(o),
                                  None if seed_arr is None else seed_arr.ctypes.data,
                                  hbm_budget, C.cast(ptrs, _vp), C.cast(reps, _vp), C.byref(br))
    _check(st)
    return labs, [reps[i].as_dict() for i in range(n)], br.as_dict()


class Server:
    """sbp_server_*: a partition server with continuous batching on the device."""

    def __init__(self, options: Optional[Options] = None, hbm_budget=0, max_active=0,
                 max_queued=0, lanes=0, lane_split=0, **kw):
        so = ServerOptions()
        _lib.sbp_server_default_options(C.byref(so))
        so.partition = options or default_options(**kw)
        so.hbm_budget = hbm_budget
        so.max_active = max_active
        so.max_queued = max_queued
        so.lanes = lanes
        so.lane_split = lane_split
        self.h = _vp()
        self._n = {}
        _check(_lib.sbp_server_create(C.byref(so), C.byref(self.h)))

    def submit(self, g: Graph, seed=0):
        jid = C.c_int64()
        _check(_lib.sbp_server_submit(self.h, C.byref(g.csr()), seed, C.byref(jid)))
        self._n[jid.value] = g.N
        return jid.value

    def poll(self, jid, timeout_ms=-1):
        """(labels, report, times) when done; None while running (BUSY)."""
        lab = np.empty(self._n.get(jid, 0), np.int32)
        rep = Report()
        t = JobTimes()
        st = _lib.sbp_server_poll(self.h, jid, timeout_ms, _p(lab), C.byref(rep), C.byref(t))
        if st == 7:  # SBP_ERR_BUSY
            return None
        self._n.pop(jid, None)
        _check(st)
        return lab, rep.as_dict(), t.as_dict()

    def stats(self):
        s = ServerStats()
        _check(_lib.sbp_server_stats_get(self.h, C.byref(s)))
        return s.as_dict()

    def close(self):
        if self.h:
            _lib.sbp_server_destroy(self.h)
            self.h = _vp()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class ResidentGraph:
    """A graph uploaded to HBM once (sbp_graph_upload) and partitioned many
    times without host-to-device copies of its arrays."""

    def __init__(self, g: Graph, device=-1):
        self.g = g
        self.h = _vp()
        _check(_lib.sbp_graph_upload(C.byref(g.csr()), device, C.byref(self.h)))

    def partition(self, options: Optional[Options] = None, **kw):
        o = options or default_options(**kw)
        lab = np.empty(self.g.N, np.int32)
        rep = Report()
        _check(_lib.sbp_partition_resident(self.h, C.byref(o), _p(lab), C.byref(rep)))
        return lab, rep.as_dict()

    def close(self):
        if self.h:
            _lib.sbp_graph_release(self.h)
            self.h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DeviceGraph(ResidentGraph):
    """A resident graph built on the device, with no host CSR: from an edge
    list in device memory (sbp_graph_from_device_edges) or by the device
    DCSBM generator (sbp_dcsbm_generate_device)."""

    def __init__(self, handle, truth=None):
        self.h = handle
        N, E = C.c_int32(), C.c_int32()
        _check(_lib.sbp_graph_shape(self.h, C.byref(N), C.byref(E)))
        self.N, self.E = N.value, E.value
        self.true_partitions = truth
        self.g = types.SimpleNamespace(N=self.N, E=self.E)  # what partition() reads

    @staticmethod
    def from_edges(N, src_ptr, dst_ptr, E, w_ptr=None, device=-1) -> "DeviceGraph":
        """src_ptr, dst_ptr, w_ptr: device addresses of E int32 / uint32
        entries (w_ptr None for unit weights)."""
        h = _vp()
        _check(_lib.sbp_graph_from_device_edges(N, E, _vp(src_ptr), _vp(dst_ptr),
                                                _vp(w_ptr) if w_ptr else None, device,
                                                C.byref(h)))
        return DeviceGraph(h)

    def download(self) -> Graph:
        """A host copy of the CSR pair."""
        N, E = self.N, self.E
        arrs = dict(out_ptr=np.zeros(N + 1, np.int32), out_idx=np.zeros(max(E, 1), np.int32),
                    out_w=np.zeros(max(E, 1), np.uint32), in_ptr=np.zeros(N + 1, np.int32),
                    in_idx=np.zeros(max(E, 1), np.int32), in_w=np.zeros(max(E, 1), np.uint32),
                    deg_out=np.zeros(N, np.uint32), deg_in=np.zeros(N, np.uint32))
        _check(_lib.sbp_graph_download(self.h, *[_p(arrs[k]) for k in (
            "out_ptr", "out_idx", "out_w", "in_ptr", "in_idx", "in_w", "deg_out", "deg_in")]))
        for k in ("out_idx", "out_w", "in_idx", "in_w"):
            arrs[k] = arrs[k][:E].copy()
        return Graph(N=N, E=E, true_partitions=self.true_partitions, **arrs)


def dcsbm_device(N, B, alpha, p_in, seed=0, deg_min=5, deg_max=50, exponent=2.5,
                 device=-1) -> DeviceGraph:
    """The graph of :func:`dcsbm` with the same arguments, generated on the
    device (sbp_dcsbm_generate_device); planted labels in true_partitions."""
    p = _DcsbmParams(N=N, B=B, alpha=float(alpha), p_in=float(p_in), deg_min=deg_min,
                     deg_max=deg_max, exponent=float(exponent), seed=seed)
    truth = np.empty(N, np.int32)
    h = _vp()
    _check(_lib.sbp_dcsbm_generate_device(C.byref(p), device, _p(truth), C.byref(h)))
    return DeviceGraph(h, truth)


def dcsbm_variant_device(variant, N, B, seed=0, device=-1) -> DeviceGraph:
    p_in, alpha = VARIANTS[variant]
    return dcsbm_device(N, B, alpha, p_in, seed=seed, device=device)


# ------------------------------------------------------------ path pieces ---
def build_blockmodel(g: Graph, part, B):
    part = np.ascontiguousarray(part, dtype=np.int32)
    cap = max(g.E, 1)
    out = dict(optr=np.zeros(B + 1, np.int32), ocol=np.zeros(cap, np.int32),
               ocnt=np.zeros(cap, np.uint32), iptr=np.zeros(B + 1, np.int32),
               icol=np.zeros(cap, np.int32), icnt=np.zeros(cap, np.uint32),
               d_out=np.zeros(B, np.uint32), d_in=np.zeros(B, np.uint32))
    nnz = C.c_int64()
    _check(_lib.sbp_build_blockmodel(C.byref(g.csr()), _p(part), B, *[_p(out[k]) for k in (
        "optr", "ocol", "ocnt", "iptr", "icol", "icnt", "d_out", "d_in")], C.byref(nnz)))
    n = nnz.value
    for k in ("ocol", "ocnt", "icol", "icnt"):
        out[k] = out[k][:n]
    return out


def delta_mdl_nodal(g: Graph, part, B, verts, props):
    part = np.ascontiguousarray(part, dtype=np.int32)
    verts = np.ascontiguousarray(verts, dtype=np.int32)
    props = np.ascontiguousarray(props, dtype=np.int32)
    dS = np.zeros(max(verts.size, 1), np.float64)
    _check(_lib.sbp_delta_mdl_nodal(C.byref(g.csr()), _p(part), B, verts.size, _p(verts),
                                    _p(props), _p(dS)))
    return dS[:verts.size]


def delta_mdl_merge(g: Graph, part, B, props, np_=10):
    part = np.ascontiguousarray(part, dtype=np.int32)
    props = np.ascontiguousarray(props, dtype=np.int32)
    dS = np.zeros(B * np_, np.float64)
    best = np.zeros(B, np.int32)
    best_dS = np.zeros(B, np.float64)
    _check(_lib.sbp_delta_mdl_merge(C.byref(g.csr()), _p(part), B, np_, _p(props), _p(dS),
                                    _p(best), _p(best_dS)))
    return dS, best, best_dS


def delta_mdl_nodal_mode(g: Graph, part, B, verts, props, exact=1, hastings=True):
    """dS of each move in a scoring mode (exact = 1: the exact change of the
    MDL) and, with hastings, each move's log Hastings ratio."""
    part = np.ascontiguousarray(part, dtype=np.int32)
    verts = np.ascontiguousarray(verts, dtype=np.int32)
    props = np.ascontiguousarray(props, dtype=np.int32)
    n = max(verts.size, 1)
    dS = np.zeros(n, np.float64)
    lh = np.zeros(n, np.float64) if hastings else None
    _check(_lib.sbp_delta_mdl_nodal_mode(C.byref(g.csr()), _p(part), B, verts.size, _p(verts),
                                         _p(props), exact, _p(dS),
                                         _p(lh) if hastings else None))
    return dS[:verts.size], (lh[:verts.size] if hastings else None)


def delta_mdl_merge_mode(g: Graph, part, B, props, np_=10, exact=1):
    part = np.ascontiguousarray(part, dtype=np.int32)
    props = np.ascontiguousarray(props, dtype=np.int32)
    dS = np.zeros(B * np_, np.float64)
    best = np.zeros(B, np.int32)
    best_dS = np.zeros(B, np.float64)
    _check(_lib.sbp_delta_mdl_merge_mode(C.byref(g.csr()), _p(part), B, np_, _p(props), exact,
                                         _p(dS), _p(best), _p(best_dS)))
    return dS, best, best_dS


def apply_merges(B, B_to_merge, best, best_dS):
    """carry_out_best_merges on the host: (map from old to new block labels,
    new block count)."""
    best = np.ascontiguousarray(best, dtype=np.int32)
    best_dS = np.ascontiguousarray(best_dS, dtype=np.float64)
    m = np.zeros(max(B, 1), np.int32)
    nb = C.c_int32()
    _check(_lib.sbp_apply_merges(B, B_to_merge, _p(best), _p(best_dS), _p(m), C.byref(nb)))
    return m[:B], nb.value


def apply_merges_device(B, B_to_merge, best, best_dS, device=-1):
    """carry_out_best_merges on the GPU, as the partition loop runs it."""
    best = np.ascontiguousarray(best, dtype=np.int32)
    best_dS = np.ascontiguousarray(best_dS, dtype=np.float64)
    m = np.zeros(max(B, 1), np.int32)
    nb = C.c_int32()
    _check(_lib.sbp_apply_merges_device(B, B_to_merge, _p(best), _p(best_dS), device, _p(m),
                                        C.byref(nb)))
    return m[:B], nb.value


def merge_proposals(g: Graph, part, B, seed, seq, np_=10):
    part = np.ascontiguousarray(part, dtype=np.int32)
    props = np.zeros(B * np_, np.int32)
    _check(_lib.sbp_merge_proposals(C.byref(g.csr()), _p(part), B, np_, seed, seq, _p(props)))
    return props


def nodal_batch(g: Graph, part, B, seed, seq, lo, hi):
    part = np.array(part, dtype=np.int32, copy=True)
    n = max(hi - lo, 1)
    dS = np.zeros(n, np.float64)
    props = np.zeros(n, np.int32)
    tot = C.c_double()
    _check(_lib.sbp_nodal_batch(C.byref(g.csr()), _p(part), B, seed, seq, lo, hi, _p(dS),
                                _p(props), C.byref(tot)))
    return part, dS[:hi - lo], props[:hi - lo], tot.value


def nodal_batch_mode(g: Graph, part, B, seed, seq, lo, hi, exact=1, mh=1, beta=3.0):
    part = np.array(part, dtype=np.int32, copy=True)
    n = max(hi - lo, 1)
    dS = np.zeros(n, np.float64)
    props = np.zeros(n, np.int32)
    tot = C.c_double()
    _check(_lib.sbp_nodal_batch_mode(C.byref(g.csr()), _p(part), B, seed, seq, lo, hi, exact, mh,
                                     beta, _p(dS), _p(props), C.byref(tot)))
    return part, dS[:hi - lo], props[:hi - lo], tot.value


def nodal_sweeps(g: Graph, part, B, seed, seq0, num_batches=4, sweeps=1, dense_max=4096):
    """`sweeps` nodal sweeps as the nodal phase runs them; returns the new
    labels and the recorded dS sum of every batch."""
    part = np.array(part, dtype=np.int32, copy=True)
    sums = np.zeros(num_batches * sweeps, np.float64)
    _check(_lib.sbp_nodal_sweeps(C.byref(g.csr()), _p(part), B, seed, seq0, num_batches, sweeps,
                                 dense_max, _p(sums)))
    return part, sums


def merge_step(g: Graph, part, B, B_to_merge, seed, seq, np_=10, ref_grid=0):
    """One merge step (sbp_merge_step_mode); ref_grid = 1 makes it the first
    merge step of a run that reproduces GSAP's merge grid."""
    part = np.array(part, dtype=np.int32, copy=True)
    best = np.zeros(B, np.int32)
    best_dS = np.zeros(B, np.float64)
    nb = C.c_int32()
    _check(_lib.sbp_merge_step_mode(C.byref(g.csr()), _p(part), B, B_to_merge, np_, seed, seq,
                                    ref_grid, _p(best), _p(best_dS), C.byref(nb)))
    return part, nb.value, best, best_dS


def mdl(g: Graph, part, B, exact=0):
    """(S, data_S): GSAP's MDL (exact = 0) or the standard description
    length in bits (exact = 1, the objective of exact mode)."""
    part = np.ascontiguousarray(part, dtype=np.int32)
    S, dS = C.c_double(), C.c_double()
    _check(_lib.sbp_mdl_mode(C.byref(g.csr()), _p(part), B, exact, C.byref(S), C.byref(dS)))
    return S.value, dS.value


def mdl_device_static(N, E, B, out_ptr, out_col, out_cnt, d_out, d_in, S, data_S, stream=0):
    """sbp_mdl_device_static on device pointers (integers); allocates nothing."""
    _check(_lib.sbp_mdl_device_static(N, E, B, out_ptr, out_col, out_cnt, d_out, d_in, S, data_S,
                                      stream))


def evaluate(truth, given):
    """(pairwise recall, pairwise precision, NMI), evaluate.hpp:18-265."""
    truth = np.ascontiguousarray(truth, dtype=np.int32)
    given = np.ascontiguousarray(given, dtype=np.int32)
    r, p, n = C.c_double(), C.c_double(), C.c_double()
    _check(_lib.sbp_evaluate(truth.size, _p(truth), _p(given), C.byref(r), C.byref(p),
                             C.byref(n)))
    return r.value, p.value, n.value


# ------------------------------------------------------- graph file format --
_MAGIC = 0x53425047


def write_graph_bin(g: Graph, path):
    """Graph file read by the reference driver (header magic, N, E, 0; then
    out_ptr, out_idx, out_w, in_ptr, in_idx, in_w, deg_out, deg_in)."""
    with open(path, "wb") as f:
        f.write(struct.pack("<4i", _MAGIC, g.N, g.E, 0))
        for a in (g.out_ptr, g.out_idx, g.out_w, g.in_ptr, g.in_idx, g.in_w, g.deg_out,
                  g.deg_in):
            f.write(np.ascontiguousarray(a).tobytes())
