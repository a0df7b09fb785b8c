"""ctypes view of the CPU oracle (oracle/sbp_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's cpu_baseline leg as the checker, never by the partitioner.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "sbp_oracle.cpp")
LIB = os.path.join(HERE, "liboracle.so")


def build(force=False):
    if force or not os.path.exists(LIB) or os.path.getmtime(SRC) > os.path.getmtime(LIB):
        tmp = LIB + ".tmp"
        subprocess.run(["g++", "-std=c++17", "-O3", "-fPIC", "-shared", SRC, "-o", tmp],
                       check=True)
        os.replace(tmp, LIB)
    return LIB


build()
_lib = C.CDLL(LIB)
_vp = C.c_void_p


class _G(C.Structure):
    _fields_ = [("N", C.c_int32), ("E", C.c_int32)] + [
        (k, C.c_void_p) for k in ("out_ptr", "out_idx", "out_w", "in_ptr", "in_idx", "in_w",
                                  "deg_out", "deg_in")]


class Options(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("num_proposals", C.c_int32),
                ("reduction_rate", C.c_float), ("max_nodal_itr", C.c_int32),
                ("num_batches", C.c_int32), ("threshold1", C.c_float),
                ("threshold2", C.c_float), ("window", C.c_int32), ("max_outer", C.c_int32),
                ("exact", C.c_int32), ("mh", C.c_int32), ("beta", C.c_double),
                ("ref_grid", C.c_int32)]


class Report(C.Structure):
    _fields_ = [("B", C.c_int32), ("S", C.c_double), ("outer_steps", C.c_int32),
                ("nodal_itrs", C.c_int32), ("nodal_proposals", C.c_int64),
                ("accepted", C.c_int64), ("ms_total", C.c_double), ("ms_merge", C.c_double),
                ("ms_nodal", C.c_double), ("ms_rebuild", C.c_double), ("status", C.c_int32)]


def _sig(name, res, *args):
    f = getattr(_lib, name)
    f.restype = res
    f.argtypes = list(args)


_GP = C.POINTER(_G)
_sig("orc_philox", None, _vp, _vp, _vp)
_sig("orc_build_blockmodel", C.c_int64, _GP, _vp, C.c_int32, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
     _vp)
_sig("orc_nodal_delta", None, _GP, _vp, C.c_int32, C.c_int32, _vp, _vp, _vp, _vp, _vp)
_sig("orc_merge_delta", None, _GP, _vp, C.c_int32, C.c_int32, _vp, _vp, _vp, _vp)
_sig("orc_mdl", C.c_double, _GP, _vp, C.c_int32, C.POINTER(C.c_double))
_sig("orc_mdl_mode", C.c_double, _GP, _vp, C.c_int32, C.c_int32, C.POINTER(C.c_double))
_sig("orc_nodal_delta_mode", None, _GP, _vp, C.c_int32, C.c_int32, _vp, _vp, C.c_int32, _vp, _vp)
_sig("orc_merge_delta_mode", None, _GP, _vp, C.c_int32, C.c_int32, _vp, C.c_int32, _vp, _vp, _vp)
_sig("orc_nodal_batch_mode", C.c_double, _GP, _vp, C.c_int32, C.c_uint64, C.c_uint32, C.c_int32,
     C.c_int32, C.c_int32, C.c_int32, C.c_double, _vp, _vp)
_sig("orc_merge_proposals", None, _GP, _vp, C.c_int32, C.c_int32, C.c_uint64, C.c_uint32, _vp)
_sig("orc_nodal_batch", C.c_double, _GP, _vp, C.c_int32, C.c_uint64, C.c_uint32, C.c_int32,
     C.c_int32, _vp, _vp)
_sig("orc_merge_step", C.c_int32, _GP, _vp, C.c_int32, C.c_int32, C.c_int32, C.c_uint64,
     C.c_uint32, _vp, _vp)
_sig("orc_merge_step_mode", C.c_int32, _GP, _vp, C.c_int32, C.c_int32, C.c_int32, C.c_uint64,
     C.c_uint32, C.c_int32, _vp, _vp)
_sig("orc_apply_merges", C.c_int32, C.c_int32, _vp, C.c_int32, C.c_int32, _vp, _vp)
_sig("orc_partition", C.c_int, _GP, C.POINTER(Options), _vp, C.POINTER(Report))
_sig("orc_partition_trace", C.c_int, _GP, C.POINTER(Options), _vp, _vp, _vp, _vp, C.c_int32)
_sig("orc_time_nodal", C.c_double, _GP, _vp, C.c_int32, C.c_uint64, C.c_int32, C.c_int32)
_sig("orc_evaluate", None, C.c_int32, _vp, _vp, _vp)


def _p(a):
    return a.ctypes.data_as(_vp)


def _g(g):
    s = _G()
    s.N, s.E = g.N, g.E
    for k in ("out_ptr", "out_idx", "out_w", "in_ptr", "in_idx", "in_w", "deg_out", "deg_in"):
        setattr(s, k, _p(getattr(g, k)))
    return s


def philox(ctr, key):
    c = np.ascontiguousarray(ctr, dtype=np.uint32)
    k = np.ascontiguousarray(key, dtype=np.uint32)
    o = np.zeros(4, np.uint32)
    _lib.orc_philox(_p(c), _p(k), _p(o))
    return o


def build_blockmodel(g, part, B):
    part = np.ascontiguousarray(part, dtype=np.int32)
    cap = max(g.E, 1)
    out = dict(optr=np.zeros(B + 1, np.int32), ocol=np.zeros(cap, np.int32),
               ocnt=np.zeros(cap, np.uint32), iptr=np.zeros(B + 1, np.int32),
               icol=np.zeros(cap, np.int32), icnt=np.zeros(cap, np.uint32),
               d_out=np.zeros(B, np.uint32), d_in=np.zeros(B, np.uint32))
    n = _lib.orc_build_blockmodel(C.byref(_g(g)), _p(part), B, *[_p(out[k]) for k in (
        "optr", "ocol", "ocnt", "iptr", "icol", "icnt", "d_out", "d_in")])
    for k in ("ocol", "ocnt", "icol", "icnt"):
        out[k] = out[k][:n]
    return out


def nodal_delta(g, part, B, verts, props):
    part = np.ascontiguousarray(part, dtype=np.int32)
    verts = np.ascontiguousarray(verts, dtype=np.int32)
    props = np.ascontiguousarray(props, dtype=np.int32)
    dS = np.zeros(max(verts.size, 1))
    q3 = np.zeros(max(verts.size, 1), np.uint8)
    _lib.orc_nodal_delta(C.byref(_g(g)), _p(part), B, verts.size, _p(verts), _p(props), _p(dS),
                         _p(q3), None)
    return dS[:verts.size], q3[:verts.size].astype(bool)


def nodal_delta_scale(g, part, B, verts, props):
    """GSAP's dS of the moves and the sum of the magnitudes of the eight row
    sums each is the difference of (FP64 rounding grows with them)."""
    part = np.ascontiguousarray(part, dtype=np.int32)
    verts = np.ascontiguousarray(verts, dtype=np.int32)
    props = np.ascontiguousarray(props, dtype=np.int32)
    n = max(verts.size, 1)
    dS, q3, mag = np.zeros(n), np.zeros(n, np.uint8), np.zeros(n)
    _lib.orc_nodal_delta(C.byref(_g(g)), _p(part), B, verts.size, _p(verts), _p(props), _p(dS),
                         _p(q3), _p(mag))
    return dS[:verts.size], mag[:verts.size]


def nodal_delta_exact(g, part, B, verts, props):
    """Exact-mode dS of the moves and their log Hastings ratios."""
    part = np.ascontiguousarray(part, dtype=np.int32)
    verts = np.ascontiguousarray(verts, dtype=np.int32)
    props = np.ascontiguousarray(props, dtype=np.int32)
    dS = np.zeros(max(verts.size, 1))
    lh = np.zeros(max(verts.size, 1))
    _lib.orc_nodal_delta_mode(C.byref(_g(g)), _p(part), B, verts.size, _p(verts), _p(props), 1,
                              _p(dS), _p(lh))
    return dS[:verts.size], lh[:verts.size]


def merge_delta_exact(g, part, B, props, np_=10):
    part = np.ascontiguousarray(part, dtype=np.int32)
    props = np.ascontiguousarray(props, dtype=np.int32)
    dS = np.zeros(B * np_)
    best = np.zeros(B, np.int32)
    bds = np.zeros(B)
    _lib.orc_merge_delta_mode(C.byref(_g(g)), _p(part), B, np_, _p(props), 1, _p(dS), _p(best),
                              _p(bds))
    return dS, best, bds


def nodal_batch_mode(g, part, B, seed, seq, lo, hi, exact=1, mh=1, beta=3.0):
    part = np.array(part, dtype=np.int32, copy=True)
    n = max(hi - lo, 1)
    dS = np.zeros(n)
    props = np.zeros(n, np.int32)
    tot = _lib.orc_nodal_batch_mode(C.byref(_g(g)), _p(part), B, seed, seq, lo, hi, exact, mh,
                                    beta, _p(dS), _p(props))
    return part, dS[:hi - lo], props[:hi - lo], tot


def merge_delta(g, part, B, props, np_=10):
    part = np.ascontiguousarray(part, dtype=np.int32)
    props = np.ascontiguousarray(props, dtype=np.int32)
    dS = np.zeros(B * np_)
    best = np.zeros(B, np.int32)
    bds = np.zeros(B)
    _lib.orc_merge_delta(C.byref(_g(g)), _p(part), B, np_, _p(props), _p(dS), _p(best), _p(bds))
    return dS, best, bds


def mdl(g, part, B):
    part = np.ascontiguousarray(part, dtype=np.int32)
    d = C.c_double()
    S = _lib.orc_mdl(C.byref(_g(g)), _p(part), B, C.byref(d))
    return S, d.value


def mdl_mode(g, part, B, exact=1):
    """exact = 1: the standard description length in bits; 0: GSAP's (Q6)."""
    part = np.ascontiguousarray(part, dtype=np.int32)
    d = C.c_double()
    S = _lib.orc_mdl_mode(C.byref(_g(g)), _p(part), B, exact, C.byref(d))
    return S, d.value


def merge_proposals(g, part, B, seed, seq, np_=10):
    part = np.ascontiguousarray(part, dtype=np.int32)
    props = np.zeros(B * np_, np.int32)
    _lib.orc_merge_proposals(C.byref(_g(g)), _p(part), B, np_, seed, seq, _p(props))
    return props


def nodal_batch(g, part, B, seed, seq, lo, hi):
    part = np.array(part, dtype=np.int32, copy=True)
    n = max(hi - lo, 1)
    dS = np.zeros(n)
    props = np.zeros(n, np.int32)
    tot = _lib.orc_nodal_batch(C.byref(_g(g)), _p(part), B, seed, seq, lo, hi, _p(dS), _p(props))
    return part, dS[:hi - lo], props[:hi - lo], tot


def merge_step(g, part, B, B_to_merge, seed, seq, np_=10, ref_grid=0):
    part = np.array(part, dtype=np.int32, copy=True)
    best = np.zeros(B, np.int32)
    bds = np.zeros(B)
    nb = _lib.orc_merge_step_mode(C.byref(_g(g)), _p(part), B, B_to_merge, np_, seed, seq,
                                  ref_grid, _p(best), _p(bds))
    return part, nb, best, bds


def apply_merges(part, B, B_to_merge, best, best_dS):
    part = np.array(part, dtype=np.int32, copy=True)
    best = np.ascontiguousarray(best, dtype=np.int32)
    best_dS = np.ascontiguousarray(best_dS, dtype=np.float64)
    nb = _lib.orc_apply_merges(part.size, _p(part), B, B_to_merge, _p(best), _p(best_dS))
    return part, nb


def default_options(**kw):
    o = Options(seed=0, num_proposals=10, reduction_rate=0.35, max_nodal_itr=100, num_batches=4,
                threshold1=5e-4, threshold2=1e-4, window=3, max_outer=1000, exact=0, mh=0,
                beta=3.0, ref_grid=-1)
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def partition(g, **kw):
    o = default_options(**kw)
    lab = np.zeros(g.N, np.int32)
    r = Report()
    st = _lib.orc_partition(C.byref(_g(g)), C.byref(o), _p(lab), C.byref(r))
    return lab, {k: getattr(r, k) for k, _ in r._fields_}, st


def partition_trace(g, max_steps=1000, **kw):
    """orc_partition with its outer-step trace: labels and a list of (B, S,
    cumulative sweeps) per outer step, in the order the golden section saw
    them."""
    o = default_options(**kw)
    lab = np.zeros(g.N, np.int32)
    sb = np.zeros(max_steps, np.int32)
    ss = np.zeros(max_steps, np.float64)
    si = np.zeros(max_steps, np.int32)
    n = _lib.orc_partition_trace(C.byref(_g(g)), C.byref(o), _p(lab), _p(sb), _p(ss), _p(si),
                                 max_steps)
    if n < 0:
        raise RuntimeError("oracle partition failed")
    n = min(n, max_steps)
    return lab, [(int(sb[i]), float(ss[i]), int(si[i])) for i in range(n)]


def time_nodal(g, part, B, seed, batches, num_batches=4):
    part = np.array(part, dtype=np.int32, copy=True)
    ms = _lib.orc_time_nodal(C.byref(_g(g)), _p(part), B, seed, batches, num_batches)
    return ms, part


def evaluate(truth, given):
    t = np.ascontiguousarray(truth, dtype=np.int32)
    g = np.ascontiguousarray(given, dtype=np.int32)
    o = np.zeros(3)
    _lib.orc_evaluate(t.size, _p(t), _p(g), _p(o))
    return tuple(o)


# ------------------------------------------------------- benchmark graphs --
_sig("orc_dcsbm", C.c_int64, C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_int32, C.c_int32,
     C.c_double, C.c_uint64, _vp, _vp, C.c_int64, _vp)

# (p_in, Dirichlet alpha) of the GraphChallenge-style variants
VARIANTS = {"LL": (0.8, 20.0), "LH": (0.8, 1.0), "HL": (0.5, 20.0), "HH": (0.5, 1.0)}


class Graph:
    """Both CSR directions of a directed graph, N+1 row pointers, the way
    GSAP/load.hpp:86-117 orders them (each row in edge order), weighted
    degrees, and the planted labels."""

    def __init__(self, N, src, dst, w=None, truth=None):
        src = np.ascontiguousarray(src, dtype=np.int32)
        dst = np.ascontiguousarray(dst, dtype=np.int32)
        w = np.ones(src.size, np.uint32) if w is None else np.ascontiguousarray(w, np.uint32)
        self.N, self.E = int(N), int(src.size)
        o = np.argsort(src, kind="stable")
        i = np.argsort(dst, kind="stable")
        self.out_ptr = np.zeros(N + 1, np.int32)
        self.out_ptr[1:] = np.cumsum(np.bincount(src, minlength=N))
        self.in_ptr = np.zeros(N + 1, np.int32)
        self.in_ptr[1:] = np.cumsum(np.bincount(dst, minlength=N))
        self.out_idx, self.out_w = dst[o].copy(), w[o].copy()
        self.in_idx, self.in_w = src[i].copy(), w[i].copy()
        self.deg_out = np.bincount(src, weights=w, minlength=N).astype(np.uint32)
        self.deg_in = np.bincount(dst, weights=w, minlength=N).astype(np.uint32)
        self.true_partitions = None if truth is None else np.ascontiguousarray(truth, np.int32)


def dcsbm(N, B, alpha, p_in, seed=0, deg_min=5, deg_max=50, exponent=2.5):
    """The seeded DCSBM graph of the benchmarks (orc_dcsbm)."""
    cap = N * deg_max
    src = np.zeros(cap, np.int32)
    dst = np.zeros(cap, np.int32)
    truth = np.zeros(N, np.int32)
    E = _lib.orc_dcsbm(N, B, float(alpha), float(p_in), deg_min, deg_max, float(exponent), seed,
                       _p(src), _p(dst), cap, _p(truth))
    if E < 0:
        raise ValueError("bad DCSBM parameters")
    return Graph(N, src[:E], dst[:E], truth=truth)


def dcsbm_variant(variant, N, B, seed=0):
    p_in, alpha = VARIANTS[variant]
    return dcsbm(N, B, alpha, p_in, seed=seed)


def write_graph_bin(g, path):
    """The graph file oracle/gsap_ref_main.cu reads: int32 magic 0x53425047,
    N, E, 0, then out_ptr (N+1), out_idx, out_w, in_ptr (N+1), in_idx, in_w,
    deg_out, deg_in."""
    import struct
    with open(path, "wb") as f:
        f.write(struct.pack("<4i", 0x53425047, g.N, g.E, 0))
        for a in (g.out_ptr, g.out_idx, g.out_w, g.in_ptr, g.in_idx, g.in_w, g.deg_out,
                  g.deg_in):
            f.write(np.ascontiguousarray(a).tobytes())
