"""ctypes view of the reference's own kernels compiled for the host
(oracle/_ref/libref_kernels.so, built by oracle/build_ref.sh from GSAP's
kernels.hpp).  Test infrastructure: present only where the reference tree
was available at build time."""
import ctypes as C
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "oracle", "_ref", "libref_kernels.so")
available = os.path.exists(LIB)
_lib = C.CDLL(LIB) if available else None
_vp = C.c_void_p


def _p(a):
    return a.ctypes.data_as(_vp)


def _ref_layout(bm):
    """Row pointers with B entries (the reference's layout) and nnz."""
    return bm["optr"][:-1].copy(), bm["iptr"][:-1].copy(), int(bm["ocol"].size)


def nodal_batch(g, part, B, bm, props_by_vertex, BS, itr):
    """Runs the reference's nodal kernel chain for batch `itr` of size BS.
    Returns (dS_out_blocks[B], terms[6, BS], dS_accepted[BS], new part)."""
    part = np.array(part, dtype=np.int32, copy=True)
    optr, iptr, nnz = _ref_layout(bm)
    gop = np.ascontiguousarray(g.out_ptr[:-1])
    gip = np.ascontiguousarray(g.in_ptr[:-1])
    dso = np.zeros(B, np.float32)
    terms = np.zeros(6 * BS, np.float32)
    acc = np.zeros(BS, np.float32)
    props = np.ascontiguousarray(props_by_vertex, dtype=np.int32)
    f = _lib.ref_nodal_batch
    f.restype = None
    f(C.c_int(g.N), C.c_int(g.E), _p(gop), _p(g.out_idx), _p(g.out_w), _p(gip), _p(g.in_idx),
      _p(g.in_w), _p(g.deg_out), _p(g.deg_in), C.c_int(B), _p(optr), _p(bm["ocol"]),
      _p(bm["ocnt"]), _p(iptr), _p(bm["icol"]), _p(bm["icnt"]), C.c_long(nnz), _p(bm["d_out"]),
      _p(bm["d_in"]), _p(part), _p(props), C.c_int(BS), C.c_int(itr), _p(dso), _p(terms),
      _p(acc))
    return dso, terms.reshape(6, BS), acc, part


def merge_delta(B, bm, props, np_=10):
    optr, iptr, nnz = _ref_layout(bm)
    props = np.ascontiguousarray(props, dtype=np.int32)
    dS = np.zeros(B * np_, np.float32)
    f = _lib.ref_merge_delta
    f.restype = None
    f(C.c_int(B), C.c_int(np_), _p(optr), _p(bm["ocol"]), _p(bm["ocnt"]), _p(iptr),
      _p(bm["icol"]), _p(bm["icnt"]), C.c_long(nnz), _p(bm["d_out"]), _p(bm["d_in"]), _p(props),
      _p(dS))
    return dS


def mdl(B, N, E, bm):
    optr, _, nnz = _ref_layout(bm)
    dS = C.c_double()
    S = C.c_float()
    f = _lib.ref_mdl
    f.restype = None
    f(C.c_int(B), C.c_int(N), C.c_int(E), _p(optr), _p(bm["ocol"]), _p(bm["ocnt"]), C.c_long(nnz),
      _p(bm["d_out"]), _p(bm["d_in"]), C.byref(dS), C.byref(S))
    return S.value, dS.value


def accepted_prob(B, bm):
    out = np.zeros(B, np.float32)
    f = _lib.ref_accepted_prob
    f.restype = None
    f(C.c_int(B), _p(bm["d_out"]), _p(bm["d_in"]), _p(out))
    return out
