"""CPU oracle for the Invariant Bit Packing codec (numpy front end over libibp_oracle.so).

TEST INFRASTRUCTURE ONLY.  This package is the checker: tests/, the smoke()
entry point and bench.py's CPU-baseline / reference legs may call it; the
product (invariantbitpacking_b200) never imports it.

Every function restates the reference behaviour cited in oracle/ibp_oracle.h
(file:line in the reference repository).  Arrays are 2-D C-contiguous numpy
arrays of 1/2/4/8-byte words (any dtype; viewed as unsigned words).

Parity pinning: tests/golden/*.npz were dumped by the reference extension
itself (tests/golden/make_golden.py); tests/test_oracle_golden.py checks this
oracle against them.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "libibp_oracle.so")
_lib = None

_UINT = {1: np.uint8, 2: np.uint16, 4: np.uint32, 8: np.uint64}
_P = ctypes.c_void_p
_I64 = ctypes.c_int64


def build():
    """Compile the C restatement (make -C oracle)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        L = ctypes.CDLL(_LIB)
        sig = {
            "orc_count_bits": [_P, _I64, _I64, ctypes.c_int, _P],
            "orc_create_mask": [_P, _I64, _I64, ctypes.c_int, ctypes.c_float, _P, _P],
            "orc_check_feats": [_P, _I64, _I64, ctypes.c_int, _P, _P],
            "orc_preprocess": [_P, _I64, _I64, ctypes.c_int, ctypes.c_float, _P, _P, _P, _P, _P],
            "orc_compress_size": [_P, _I64, _I64, ctypes.c_int, _P, _P, _P, _I64, _P],
            "orc_compress": [_P, _I64, _I64, ctypes.c_int, _P, _P, _P, _I64, _P, _P],
            "orc_compress_condensed": [_P, _I64, _I64, ctypes.c_int, _P, _P, _P, _I64, _P, _P],
            "orc_decompress": [_P, _I64, _I64, ctypes.c_int, _P, _P, _P, _P, _I64, _P],
            "orc_kmeans_assign": [_P, _I64, _I64, ctypes.c_int, _P, ctypes.c_int, _P],
            "orc_kmeans_update": [_P, _I64, _I64, ctypes.c_int, _P, ctypes.c_int, _P],
            "orc_kmeans_masks": [_P, _I64, _I64, ctypes.c_int, _P, ctypes.c_int, ctypes.c_float, _P, _P],
            "orc_preprocess_kmeans": [_P, _I64, _I64, ctypes.c_int, ctypes.c_int, _P, _P, _P, _P],
            "orc_random_shuffle_init": [_I64, ctypes.c_int, _P, ctypes.c_int],
            "orc_set_threads": [ctypes.c_int],
            "orc_get_threads": [],
        }
        for name, args in sig.items():
            f = getattr(L, name)
            f.argtypes = args
        L.orc_check_feats.restype = ctypes.c_uint64
        L.orc_preprocess.restype = ctypes.c_int
        L.orc_get_threads.restype = ctypes.c_int
        for name in sig:
            if name not in ("orc_check_feats", "orc_preprocess", "orc_get_threads"):
                getattr(L, name).restype = None
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def words(a):
    """View a C-contiguous array as unsigned words of its own item size."""
    a = np.ascontiguousarray(a)
    return a.view(_UINT[a.dtype.itemsize])


def _rows(data):
    d = words(data)
    if d.ndim == 1:
        d = d.reshape(1, -1)
    assert d.ndim == 2
    return d, d.shape[0], d.shape[1], d.dtype.itemsize


def _like(out, data):
    """Return word arrays in the caller's dtype (so comparisons with the input are exact)."""
    dt = np.asarray(data).dtype
    return out.view(dt) if dt.itemsize == out.dtype.itemsize else out


def _idx(idx):
    return None if idx is None else np.ascontiguousarray(np.asarray(idx, dtype=np.int64))


def set_threads(t):
    lib().orc_set_threads(int(t))


def get_threads():
    return lib().orc_get_threads()


def count_bits(data):
    d, n, v, wb = _rows(data)
    c = np.zeros((v, 8 * wb), dtype=np.uint32)
    lib().orc_count_bits(_p(d), n, v, wb, _p(c))
    return c


def create_mask(counts, n, thr, itemsize):
    v = counts.shape[0]
    m = np.zeros(v, dtype=_UINT[itemsize])
    b = np.zeros(v, dtype=_UINT[itemsize])
    lib().orc_create_mask(_p(np.ascontiguousarray(counts, dtype=np.uint32)), n, v, itemsize,
                          float(thr), _p(m), _p(b))
    return m, b


def check_feats(data, mask, bitval):
    d, n, v, wb = _rows(data)
    return int(lib().orc_check_feats(_p(d), n, v, wb, _p(words(mask)), _p(words(bitval))))


def preprocess(data, threshold=None):
    """(mask, bitval, info) -- info has the per-step thresholds, saved bits and selection."""
    d, n, v, wb = _rows(data)
    m = np.zeros(v, dtype=_UINT[wb])
    b = np.zeros(v, dtype=_UINT[wb])
    saved = np.zeros(64, dtype=np.uint64)
    thrs = np.zeros(64, dtype=np.float32)
    ns = ctypes.c_int(0)
    thr = -1.0 if threshold is None else float(threshold)
    sel = lib().orc_preprocess(_p(d), n, v, wb, thr, _p(m), _p(b), _p(saved), _p(thrs),
                               ctypes.byref(ns))
    k = ns.value
    return _like(m, data), _like(b, data), {"selected": sel, "saved": saved[:k].copy(), "thresholds": thrs[:k].copy()}


def compress_size(data, mask, bitval, idx=None):
    d, n, v, wb = _rows(data)
    ix = _idx(idx)
    nout = n if ix is None else ix.shape[0]
    s = np.zeros(nout, dtype=np.int64)
    lib().orc_compress_size(_p(d), n, v, wb, _p(words(mask)), _p(words(bitval)), _p(ix), nout, _p(s))
    return s


def compress(data, mask, bitval, idx=None):
    """(compressed rows [nout, v], bitmask int32[(nout+31)//32])"""
    d, n, v, wb = _rows(data)
    ix = _idx(idx)
    nout = n if ix is None else ix.shape[0]
    out = np.zeros((nout, v), dtype=d.dtype)
    bm = np.zeros((nout + 31) // 32, dtype=np.int32)
    lib().orc_compress(_p(d), n, v, wb, _p(words(mask)), _p(words(bitval)), _p(ix), nout,
                       _p(out), _p(bm))
    return _like(out, data), bm


def compress_condensed(data, mask, bitval, idx=None):
    """(condensed words [sum(sizes)/wb], inclusive byte offsets int64[nout])"""
    d, n, v, wb = _rows(data)
    ix = _idx(idx)
    nout = n if ix is None else ix.shape[0]
    sizes = compress_size(d, mask, bitval, ix)
    offs = np.cumsum(sizes).astype(np.int64)
    total = int(offs[-1]) if nout else 0
    out = np.zeros(total // wb, dtype=d.dtype)
    lib().orc_compress_condensed(_p(d), n, v, wb, _p(words(mask)), _p(words(bitval)), _p(ix),
                                 nout, _p(offs), _p(out))
    return _like(out, data), offs


def decompress(comp, mask, bitval, bitmask, idx=None):
    d, n, v, wb = _rows(comp)
    ix = _idx(idx)
    nout = n if ix is None else ix.shape[0]
    out = np.zeros((nout, v), dtype=d.dtype)
    bm = np.ascontiguousarray(np.asarray(bitmask).view(np.int32))
    lib().orc_decompress(_p(d), n, v, wb, _p(words(mask)), _p(words(bitval)), _p(bm), _p(ix),
                         nout, _p(out))
    return _like(out, comp)


def kmeans_assign(data, centroids):
    d, n, v, wb = _rows(data)
    c = words(centroids).reshape(-1, v)
    cl = np.zeros(n, dtype=np.int32)
    lib().orc_kmeans_assign(_p(d), n, v, wb, _p(c), c.shape[0], _p(cl))
    return cl


def kmeans_update(data, clusters, c):
    d, n, v, wb = _rows(data)
    cent = np.zeros((c, v), dtype=d.dtype)
    lib().orc_kmeans_update(_p(d), n, v, wb, _p(np.ascontiguousarray(clusters, dtype=np.int32)),
                            c, _p(cent))
    return _like(cent, data)


def kmeans_masks(data, clusters, c, thr=1.0):
    d, n, v, wb = _rows(data)
    m = np.zeros((c, v), dtype=d.dtype)
    b = np.zeros((c, v), dtype=d.dtype)
    lib().orc_kmeans_masks(_p(d), n, v, wb, _p(np.ascontiguousarray(clusters, dtype=np.int32)),
                           c, float(thr), _p(m), _p(b))
    return _like(m, data), _like(b, data)


def random_shuffle_init(n, c, reseed=True):
    """Rows seeding centroids 0..min(c,n)-1 by the reference's std::random_shuffle."""
    k = min(c, n)
    init = np.zeros(max(k, 1), dtype=np.int64)
    lib().orc_random_shuffle_init(n, c, _p(init), 1 if reseed else 0)
    return init[:k]


def preprocess_kmeans(data, c, init=None):
    """(masks [c, v], bitvals [c, v], clusters int32[n]); init defaults to the reference seeding."""
    d, n, v, wb = _rows(data)
    if init is None:
        init = random_shuffle_init(n, c)
    ix = _idx(init)
    m = np.zeros((c, v), dtype=d.dtype)
    b = np.zeros((c, v), dtype=d.dtype)
    cl = np.zeros(n, dtype=np.int32)
    lib().orc_preprocess_kmeans(_p(d), n, v, wb, c, _p(ix), _p(m), _p(b), _p(cl))
    return _like(m, data), _like(b, data), cl
