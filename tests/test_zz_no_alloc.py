"""ibp_decompress_fetch_noalloc: the decompress_fetch entry point for callers that cannot
allocate device memory (it runs from a static 4 MiB scratch array inside the library).

Called through the C ABI with plain pointers and checked, bit for bit, against the regular
ibp_decompress_fetch (caller-provided scratch) on two calls in a row -- different index
arrays, word sizes and row lengths, so whatever the first call leaves in the shared scratch
must not leak into the second -- and against the source rows.  A call that needs more
scratch than the static array holds is refused before anything runs, and the status word of
a call (here: an out-of-range index) is readable through ibp_decompress_fetch_noalloc_status.
This file is named so that pytest collects it last."""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

LIMIT = 4 << 20


@pytest.fixture(scope="module")
def eng():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import invariantbitpacking_b200 as ibp
    from invariantbitpacking_b200 import _capi
    return ibp, _capi


def _compressed(ibp, d):
    x = torch.from_numpy(d).pin_memory()
    m, b = ibp.preprocess(x, None)
    bm = ibp.compress_inplace(x, m, b)
    torch.cuda.synchronize()
    return x, m, b, bm


def _regular(capi, x, m, b, bm, idx, v, wb, nrows):
    lib = capi.lib
    out = torch.empty((nrows, v), dtype=x.dtype, device="cuda")
    nidx = -1 if idx is None else idx.numel()
    wsb = lib.ibp_decompress_fetch_workspace_size(max(nidx, 0), v, wb, 0 if idx is None else 1)
    ws = torch.empty(max(wsb, 1), dtype=torch.uint8, device="cuda")
    capi.check(lib.ibp_decompress_fetch(
        x.data_ptr(), x.shape[0], v, wb, m.data_ptr(), b.data_ptr(), bm.data_ptr(),
        None if idx is None else idx.data_ptr(), nidx, -1, out.data_ptr(), -1, -1, -1,
        ws.data_ptr(), wsb, torch.cuda.current_stream().cuda_stream))
    return out


def _noalloc(capi, x, m, b, bm, idx, v, wb, nrows):
    out = torch.full((nrows, v), -7, dtype=x.dtype, device="cuda")
    capi.check(capi.lib.ibp_decompress_fetch_noalloc(
        x.data_ptr(), x.shape[0], v, wb, m.data_ptr(), b.data_ptr(), bm.data_ptr(),
        None if idx is None else idx.data_ptr(), -1 if idx is None else idx.numel(), -1,
        out.data_ptr(), torch.cuda.current_stream().cuda_stream))
    return out


def test_noalloc_matches_regular_entry_point_twice(eng):
    ibp, capi = eng
    from invariantbitpacking_b200 import synthetic
    # call 1: int64 rows of 64 words, a Zipf index with many repeats
    d1 = synthetic.graph_features(n=6000, seed=31)
    x1, m1, b1, bm1 = _compressed(ibp, d1)
    idx1 = torch.from_numpy(synthetic.Zipf(6000, 1.1, seed=3).sample(20000)).cuda()
    a = _noalloc(capi, x1, m1, b1, bm1, idx1, 64, 8, 20000)
    r = _regular(capi, x1, m1, b1, bm1, idx1, 64, 8, 20000)
    torch.cuda.synchronize()
    assert torch.equal(a, r)
    assert np.array_equal(a.cpu().numpy(), d1[idx1.cpu().numpy()])
    # call 2: int32 rows of 100 words, no index, then a short index on the same rows
    rng = np.random.default_rng(32)
    f = (rng.normal(0, 1, (3000, 100)).astype(np.float32).view(np.uint32)
         & np.uint32(0xFFFFF000)).view(np.int32)
    x2, m2, b2, bm2 = _compressed(ibp, np.ascontiguousarray(f))
    a = _noalloc(capi, x2, m2, b2, bm2, None, 100, 4, 3000)
    r = _regular(capi, x2, m2, b2, bm2, None, 100, 4, 3000)
    torch.cuda.synchronize()
    assert torch.equal(a, r)
    assert np.array_equal(a.cpu().numpy(), f)
    idx2 = torch.from_numpy(rng.integers(0, 3000, 777)).cuda()
    a = _noalloc(capi, x2, m2, b2, bm2, idx2, 100, 4, 777)
    r = _regular(capi, x2, m2, b2, bm2, idx2, 100, 4, 777)
    torch.cuda.synchronize()
    assert torch.equal(a, r)


def test_noalloc_refuses_calls_beyond_its_scratch(eng):
    ibp, capi = eng
    lib = capi.lib
    n, v = 1000, 64
    nidx = 400_000
    assert lib.ibp_decompress_fetch_workspace_size(nidx, v, 8, 1) > LIMIT
    x = torch.zeros((n, v), dtype=torch.int64, device="cuda")
    m = torch.zeros(v, dtype=torch.int64, device="cuda")
    bm = torch.zeros((n + 31) // 32, dtype=torch.int32, device="cuda")
    idx = torch.zeros(nidx, dtype=torch.int64, device="cuda")
    out = torch.full((nidx, v), 5, dtype=torch.int64, device="cuda")
    st = lib.ibp_decompress_fetch_noalloc(x.data_ptr(), n, v, 8, m.data_ptr(), m.data_ptr(),
                                          bm.data_ptr(), idx.data_ptr(), nidx, -1,
                                          out.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert st == capi.IBP_ERR_WORKSPACE
    assert b"static" in lib.ibp_last_error()
    torch.cuda.synchronize()
    assert bool((out == 5).all())


def _status(capi):
    st = ctypes.c_int32(-1)
    capi.check(capi.lib.ibp_decompress_fetch_noalloc_status(
        ctypes.byref(st), torch.cuda.current_stream().cuda_stream))
    return st.value


def test_noalloc_status_reports_out_of_range_index(eng):
    ibp, capi = eng
    from invariantbitpacking_b200 import synthetic
    assert capi.NOALLOC_SCRATCH_BYTES == LIMIT
    d = synthetic.graph_features(n=3000, seed=33)
    x, m, b, bm = _compressed(ibp, d)
    rows = np.array([5, 2999, 3000, -1, 7, 5], dtype=np.int64)
    idx = torch.from_numpy(rows).cuda()
    a = _noalloc(capi, x, m, b, bm, idx, 64, 8, len(rows))
    assert _status(capi) & 1  # bit 0: an index was out of range
    a = a.cpu().numpy()
    ok = (rows >= 0) & (rows < 3000)
    assert np.array_equal(a[ok], d[rows[ok]])
    assert (a[~ok] == -7).all()  # rows of bad indices are left untouched
    # the next call starts from a clear status word
    good = torch.from_numpy(rows[ok]).cuda()
    a = _noalloc(capi, x, m, b, bm, good, 64, 8, int(ok.sum()))
    assert _status(capi) == 0
    assert np.array_equal(a.cpu().numpy(), d[rows[ok]])
