"""Both ways decompress_fetch finds repeated rows -- radix sort, and the open-addressing hash
table it uses for sparse batches -- must give the oracle's rows bit for bit: repeats, hot
rows, out-of-range entries, empty and single-entry indices, 4- and 8-byte words, row
lengths that break 16-byte alignment, host and device sets, and the condensed layout."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ibp():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import invariantbitpacking_b200 as m
    return m


@pytest.fixture(params=[1, 2, 0], ids=["sort", "hash", "auto"])
def mode(request, ibp):
    from invariantbitpacking_b200 import _capi
    _capi.check(_capi.lib.ibp_set_fetch_dedup(request.param))
    yield request.param
    _capi.check(_capi.lib.ibp_set_fetch_dedup(0))


def make(rng, n, v, wb):
    f = rng.normal(0, 0.4, (n, v * wb // 4)).astype(np.float32)
    f = (f.view(np.uint32) & np.uint32(0xFFFF8000)).view(np.float32)
    return np.ascontiguousarray(f).view(np.int64 if wb == 8 else np.int32)


@pytest.mark.parametrize("wb,v", [(8, 64), (8, 7), (4, 33), (4, 128), (8, 300), (8, 65), (4, 131)])
@pytest.mark.parametrize("where", ["host", "device"])
def test_dedup_modes_match_oracle(ibp, oracle, mode, wb, v, where):
    rng = np.random.default_rng(v * 10 + wb)
    n = 20000
    d = make(rng, n, v, wb)
    x = torch.from_numpy(d.copy()).pin_memory()
    m, b = ibp.preprocess(x, None)
    bm = ibp.compress_inplace(x, m, b)
    cl = ibp.get_single_compress_len(x, m, b)
    if where == "device":
        x = x.cuda()
    comp = x.cpu().numpy()
    cases = [
        rng.integers(0, n, 3000),                         # sparse, some repeats
        np.repeat(rng.integers(0, n, 50), 40),            # few rows, long runs
        rng.integers(0, n, 40000),                        # denser than the set
        np.array([n - 1]), np.array([], dtype=np.int64),
        np.concatenate([rng.integers(0, n, 500), [-1, n, 10 ** 12, 5, 5]]),
    ]
    for idx in cases:
        ti = torch.from_numpy(idx.astype(np.int64)).cuda()
        out = torch.full((idx.size, v), 7, dtype=x.dtype, device="cuda")
        ibp.decompress_fetch(x, m, b, bm, "cuda", cl, ti, output_tensor=out)
        got = out.cpu().numpy()
        ok = (idx >= 0) & (idx < n)
        want = oracle.decompress(comp, m.cpu().numpy(), b.cpu().numpy(), bm.cpu().numpy(),
                                 np.where(ok, idx, 0))
        assert np.array_equal(got[ok], want[ok])
        assert (got[~ok] == 7).all()   # skipped rows are left untouched


def test_dedup_modes_condensed(ibp, mode):
    rng = np.random.default_rng(5)
    n, v = 9000, 40
    d = make(rng, n, v, 8)
    x = torch.from_numpy(d.copy()).pin_memory()
    m, b = ibp.preprocess(x, None)
    comp, offs = ibp.compress_condensed(x, m, b)
    for idx in (rng.integers(0, n, 1500), np.repeat(rng.integers(0, n, 30), 17)):
        out = ibp.decompress_fetch_condensed(comp, offs.cuda(), m, b, v, "cuda",
                                             torch.from_numpy(idx).cuda())
        assert np.array_equal(out.cpu().numpy(), d[idx])


@pytest.mark.parametrize("pattern", ["zipf", "one_row", "pairs"])
@pytest.mark.parametrize("aligned", [True, False], ids=["out16", "out8"])
@pytest.mark.parametrize("where", ["host", "device"])
@pytest.mark.parametrize("layout", ["fixed", "condensed"])
def test_in_fetch_repeats(ibp, oracle, pattern, aligned, where, layout):
    """Hash claims (made inside the fetch for host rows, by a claim pass for device rows):
    each repeat copies its first occurrence's output row once that row is published in the
    table.  Every row must be exact, for fixed-stride and condensed rows, into 16-byte aligned
    and unaligned outputs, and no wait may give up (status bit 3)."""
    import ctypes
    from invariantbitpacking_b200 import _capi
    lib = _capi.lib
    rng = np.random.default_rng(77)
    n, v = 30000, 64
    d = make(rng, n, v, 8)
    x = torch.from_numpy(d.copy()).pin_memory()
    m, b = ibp.preprocess(x, None)
    if layout == "condensed":
        ccomp, offs = ibp.compress_condensed(x, m, b)
        offs = offs.cuda()
    bm = ibp.compress_inplace(x, m, b)
    cl = ibp.get_single_compress_len(x, m, b)
    torch.cuda.synchronize()
    comp = x.numpy().copy()
    if pattern == "zipf":
        idx = np.minimum(rng.zipf(1.1, 120000) - 1, n - 1)
    elif pattern == "one_row":
        idx = np.full(50000, 1234)
    else:  # each row twice, the two occurrences next to each other or far apart
        r = rng.permutation(n)[:20000]
        idx = np.concatenate([np.repeat(r[:10000], 2), r[10000:], r[10000:][::-1]])
    idx = idx.astype(np.int64)
    if where == "device":
        x = x.cuda()
        if layout == "condensed":
            ccomp = ccomp.cuda()
    ti = torch.from_numpy(idx).cuda()
    nidx = idx.size
    buf = torch.full((nidx * v + 1,), 7, dtype=torch.int64, device="cuda")
    out = buf[:nidx * v] if aligned else buf[1:]
    wsb = lib.ibp_decompress_fetch_workspace_size(nidx, v, 8, 1)
    ws = torch.empty(wsb, dtype=torch.uint8, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    _capi.check(lib.ibp_set_fetch_dedup(2))
    try:
        if layout == "fixed":
            _capi.check(lib.ibp_decompress_fetch(
                x.data_ptr(), n, v, 8, m.data_ptr(), b.data_ptr(), bm.data_ptr(), ti.data_ptr(),
                nidx, cl, out.data_ptr(), -1, -1, -1, ws.data_ptr(), wsb, st))
        else:
            _capi.check(lib.ibp_decompress_fetch_condensed(
                ccomp.data_ptr(), ccomp.numel(), offs.data_ptr(), n, v, 8, m.data_ptr(),
                b.data_ptr(), ti.data_ptr(), nidx, out.data_ptr(), ws.data_ptr(), wsb, st))
        status = ctypes.c_int32(-1)
        _capi.check(lib.ibp_read_status(ws.data_ptr(), ctypes.byref(status), st))
    finally:
        _capi.check(lib.ibp_set_fetch_dedup(0))
    assert status.value == 0
    want = oracle.decompress(comp, m.cpu().numpy(), b.cpu().numpy(), bm.cpu().numpy(), idx)
    assert np.array_equal(out.view(nidx, v).cpu().numpy(), want)


@pytest.mark.parametrize("pattern", ["zipf", "one_row"])
@pytest.mark.parametrize("layout", ["fixed", "condensed"])
def test_repeat_wait_gives_up_and_decodes_from_source(ibp, oracle, pattern, layout):
    """A repeat of a hashed host-row fetch whose first occurrence is not published within the
    wait limit decodes its own row from the source.  With the limit at 0 polls every repeat
    takes that path: status bit 3 reports it, and every output row is still the oracle's (a
    bounded device wait made to run out; nothing faults)."""
    import ctypes
    from invariantbitpacking_b200 import _capi
    lib = _capi.lib
    rng = np.random.default_rng(78)
    n, v = 30000, 64
    d = make(rng, n, v, 8)
    x = torch.from_numpy(d.copy()).pin_memory()
    m, b = ibp.preprocess(x, None)
    if layout == "condensed":
        ccomp, offs = ibp.compress_condensed(x, m, b)
        offs = offs.cuda()
    bm = ibp.compress_inplace(x, m, b)
    cl = ibp.get_single_compress_len(x, m, b)
    torch.cuda.synchronize()
    comp = x.numpy().copy()
    if pattern == "zipf":
        idx = np.minimum(rng.zipf(1.1, 120000) - 1, n - 1).astype(np.int64)
    else:
        idx = np.full(20000, 4321, dtype=np.int64)
    ti = torch.from_numpy(idx).cuda()
    nidx = idx.size
    out = torch.full((nidx, v), 7, dtype=torch.int64, device="cuda")
    wsb = lib.ibp_decompress_fetch_workspace_size(nidx, v, 8, 1)
    ws = torch.empty(wsb, dtype=torch.uint8, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    status = ctypes.c_int32(-1)
    _capi.check(lib.ibp_set_fetch_dedup(2))
    _capi.check(lib.ibp_set_repeat_wait_limit(0))
    try:
        if layout == "fixed":
            _capi.check(lib.ibp_decompress_fetch(
                x.data_ptr(), n, v, 8, m.data_ptr(), b.data_ptr(), bm.data_ptr(), ti.data_ptr(),
                nidx, cl, out.data_ptr(), -1, -1, -1, ws.data_ptr(), wsb, st))
        else:
            _capi.check(lib.ibp_decompress_fetch_condensed(
                ccomp.data_ptr(), ccomp.numel(), offs.data_ptr(), n, v, 8, m.data_ptr(),
                b.data_ptr(), ti.data_ptr(), nidx, out.data_ptr(), ws.data_ptr(), wsb, st))
        _capi.check(lib.ibp_read_status(ws.data_ptr(), ctypes.byref(status), st))
    finally:
        _capi.check(lib.ibp_set_repeat_wait_limit(-1))
        _capi.check(lib.ibp_set_fetch_dedup(0))
    assert status.value == 8  # bit 3 only: repeats gave up, nothing else went wrong
    want = oracle.decompress(comp, m.cpu().numpy(), b.cpu().numpy(), bm.cpu().numpy(), idx)
    assert np.array_equal(out.cpu().numpy(), want)


def test_check_raises_for_out_of_range_index(ibp):
    """check=True turns the status word into an error; the default stays non-blocking and
    leaves the bad rows unwritten."""
    rng = np.random.default_rng(79)
    n, v = 5000, 64
    d = make(rng, n, v, 8)
    x = torch.from_numpy(d.copy()).pin_memory()
    m, b = ibp.preprocess(x, None)
    bm = ibp.compress_inplace(x, m, b)
    good = torch.from_numpy(rng.integers(0, n, 700)).cuda()
    out = ibp.decompress_fetch(x, m, b, bm, "cuda", None, good, check=True)
    assert np.array_equal(out.cpu().numpy(), d[good.cpu().numpy()])
    bad = torch.cat([good, torch.tensor([n], device="cuda")])
    with pytest.raises(RuntimeError, match="out of range"):
        ibp.decompress_fetch(x, m, b, bm, "cuda", None, bad, check=True)
    out = ibp.decompress_fetch(x, m, b, bm, "cuda", None, bad)
    assert np.array_equal(out[:-1].cpu().numpy(), d[good.cpu().numpy()])
