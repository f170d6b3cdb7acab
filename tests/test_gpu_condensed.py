"""Fetch from the condensed layout (rows packed back to back, inclusive byte offsets): the
layout is the reference's compress_condensed output (pinned against the reference's goldens
through the oracle); every fetched row must equal its source row bit for bit, for both word
sizes, rows of any length (unaligned row starts), raw rows among compressed ones, repeats,
out-of-range indices and offsets that cannot describe a row."""
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


def source(rng, n, v, wb, outliers=0.05):
    """Rows of quantised normals viewed as `wb`-byte words; a share of outlier rows that do
    not compress, so raw and compressed rows alternate in the condensed layout."""
    f = rng.normal(0, 0.5, (n, v * wb // 4)).astype(np.float32)
    f = (f.view(np.uint32) & np.uint32(0xFFFF0000)).view(np.float32)
    k = int(n * outliers)
    rows = rng.choice(n, k, replace=False)
    f[rows] = rng.normal(0, 1e4, (k, f.shape[1])).astype(np.float32)
    return np.ascontiguousarray(f).view(np.int64 if wb == 8 else np.int32)


def condensed(ibp, d, where):
    x = torch.from_numpy(d.copy())
    x = x.pin_memory() if where == "host" else x.cuda()
    m, b = ibp.preprocess(x, None)
    comp, offs = ibp.compress_condensed(x, m, b)
    return comp, offs.cuda(), m, b


@pytest.mark.parametrize("wb", [8, 4])
@pytest.mark.parametrize("v", [1, 3, 17, 64, 100, 512])
@pytest.mark.parametrize("where", ["host", "device"])
def test_condensed_fetch_matches_sources(ibp, wb, v, where):
    rng = np.random.default_rng(100 * v + wb)
    n = 3000 if v < 512 else 600
    d = source(rng, n, v, wb)
    comp, offs, m, b = condensed(ibp, d, where)
    sizes = np.diff(np.concatenate([[0], offs.cpu().numpy()]))
    assert (sizes < v * wb).any() or v < 4  # some rows compressed
    # every row, in order
    out = ibp.decompress_fetch_condensed(comp, offs, m, b, v, "cuda")
    assert np.array_equal(out.cpu().numpy(), d)
    # a shuffled index with repeats
    idx = rng.integers(0, n, 5000)
    out = ibp.decompress_fetch_condensed(comp, offs, m, b, v, "cuda", torch.from_numpy(idx).cuda())
    assert np.array_equal(out.cpu().numpy(), d[idx])
    # empty index
    out = ibp.decompress_fetch_condensed(comp, offs, m, b, v, "cuda",
                                         torch.empty(0, dtype=torch.int64, device="cuda"))
    assert out.shape == (0, v)


def test_condensed_fetch_small_batches_and_pinned_output(ibp):
    rng = np.random.default_rng(9)
    d = source(rng, 20000, 64, 8)
    comp, offs, m, b = condensed(ibp, d, "host")
    for k in (1, 2, 31, 33, 257, 4096):
        idx = rng.integers(0, d.shape[0], k)
        out = ibp.decompress_fetch_condensed(comp, offs, m, b, 64, "cpu",
                                             torch.from_numpy(idx).cuda())
        torch.cuda.synchronize()
        assert out.is_pinned() and np.array_equal(out.numpy(), d[idx])


def test_condensed_fetch_flags_bad_indices_and_offsets(ibp):
    import ctypes
    from invariantbitpacking_b200 import _capi
    lib = _capi.lib
    rng = np.random.default_rng(3)
    n, v = 1000, 40
    d = source(rng, n, v, 8)
    comp, offs, m, b = condensed(ibp, d, "device")
    stream = torch.cuda.current_stream().cuda_stream

    def fetch(offsets, idx):
        out = torch.zeros((idx.shape[0], v), dtype=torch.int64, device="cuda")
        ws = torch.zeros(lib.ibp_decompress_fetch_workspace_size(idx.shape[0], v, 8, 1),
                         dtype=torch.uint8, device="cuda")
        _capi.check(lib.ibp_decompress_fetch_condensed(
            comp.data_ptr(), comp.numel(), offsets.data_ptr(), n, v, 8, m.data_ptr(),
            b.data_ptr(), idx.data_ptr(), idx.shape[0], out.data_ptr(), ws.data_ptr(),
            ws.numel(), stream))
        st = ctypes.c_int32()
        _capi.check(lib.ibp_read_status(ws.data_ptr(), ctypes.byref(st), stream))
        return out.cpu().numpy(), st.value

    idx = torch.tensor([5, -1, 7, n, 5, 10 ** 9, 999], dtype=torch.int64, device="cuda")
    got, st = fetch(offs, idx)
    assert st & 1 and not st & 2
    for k, r in enumerate([5, -1, 7, n, 5, 10 ** 9, 999]):
        if 0 <= r < n:
            assert np.array_equal(got[k], d[r])
        else:
            assert not got[k].any()
    # offsets that cannot describe a row: decreasing, past the end, not whole words
    bad = offs.clone()
    o = bad.cpu().numpy()
    bad[100] = int(o[98])                 # row 100 ends before it starts
    bad[200] = int(comp.numel() * 8 + 64) # row 200 ends past the buffer
    bad[300] = int(o[300]) - 3            # not a whole number of words
    idx = torch.tensor([100, 200, 300, 301, 50], dtype=torch.int64, device="cuda")
    got, st = fetch(bad, idx)
    assert st & 2
    assert np.array_equal(got[4], d[50])
    assert not got[0].any() and not got[1].any() and not got[2].any()
