"""Caller shims: FlexGen-style general_copy of compressed weights into GPU tensors (whole
tensors, row ranges, column slices, other dtypes) must equal a plain copy, and the cached,
compressed embedding bag must equal torch's embedding bag over the full table while its cache
evicts and refetches rows."""
import numpy as np
import pytest
import torch
import torch.nn.functional as F

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def callers():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from invariantbitpacking_b200 import callers as c
    return c


@pytest.mark.parametrize("dtype", [torch.float16, torch.bfloat16, torch.float32])
def test_general_copy_matches_plain_copy(callers, dtype):
    g = torch.Generator().manual_seed(4)
    w = (torch.randn(300, 256, generator=g) * 0.02).to(dtype)
    src = callers.IBPTensor(w.clone().pin_memory())
    src.ibp_preprocess()
    src.ibp_compress()
    assert src.compressed
    # whole tensor
    dst = torch.empty_like(w, device="cuda")
    callers.general_copy(dst, None, src, None)
    assert torch.equal(dst.cpu(), w)
    # row range into a row range of a larger destination
    big = torch.zeros((400, 256), dtype=dtype, device="cuda")
    callers.general_copy(big, (slice(50, 150),), src, (slice(100, 200),))
    assert torch.equal(big[50:150].cpu(), w[100:200]) and not big[:50].any()
    # column slice (non-contiguous destination and selection)
    d2 = torch.zeros((300, 64), dtype=dtype, device="cuda")
    callers.general_copy(d2, None, src, (slice(None), slice(64, 128)))
    assert torch.equal(d2.cpu(), w[:, 64:128])
    # an uncompressed source takes the plain copy
    plain = callers.IBPTensor(w.clone().pin_memory())
    d3 = torch.empty_like(w, device="cuda")
    callers.general_copy(d3, None, plain, None)
    assert torch.equal(d3.cpu(), w)


@pytest.mark.parametrize("comp", [True, False])
def test_compressed_embedding_bag_matches_full_table(callers, comp):
    rng = np.random.default_rng(8)
    rows, dim = 20000, 64
    t = rng.normal(0, 0.5, (rows, dim)).astype(np.float32)
    t = (t.view(np.uint32) & np.uint32(0xFFFF0000)).view(np.float32)
    table = torch.from_numpy(t)
    bag = callers.CompressedEmbeddingBag(rows, dim, cache_ratio=0.05, _weight=table, comp=comp)
    full = table.cuda()
    for step in range(6):
        n = 700
        idx = torch.from_numpy(rng.zipf(1.2, n) % rows).cuda()
        lens = rng.integers(1, 6, 200)
        lens = lens[np.cumsum(lens) <= n]
        offsets = torch.from_numpy(np.concatenate([[0], np.cumsum(lens)[:-1]])).cuda()
        idx = idx[:int(lens.sum())]
        got = bag(idx, offsets)
        want = F.embedding_bag(idx, full, offsets, mode="sum")
        torch.cuda.synchronize()
        assert torch.allclose(got, want, rtol=1e-6, atol=1e-6), step
        # cached rows are bit-identical to the table
        live = bag.row_of_slot >= 0
        assert torch.equal(bag.cache[live], full[bag.row_of_slot[live]])
    st = bag.stats
    assert st["misses"] > 0 and st["hits"] > 0
    assert st["lookups"] == st["hits"] + st["misses"]


def test_sharded_fetcher_single_rank(callers):
    import invariantbitpacking_b200 as ibp
    from invariantbitpacking_b200.shard import ShardedFetcher
    rng = np.random.default_rng(2)
    f = rng.normal(0, 0.5, (5000, 64)).astype(np.float32)
    d = (f.view(np.uint32) & np.uint32(0xFFFF0000)).view(np.int64)
    x = torch.from_numpy(d.copy()).pin_memory()
    m, b = ibp.preprocess(x, None)
    bm = ibp.compress_inplace(x, m, b)
    sf = ShardedFetcher(x, m, b, bm, ibp.get_single_compress_len(x, m, b))
    idx = torch.from_numpy(rng.integers(0, 5000, 777))
    rows, (lo, hi) = sf(idx)
    assert (lo, hi) == (0, 777) and np.array_equal(rows.cpu().numpy(), d[idx.numpy()])
    assert np.array_equal(sf(idx, gather=True).cpu().numpy(), d[idx.numpy()])
