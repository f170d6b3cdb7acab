"""decompress_fetch captured in a CUDA graph: the call's kernels (the prep kernel, the fetch
with its in-fetch claims for host rows; the claim pass, the whole-row decode and the repeat
copies for device rows), launched as dependent launches, replayed with new index contents
and checked bit-exact against the source rows."""
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


def masked_rows(rng, n, v):
    """int64 rows whose words mostly agree with a random mask (a few words and rows not)."""
    bits = rng.random((v, 64)) < 0.6
    m = np.zeros(v, dtype=np.uint64)
    for b in range(64):
        m |= bits[:, b].astype(np.uint64) << np.uint64(b)
    base = rng.integers(0, 2**63, v, dtype=np.uint64) & m
    noise = rng.integers(0, 2**63, (n, v), dtype=np.uint64)
    data = (noise & ~m) | base
    data = np.where(rng.random((n, v)) < 0.02, noise, data)
    return data.view(np.int64), m.view(np.int64), base.view(np.int64)


@pytest.mark.parametrize("where", ["host", "device"])
def test_decompress_fetch_replays_in_a_cuda_graph(ibp, where):
    rng = np.random.default_rng(77 if where == "host" else 78)
    n, v, k = 20000, 64, 3000
    d, m, b = masked_rows(rng, n, v)
    dm, db = torch.from_numpy(m).cuda(), torch.from_numpy(b).cuda()
    x = torch.from_numpy(d.copy()).pin_memory()
    bm = ibp.compress_inplace(x, dm, db)
    xs = x if where == "host" else x.cuda()
    # skewed batches: a few hot rows repeated many times, the rest spread out
    def batch():
        hot = rng.integers(0, n, 16)
        return np.where(rng.random(k) < 0.5, hot[rng.integers(0, 16, k)],
                        rng.integers(0, n, k)).astype(np.int64)
    first = batch()
    idx = torch.from_numpy(first).cuda()
    out = torch.empty((k, v), dtype=torch.int64, device="cuda")
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):  # warm-up outside the capture (launch shapes, modules)
        ibp.decompress_fetch(xs, dm, db, bm, "cuda", None, idx, output_tensor=out)
    torch.cuda.current_stream().wait_stream(side)
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), d[first])
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        ibp.decompress_fetch(xs, dm, db, bm, "cuda", None, idx, output_tensor=out)
    for _ in range(3):
        new = batch()
        idx.copy_(torch.from_numpy(new))
        out.fill_(-1)
        graph.replay()
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy(), d[new])
    del graph
