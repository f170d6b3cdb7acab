"""Batched multi-set fetch: one launch over many (set, rows) requests with different row
lengths, masks and residency, plain and CUDA-graph replayed, checked bit for bit against the
source rows (whose compressed form the oracle-pinned engine produced)."""
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


def make_set(ibp, rng, n, v, where, scale):
    f = rng.normal(0, scale, (n, 2 * v)).astype(np.float32)
    f = (f.view(np.uint32) & np.uint32(0xFFFF0000)).view(np.float32)
    d = np.ascontiguousarray(f).view(np.int64)
    x = torch.from_numpy(d).pin_memory()
    m, b = ibp.preprocess(x, None)
    bm = ibp.compress_inplace(x, m, b)
    comp_len = ibp.get_single_compress_len(x, m, b)
    if where == "device":
        x = x.cuda()
    return d, (x, m, b, bm, comp_len)


@pytest.fixture(scope="module")
def sets(ibp):
    rng = np.random.default_rng(77)
    out = []
    for i, (n, v, where, sc) in enumerate([(5000, 32, "host", 0.5), (3000, 64, "host", 2.0),
                                           (2000, 100, "device", 0.1), (700, 512, "host", 1.0),
                                           (4000, 48, "device", 0.01)]):
        out.append(make_set(ibp, rng, n, v, where, sc))
    return out


def check(outs, reqs, sets):
    torch.cuda.synchronize()
    for o, (sid, idx, first, count) in zip(outs, reqs):
        d = sets[sid][0]
        want = d[idx.cpu().numpy()] if idx is not None else d[first:first + count]
        assert np.array_equal(o.cpu().numpy(), want), (sid, count)


def requests(rng, sets, k):
    reqs = []
    for j in range(k):
        sid = int(rng.integers(0, len(sets)))
        n = sets[sid][0].shape[0]
        if j % 3 == 2:
            first = int(rng.integers(0, n // 2))
            reqs.append((sid, None, first, int(rng.integers(1, n - first))))
        else:
            cnt = int(rng.integers(1, 3000))
            reqs.append((sid, torch.from_numpy(rng.integers(0, n, cnt)).cuda(), 0, cnt))
    return reqs


def test_batch_fetch_matches_sources(ibp, sets):
    from invariantbitpacking_b200.batch import BatchFetcher, SetRegistry
    reg = SetRegistry([s[1] for s in sets])
    bf = BatchFetcher(reg, max_requests=40)
    rng = np.random.default_rng(1)
    for _ in range(3):
        reqs = requests(rng, sets, 25)
        outs = bf.fetch(reqs)
        check(outs, reqs, sets)
    assert bf.status() == 0


def test_batch_graph_replay_with_new_requests(ibp, sets):
    from invariantbitpacking_b200.batch import BatchFetcher, SetRegistry
    reg = SetRegistry([s[1] for s in sets])
    bf = BatchFetcher(reg, max_requests=64)
    bf.capture()
    rng = np.random.default_rng(2)
    for k in (1, 17, 64, 5):
        reqs = requests(rng, sets, k)
        outs = bf.fetch(reqs)
        check(outs, reqs, sets)


def test_batch_autotune_keeps_results_exact(ibp, sets):
    from invariantbitpacking_b200.batch import BatchFetcher, SetRegistry
    reg = SetRegistry([s[1] for s in sets])
    bf = BatchFetcher(reg, max_requests=32)
    rng = np.random.default_rng(3)
    reqs = requests(rng, sets, 20)
    shape = bf.autotune(reqs)
    assert shape["threads"] in (128, 256) and shape["rows_in_flight"] in (1, 2, 4)
    outs = bf.fetch(reqs)
    check(outs, reqs, sets)


def test_batch_bad_rows_and_sets_are_flagged(ibp, sets):
    from invariantbitpacking_b200.batch import BatchFetcher, SetRegistry
    reg = SetRegistry([s[1] for s in sets[:2]])
    bf = BatchFetcher(reg, max_requests=4)
    good = torch.tensor([0, 1, 2], dtype=torch.int64, device="cuda")
    bad = torch.tensor([1, 10 ** 9, -5], dtype=torch.int64, device="cuda")
    outs = bf.fetch([(0, good, 0, 3), (1, bad, 0, 3)])
    torch.cuda.synchronize()
    assert bf.status() & 1
    assert np.array_equal(outs[0].cpu().numpy(), sets[0][0][[0, 1, 2]])
    assert np.array_equal(outs[1][0].cpu().numpy(), sets[1][0][1])
    o2 = torch.zeros((2, 32), dtype=torch.int64, device="cuda")
    bf.fetch([(7, None, 0, 2)], [o2])
    assert bf.status() & 1 and not o2.any()
