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


def dup_requests(rng, sets, k):
    """Requests whose rows repeat heavily (a few hundred distinct rows per request)."""
    reqs = []
    for j in range(k):
        sid = int(rng.integers(0, len(sets)))
        n = sets[sid][0].shape[0]
        if j % 5 == 4:
            first = int(rng.integers(0, n // 2))
            reqs.append((sid, None, first, int(rng.integers(0, n - first))))
        else:
            cnt = int(rng.integers(1, 4000))
            hot = rng.integers(0, n, int(rng.integers(1, 300)))
            reqs.append((sid, torch.from_numpy(hot[rng.integers(0, hot.size, cnt)]).cuda(), 0, cnt))
    return reqs


def test_batch_sorted_dedup_matches_sources(ibp, sets):
    from invariantbitpacking_b200.batch import BatchFetcher, SetRegistry
    reg = SetRegistry([s[1] for s in sets])
    bf = BatchFetcher(reg, max_requests=64)
    rng = np.random.default_rng(11)
    for k in (1, 7, 40, 64):
        reqs = dup_requests(rng, sets, k)
        outs = bf.fetch(reqs, dedup=True)
        check(outs, reqs, sets)
        assert bf.status() == 0
    # the same requests through the listed-order path agree
    reqs = dup_requests(rng, sets, 30)
    a = bf.fetch(reqs, dedup=True)
    torch.cuda.synchronize()
    b = bf.fetch(reqs)
    torch.cuda.synchronize()
    for x, y in zip(a, b):
        assert torch.equal(x, y)


def test_batch_sorted_after_capture_and_bad_rows(ibp, sets):
    from invariantbitpacking_b200.batch import BatchFetcher, SetRegistry
    reg = SetRegistry([s[1] for s in sets[:2]])
    bf = BatchFetcher(reg, max_requests=8)
    bf.capture()
    good = torch.tensor([2, 0, 2, 1, 0], dtype=torch.int64, device="cuda")
    bad = torch.tensor([1, 10 ** 9, -5, 1, 10 ** 9], dtype=torch.int64, device="cuda")
    o2 = torch.zeros((2, 32), dtype=torch.int64, device="cuda")
    reqs = [(0, good, 0, 5), (1, bad, 0, 5), (7, None, 0, 2), (1, None, 0, 0)]
    outs = bf.outputs_for([reqs[0], reqs[1]]) + [o2] + bf.outputs_for([reqs[3]])
    outs = bf.fetch(reqs, outs, dedup=True)
    torch.cuda.synchronize()
    assert bf.status() & 1
    assert np.array_equal(outs[0].cpu().numpy(), sets[0][0][[2, 0, 2, 1, 0]])
    o = outs[1].cpu().numpy()
    assert np.array_equal(o[0], sets[1][0][1]) and np.array_equal(o[3], sets[1][0][1])
    assert outs[3].shape[0] == 0 and not o2.any()
    # graph replays still serve the listed-order path afterwards
    outs = bf.fetch([(0, good, 0, 5)])
    check(outs, [(0, good, 0, 5)], sets)


def test_batch_sorted_total_mismatch_is_flagged(ibp, sets):
    from invariantbitpacking_b200 import _capi
    from invariantbitpacking_b200.batch import SetRegistry
    reg = SetRegistry([s[1] for s in sets[:1]])
    idx = torch.arange(0, 600, 3, dtype=torch.int64, device="cuda")
    out = torch.zeros((200, 32), dtype=torch.int64, device="cuda")
    rec = (_capi.Request * 1)()
    rec[0].set, rec[0].index, rec[0].first, rec[0].count, rec[0].out = 0, idx.data_ptr(), 0, 200, out.data_ptr()
    dreq = torch.frombuffer(bytearray(bytes(rec)), dtype=torch.uint8).cuda()
    lib = _capi.lib
    for total in (150, 260):
        ws = torch.empty(lib.ibp_batch_fetch_sorted_workspace_size(total, 1), dtype=torch.uint8,
                         device="cuda")
        out.zero_()
        _capi.check(lib.ibp_batch_fetch_sorted(reg.buf.data_ptr(), dreq.data_ptr(), 1, total,
                                               ws.data_ptr(), ws.numel(),
                                               torch.cuda.current_stream().cuda_stream))
        torch.cuda.synchronize()
        assert int(ws[:4].view(torch.int32).item()) & 4
        got = out.cpu().numpy()
        want = sets[0][0][idx.cpu().numpy()]
        k = min(total, 200)
        assert np.array_equal(got[:k], want[:k])
        assert not got[k:].any()
    with pytest.raises(_capi.IBPError):
        _capi.check(lib.ibp_batch_fetch_sorted(reg.buf.data_ptr(), dreq.data_ptr(), 1, 100,
                                               ws.data_ptr(), 16,
                                               torch.cuda.current_stream().cuda_stream))


def test_batch_hashed_dedup_matches_sources(ibp, sets):
    """Hash-claimed batches (ibp_batch_fetch_hashed): rows repeated within and across requests
    of one set are fetched once and copied; every output row matches the source, and the
    listed-order path agrees."""
    from invariantbitpacking_b200.batch import BatchFetcher, SetRegistry
    reg = SetRegistry([s[1] for s in sets])
    bf = BatchFetcher(reg, max_requests=64)
    rng = np.random.default_rng(12)
    for k in (1, 7, 40, 64):
        reqs = dup_requests(rng, sets, k)
        outs = bf.fetch(reqs, dedup="hash")
        check(outs, reqs, sets)
        assert bf.status() == 0
    reqs = dup_requests(rng, sets, 30)
    # the same rows in two requests of one set share their claims
    reqs.append((reqs[0][0],) + reqs[0][1:])
    a = bf.fetch(reqs, dedup="hash")
    torch.cuda.synchronize()
    b = bf.fetch(reqs)
    torch.cuda.synchronize()
    for x, y in zip(a, b):
        assert torch.equal(x, y)


def test_batch_hashed_bad_rows_and_waits(ibp, sets):
    """Bad rows and set ids are flagged and skipped; with the repeat wait limit at 0 every
    repeat decodes its own row (status bit 3) and the rows are still exact."""
    from invariantbitpacking_b200.batch import BatchFetcher, SetRegistry
    reg = SetRegistry([s[1] for s in sets[:2]])
    bf = BatchFetcher(reg, max_requests=8)
    good = torch.tensor([2, 0, 2, 1, 0], dtype=torch.int64, device="cuda")
    bad = torch.tensor([1, 10 ** 9, -5, 1, 10 ** 9], dtype=torch.int64, device="cuda")
    o2 = torch.zeros((2, 32), dtype=torch.int64, device="cuda")
    reqs = [(0, good, 0, 5), (1, bad, 0, 5), (7, None, 0, 2), (1, None, 0, 0)]
    outs = bf.outputs_for([reqs[0], reqs[1]]) + [o2] + bf.outputs_for([reqs[3]])
    outs = bf.fetch(reqs, outs, dedup="hash")
    torch.cuda.synchronize()
    assert bf.status() & 1
    assert np.array_equal(outs[0].cpu().numpy(), sets[0][0][[2, 0, 2, 1, 0]])
    o = outs[1].cpu().numpy()
    assert np.array_equal(o[0], sets[1][0][1]) and np.array_equal(o[3], sets[1][0][1])
    assert outs[3].shape[0] == 0 and not o2.any()
    ibp.set_repeat_wait_limit(0)
    try:
        rng = np.random.default_rng(13)
        reqs = dup_requests(rng, sets[:2], 8)
        outs = bf.fetch(reqs, dedup="hash")
        check(outs, reqs, sets)
        assert bf.status() == 8
    finally:
        ibp.set_repeat_wait_limit(None)


def test_batch_hashed_understated_total(ibp, sets):
    """A stated total below the requests' rows sets status bit 2; the claim table is then
    undersized, and rows whose claim finds it full are fetched without one: every row is
    still written."""
    from invariantbitpacking_b200 import _capi
    from invariantbitpacking_b200.batch import SetRegistry
    reg = SetRegistry([s[1] for s in sets[:1]])
    idx = torch.arange(0, 600, 3, dtype=torch.int64, device="cuda")
    out = torch.zeros((200, 32), dtype=torch.int64, device="cuda")
    rec = (_capi.Request * 1)()
    rec[0].set, rec[0].index, rec[0].first, rec[0].count, rec[0].out = 0, idx.data_ptr(), 0, 200, out.data_ptr()
    dreq = torch.frombuffer(bytearray(bytes(rec)), dtype=torch.uint8).cuda()
    lib = _capi.lib
    want = sets[0][0][idx.cpu().numpy()]
    for total in (10, 150, 200):
        ws = torch.empty(lib.ibp_batch_fetch_hashed_workspace_size(total), dtype=torch.uint8,
                         device="cuda")
        out.zero_()
        _capi.check(lib.ibp_batch_fetch_hashed(reg.buf.data_ptr(), dreq.data_ptr(), 1, total,
                                               ws.data_ptr(), ws.numel(),
                                               torch.cuda.current_stream().cuda_stream))
        torch.cuda.synchronize()
        st = int(ws[:4].view(torch.int32).item())
        assert (st & 4) == (4 if total != 200 else 0)
        assert np.array_equal(out.cpu().numpy(), want)
    with pytest.raises(_capi.IBPError):
        _capi.check(lib.ibp_batch_fetch_hashed(reg.buf.data_ptr(), dreq.data_ptr(), 1, 100,
                                               ws.data_ptr(), 16,
                                               torch.cuda.current_stream().cuda_stream))
