"""Continuous-batching server: a burst of mixed requests from two client threads, with an
output arena small enough that admission has to wait for releases, rows that repeat inside
a request, with the default batch limits and with small ones; every result must equal the
same request fetched alone by plain decompress_fetch, and the source rows."""
import threading

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


@pytest.mark.parametrize("dedup", ["hash", "sort"])
@pytest.mark.parametrize("limits", [None, (2000, 256 << 10)])
def test_server_results_equal_solo_fetches(ibp, limits, dedup):
    from invariantbitpacking_b200.batch import SetRegistry
    from invariantbitpacking_b200.serve import Server
    rng = np.random.default_rng(5)
    srcs, sets = [], []
    for n, v in [(20000, 64), (8000, 128), (3000, 256), (1500, 512)]:
        f = rng.normal(0, 0.3, (n, 2 * v)).astype(np.float32)
        f = (f.view(np.uint32) & np.uint32(0xFFFF8000)).view(np.float32)
        d = np.ascontiguousarray(f).view(np.int64)
        x = torch.from_numpy(d).pin_memory()
        m, b = ibp.preprocess(x, None)
        bm = ibp.compress_inplace(x, m, b)
        srcs.append(d)
        sets.append((x, m, b, bm, ibp.get_single_compress_len(x, m, b)))
    reg = SetRegistry(sets)
    srv = Server(reg, arena_bytes=64 << 20, index_capacity=1 << 20, max_batch=16,
                 max_inflight=2)
    srv.set_dedup(dedup)
    if limits:
        srv.set_batch_limits(*limits)
    reqs = []
    for j in range(60):
        sid = int(rng.integers(0, 4))
        n = srcs[sid].shape[0]
        cnt = int(np.exp(rng.uniform(np.log(16), np.log(4000))))
        if j % 4 == 3:
            first = int(rng.integers(0, n - cnt)) if cnt < n else 0
            cnt = min(cnt, n - first)
            reqs.append((sid, None, first, cnt))
        elif j % 4 == 2:  # rows repeat: a few dozen hot rows
            hot = rng.integers(0, n, int(rng.integers(1, 40))).astype(np.int64)
            reqs.append((sid, hot[rng.integers(0, hot.size, cnt)], 0, cnt))
        else:
            reqs.append((sid, rng.integers(0, n, cnt).astype(np.int64), 0, cnt))
    ids = [None] * len(reqs)

    def client(part):
        for j in range(part, len(reqs), 2):
            sid, rows, first, cnt = reqs[j]
            while True:
                try:
                    ids[j] = srv.submit(sid, rows, first, cnt)
                    break
                except RuntimeError:  # index staging full: let the server drain
                    threading.Event().wait(0.001)

    ths = [threading.Thread(target=client, args=(p,)) for p in (0, 1)]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    for j, (sid, rows, first, cnt) in enumerate(reqs):
        out, times = srv.wait(ids[j], 20000)
        got = out.cpu().numpy()
        srv.release(ids[j])
        want = srcs[sid][rows] if rows is not None else srcs[sid][first:first + cnt]
        assert np.array_equal(got, want), j
        x, m, b, bm, cl = sets[sid]
        idx = None if rows is None else torch.from_numpy(rows).cuda()
        solo = ibp.decompress_fetch(x, m, b, bm, "cuda", cl, idx)
        if rows is None:
            solo = solo[first:first + cnt]
        assert np.array_equal(solo.cpu().numpy(), got), j
        assert times[0] <= times[1] <= times[2]
    st = srv.stats()
    assert st["rows_done"] == sum(r[3] for r in reqs) and st["pending"] == 0
    assert st["batches"] < len(reqs)  # requests were batched
    if limits:
        big = max(r[3] * sets[r[0]][0].shape[1] * 8 for r in reqs)
        assert st["batches"] >= sum(r[3] * sets[r[0]][0].shape[1] * 8 for r in reqs) // (
            limits[1] + big)
    srv.close()


def test_server_cancel_and_admission_wait(ibp):
    """A request that cannot be admitted (its output does not fit the arena beside an
    unreleased one) stays queued and can be withdrawn; an admitted one cannot; the server
    keeps serving afterwards."""
    from invariantbitpacking_b200.batch import SetRegistry
    from invariantbitpacking_b200.serve import Server
    rng = np.random.default_rng(9)
    n, v = 4000, 64
    f = rng.normal(0, 0.3, (n, 2 * v)).astype(np.float32)
    f = (f.view(np.uint32) & np.uint32(0xFFFF8000)).view(np.float32)
    d = np.ascontiguousarray(f).view(np.int64)
    x = torch.from_numpy(d.copy()).pin_memory()
    m, b = ibp.preprocess(x, None)
    cl = ibp.get_single_compress_len(x, m, b)
    bm = ibp.compress_inplace(x, m, b)
    reg = SetRegistry([(x, m, b, bm, cl)])
    rows = 3000
    srv = Server(reg, arena_bytes=rows * v * 8 + 4096, index_capacity=1 << 16, max_batch=4)
    ra = rng.integers(0, n, rows)
    a = srv.submit(0, ra)
    out_a, _ = srv.wait(a, 20000)             # admitted and done; its rows hold the arena
    b_id = srv.submit(0, rng.integers(0, n, rows))
    import time
    time.sleep(0.05)
    assert srv.stats()["pending"] == 1        # cannot fit until `a` is released
    srv.cancel(b_id)
    assert srv.stats()["pending"] == 0
    with pytest.raises(RuntimeError):
        srv.cancel(a)                          # already admitted
    with pytest.raises(RuntimeError):
        srv.wait(b_id, 100)                    # withdrawn: unknown now
    assert np.array_equal(out_a.cpu().numpy(), d[ra])
    srv.release(a)
    rc = rng.integers(0, n, 100)
    c = srv.submit(0, rc)
    out_c, _ = srv.wait(c, 20000)
    assert np.array_equal(out_c.cpu().numpy(), d[rc])
    srv.release(c)
    srv.close()
