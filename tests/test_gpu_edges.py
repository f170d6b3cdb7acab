"""GPU edge cases and full-size properties, checked against the CPU oracle (which the
golden vectors pin to the reference): empty inputs, tiny and ragged rows, repeated and
out-of-range indices, host outputs, the raw-gather knob, direct C-ABI calls, and
bit-exact round trips at the benchmark sizes."""
import ctypes

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


def npy(t):
    torch.cuda.synchronize()
    return t.detach().cpu().numpy()


def same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return a.shape == b.shape and a.tobytes() == b.tobytes()


def masked_rows(rng, n, v, wb, frac=0.6, flip=0.2):
    W = 8 * wb
    it = {4: np.int32, 8: np.int64}[wb]
    ut = {4: np.uint32, 8: np.uint64}[wb]
    bits = rng.random((v, W)) < frac
    m = np.zeros(v, dtype=np.uint64)
    for b in range(W):
        m |= bits[:, b].astype(np.uint64) << np.uint64(b)
    m = m.astype(ut)
    base = rng.integers(0, 2**63, v, dtype=np.uint64).astype(ut) & m
    noise = rng.integers(0, 2**63, (n, v), dtype=np.uint64).astype(ut)
    data = (noise & ~m) | base
    data = np.where(rng.random((n, v)) < flip, noise, data)
    return data.view(it), m.view(it), base.view(it)


@pytest.mark.parametrize("wb", [4, 8])
@pytest.mark.parametrize("v", [1, 2, 3, 31, 32, 33, 200])
def test_small_and_ragged_rows(ibp, oracle, wb, v):
    rng = np.random.default_rng(100 * v + wb)
    n = 301
    d, m, b = masked_rows(rng, n, v, wb)
    dm, db = torch.from_numpy(m).cuda(), torch.from_numpy(b).cuda()
    x = torch.from_numpy(d).pin_memory()
    assert same(npy(ibp.get_compress_size(x, dm, db)), oracle.compress_size(d, m, b))
    ocomp, obm = oracle.compress(d, m, b)
    bm = ibp.compress_inplace(x, dm, db)
    assert same(npy(bm), obm)
    assert same(npy(x), ocomp.view(d.dtype))
    idx = rng.integers(0, n, 777).astype(np.int64)
    out = ibp.decompress_fetch(x, dm, db, bm, "cuda", None, torch.from_numpy(idx).cuda())
    assert same(npy(out), d[idx])
    out = ibp.decompress_fetch(x.cuda(), dm, db, bm, "cuda")
    assert same(npy(out), d)


def test_empty_inputs(ibp):
    d = np.zeros((0, 64), dtype=np.int64)
    x = torch.from_numpy(d).cuda()
    m, b = ibp.preprocess(x, 0.9)
    assert same(npy(m), np.zeros(64, np.int64))
    assert npy(ibp.get_compress_size(x, m, b)).shape == (0,)
    bm = ibp.compress_inplace(x, m, b)
    assert npy(bm).shape == (0,)
    out = ibp.decompress_fetch(x, m, b, bm, "cuda")
    assert npy(out).shape == (0, 64)
    rng = np.random.default_rng(1)
    d2, m2, b2 = masked_rows(rng, 50, 64, 8)
    y = torch.from_numpy(d2).pin_memory()
    dm, db = torch.from_numpy(m2).cuda(), torch.from_numpy(b2).cuda()
    bm2 = ibp.compress_inplace(y, dm, db)
    out = ibp.decompress_fetch(y, dm, db, bm2, "cuda", None,
                               torch.zeros(0, dtype=torch.int64, device="cuda"))
    assert npy(out).shape == (0, 64)


def test_preprocess_nothing_saved_gives_zero_mask(ibp):
    rng = np.random.default_rng(5)
    d = rng.integers(-2**63, 2**63 - 1, (64, 40), dtype=np.int64)
    m, b = ibp.preprocess(torch.from_numpy(d).cuda(), None)
    assert not npy(m).any() and not npy(b).any()


def test_repeated_indices_and_host_output(ibp, oracle):
    rng = np.random.default_rng(7)
    d, m, b = masked_rows(rng, 1000, 64, 8, frac=0.7, flip=0.1)
    x = torch.from_numpy(d).pin_memory()
    dm, db = torch.from_numpy(m).cuda(), torch.from_numpy(b).cuda()
    bm = ibp.compress_inplace(x, dm, db)
    hot = np.concatenate([np.full(5000, 17), np.full(300, 999), rng.integers(0, 1000, 4000)])
    idx = rng.permutation(hot).astype(np.int64)
    out = ibp.decompress_fetch(x, dm, db, bm, "cuda", None, torch.from_numpy(idx).cuda())
    assert same(npy(out), d[idx])
    out = ibp.decompress_fetch(x, dm, db, bm, "cpu", None, torch.from_numpy(idx[:100]).cuda())
    torch.cuda.synchronize()
    assert out.device.type == "cpu" and out.is_pinned()
    assert same(out.numpy(), d[idx[:100]])
    buf = torch.empty((100, 64), dtype=torch.int64, device="cuda")
    out = ibp.decompress_fetch(x, dm, db, bm, "cuda", None,
                               torch.from_numpy(idx[:100]).int().cuda(), None, None, None, buf)
    assert out.data_ptr() == buf.data_ptr()
    assert same(npy(buf), d[idx[:100]])
    raw = ibp.decompress_fetch(x, dm, db, bm, "cuda", None, torch.from_numpy(idx[:64]).cuda(),
                               None, None, 2)
    assert same(npy(raw), npy(x)[idx[:64]])


def test_bad_index_is_flagged_not_read(ibp):
    """An out-of-range row index is skipped and reported through the status word."""
    from invariantbitpacking_b200 import _capi
    rng = np.random.default_rng(9)
    d, m, b = masked_rows(rng, 100, 64, 8)
    x = torch.from_numpy(d).pin_memory()
    dm, db = torch.from_numpy(m).cuda(), torch.from_numpy(b).cuda()
    bm = ibp.compress_inplace(x, dm, db)
    idx = torch.tensor([3, 100, -1, 5, 1 << 40], dtype=torch.int64, device="cuda")
    out = torch.zeros((5, 64), dtype=torch.int64, device="cuda")
    lib = _capi.lib
    wsb = lib.ibp_decompress_fetch_workspace_size(5, 64, 8, 1)
    ws = torch.empty(wsb, dtype=torch.uint8, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    _capi.check(lib.ibp_decompress_fetch(x.data_ptr(), 100, 64, 8, dm.data_ptr(), db.data_ptr(),
                                         bm.data_ptr(), idx.data_ptr(), 5, -1, out.data_ptr(),
                                         -1, -1, -1, ws.data_ptr(), wsb, st))
    status = ctypes.c_int32(0)
    _capi.check(lib.ibp_read_status(ws.data_ptr(), ctypes.byref(status), st))
    assert status.value & 1
    o = npy(out)
    assert same(o[0], d[3]) and same(o[3], d[5])
    assert not o[1].any() and not o[2].any() and not o[4].any()


def test_capi_direct_matches_oracle(ibp, oracle):
    """Plain pointers through the C ABI (no torch layer) on device buffers."""
    from invariantbitpacking_b200 import _capi
    lib = _capi.lib
    rng = np.random.default_rng(21)
    n, v = 4000, 96
    d, m, b = masked_rows(rng, n, v, 4, frac=0.5, flip=0.3)
    st = torch.cuda.current_stream().cuda_stream
    x = torch.from_numpy(d).cuda()
    dm, db = torch.from_numpy(m).cuda(), torch.from_numpy(b).cuda()
    bm = torch.empty((n + 31) // 32, dtype=torch.int32, device="cuda")
    wsb = lib.ibp_compress_inplace_workspace_size(n, v, 4, 0)
    ws = torch.empty(wsb, dtype=torch.uint8, device="cuda")
    _capi.check(lib.ibp_compress_inplace(x.data_ptr(), n, v, 4, dm.data_ptr(), db.data_ptr(),
                                         None, -1, bm.data_ptr(), ws.data_ptr(), wsb, st))
    ocomp, obm = oracle.compress(d, m, b)
    assert same(npy(x), ocomp.view(np.int32)) and same(npy(bm), obm)
    out = torch.empty((n, v), dtype=torch.int32, device="cuda")
    wsb = lib.ibp_decompress_fetch_workspace_size(n, v, 4, 0)
    ws = torch.empty(max(wsb, 1), dtype=torch.uint8, device="cuda")
    _capi.check(lib.ibp_decompress_fetch(x.data_ptr(), n, v, 4, dm.data_ptr(), db.data_ptr(),
                                         bm.data_ptr(), None, -1, -1, out.data_ptr(), -1, -1, -1,
                                         ws.data_ptr(), wsb, st))
    assert same(npy(out), d)


def test_compress_with_index_reads_sources_first(ibp, oracle):
    rng = np.random.default_rng(31)
    d, m, b = masked_rows(rng, 500, 64, 8)
    idx = rng.permutation(500)[:400].astype(np.int64)
    x = torch.from_numpy(d.copy()).pin_memory()
    dm, db = torch.from_numpy(m).cuda(), torch.from_numpy(b).cuda()
    bm = ibp.compress_inplace(x, dm, db, torch.from_numpy(idx).cuda())
    ocomp, obm = oracle.compress(d, m, b, idx)
    got = npy(x)
    assert same(npy(bm), obm)
    assert same(got[:400], ocomp.view(np.int64))
    assert same(got[400:], d[400:])


def test_plain_small_full_size(ibp, oracle):
    """16384 x 128 int64 rows: preprocess(0.9) -> compress -> fetch 2048 rows, vs oracle."""
    from invariantbitpacking_b200 import synthetic
    d, idx = synthetic.plain_small()
    om, ob, _ = oracle.preprocess(d, 0.9)
    x = torch.from_numpy(d).pin_memory()
    m, b = ibp.preprocess(x, 0.9)
    assert same(npy(m), om.view(np.int64)) and same(npy(b), ob.view(np.int64))
    ocomp, obm = oracle.compress(d, om, ob)
    bm = ibp.compress_inplace(x, m, b)
    assert same(npy(bm), obm) and same(npy(x), ocomp.view(np.int64))
    out = ibp.decompress_fetch(x, m, b, bm, "cuda", None, torch.from_numpy(idx).cuda())
    assert same(npy(out), d[idx])


def test_graph_features_full_size_round_trip(ibp, oracle):
    """2.4M x 64 int64 rows (1.2 GB pinned): sweep preprocess, compress, and Zipf batches of
    100k/200k/400k rows decompressed bit-exact; sizes checked against the oracle."""
    from invariantbitpacking_b200 import synthetic
    d = synthetic.graph_features()
    x = torch.from_numpy(d).pin_memory()
    m, b = ibp.preprocess(x, None)
    mm = npy(m)
    assert mm.any(), "the sweep found no invariant bits"
    sz = npy(ibp.get_compress_size(x, m, b))
    samp = np.random.default_rng(0).integers(0, d.shape[0], 20000)
    assert same(sz[samp], oracle.compress_size(d, mm, npy(b), samp))
    comp_len = ibp.get_single_compress_len(x, m, b)
    assert 0 < comp_len < 64
    ref = torch.from_numpy(d).cuda()
    bm = ibp.compress_inplace(x, m, b)
    z = synthetic.Zipf(d.shape[0], 1.1, seed=12)
    for k in (100_000, 200_000, 400_000):
        idx = torch.from_numpy(z.sample(k)).cuda()
        out = ibp.decompress_fetch(x, m, b, bm, "cuda", comp_len, idx)
        assert torch.equal(out, ref[idx])


@pytest.mark.parametrize("wb", [4, 8])
@pytest.mark.parametrize("where", ["host", "device"])
def test_long_rows_longer_than_their_slot(ibp, oracle, wb, where):
    """Long rows whose compressed lengths vary a lot around the hint: most rows compress to a
    few words, a few keep almost every bit, so some rows outgrow the fetch's shared-memory
    slot (sized from the hint) and are decoded from their source instead; all must match."""
    rng = np.random.default_rng(21 + wb)
    n, v = 3000, 1100
    d = np.zeros((n, v), dtype=np.int64 if wb == 8 else np.int32)
    noisy = rng.choice(n, 150, replace=False)
    span = 30 if wb == 8 else 14
    d[noisy] = rng.integers(0, 1 << span, (noisy.size, v))
    d[noisy, ::7] = 0  # still compressible: those rows are compressed, but long
    x = torch.from_numpy(d.copy()).pin_memory()
    m, b = ibp.preprocess(x, 0.9)
    sizes = ibp.get_compress_size(x, m, b)
    torch.cuda.synchronize()
    cl = ibp.get_single_compress_len(x, m, b)
    bm = ibp.compress_inplace(x, m, b)
    sz = sizes.numpy()
    assert (sz < v * wb).all() and sz.max() > 4 * cl * wb  # long compressed rows exist
    if where == "device":
        x = x.cuda()
    comp = x.cpu().numpy()
    idx = np.concatenate([noisy[:40], rng.integers(0, n, 500)])
    for ix in (None, idx):
        ti = None if ix is None else torch.from_numpy(ix).cuda()
        out = ibp.decompress_fetch(x, m, b, bm, "cuda", cl, ti)
        want = d if ix is None else d[ix]
        assert np.array_equal(out.cpu().numpy(), want)
    ref = oracle.decompress(comp, m.cpu().numpy(), b.cpu().numpy(), bm.cpu().numpy(), idx)
    assert np.array_equal(ref, d[idx])


@pytest.mark.parametrize("wb", [4, 8])
@pytest.mark.parametrize("kept", [(1, 4), (5, 20)], ids=["few", "many"])
@pytest.mark.parametrize("where", ["host", "device"])
def test_long_rows_few_and_many_kept_bits(ibp, wb, kept, where):
    """Rows of 300 and 1100 words under masks that keep 1-4 bits per word (each kept bit
    placed straight from the mask) or 5-20 (the move-mask scatter), with random values in
    the kept bits, a few words stored whole and a few rows stored raw: whole sets and
    batches decode to the source rows.  The first word of each row ends within the stream's
    first word, so its read window starts in the row's bitmap."""
    rng = np.random.default_rng(40 + wb + kept[0])
    W = 8 * wb
    it = {4: np.int32, 8: np.int64}[wb]
    ut = {4: np.uint32, 8: np.uint64}[wb]
    for v in (300, 1100):
        n = 2000
        keep = np.zeros(v, dtype=np.uint64)
        for j in range(v):
            for bit in rng.choice(W, rng.integers(kept[0], kept[1] + 1), replace=False):
                keep[j] |= np.uint64(1) << np.uint64(bit)
        keep = keep.astype(ut)
        base = rng.integers(0, 2**63, v, dtype=np.uint64).astype(ut) & ~keep
        noise = rng.integers(0, 2**63, (n, v), dtype=np.uint64).astype(ut)
        data = (noise & keep) | base
        whole = rng.random((n, v)) < 0.01
        data = np.where(whole, noise, data)
        data[rng.choice(n, 20, replace=False)] = noise[:20]
        d = data.view(it)
        m = torch.from_numpy((~keep).view(it)).cuda()
        b = torch.from_numpy(base.view(it)).cuda()
        x = torch.from_numpy(d.copy()).pin_memory()
        cl = ibp.get_single_compress_len(x, m, b)
        bm = ibp.compress_inplace(x, m, b)
        xs = x if where == "host" else x.cuda()
        idx = rng.integers(0, n, 700)
        for ix in (None, idx):
            ti = None if ix is None else torch.from_numpy(ix).cuda()
            out = ibp.decompress_fetch(xs, m, b, bm, "cuda", cl, ti, check=True)
            assert np.array_equal(out.cpu().numpy(), d if ix is None else d[ix])


@pytest.mark.parametrize("wb,v", [(8, 64), (8, 65), (4, 131), (8, 600)])
def test_device_rows_whole_set_and_small_batches(ibp, oracle, wb, v):
    """Device-resident rows of 512 bytes and up take the double-buffered read path; rows whose
    length is not a multiple of 16 bytes alternate alignment (the unaligned ones fall back to
    plain loads).  Whole sets, tiny batches and repeats must all match the oracle."""
    rng = np.random.default_rng(v + wb)
    n = 4000
    f = rng.normal(0, 0.4, (n, v * wb // 4)).astype(np.float32)
    f = (f.view(np.uint32) & np.uint32(0xFFFF8000)).view(np.float32)
    d = np.ascontiguousarray(f).view(np.int64 if wb == 8 else np.int32)
    x = torch.from_numpy(d.copy()).pin_memory()
    m, b = ibp.preprocess(x, None)
    cl = ibp.get_single_compress_len(x, m, b)
    bm = ibp.compress_inplace(x, m, b)
    xd = x.cuda()
    out = ibp.decompress_fetch(xd, m, b, bm, "cuda", cl, None)
    assert np.array_equal(out.cpu().numpy(), d)
    for k in (1, 5, 33, 1000):
        idx = rng.integers(0, n, k)
        out = ibp.decompress_fetch(xd, m, b, bm, "cuda", cl, torch.from_numpy(idx).cuda())
        assert np.array_equal(out.cpu().numpy(), d[idx])


@pytest.mark.parametrize("wb,v", [(8, 2), (8, 16), (8, 48), (8, 64), (4, 4), (4, 32), (4, 64)])
@pytest.mark.parametrize("mode", [0, 1, 2], ids=["auto", "sort", "hash"])
def test_device_rows_up_to_64_words(ibp, oracle, wb, v, mode):
    """Device rows of at most 64 words, 16-byte aligned (the whole-row HBM decode kernel for
    unindexed and hash-listed fetches; the sort mode keeps the general kernel): raw and
    compressed rows mixed, whole sets and batches with repeats, all exact."""
    from invariantbitpacking_b200 import _capi
    rng = np.random.default_rng(1000 + 10 * v + wb)
    n = 3000
    d, m, b = masked_rows(rng, n, v, wb, frac=0.7, flip=0.15)
    dm, db = torch.from_numpy(m).cuda(), torch.from_numpy(b).cuda()
    x = torch.from_numpy(d.copy()).pin_memory()
    bm = ibp.compress_inplace(x, dm, db)
    xd = x.cuda()
    _capi.check(_capi.lib.ibp_set_fetch_dedup(mode))
    try:
        out = ibp.decompress_fetch(xd, dm, db, bm, "cuda", None, None, check=True)
        assert same(npy(out), d)
        for k in (1, 31, 33, 700, 9000):
            idx = rng.integers(0, n, k).astype(np.int64)
            out = ibp.decompress_fetch(xd, dm, db, bm, "cuda", None, torch.from_numpy(idx).cuda(),
                                       check=True)
            assert same(npy(out), d[idx])
    finally:
        _capi.check(_capi.lib.ibp_set_fetch_dedup(0))


@pytest.mark.parametrize("wb", [4, 8])
def test_device_rows_large_batches(ibp, oracle, wb):
    """Device-resident batches larger than one wave of claim-pass blocks (two positions per
    thread there; 8-row chunks in the HBM-row kernel), Zipf-skewed and uniform: most rows have
    every word compressible (the fixed-offset decode), a fifth have some words stored whole
    (the prefix-sum decode), a few are stored raw; all exact, with the repeat copies."""
    from invariantbitpacking_b200 import synthetic
    rng = np.random.default_rng(3000 + wb)
    n, v = 150_000, 64
    d, m, b = masked_rows(rng, n, v, wb, frac=0.7, flip=0.0)
    ut = {4: np.uint32, 8: np.uint64}[wb]
    mixed = rng.choice(n, n // 5, replace=False)
    words = rng.integers(0, v, (mixed.size, 3))
    noise = rng.integers(0, 2**63, (mixed.size, 3), dtype=np.uint64).astype(ut).view(d.dtype)
    d[mixed[:, None], words] = noise
    raw = rng.choice(n, n // 50, replace=False)
    d[raw] = rng.integers(0, 2**63, (raw.size, v), dtype=np.uint64).astype(ut).view(d.dtype)
    dm, db = torch.from_numpy(m).cuda(), torch.from_numpy(b).cuda()
    x = torch.from_numpy(d.copy()).pin_memory()
    bm = ibp.compress_inplace(x, dm, db)
    xd = x.cuda()
    z = synthetic.Zipf(n, 1.1, seed=31)
    for idx in (z.sample(400_000), rng.integers(0, n, 320_000).astype(np.int64)):
        out = ibp.decompress_fetch(xd, dm, db, bm, "cuda", None, torch.from_numpy(idx).cuda(),
                                   check=True)
        assert same(npy(out), d[idx])


@pytest.mark.parametrize("where", ["host", "device"])
@pytest.mark.parametrize("wb,v", [(8, 64), (4, 64), (8, 24), (8, 200)])
def test_corrupt_rows_are_flagged_and_skipped(ibp, oracle, where, wb, v):
    """Rows stored raw but marked compressed in a doctored bitmask: a row whose bitmap claims
    a stream as long as the raw row is reported (status bit 1, check=True raises) and its
    output row left untouched; a row whose bitmap happens to fit is decoded as the oracle
    decodes it."""
    rng = np.random.default_rng(2000 + v + wb)
    n = 2000
    W = 8 * wb
    d, m, b = masked_rows(rng, n, v, wb, frac=0.8, flip=0.05)
    mw = -(-(-(-v // 8)) // wb)
    # a tenth of the rows random (stored raw); half of those with a zero first (bitmap) part,
    # which, marked compressed, claims every word raw: a stream longer than the row
    noisy = rng.choice(n, n // 10, replace=False)
    d[noisy] = rng.integers(-(2 ** 62), 2 ** 62, (noisy.size, v)).astype(d.dtype)
    d.view(np.uint32).reshape(n, -1)[noisy[: noisy.size // 2], : mw * wb // 4] = 0
    dm, db = torch.from_numpy(m).cuda(), torch.from_numpy(b).cuda()
    x = torch.from_numpy(d.copy()).pin_memory()
    bm = ibp.compress_inplace(x, dm, db)
    comp = x.numpy().copy()
    bits = npy(bm).view(np.uint32)
    raw = np.array([not (bits[r // 32] >> (r % 32)) & 1 for r in range(n)])
    assert raw.any() and not raw.all()
    bad_bits = bits.copy()
    for r in np.flatnonzero(raw):
        bad_bits[r // 32] |= np.uint32(1) << np.uint32(r % 32)
    bm2 = torch.from_numpy(bad_bits.view(np.int32)).cuda()
    # which doctored rows claim a stream too long for the row
    ut = {4: np.uint32, 8: np.uint64}[wb]
    nb = np.array([W - bin(int(x)).count("1") for x in m.view(ut)])
    units = comp.view(np.uint32).reshape(n, -1)
    too_long = np.zeros(n, dtype=bool)
    for r in np.flatnonzero(raw):
        cj = np.array([(units[r, j // 32] >> (j % 32)) & 1 for j in range(v)], dtype=bool)
        total = int(np.where(cj, nb, W).sum())
        too_long[r] = mw + -(-total // W) >= v
    assert too_long.any()
    src = x.cuda() if where == "device" else x
    for idx in (None, rng.integers(0, n, 1500).astype(np.int64)):
        rows = np.arange(n) if idx is None else idx
        out = torch.full((rows.size, v), 7, dtype=x.dtype, device="cuda")
        ti = None if idx is None else torch.from_numpy(idx).cuda()
        with pytest.raises(RuntimeError, match="bitmap"):
            ibp.decompress_fetch(src, dm, db, bm2, "cuda", None, ti, output_tensor=out,
                                 check=True)
        out.fill_(7)
        ibp.decompress_fetch(src, dm, db, bm2, "cuda", None, ti, output_tensor=out)
        got = npy(out)
        skip = too_long[rows]
        assert (got[skip] == 7).all()
        keep = ~skip
        want = oracle.decompress(comp, m, b, bad_bits.view(np.int32), rows[keep])
        assert same(got[keep], want.view(d.dtype))


def test_read_rows_probe_reads_the_listed_rows(ibp):
    """The access-pattern probe (a measurement aid) runs over host and device rows, takes
    every listed row (its work counter ends at or past the list), and refuses reads that would
    leave a row's stride."""
    from invariantbitpacking_b200 import _capi
    lib = _capi.lib
    n, v = 5000, 64
    x = torch.zeros((n, v), dtype=torch.int64).pin_memory()
    rows = torch.randint(0, n, (3000,), device="cuda")
    ws = torch.zeros(256, dtype=torch.uint8, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    for base in (x, x.cuda()):
        for nbytes in (16, 288, 512):
            _capi.check(lib.ibp_read_rows_probe(base.data_ptr(), v * 8, rows.data_ptr(), 3000,
                                                nbytes, ws.data_ptr(), 256, st))
            torch.cuda.synchronize()
            assert int(ws[64:72].view(torch.int64).item()) >= 3000
    assert lib.ibp_read_rows_probe(x.data_ptr(), v * 8, rows.data_ptr(), 3000, 600, ws.data_ptr(),
                                   256, st) == _capi.IBP_ERR_ARGUMENT
    assert lib.ibp_read_rows_probe(x.data_ptr(), v * 8, rows.data_ptr(), 3000, 288, ws.data_ptr(),
                                   16, st) == _capi.IBP_ERR_WORKSPACE
