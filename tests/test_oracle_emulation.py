"""The oracle's restatement of the compressed layout agrees with a literal replay of the
reference device loops (tests/ref_emulation.py) on small random cases, including the
mask extremes where the reference depends on PTX shift clamping."""
import numpy as np
import pytest

import ref_emulation as emu

UT = {4: np.uint32, 8: np.uint64}


def _case(rng, n, v, wb, kind):
    W = 8 * wb
    full = (1 << W) - 1
    if kind == "random":
        m = [int(x) for x in rng.integers(0, 2**63, v, dtype=np.uint64) & np.uint64(full)]
        m = [x | int(rng.integers(0, 2)) << (W - 1) for x in m]
    else:
        pool = [0, full, full ^ 1, 1 << (W - 1), (1 << (W - 1)) | 1, 0xAAAAAAAAAAAAAAAA & full,
                0x5555555555555555 & full, 0x0F0F0F0F0F0F0F0F & full, full >> 1, full << 1 & full,
                0xFFFF000000000000 & full]
        m = [pool[int(rng.integers(0, len(pool)))] for _ in range(v)]
    bv = [int(rng.integers(0, 2**62)) * 3 & m[j] for j in range(v)]
    rows = []
    for _ in range(n):
        r = []
        for j in range(v):
            noise = int(rng.integers(0, 2**63)) * 2 + int(rng.integers(0, 2))
            noise &= full
            r.append(((noise & ~m[j]) | bv[j]) & full if rng.random() < 0.8 else noise)
        rows.append(r)
    return m, bv, rows


@pytest.mark.parametrize("wb", [4, 8])
@pytest.mark.parametrize("v", [1, 5, 32, 33, 70])
@pytest.mark.parametrize("kind", ["random", "extremes"])
def test_codec_matches_reference_loops(oracle, wb, v, kind):
    rng = np.random.default_rng(1000 * wb + v + (0 if kind == "random" else 7))
    W = 8 * wb
    n = 12
    m, bv, rows = _case(rng, n, v, wb, kind)
    data = np.array(rows, dtype=UT[wb]).reshape(n, v)
    mask = np.array(m, dtype=UT[wb])
    bitval = np.array(bv, dtype=UT[wb])
    sizes = oracle.compress_size(data, mask, bitval)
    comp, bm = oracle.compress(data, mask, bitval)
    for i in range(n):
        es = emu.compressed_size(rows[i], m, bv, W)
        assert sizes[i] == es
        compressed = es < v * wb
        assert bool((int(bm[i // 32]) >> (i % 32)) & 1) == compressed
        if compressed:
            assert [int(x) for x in comp[i]] == emu.compress_and_write(rows[i], m, bv, W)
            assert emu.decompress_row([int(x) for x in comp[i]], m, bv, W) == rows[i]
        else:
            assert [int(x) for x in comp[i]] == rows[i]
    dec = oracle.decompress(comp, mask, bitval, bm)
    assert np.array_equal(dec, data)
