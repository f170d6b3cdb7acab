"""Pins the CPU oracle to the reference: every vector in tests/golden/ was produced by the
reference extension itself (tests/golden/make_golden.py, run on a B200), and the oracle
must reproduce each of them bit for bit."""
import glob
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CODEC = sorted(os.path.basename(f)[:-4] for f in glob.glob(os.path.join(GOLDEN, "*.npz"))
               if not os.path.basename(f).startswith("km_"))
KMEANS = sorted(os.path.basename(f)[:-4] for f in glob.glob(os.path.join(GOLDEN, "km_*.npz")))


def load(name):
    return np.load(os.path.join(GOLDEN, name + ".npz"))


def same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return a.shape == b.shape and a.tobytes() == b.tobytes()


def test_golden_files_present():
    assert len(CODEC) >= 15 and len(KMEANS) >= 2


@pytest.mark.parametrize("name", CODEC)
def test_preprocess_matches_reference(oracle, name):
    z = load(name)
    d = z["data"]
    keys = [k for k in z.files if k.startswith("mask_")]
    assert keys
    for k in keys:
        tag = k[5:]
        thr = None if tag == "sweep" else float(tag[1:])
        m, b, _ = oracle.preprocess(d, thr)
        assert same(m.view(d.dtype), z[k]), (name, k)
        assert same(b.view(d.dtype), z["bitval_" + tag]), (name, k)


@pytest.mark.parametrize("name", CODEC)
def test_sizes_match_reference(oracle, name):
    z = load(name)
    d, mask, bitval = z["data"], z["mask"], z["bitval"]
    assert same(oracle.compress_size(d, mask, bitval), z["sizes"])
    if "idx" in z.files:
        s = oracle.compress_size(d, mask, bitval, z["idx"])
        assert same(s, z["sizes_idx"])
        assert int(z["total_idx"][0]) == int(s.sum())


@pytest.mark.parametrize("name", [n for n in CODEC if n not in ("bytes_w1", "half_w2")])
def test_codec_matches_reference(oracle, name):
    z = load(name)
    d, mask, bitval = z["data"], z["mask"], z["bitval"]
    comp, bm = oracle.compress(d, mask, bitval)
    assert same(comp.view(d.dtype), z["comp"])
    assert same(bm, z["bitmask"])
    dec = oracle.decompress(z["comp"], mask, bitval, z["bitmask"])
    ref_dec = d if "decomp_is_data" in z.files or "decomp" not in z.files else z["decomp"]
    assert same(dec.view(d.dtype), ref_dec)
    if "idx" in z.files:
        idx = z["idx"]
        dec2 = oracle.decompress(z["comp"], mask, bitval, z["bitmask"], idx)
        ref2 = d[idx] if "decomp_idx" not in z.files else z["decomp_idx"]
        assert same(dec2.view(d.dtype), ref2)
    if "condensed" in z.files:
        cc, offs = oracle.compress_condensed(d, mask, bitval)
        assert same(cc.view(d.dtype), z["condensed"])
        assert same(offs, z["condensed_offsets"])


@pytest.mark.parametrize("name", KMEANS)
def test_kmeans_masks_from_reference_clusters(oracle, name):
    """create_mask_many at the final threshold, from the reference's own assignment."""
    z = load(name)
    d, c = z["data"], int(z["c"])
    m, b = oracle.kmeans_masks(d, z["clusters"], c, 1.0)
    assert same(m.view(d.dtype), z["kmasks"])
    assert same(b.view(d.dtype), z["kbitvals"])


@pytest.mark.parametrize("name", [n for n in KMEANS if "_sep_" in n])
def test_kmeans_full_matches_reference_without_ties(oracle, name):
    """Tie-free inputs: seeding (srand(1) + std::random_shuffle), ten assignment/update
    rounds with the OR quirk, and the final masks all match the reference exactly."""
    z = load(name)
    d, c = z["data"], int(z["c"])
    init = oracle.random_shuffle_init(d.shape[0], c, reseed=True)
    m, b, cl = oracle.preprocess_kmeans(d, c, init)
    assert same(cl, z["clusters"])
    assert same(m.view(d.dtype), z["kmasks"])
    assert same(b.view(d.dtype), z["kbitvals"])
