"""GPU parity: the engine (libibp_b200.so through its C ABI, via the drop-in torch layer)
against the reference's own outputs (tests/golden/) and the CPU oracle, bit for bit."""
import glob
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CODEC = sorted(os.path.basename(f)[:-4] for f in glob.glob(os.path.join(GOLDEN, "*.npz"))
               if not os.path.basename(f).startswith("km_"))
CODEC48 = [n for n in CODEC if n not in ("bytes_w1", "half_w2")]
KMEANS = sorted(os.path.basename(f)[:-4] for f in glob.glob(os.path.join(GOLDEN, "km_*.npz")))


@pytest.fixture(scope="module")
def ibp():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import invariantbitpacking_b200 as m
    return m


def load(name):
    return np.load(os.path.join(GOLDEN, name + ".npz"))


def place(a, where):
    t = torch.from_numpy(np.ascontiguousarray(a))
    return t.pin_memory() if where == "host" else t.cuda()


def npy(t):
    torch.cuda.synchronize()
    return t.detach().cpu().numpy()


def same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return a.shape == b.shape and a.tobytes() == b.tobytes()


@pytest.mark.parametrize("where", ["host", "device"])
@pytest.mark.parametrize("name", CODEC)
def test_preprocess(ibp, name, where):
    z = load(name)
    x = place(z["data"], where)
    for k in [k for k in z.files if k.startswith("mask_")]:
        tag = k[5:]
        thr = None if tag == "sweep" else float(tag[1:])
        m, b = ibp.preprocess(x, thr)
        assert same(npy(m), z[k]), (k, "mask")
        assert same(npy(b), z["bitval_" + tag]), (k, "bitval")


@pytest.mark.parametrize("where", ["host", "device"])
@pytest.mark.parametrize("name", CODEC)
def test_get_compress_size(ibp, name, where):
    z = load(name)
    x = place(z["data"], where)
    m, b = torch.from_numpy(z["mask"]).cuda(), torch.from_numpy(z["bitval"]).cuda()
    assert same(npy(ibp.get_compress_size(x, m, b)), z["sizes"])
    if "idx" in z.files:
        tot = torch.zeros(1, dtype=torch.int64, device="cuda")
        s = ibp.get_compress_size(x, m, b, torch.from_numpy(z["idx"]).cuda(), tot)
        assert same(npy(s), z["sizes_idx"])
        assert int(npy(tot)[0]) == int(z["total_idx"][0])


@pytest.mark.parametrize("where", ["host", "device"])
@pytest.mark.parametrize("name", CODEC48)
def test_compress_inplace(ibp, name, where):
    z = load(name)
    x = place(z["data"], where)
    m, b = torch.from_numpy(z["mask"]).cuda(), torch.from_numpy(z["bitval"]).cuda()
    bm = ibp.compress_inplace(x, m, b)
    assert same(npy(bm), z["bitmask"])
    assert same(npy(x), z["comp"])


@pytest.mark.parametrize("where", ["host", "device"])
@pytest.mark.parametrize("name", CODEC48)
def test_decompress_fetch(ibp, name, where):
    z = load(name)
    d = z["data"]
    comp = place(z["comp"], where)
    m, b = torch.from_numpy(z["mask"]).cuda(), torch.from_numpy(z["bitval"]).cuda()
    bm = torch.from_numpy(z["bitmask"]).cuda()
    out = ibp.decompress_fetch(comp, m, b, bm, torch.device("cuda"))
    assert same(npy(out), d)
    if "idx" in z.files:
        idx = torch.from_numpy(z["idx"]).cuda()
        out = ibp.decompress_fetch(comp, m, b, bm, torch.device("cuda"), None, idx)
        assert same(npy(out), d[z["idx"]])


@pytest.mark.parametrize("name", [n for n in CODEC48 if n != "large_v4096_w4"])
def test_compress_condensed(ibp, name):
    z = load(name)
    if "condensed" not in z.files:
        pytest.skip("no condensed golden")
    x = torch.from_numpy(z["data"]).cuda()
    m, b = torch.from_numpy(z["mask"]).cuda(), torch.from_numpy(z["bitval"]).cuda()
    cc, offs = ibp.compress_condensed(x, m, b)
    assert same(npy(cc), z["condensed"])
    assert same(npy(offs), z["condensed_offsets"])


@pytest.mark.parametrize("name", KMEANS)
def test_kmeans_vs_oracle(ibp, oracle, name):
    z = load(name)
    d, c = z["data"], int(z["c"])
    init = oracle.random_shuffle_init(d.shape[0], c, reseed=True)
    om, ob, ocl = oracle.preprocess_kmeans(d, c, init)
    for where in ("host", "device"):
        m, b, cl = ibp.preprocess_kmeans(place(d, where), c, 0.9, seed_rows=init)
        assert same(npy(cl), ocl)
        assert same(npy(m), om.view(d.dtype))
        assert same(npy(b), ob.view(d.dtype))
    if "_sep_" in name:  # tie-free case: the reference's own outputs too
        assert same(ocl, z["clusters"])
        assert same(npy(m), z["kmasks"])


def test_kmeans_int64_vs_oracle(ibp, oracle):
    """8-byte words (not run through the reference: its create_mask_many indexes past its
    shared array there); the oracle restates the intended arithmetic."""
    rng = np.random.default_rng(11)
    c, v, n = 16, 32, 5000
    cent = rng.normal(0, 1, (c, 2 * v)).astype(np.float32) * 3
    lab = rng.integers(0, c, n)
    x = (cent[lab] + rng.normal(0, 0.05, (n, 2 * v)).astype(np.float32)).view(np.int64)
    init = oracle.random_shuffle_init(n, c, reseed=True)
    om, ob, ocl = oracle.preprocess_kmeans(x, c, init)
    m, b, cl = ibp.preprocess_kmeans(place(x, "host"), c, None, seed_rows=init)
    assert same(npy(cl), ocl)
    assert same(npy(m), om.view(np.int64))
    assert same(npy(b), ob.view(np.int64))
