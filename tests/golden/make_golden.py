"""Dump golden vectors from the REFERENCE implementation (its own ibp_cuda extension).

Runs on a GPU box: it imports the reference extension that oracle/build_ref.py
compiled from the reference sources for sm_100a (oracle/_ref/ibp_cuda*.so) and
calls it through its own positional API (src/ibp_api.cu:124-135) on small
seeded inputs.  Every array the reference returns or writes is saved to
<out>/<case>.npz together with its inputs; tests/test_oracle_golden.py checks
the CPU oracle against these files, and the GPU parity tests reuse them.

Nothing here touches the product package.  Atomics of the reference land in
device memory except the k-means cluster ids (written by the reference into its
pinned output, as it always does), so k-means runs as a separate --part.  Inputs are chosen so that every
reference row is at least 128 bytes (its warp row copy reads and writes up to
32 four-byte words past a shorter row) and k-means runs only on 4-byte words
(its create_mask_many indexes past its shared array for 8-byte words).

Usage (on a machine with a B200 and the reference built into oracle/_ref):
    python tests/golden/make_golden.py --out <dir>   # then copy the .npz files here
"""
import argparse
import ctypes
import glob
import importlib.util
import json
import os

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def _reference_extension():
    """The reference extension, loaded by explicit file path from oracle/_ref (never whatever
    module named ibp_cuda happens to be importable)."""
    mods = glob.glob(os.path.join(REPO, "oracle", "_ref", "ibp_cuda*.so"))
    if not mods:
        raise SystemExit("oracle/_ref/ibp_cuda*.so is missing: run oracle/build_ref.py first")
    spec = importlib.util.spec_from_file_location("ibp_cuda", mods[0])
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


ibp_cuda = _reference_extension()
ibp_cuda.print_debug(False)
LIBC = ctypes.CDLL("libc.so.6")

TO_TORCH = {np.dtype(np.int8): torch.int8, np.dtype(np.int16): torch.int16,
            np.dtype(np.int32): torch.int32, np.dtype(np.int64): torch.int64}


def pinned(a):
    return torch.from_numpy(np.ascontiguousarray(a)).pin_memory()


def to_np(t):
    torch.cuda.synchronize()
    return t.detach().cpu().numpy().copy()


def codec_case(name, words, thresholds, idx=None, mask=None, bitval=None, comp_len=None,
               condensed=True):
    """preprocess (each threshold) -> sizes -> compress_inplace -> decompress_fetch."""
    out = {"data": words}
    x = pinned(words)
    for thr in thresholds:
        key = "sweep" if thr is None else f"t{thr:g}"
        m, b = ibp_cuda.preprocess(x, thr)
        out[f"mask_{key}"] = to_np(m)
        out[f"bitval_{key}"] = to_np(b)
    if mask is None:
        key = "sweep" if thresholds[0] is None else f"t{thresholds[0]:g}"
        mask, bitval = out[f"mask_{key}"], out[f"bitval_{key}"]
    out["mask"], out["bitval"] = mask, bitval
    if words.dtype.itemsize not in (4, 8):
        sizes = ibp_cuda.get_compress_size(x, torch.from_numpy(mask).cuda(),
                                           torch.from_numpy(bitval).cuda(), None, None)
        out["sizes"] = to_np(sizes)
        return out
    dm, db = torch.from_numpy(mask).cuda(), torch.from_numpy(bitval).cuda()
    sizes = ibp_cuda.get_compress_size(x, dm, db, None, None)
    out["sizes"] = to_np(sizes)
    tot = torch.zeros(1, dtype=torch.int64, device="cuda")
    if idx is not None:
        di = torch.from_numpy(idx).cuda()
        out["idx"] = idx
        s2 = ibp_cuda.get_compress_size(x, dm, db, di, tot)
        out["sizes_idx"] = to_np(s2)
        out["total_idx"] = to_np(tot)
    if condensed:
        # device-resident input: the condensed packer ORs into its output with atomics
        comp_c, offs = ibp_cuda.compress_condensed(x.cuda(), dm, db, None)
        out["condensed"] = to_np(comp_c)
        out["condensed_offsets"] = to_np(offs)
    y = x.clone().pin_memory()
    bm = ibp_cuda.compress_inplace(y, dm, db, None)
    out["comp"] = to_np(y)
    out["bitmask"] = to_np(bm)
    dec = to_np(ibp_cuda.decompress_fetch(y, dm, db, bm, torch.device("cuda"), comp_len, None,
                                          None, None, None, None))
    # a faithful round trip is stored as a flag (the rows are already in "data")
    if np.array_equal(dec, words):
        out["decomp_is_data"] = np.array(True)
    else:
        out["decomp"] = dec
    if idx is not None:
        dec2 = to_np(ibp_cuda.decompress_fetch(y, dm, db, bm, torch.device("cuda"), comp_len,
                                               torch.from_numpy(idx).cuda(), None, None, None,
                                               None))
        if np.array_equal(dec2, words[idx]):
            out["decomp_idx_is_data"] = np.array(True)
        else:
            out["decomp_idx"] = dec2
    return out


def kmeans_case(words, c, repeat=False):
    x = pinned(words)
    LIBC.srand(1)  # the reference seeds with std::random_shuffle on the process rand() state
    m, b, cl = ibp_cuda.preprocess_kmeans(x, c, 0.9)
    out = {"data": words, "c": np.array(c), "kmasks": to_np(m), "kbitvals": to_np(b),
           "clusters": to_np(cl), "srand": np.array(1)}
    if repeat:  # same call again: shows whether tied assignments change run to run
        LIBC.srand(1)
        _, _, cl2 = ibp_cuda.preprocess_kmeans(x, c, 0.9)
        out["clusters_run2"] = to_np(cl2)
    return out


def shuffle_seed_rows(n, c):
    """Rows the reference seeds its centroids with after srand(1): libstdc++'s
    random_shuffle over 0..n-1 (swap i with rand() % (i + 1)), first min(c, n) entries."""
    LIBC.srand(1)
    ind = list(range(n))
    for i in range(1, n):
        j = LIBC.rand() % (i + 1)
        ind[i], ind[j] = ind[j], ind[i]
    return ind[:min(c, n)]


def f32_words(a, wb):
    a = np.ascontiguousarray(a.astype(np.float32))
    return a.view(np.int32) if wb == 4 else a.view(np.int64)


def random_mask(rng, v, wb, frac):
    """Arbitrary mask/bitval (not from preprocess), like the reference's throughput test."""
    W = 8 * wb
    ut = {4: np.uint32, 8: np.uint64}[wb]
    bits = rng.random((v, W)) < frac
    m = np.zeros(v, dtype=np.uint64)
    for b in range(W):
        m |= bits[:, b].astype(np.uint64) << np.uint64(b)
    return m.astype(ut).view({4: np.int32, 8: np.int64}[wb])


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(REPO, "golden_out"))
    ap.add_argument("--part", choices=["codec", "kmeans"], default="codec")
    a = ap.parse_args()
    os.makedirs(a.out, exist_ok=True)
    torch.cuda.init()
    cases = {}
    if a.part == "kmeans":
        kmeans_cases(cases)
    else:
        codec_cases(cases)
    save(a.out, cases, a.part)


def codec_cases(cases):
    # 1. the reference's own round-trip test shapes (tests/compress_test.py:30-46), seeded
    rng = np.random.default_rng(101)
    u = rng.random((1200, 128), dtype=np.float32)
    u = u[:600]
    cases["rand_f32_w4"] = codec_case("rand_f32_w4", f32_words(u, 4), [None, 0.9],
                                      idx=rng.integers(0, 600, 300).astype(np.int64))
    cases["rand_f32_w8"] = codec_case("rand_f32_w8", f32_words(u, 8), [None, 0.9],
                                      idx=rng.integers(0, 600, 300).astype(np.int64))
    d = rng.integers(0, 2147483647, (100, 100), dtype=np.int64).astype(np.int32)
    cases["dense_w4"] = codec_case("dense_w4", d, [None])
    cases["dense_w8"] = codec_case("dense_w8", d.view(np.int64), [None])
    s = rng.integers(0, 2147483647 // 100, (6, 100), dtype=np.int64).astype(np.int32)
    cases["semidense_w4"] = codec_case("semidense_w4", s, [None])
    cases["semidense_w8"] = codec_case("semidense_w8", s.view(np.int64), [None])

    # 2. plain-IBP shape: N(0, 0.5^2) with 5% rows from N(0, 100^2), int64 rows of 128 words
    rng = np.random.default_rng(1)
    x = rng.normal(0, 0.5, (512, 256)).astype(np.float32)
    out_rows = rng.choice(512, 26, replace=False)
    x[out_rows] = rng.normal(0, 100, (26, 256)).astype(np.float32)
    cases["cfg1_small"] = codec_case("cfg1_small", f32_words(x, 8), [0.9, None],
                                     idx=rng.permutation(512)[:128].astype(np.int64),
                                     comp_len=96)

    # 3. graph-feature shape: N(0, 0.3^2), 8 mantissa bits kept, 30% zeros, int64 rows of 64
    rng = np.random.default_rng(2)
    x = rng.normal(0, 0.3, (2048, 128)).astype(np.float32)
    x = (x.view(np.uint32) & np.uint32(0xFFFF8000)).view(np.float32)
    x[rng.random(x.shape) < 0.3] = 0.0
    idx = rng.integers(0, 2048, 700).astype(np.int64)
    cases["cfg2_small"] = codec_case("cfg2_small", f32_words(x, 8), [None, 0.7, 0.95], idx=idx,
                                     comp_len=40)

    # 4. odd vector sizes and arbitrary masks (bitval bits outside the mask included)
    rng = np.random.default_rng(7)
    for v, wb, frac in [(33, 8, 0.6), (65, 8, 0.3), (47, 4, 0.5), (100, 4, 0.9), (129, 8, 0.95)]:
        n = 257
        base = rng.integers(-2**62, 2**62, (1, v)).astype(np.int64)
        if wb == 4:
            base = base.astype(np.int32)
        m = random_mask(rng, v, wb, frac)
        noise = rng.integers(-2**62, 2**62, (n, v)).astype(np.int64)
        if wb == 4:
            noise = noise.astype(np.int32)
        data = (base & m) | (noise & ~m)
        flip = rng.random((n, v)) < 0.15
        data = np.where(flip, noise, data)
        bv = base[0] & m
        bv[::7] = base[0][::7]  # some bitvals with bits outside the mask: never compressible
        cases[f"odd_v{v}_w{wb}"] = codec_case(
            f"odd_v{v}_w{wb}", np.ascontiguousarray(data), [None], mask=m, bitval=bv,
            idx=rng.integers(0, n, 100).astype(np.int64))

    # 5. mask extremes: all ones, all zeros, MSB-set runs, alternating bits
    rng = np.random.default_rng(8)
    v, n = 64, 200
    m = np.zeros(v, dtype=np.uint64)
    m[0:8] = 0xFFFFFFFFFFFFFFFF
    m[8:16] = 0
    m[16:24] = 0xFFFF000000000000
    m[24:32] = 0xAAAAAAAAAAAAAAAA
    m[32:40] = 0x5555555555555555
    m[40:48] = 0x8000000000000001
    m[48:56] = 0x7FFFFFFFFFFFFFFE
    m[56:64] = 0x0F0F0F0F0F0F0F0F
    m = m.view(np.int64)
    noise = rng.integers(-2**63, 2**63 - 1, (n, v), dtype=np.int64)
    bv = rng.integers(-2**63, 2**63 - 1, v, dtype=np.int64) & m
    data = np.where(rng.random((n, v)) < 0.9, (noise & ~m) | bv, noise)
    cases["mask_extremes_w8"] = codec_case("mask_extremes_w8", np.ascontiguousarray(data), [None],
                                           mask=m, bitval=bv,
                                           idx=rng.integers(0, n, 64).astype(np.int64))

    # 6. large vectors (block-parallel reference path): 4096 int32 words per row
    rng = np.random.default_rng(9)
    x = rng.normal(0, 1.0, (48, 4096)).astype(np.float32)
    x = (x.view(np.uint32) & np.uint32(0xFFFFF000)).view(np.float32)
    cases["large_v4096_w4"] = codec_case("large_v4096_w4", f32_words(x, 4), [0.9],
                                         idx=rng.integers(0, 48, 20).astype(np.int64),
                                         condensed=False)

    # 7. 1- and 2-byte words: preprocess + sizes only (the codec takes 4/8-byte words)
    rng = np.random.default_rng(10)
    b8 = (rng.integers(0, 16, (500, 256)) | 0x40).astype(np.int8)
    cases["bytes_w1"] = codec_case("bytes_w1", b8, [None, 0.8])
    h16 = (rng.normal(0, 0.1, (400, 130)).astype(np.float16)).view(np.int16)
    cases["half_w2"] = codec_case("half_w2", np.ascontiguousarray(h16), [None, 0.9])



def kmeans_cases(cases):
    # 8. k-means (4-byte words): separated Gaussian mixtures
    rng = np.random.default_rng(3)
    for name, n, v, c in [("km_v64_w4", 3000, 64, 16), ("km_v16_w4", 2000, 16, 8)]:
        cent = rng.normal(0, 1, (c, v)).astype(np.float32) * 4
        lab = rng.integers(0, c, n)
        scale = (10.0 ** rng.uniform(-3, 0, c)).astype(np.float32)
        x = cent[lab] + rng.normal(0, 1, (n, v)).astype(np.float32) * scale[lab, None]
        cases[name] = kmeans_case(f32_words(x, 4), c, repeat=True)

    # tie-free k-means: C binary patterns with 2% bit noise, and the rows the reference
    # seeds its centroids with (srand(1) + random_shuffle) placed in C distinct clusters,
    # so every assignment has a unique nearest centroid and the result is deterministic
    rng = np.random.default_rng(4)
    for name, n, v, c in [("km_sep_v16_w4", 1500, 16, 8), ("km_sep_v64_w4", 1500, 64, 12)]:
        seeds = shuffle_seed_rows(n, c)
        assert 0 not in seeds[1:], "a seed row repeats row 0: pick another n"
        pat = rng.integers(-2**31, 2**31 - 1, (c, v), dtype=np.int64).astype(np.int32)
        lab = rng.integers(0, c, n)
        lab[0] = 0
        for i in range(1, c):
            lab[seeds[i]] = i
        noise = (rng.random((n, v, 32)) < 0.02)
        flips = np.zeros((n, v), dtype=np.uint32)
        for b in range(32):
            flips |= noise[:, :, b].astype(np.uint32) << np.uint32(b)
        x = (pat[lab].view(np.uint32) ^ flips).view(np.int32)
        cases[name] = kmeans_case(np.ascontiguousarray(x), c)


def save(out, cases, part):
    manifest = {}
    for k, val in cases.items():
        np.savez_compressed(os.path.join(out, f"{k}.npz"), **val)
        manifest[k] = sorted(val.keys())
    info = {"torch": torch.__version__, "gpu": torch.cuda.get_device_name(0),
            "reference_module": os.path.basename(ibp_cuda.__file__), "cases": manifest}
    with open(os.path.join(out, f"manifest_{part}.json"), "w") as f:
        json.dump(info, f, indent=1)
    print("wrote", len(cases), "cases to", out)


if __name__ == "__main__":
    main()
