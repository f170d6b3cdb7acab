"""Seeded synthetic tensor sets with the shapes and value distributions of the benchmark
workloads (no datasets are downloaded).  All generators return numpy arrays of int64 words
(the view the codec works on) plus the metadata a benchmark needs.

  plain_small        16384 x 256 fp32 N(0, 0.5^2), 5% of rows redrawn from N(0, 100^2)
                     -> int64 [16384, 128]; fetch 2048 distinct rows
  graph_features     2.4M x 128 fp32 N(0, 0.3^2), low 15 mantissa bits cleared, 30% zeros
                     -> int64 [2.4M, 64]; Zipf(s=1.1) mini-batches of 100k-400k rows
  embedding_tables   26 tables of 64 fp32, rows log-uniform in [1e4, 4e6], mixtures of 16
                     Gaussians with per-cluster scale 10^U(-3, 1) -> int64 [rows, 32]
  decoder_layer      fp16 weights of a 4096-hidden layer + one layer of a 32 x 32 x 4096 x 128
                     fp16 KV cache -> 9 sets of int64 rows of 512 words
"""
import numpy as np


def _f32_to_i64(x):
    x = np.ascontiguousarray(x, dtype=np.float32)
    return x.view(np.int64)


def plain_small(n=16384, seed=1):
    rng = np.random.default_rng(seed)
    x = rng.normal(0.0, 0.5, (n, 256)).astype(np.float32)
    k = int(round(0.05 * n))
    rows = rng.choice(n, k, replace=False)
    x[rows] = rng.normal(0.0, 100.0, (k, 256)).astype(np.float32)
    idx = rng.permutation(n)[:2048].astype(np.int64)
    return _f32_to_i64(x), idx


def graph_features(n=2_400_000, seed=2):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((n, 128), dtype=np.float32)
    x *= np.float32(0.3)
    xi = x.view(np.uint32)
    xi &= np.uint32(0xFFFF8000)
    zero = rng.random((n, 128), dtype=np.float32) < np.float32(0.3)
    x[zero] = 0.0
    del zero
    return _f32_to_i64(x)


class Zipf:
    """Finite Zipf(s) over ranks 1..n mapped to rows through a seeded permutation;
    inverse-CDF sampling with replacement."""

    def __init__(self, n, s, seed):
        rng = np.random.default_rng(seed)
        w = np.arange(1, n + 1, dtype=np.float64) ** (-s)
        self.cdf = np.cumsum(w)
        self.cdf /= self.cdf[-1]
        self.perm = rng.permutation(n).astype(np.int64)
        self.rng = np.random.default_rng(seed + 1)

    def sample(self, k):
        u = self.rng.random(k)
        ranks = np.searchsorted(self.cdf, u, side="right")
        ranks = np.minimum(ranks, len(self.cdf) - 1)
        return self.perm[ranks]


def embedding_tables(num_tables=26, dim=64, clusters=16, seed=3, max_rows=4_000_000,
                     min_rows=10_000):
    rng = np.random.default_rng(seed)
    rows = np.round(np.exp(rng.uniform(np.log(min_rows), np.log(max_rows), num_tables)))
    tables = []
    for r in rows.astype(np.int64):
        cent = rng.standard_normal((clusters, dim), dtype=np.float32)
        scale = (10.0 ** rng.uniform(-3, 1, clusters)).astype(np.float32)
        lab = rng.integers(0, clusters, r)
        x = rng.standard_normal((r, dim), dtype=np.float32)
        x *= scale[lab, None]
        x += cent[lab]
        tables.append(_f32_to_i64(x))
    return tables


def decoder_layer(seed=4, hidden=4096, inter=11008, heads=32, tokens=4096, head_dim=128):
    """The 9 tensor sets of one decoder layer, as int64 rows of 512 words (4 KiB)."""
    rng = np.random.default_rng(seed)

    def f16(shape, std):
        a = (rng.standard_normal(shape, dtype=np.float32) * np.float32(std)).astype(np.float16)
        return np.ascontiguousarray(a).view(np.int64).reshape(-1, 512)

    sets = {}
    for name in ("q", "k", "v", "o"):
        sets[name] = f16((hidden, hidden), 0.02)
    sets["gate"] = f16((hidden, inter), 0.02)
    sets["up"] = f16((hidden, inter), 0.02)
    sets["down"] = f16((inter, hidden), 0.02)
    sets["kcache"] = f16((heads, tokens, head_dim), 1.0)
    sets["vcache"] = f16((heads, tokens, head_dim), 1.0)
    return sets
