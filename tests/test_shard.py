"""Sharded fetch host logic: shard bounds, NUMA CPU lists, and the fetch + all-gather of a
batch split across two gloo ranks on CPU (each rank's fetch is the oracle's decompress, so
the gathered rows must equal the oracle's whole-batch decompress)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from invariantbitpacking_b200.shard import (ShardedFetcher, local_cpus_of_bus, parse_cpulist,
                                            shard_bounds)


def test_shard_bounds_cover_contiguously():
    for n in range(0, 40):
        for world in range(1, 6):
            spans = [shard_bounds(n, world, r) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            for (a, b), (c, _) in zip(spans, spans[1:]):
                assert b == c
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1 and sizes == sorted(sizes, reverse=True)
    with pytest.raises(ValueError):
        shard_bounds(5, 2, 2)


def test_parse_cpulist_and_sysfs(tmp_path):
    assert parse_cpulist("0-3,8,10-11\n") == [0, 1, 2, 3, 8, 10, 11]
    assert parse_cpulist("") == []
    d = tmp_path / "0000:1b:00.0"
    d.mkdir()
    (d / "local_cpulist").write_text("4-7,12\n")
    assert local_cpus_of_bus("0000:1b:00.0", str(tmp_path)) == [4, 5, 6, 7, 12]
    assert local_cpus_of_bus("0000:ff:00.0", str(tmp_path)) == []


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port):
    import oracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        rng = np.random.default_rng(12)
        f = rng.normal(0, 0.5, (3000, 32)).astype(np.float32)
        d = (f.view(np.uint32) & np.uint32(0xFFFF0000)).view(np.int64)
        m, b, _ = oracle.preprocess(d, None)
        comp, bm = oracle.compress(d, m, b)
        idx = rng.integers(0, d.shape[0], 1001)

        def fetch(ix):
            return torch.from_numpy(oracle.decompress(comp, m, b, bm, ix.numpy()))

        sf = ShardedFetcher(fetch=fetch)
        rows, (lo, hi) = sf(torch.from_numpy(idx))
        assert (lo, hi) == shard_bounds(1001, world, rank)
        assert np.array_equal(rows.numpy(), d[idx[lo:hi]])
        full = sf(torch.from_numpy(idx), gather=True)
        assert np.array_equal(full.numpy(), d[idx])
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_sharded_fetch_gathers_across_two_gloo_ranks():
    mp.spawn(_rank_main, args=(2, _free_port()), nprocs=2, join=True)
