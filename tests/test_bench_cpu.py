"""bench.py's CPU-only leg (the reference arm: the oracle's decompress on the host cores) on a
small set: it runs without a GPU and prints one JSON line with the contract's keys."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_contract_line():
    """The reference arm runs the GPU arm's exact configuration (whole-set mask sweep, whole
    mini-batches) and loads nothing of the engine: the process never maps libibp_b200.so."""
    code = ("import runpy, sys; sys.argv = ['bench.py', '--impl', 'reference', '--rows', '60000', "
            "'--steps', '2', '--warmup', '1']; runpy.run_path('bench.py', run_name='__main__'); "
            "maps = open('/proc/self/maps').read(); "
            "print('ENGINE_MAPPED' if 'libibp_b200' in maps else 'ENGINE_NOT_MAPPED')")
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                         timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = out.stdout.strip().splitlines()
    assert lines[-1] == "ENGINE_NOT_MAPPED"
    line = json.loads(lines[-2])
    for key in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0
    # the same config dict the GPU arm builds for this run (mask and sizes from the oracle,
    # which is bit-exact with the engine)
    sys.path.insert(0, ROOT)
    import bench
    import oracle
    d, _ = bench.make_workload(60000)
    m, b, _ = oracle.preprocess(d, None)
    sizes = oracle.compress_size(d, m, b)

    class A:
        rows = 60000
    want = bench.headline_config(A, 1, False, 2, int(int(sizes.sum()) / d.nbytes * bench.V),
                                 float(sizes.sum()) / d.nbytes)
    assert line["config"] == json.loads(json.dumps(want))
    assert "sample_rows_per_step" not in line["config"]


def test_cpu_core_sweep_small():
    """The host-side cores sweep (oracle decompress, uncompressed gather, oracle compress) on a
    small set: one entry per thread count, positive rates."""
    import numpy as np
    import torch
    sys.path.insert(0, ROOT)
    import bench
    import oracle
    from invariantbitpacking_b200 import synthetic
    d = synthetic.graph_features(n=3000)
    m, b, _ = oracle.preprocess(d, None)
    comp, bm = oracle.compress(d, m, b)
    rng = np.random.default_rng(1)
    batches = [rng.integers(0, 3000, 500), rng.integers(0, 3000, 900)]
    r = bench.cpu_core_sweep(torch, d, m, b, comp, bm, batches, 1.5)
    cores = sorted({1, min(8, os.cpu_count() or 1), os.cpu_count() or 1})
    assert [e["cores"] for e in r["decompress"]] == cores
    assert [e["cores"] for e in r["gather_copy"]] == cores
    assert all(e["value"] > 0 for e in r["decompress"] + r["gather_copy"])
    assert r["compress"]["value"] > 0


def test_clock_summary_keeps_samples_inside_the_region():
    """bench.Clocks.summary on fake nvidia-smi lines: only samples taken inside the timed
    region count, throttle reasons are collected from them, and a region shorter than one
    sampling period keeps the sample nearest its middle."""
    sys.path.insert(0, ROOT)
    import bench
    c = bench.Clocks(0)
    c.t0, c.t1 = 10.0, 10.1
    c.lines = [
        (9.90, "1000, 1965, 500, Not Active, Not Active, Not Active, Active"),  # before
        (10.02, "1965, 1965, 900, Not Active, Not Active, Not Active, Not Active"),
        (10.06, "1900, 1965, 950, Not Active, Not Active, Not Active, Active"),
        (10.09, "1950, 1965, 940, Not Active, Not Active, Not Active, Not Active"),
        (10.30, "700, 1965, 300, Active, Not Active, Not Active, Not Active"),  # after
        (10.31, "garbage line"),
    ]
    s = c.summary()
    assert s["samples"] == 3 and s["sm_mhz"] == 1950.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap"]
    c.t0, c.t1 = 10.03, 10.035
    s = c.summary()
    assert s["samples"] == 1 and s["sm_mhz"] == 1965.0
    c.lines = []
    assert bench.Clocks(0).summary()["samples"] == 0
