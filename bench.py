"""decompress_fetch benchmark on the graph-feature workload (2.4M x 128 fp32 rows viewed as
int64 [2.4M x 64], 1.2 GB in pinned host memory, Zipf(s=1.1) mini-batches of 100k-400k rows).

python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is one decompress_fetch of one mini-batch (cycling 100k, 200k, 400k rows).  The
line's `value` is delivered (uncompressed) GB/s of the engine call made through the C ABI
with the index array already on the device; `e2e` is the same through the public API with
the index uploaded from pinned host memory and the last output row read back each step.
`roofline` is for the row-fetch kernel: compressed bytes of the distinct rows it reads over
PCIe per launch / its CUDA-event duration, against the PCIe host-to-device copy bandwidth
measured in the same run.  `--impl reference` times the CPU restatement of the reference
algorithm on the host cores, on exactly this configuration (whole-set mask sweep, whole
mini-batches) and without loading the engine (the reference implementation has no CPU path
of its own).  Under torchrun every rank runs an independent replica on its own GPU (the path
has no exchange step); time is the max over ranks.

The default line also carries the other named configurations, each measured in the same
run: `plain_small` (16384 x 128 int64, 2048-row fetches: microseconds per call),
`served_mix` (the continuous-batching server against per-request fetches, ours and the
reference's, p50/p99 and GB/s at three arrival rates), `embedding_tables` and `decoder_layer`
(batched multi-set fetches), and `value_1000_steps` (the headline over a long region).
`--no-extras` leaves them out.

Other lines (`--config`): embedding_tables and decoder_layer (batched multi-set fetch),
served_mix (the server against per-request fetches), embedding_bag (cache-miss fetch shim),
host_rows and device_rows (whole-set decompression against the reference's GPU build), and
device_graph_features (the graph-feature batches from a device-resident copy of the set,
against the HBM roofline).
"""
import argparse
import ctypes
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

ROWS = 2_400_000
V = 64
BATCHES = (100_000, 200_000, 400_000)
METRIC = "decompress_fetch delivered GB/s (graph features, Zipf 1.1 mini-batches, host-resident)"


_REF_MODULE = None


def reference_module():
    """The reference's own extension module (its sources built for sm_100a into
    oracle/_ref/ibp_cuda*.so), loaded by explicit file path so that no other module named
    ibp_cuda on sys.path (a drop-in shim, say) can stand in for it; None when not built."""
    global _REF_MODULE
    if _REF_MODULE is None:
        import glob
        import importlib.util
        mods = glob.glob(os.path.join(REPO, "oracle", "_ref", "ibp_cuda*.so"))
        if not mods:
            return None
        spec = importlib.util.spec_from_file_location("ibp_cuda", mods[0])
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        assert os.path.samefile(mod.__file__, mods[0])
        mod.print_debug(False)
        _REF_MODULE = mod
    return _REF_MODULE


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--rows", type=int, default=ROWS)
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-reference-gpu", action="store_true")
    ap.add_argument("--config", default="graph_features",
                    choices=["graph_features", "embedding_tables", "decoder_layer",
                             "served_mix", "embedding_bag", "device_rows", "host_rows",
                             "device_graph_features"])
    ap.add_argument("--rates", default="1000,2000,5000,10000,20000,50000")
    ap.add_argument("--requests", type=int, default=300)
    ap.add_argument("--served-reps", type=int, default=3,
                    help="served_mix: rounds of each arm per rate (medians reported)")
    ap.add_argument("--shard", action="store_true",
                    help="graph_features under torchrun: split every batch across the ranks "
                         "(strong scaling) instead of one replica per rank")
    ap.add_argument("--inflight", type=int, default=4,
                    help="served_mix: batches the server keeps on the GPU")
    ap.add_argument("--no-extras", action="store_true",
                    help="graph_features: skip the other configurations' summaries")
    ap.add_argument("--server-dedup", choices=["hash", "sort"], default="hash",
                    help="served_mix: how the server's batches find repeated rows")
    ap.add_argument("--batch-mb", type=int, default=128,
                    help="served_mix: output MiB one server batch admits")
    return ap.parse_args()


def dist_setup(args):
    import torch
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    else:
        torch.cuda.set_device(0)
    return ws, rank


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, ws):
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class Clocks:
    """nvidia-smi samples (every 20 ms) during the timed region: the sampler is running, with
    its first sample in, before the region starts; samples outside the region are dropped
    (a region shorter than one period keeps the sample nearest to its middle)."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []
        self.t0 = self.t1 = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "20"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            deadline = time.monotonic() + 5.0
            while not self.lines and time.monotonic() < deadline and self.proc.poll() is None:
                time.sleep(0.005)
        except Exception:
            self.proc = None
        self.t0 = time.monotonic()
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.monotonic(), line.strip()))

    def __exit__(self, *a):
        self.t1 = time.monotonic()
        if self.proc:
            time.sleep(0.05)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        rows = []
        for t, ln in self.lines:
            p = [q.strip() for q in ln.split(",")]
            if len(p) < 7:
                continue
            try:
                rows.append((t, float(p[0]), float(p[1]), p[3:7]))
            except ValueError:
                continue
        if not rows or self.t0 is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        t1 = self.t1 if self.t1 is not None else rows[-1][0]
        inside = [r for r in rows if self.t0 <= r[0] <= t1 + 0.02]
        if not inside:
            mid = 0.5 * (self.t0 + t1)
            inside = [min(rows, key=lambda r: abs(r[0] - mid))]
        for t, clk, cmax, flags in inside:
            sm.append(clk)
            mx = max(mx, cmax)
            for nm, val in zip(names, flags):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm), "region_ms": round((t1 - self.t0) * 1e3, 1)}


def synthetic_module():
    """invariantbitpacking_b200/synthetic.py (numpy only), loaded by file path: importing it
    through the package would load the engine's library, which the reference arm must not."""
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "_ibp_synthetic", os.path.join(REPO, "invariantbitpacking_b200", "synthetic.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def make_workload(rows, seed_batches=12):
    synthetic = synthetic_module()
    d = synthetic.graph_features(n=rows)
    z = synthetic.Zipf(rows, 1.1, seed=12)
    batches = [z.sample(BATCHES[i % len(BATCHES)]) for i in range(seed_batches)]
    return d, batches


def measured_pcie_h2d(torch):
    """Pinned host -> device copy bandwidth (copy engine), best of 5, 1 GiB."""
    n = 1 << 30
    h = torch.empty(n, dtype=torch.uint8).pin_memory()
    dv = torch.empty(n, dtype=torch.uint8, device="cuda")
    best = 1e9
    for _ in range(5):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        dv.copy_(h, non_blocking=True)
        b.record()
        b.synchronize()
        best = min(best, a.elapsed_time(b))
    del h, dv
    return n / best / 1e6


def cpu_baseline(d, mask, bitval, comp, bitmask, batches, seconds):
    """The oracle's decompress (OpenMP, all host threads) on bounded samples of the same
    mini-batches: delivered GB/s on the host."""
    import oracle
    oracle.set_threads(os.cpu_count() or 1)
    t0 = time.perf_counter()
    rows = 0
    k = 0
    while time.perf_counter() - t0 < seconds:
        idx = batches[k % len(batches)][:50_000]
        out = oracle.decompress(comp, mask, bitval, bitmask, idx)
        rows += len(idx)
        k += 1
    el = time.perf_counter() - t0
    assert np.array_equal(out, d[idx])
    return {"value": rows * V * 8 / el / 1e9, "unit": "GB/s", "cores": oracle.get_threads(),
            "kind": "port",
            "sample": f"{k} mini-batch prefixes of 50k rows ({rows} rows, {el:.1f} s) "
                      "decompressed by the oracle's C restatement"}


def host_gather_copy_baseline(torch, d, batches, seconds=5.0):
    """Uncompressed host gather (numpy take into pinned staging) + one H2D copy."""
    dv = torch.empty((max(len(b) for b in batches), V), dtype=torch.int64, device="cuda")
    stage = torch.empty((max(len(b) for b in batches), V), dtype=torch.int64).pin_memory()
    sn = stage.numpy()
    t0 = time.perf_counter()
    rows, k = 0, 0
    while time.perf_counter() - t0 < seconds:
        idx = batches[k % len(batches)]
        np.take(d, idx, axis=0, out=sn[:len(idx)])
        dv[:len(idx)].copy_(stage[:len(idx)], non_blocking=True)
        torch.cuda.synchronize()
        rows += len(idx)
        k += 1
    el = time.perf_counter() - t0
    return {"value": rows * V * 8 / el / 1e9, "unit": "GB/s", "cores": 1,
            "kind": "uncompressed host gather + H2D copy", "steps": k}


def cpu_core_sweep(torch, d, mask, bitval, comp, bitmask, batches, seconds):
    """The host-side baselines at 1, 8 and all host threads (the reference's cores sweep):
    the oracle's decompress of mini-batch prefixes, the uncompressed gather (torch
    index_select into pinned staging, then one H2D copy) of whole mini-batches, and the
    oracle's compress of the first 200k rows; each sample bounded to about seconds/3."""
    import oracle
    allc = os.cpu_count() or 1
    cores = sorted({1, min(8, allc), allc})
    each = max(0.5, min(3.0, seconds / 3))
    dt = torch.from_numpy(d)
    nmax = max(len(b) for b in batches)
    stage = torch.empty((nmax, V), dtype=torch.int64)
    if torch.cuda.is_available():
        stage = stage.pin_memory()
    dv = (torch.empty((nmax, V), dtype=torch.int64, device="cuda")
          if torch.cuda.is_available() else None)
    tidx = [torch.from_numpy(b) for b in batches]
    threads0 = torch.get_num_threads()

    def timed(fn):
        t0 = time.perf_counter()
        nbytes, k = 0, 0
        while time.perf_counter() - t0 < each:
            nbytes += fn(k)
            k += 1
        return nbytes / (time.perf_counter() - t0) / 1e9

    def dec(k):
        idx = batches[k % len(batches)][:50_000]
        oracle.decompress(comp, mask, bitval, bitmask, idx)
        return len(idx) * V * 8

    def gather(k):
        idx = tidx[k % len(tidx)]
        torch.index_select(dt, 0, idx, out=stage[:len(idx)])
        if dv is not None:
            dv[:len(idx)].copy_(stage[:len(idx)], non_blocking=True)
            torch.cuda.synchronize()
        return len(idx) * V * 8

    sample = d[:200_000]

    def cmp(k):
        oracle.compress(sample, mask, bitval)
        return sample.nbytes

    out = {"unit": "GB/s", "cores_available": allc, "decompress": [], "gather_copy": []}
    try:
        for c in cores:
            oracle.set_threads(c)
            out["decompress"].append({"cores": c, "value": round(timed(dec), 3)})
            torch.set_num_threads(c)
            out["gather_copy"].append({"cores": c, "value": round(timed(gather), 3)})
        oracle.set_threads(allc)
        out["compress"] = {"cores": allc, "value": round(timed(cmp), 3),
                           "sample": "the first 200k rows (102 MB), oracle compress"}
    finally:
        torch.set_num_threads(threads0)
        oracle.set_threads(allc)
    out["what"] = ("decompress: oracle on 50k-row prefixes of the mini-batches; gather_copy: "
                   "uncompressed rows of whole mini-batches gathered on the host and copied "
                   "to the GPU; compress: oracle compress; delivered (uncompressed) GB/s")
    return out


WORKLOAD = ("graph_features: 2.4M x 128 fp32 N(0,0.3^2), 8 mantissa bits, 30% zeros -> "
            "int64 [2.4M x 64], pinned host (1.2 GB)")
BATCH_DESC = "Zipf(1.1) mini-batches cycling 100k/200k/400k rows"


def headline_config(args, ws, shard, steps, comp_len, compressed_fraction):
    """The `config` of the graph-feature line, shared by both arms so that they describe the
    same workload: the batches a K-step run cycles through, the set and its compression."""
    nrows_avg = sum(BATCHES[k % len(BATCHES)] for k in range(steps)) / steps
    return {"workload": WORKLOAD, "rows": args.rows, "vec_words": V, "batches": BATCH_DESC,
            "avg_rows_per_step": nrows_avg, "comp_len_words": int(comp_len),
            "compressed_fraction": round(float(compressed_fraction), 4),
            "mask": "preprocess threshold sweep (0.7..1.0) over the whole set",
            "l2": "inputs larger than L2 (1.2 GB host set; 51-205 MB outputs)",
            "parallelism": (f"each batch split into {ws} contiguous shards" if shard
                            else f"{ws} independent replica(s)")}


def run_reference_arm(args, ws, rank):
    """The reference algorithm on the host cores, on exactly the GPU arm's configuration: the
    mask from the threshold sweep over the whole set, the whole set compressed in place, and
    every step one whole mini-batch decompressed.  The reference implements decompress_fetch
    only as a CUDA kernel (src/decompress.cu:10-156), so its CPU implementation is the oracle's
    C restatement, run on all host threads.  Nothing of the engine is imported or loaded."""
    if rank != 0:
        return
    import oracle
    d, batches = make_workload(args.rows)
    oracle.set_threads(os.cpu_count() or 1)
    m, b, _ = oracle.preprocess(d, None)
    sizes = oracle.compress_size(d, m, b)
    comp_len = int(int(sizes.sum()) / d.nbytes * V)  # get_single_compress_len (ibp/__init__.py:22-29)
    comp, bm = oracle.compress(d, m, b)
    for k in range(len(batches)):  # the configuration is checked before it is timed
        assert np.array_equal(oracle.decompress(comp, m, b, bm, batches[k]), d[batches[k]])
    for k in range(args.warmup):
        oracle.decompress(comp, m, b, bm, batches[k % len(batches)])
    t0 = time.perf_counter()
    rows = 0
    for k in range(args.steps):
        idx = batches[k % len(batches)]
        oracle.decompress(comp, m, b, bm, idx)
        rows += len(idx)
    el = time.perf_counter() - t0
    val = rows * V * 8 / el / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": round(val, 3), "unit": "GB/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(el * 1e3 / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic",
        "config": headline_config(args, ws, args.shard and ws > 1, args.steps, comp_len,
                                  float(sizes.sum()) / d.nbytes),
        "cpu_baseline": {"value": round(val, 3), "unit": "GB/s",
                         "cores": oracle.get_threads(), "kind": "port",
                         "sample": f"{args.steps} steps, each one whole mini-batch "
                                   f"({rows} rows in all) decompressed on the host by the "
                                   "oracle's C restatement of the reference's decompress_fetch "
                                   "(which exists only as a CUDA kernel); on rank 0 only"},
        "e2e": {"value": round(val, 3), "unit": "GB/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def plain_small_summary(torch, ibp, lib, capi, pcie, steps, warmup):
    """The small plain configuration: 16384 x 256 fp32 N(0, 0.5^2) with 5% of rows redrawn
    from N(0, 100^2), viewed as int64 [16384 x 128], host-resident; preprocess at threshold
    0.9, compress_inplace, then one decompress_fetch of 2048 distinct rows per call.  A latency
    case: microseconds per call through the C ABI (index on the device) and through the
    public API (index uploaded from pinned host memory, the last row read back, synchronised
    every call), the fetch kernel's PCIe fraction, the reference's own decompress_fetch per
    call on the same rows, and the setup's outputs against the oracle."""
    import oracle
    d, idx = synthetic_module().plain_small()
    n, v = d.shape
    x = torch.from_numpy(d.copy()).pin_memory()
    m, b = ibp.preprocess(x, 0.9)
    bm = ibp.compress_inplace(x, m, b)
    torch.cuda.synchronize()
    om, ob, _ = oracle.preprocess(d, 0.9)
    ocomp, obm = oracle.compress(d, om, ob)
    sizes = oracle.compress_size(d, om, ob)
    setup_exact = bool(np.array_equal(m.cpu().numpy(), om.view(np.int64))
                       and np.array_equal(b.cpu().numpy(), ob.view(np.int64))
                       and np.array_equal(bm.cpu().numpy(), obm)
                       and np.array_equal(x.numpy(), ocomp.view(np.int64)))
    cl = int(int(sizes.sum()) / d.nbytes * v)
    ti = torch.from_numpy(idx).cuda()
    k = idx.size
    out = torch.empty((k, v), dtype=torch.int64, device="cuda")
    wsb = lib.ibp_decompress_fetch_workspace_size(k, v, 8, 1)
    ws = torch.empty(wsb, dtype=torch.uint8, device="cuda")
    st = torch.cuda.current_stream().cuda_stream

    def call():
        capi.check(lib.ibp_decompress_fetch(x.data_ptr(), n, v, 8, m.data_ptr(), b.data_ptr(),
                                            bm.data_ptr(), ti.data_ptr(), k, cl, out.data_ptr(),
                                            -1, -1, -1, ws.data_ptr(), wsb, st))
    call()
    torch.cuda.synchronize()
    exact = bool(np.array_equal(out.cpu().numpy(), d[idx]))
    for _ in range(warmup):
        call()
    torch.cuda.synchronize()
    capi.check(lib.ibp_profile_enable(steps))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        call()
    e1.record()
    e1.synchronize()
    buf = (ctypes.c_float * steps)()
    got = lib.ibp_profile_take(buf, steps)
    kms = float(np.mean(buf[:got])) if got else None
    us = e0.elapsed_time(e1) * 1e3 / steps
    comp_b = int(sizes[idx].sum())
    # public API, one synchronised call at a time (what a latency-bound caller sees)
    hidx = torch.from_numpy(idx).pin_memory()
    res = torch.empty(v, dtype=torch.int64).pin_memory()
    lat = []
    for j in range(steps + warmup):
        t0 = time.perf_counter()
        o = ibp.decompress_fetch(x, m, b, bm, torch.device("cuda"), cl,
                                 hidx.to("cuda", non_blocking=True))
        res.copy_(o[-1], non_blocking=True)
        torch.cuda.current_stream().synchronize()
        if j >= warmup:
            lat.append((time.perf_counter() - t0) * 1e6)
    ref = reference_module()
    ref_us = None
    if ref is not None:
        dev = torch.device("cuda", torch.cuda.current_device())
        ro = ref.decompress_fetch(x, m, b, bm, dev, cl, ti, None, None, None, None)
        torch.cuda.synchronize()
        ref_exact = bool(np.array_equal(ro.cpu().numpy(), d[idx]))
        for _ in range(warmup):
            ref.decompress_fetch(x, m, b, bm, dev, cl, ti, None, None, None, None)
        torch.cuda.synchronize()
        r0, r1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        r0.record()
        for _ in range(steps):
            ref.decompress_fetch(x, m, b, bm, dev, cl, ti, None, None, None, None)
        r1.record()
        r1.synchronize()
        ref_us = {"us_per_call": round(r0.elapsed_time(r1) * 1e3 / steps, 2),
                  "bit_exact": ref_exact}
    return {"workload": "plain_small: 16384 x 256 fp32 N(0,0.5^2), 5% rows N(0,100^2) -> int64 "
                        "[16384 x 128] pinned host; threshold 0.9; 2048 distinct rows per call",
            "us_per_call": round(us, 2), "GBps": round(k * v * 8 / us / 1e3, 3),
            "kernel_us": None if kms is None else round(kms * 1e3, 2),
            "kernel_pcie_frac": None if kms is None else round(comp_b / kms / 1e6 / pcie, 4),
            "e2e_api_us": {"p50": round(float(np.percentile(lat, 50)), 2),
                           "p99": round(float(np.percentile(lat, 99)), 2)},
            "compressed_fraction": round(float(sizes.sum()) / d.nbytes, 4),
            "setup_bit_exact_vs_oracle": setup_exact, "round_trip_bit_exact": exact,
            "reference_gpu": ref_us, "steps": steps}


def subconfig_line(config, extra_args, timeout):
    """Run `bench.py --config <config>` in a child process (its own CUDA context and host
    memory) and return its JSON line, or an error description."""
    cmd = [sys.executable, os.path.abspath(__file__), "--config", config] + extra_args
    try:
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout, cwd=REPO)
    except subprocess.TimeoutExpired:
        return {"error": f"timed out after {timeout} s"}
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    if r.returncode != 0 or not lines:
        return {"error": f"rc {r.returncode}: {r.stderr[-300:]}"}
    return json.loads(lines[-1])


def served_summary(line):
    """The served-vs-per-call comparison of a served_mix line, rate by rate."""
    if "rates" not in line:
        return line
    out = []
    for e in line["rates"]:
        srv, own = e["served"], e["per_request"]
        ref = e.get("per_request_reference")
        # requests per second each arm completes without a growing queue: its delivered
        # bytes per second over the mean request's output
        mean_req = e["output_GB"] * 1e9 / e["requests"]
        for arm in (srv, own, ref):
            if arm is not None:
                arm["sustainable_rate_per_s"] = round(arm["GBps"] * 1e9 / mean_req, 1)
        row = {"rate_per_s": e["rate_per_s"], "requests": e["requests"],
               "served": srv, "per_request": own,
               "served_beats_per_request": bool(srv["GBps"] >= own["GBps"]
                                                 and srv["p99_ms"] <= own["p99_ms"])}
        if ref is not None:
            row["per_request_reference"] = ref
            row["served_beats_reference_per_request"] = bool(
                srv["GBps"] >= ref["GBps"] and srv["p99_ms"] <= ref["p99_ms"])
        out.append(row)
    return {"what": "continuous-batching server (hash-claimed batches) against one "
                    "decompress_fetch per request, ours and the reference's, on Poisson "
                    "arrivals; latency = completion - scheduled arrival",
            "config": line.get("config"), "rates": out}


def batched_summary(line):
    """The batched line's headline numbers: graph-replayed batch, hashed and sorted batches,
    one call per set (ours and the reference's), and the batch kernel's PCIe fraction."""
    if "value" not in line:
        return line
    pick = lambda d: None if not isinstance(d, dict) else {  # noqa: E731
        k: d[k] for k in ("value", "ms_per_step", "error") if k in d}
    return {"metric": line["metric"], "value": line["value"], "unit": line["unit"],
            "ms_per_step": line["ms_per_step"], "steps": line["steps"],
            "hashed_batch": pick(line.get("hashed_batch")),
            "sorted_batch": pick(line.get("sorted_batch")),
            "per_call": pick(line.get("per_call")),
            "reference_per_call": pick(line.get("reference_per_call")),
            "kernel_pcie_frac": line.get("roofline", {}).get("frac"),
            "compressed_fraction": line["config"].get("compressed_fraction")}


def setup_vs_reference(torch, ibp, d, x_comp, m, b, bm, sizes):
    """preprocess (threshold sweep), get_compress_size and compress_inplace of the whole
    host-resident set, ours against the reference's (built from its sources for sm_100a),
    each timed on a fresh pinned copy of the uncompressed rows; the reference's masks, sizes,
    bitmask and compressed bytes are checked against ours bit for bit."""
    ref = reference_module()
    y = torch.from_numpy(d).pin_memory()

    def run(pre, size, comp):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        mm, bb = pre(y)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        sz = size(y, mm, bb)
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        bmk = comp(y, mm, bb)
        torch.cuda.synchronize()
        t3 = time.perf_counter()
        ms = {"preprocess_ms": round((t1 - t0) * 1e3, 2),
              "get_compress_size_ms": round((t2 - t1) * 1e3, 2),
              "compress_inplace_ms": round((t3 - t2) * 1e3, 2)}
        return ms, (mm, bb, sz, bmk)

    ours, _ = run(lambda t: ibp.preprocess(t, None), lambda t, mm, bb: ibp.get_compress_size(t, mm, bb),
                  lambda t, mm, bb: ibp.compress_inplace(t, mm, bb))
    res = {"ours": ours, "what": "whole 1.2 GB host-resident set, fresh pinned copy each, "
                                 "wall time with device synchronisation"}
    if ref is not None:
        y.copy_(torch.from_numpy(d))
        theirs, (rm, rb, rsz, rbm) = run(
            lambda t: ref.preprocess(t, None),
            lambda t, mm, bb: ref.get_compress_size(t, mm, bb, None, None),
            lambda t, mm, bb: ref.compress_inplace(t, mm, bb, None))
        res["reference"] = theirs
        res["bit_exact_vs_reference"] = bool(
            torch.equal(rm.cpu(), m.cpu()) and torch.equal(rb.cpu(), b.cpu())
            and torch.equal(rsz.cpu(), sizes.cpu()) and torch.equal(rbm.cpu(), bm.cpu())
            and torch.equal(y, x_comp))
        res["speedup"] = {k: round(theirs[k] / max(ours[k], 1e-6), 2) for k in ours}
    del y
    return res


def reference_gpu(torch, comp, m, b, bm, comp_len, batches_dev, steps):
    """The reference extension (built from its sources for sm_100a, oracle/_ref) on the same
    compressed rows, through its own positional API; None when it is not built."""
    ref = reference_module()
    if ref is None:
        return None
    dev = torch.device("cuda")
    for k in range(3):
        ref.decompress_fetch(comp, m, b, bm, dev, comp_len, batches_dev[k % len(batches_dev)],
                             None, None, None, None)
    torch.cuda.synchronize()
    a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    rows = 0
    a.record()
    for k in range(steps):
        idx = batches_dev[k % len(batches_dev)]
        ref.decompress_fetch(comp, m, b, bm, dev, comp_len, idx, None, None, None, None)
        rows += idx.shape[0]
    e.record()
    e.synchronize()
    ms = a.elapsed_time(e)
    out = ref.decompress_fetch(comp, m, b, bm, dev, comp_len, batches_dev[0], None, None, None,
                               None)
    return {"value": round(rows * V * 8 / ms / 1e6, 3), "unit": "GB/s",
            "ms_per_step": round(ms / steps, 3), "steps": steps,
            "what": "reference decompress_fetch (its sources built for sm_100a, default impl, "
                    "nblks=2*SMs) on the same compressed rows and index arrays"}, out


def run_device_graph(args):
    """The graph-feature fetch from a device-resident copy of the compressed set (the
    `--rows` rows compressed in place on the host, then copied to HBM): the same Zipf(1.1)
    mini-batches, index on the device, one decompress_fetch per step.  Reports delivered
    GB/s, the call against the HBM roofline (compressed bytes of the distinct rows read +
    every output row written, over the measured HBM copy bandwidth), the row-fetch kernel
    alone, and the reference's decompress_fetch on the same device rows."""
    import torch
    import invariantbitpacking_b200 as ibp
    from invariantbitpacking_b200 import _capi
    lib = _capi.lib
    d, batches = make_workload(args.rows)
    x = torch.from_numpy(d).pin_memory()
    m, b = ibp.preprocess(x, None)
    comp_len = ibp.get_single_compress_len(x, m, b)
    sizes = ibp.get_compress_size(x, m, b)
    bm = ibp.compress_inplace(x, m, b)
    torch.cuda.synchronize()
    sizes_np = sizes.cpu().numpy()
    xd = x.cuda()
    bdev = [torch.from_numpy(bt).cuda() for bt in batches]
    uniq = [np.unique(bt) for bt in batches]
    # per batch, outside the timed region: compressed bytes of its distinct rows, and the
    # algorithmic bytes of the whole call / of the fetch kernel alone
    comp_b = [int(sizes_np[u].sum()) for u in uniq]
    call_b = [comp_b[j] + len(batches[j]) * V * 8 for j in range(len(batches))]
    kern_b = [comp_b[j] + len(uniq[j]) * V * 8 for j in range(len(batches))]
    nmax = max(len(bt) for bt in batches)
    out = torch.empty((nmax, V), dtype=torch.int64, device="cuda")
    wsb = lib.ibp_decompress_fetch_workspace_size(nmax, V, 8, 1)
    wsp = torch.empty(wsb, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()

    def step(k):
        idx = bdev[k % len(bdev)]
        _capi.check(lib.ibp_decompress_fetch(
            xd.data_ptr(), args.rows, V, 8, m.data_ptr(), b.data_ptr(), bm.data_ptr(),
            idx.data_ptr(), idx.shape[0], comp_len, out.data_ptr(), -1, -1, -1, wsp.data_ptr(),
            wsb, stream.cuda_stream))
        return k % len(bdev)

    for k in range(len(batches)):
        step(k)
        torch.cuda.synchronize()
        assert np.array_equal(out[:len(batches[k])].cpu().numpy(), d[batches[k]]), \
            "device-resident fetch mismatch"
    for k in range(args.warmup):
        step(k)
    torch.cuda.synchronize()
    try:
        peaks = json.load(open(os.path.join(REPO, "MEASURED_PEAKS.json")))
        hbm_peak, hbm_src = float(peaks["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs"
    except Exception:
        hbm_peak, hbm_src = 6650.0, "fallback 6.65 TB/s"
    n0 = lib.ibp_kernel_launch_count()
    _capi.check(lib.ibp_profile_enable(args.steps))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    rows = call_bytes = kern_bytes = 0
    with Clocks(torch.cuda.current_device()) as clk:
        e0.record()
        for k in range(args.steps):
            j = step(k)
            rows += len(batches[j])
            call_bytes += call_b[j]
            kern_bytes += kern_b[j]
        e1.record()
        e1.synchronize()
    launches = lib.ibp_kernel_launch_count() - n0
    ms = e0.elapsed_time(e1)
    buf = (ctypes.c_float * args.steps)()
    got = lib.ibp_profile_take(buf, args.steps)
    kms = sum(buf[i] for i in range(got))
    kern_share = got / args.steps
    call_gbs = call_bytes / ms / 1e6
    kern_gbs = kern_bytes * kern_share / kms / 1e6
    ref = None
    if not args.no_reference_gpu:
        try:
            r = reference_gpu(torch, xd, m, b, bm, comp_len, bdev, args.steps)
            if r is not None:
                ref, rout = r
                torch.cuda.synchronize()
                ref["bit_exact_vs_input"] = bool(
                    np.array_equal(rout.cpu().numpy(), d[batches[0]]))
        except Exception as exc:  # reported, not fatal
            ref = {"error": repr(exc)[:200]}
    line = {
        "metric": "decompress_fetch delivered GB/s (graph features, Zipf 1.1 mini-batches, "
                  "device-resident)",
        "value": round(rows * V * 8 / ms / 1e6, 3), "unit": "GB/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
        "data": "synthetic",
        "config": {"workload": f"device_graph_features: {args.rows} graph-feature rows of 64 "
                               "int64 words compressed in place, copied to HBM",
                   "rows": args.rows, "vec_words": V, "batches": BATCH_DESC,
                   "comp_len_words": comp_len,
                   "l2": "outputs of 51-205 MB per step; the compressed set is "
                         f"{x.numel() * 8 / 1e9:.2f} GB"},
        "roofline": {"bound": "hbm", "achieved": round(call_gbs, 1), "peak": hbm_peak,
                     "unit": "GB/s", "frac": round(call_gbs / hbm_peak, 4), "traffic": None,
                     "what": "whole call: compressed bytes of the distinct rows read + every "
                             "output row written, over the call's CUDA-event time",
                     "peak_source": hbm_src},
        "fetch_kernel": {"achieved": round(kern_gbs, 1), "frac": round(kern_gbs / hbm_peak, 4),
                         "unit": "GB/s",
                         "ms_per_launch": round(kms / max(got, 1), 4),
                         "what": "row-fetch kernel alone: compressed bytes read + decoded "
                                 "bytes written of the distinct rows / its CUDA-event time"},
        "reference_gpu": ref,
        "clocks": clk.summary(),
        "gpu_launches": int(launches),
    }
    print(json.dumps(line), flush=True)


def reference_per_call(torch, sets, variants, outs, step_bytes, arrays, warmup, steps):
    """The reference's decompress_fetch (its sources built for sm_100a, oracle/_ref) called
    the way its callers do: one call per tensor set per step, on the same compressed sets,
    index arrays and output tensors; None when the reference is not built.  Every output of
    the first pass over the request variants is checked against the source rows."""
    ref = reference_module()
    if ref is None:
        return None
    # the reference compares the output tensor's device with this one, index included
    dev = torch.device("cuda", torch.cuda.current_device())

    def step(j):
        for (sid, idx, first, count), oo in zip(variants[j], outs[j]):
            x, m, b, bm, cl = sets[sid]
            ref.decompress_fetch(x, m, b, bm, dev, cl, idx, None, None, None, oo)

    exact = True
    for j in range(len(variants)):
        for oo in outs[j]:
            oo.zero_()
        step(j)
        torch.cuda.synchronize()
        for (sid, idx, first, count), oo in zip(variants[j], outs[j]):
            want = (arrays[sid][idx.cpu().numpy()] if idx is not None
                    else arrays[sid][first:first + count])
            exact = exact and bool(np.array_equal(oo.cpu().numpy(), want))
    for k in range(warmup):
        step(k % len(variants))
    torch.cuda.synchronize()
    a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    tot = 0
    a.record()
    for k in range(steps):
        j = k % len(variants)
        step(j)
        tot += step_bytes[j]
    e.record()
    e.synchronize()
    ms = a.elapsed_time(e)
    return {"value": round(tot / ms / 1e6, 3), "unit": "GB/s", "ms_per_step": round(ms / steps, 4),
            "steps": steps, "bit_exact_vs_input": exact,
            "what": f"reference decompress_fetch, one call per set per step (its sources built "
                    f"for sm_100a, default impl, nblks=2*SMs), same sets, indices and outputs"}


def kmeans_vs_reference(torch, ibp, arrays):
    """preprocess_kmeans (16 clusters) on the three smallest tables viewed as int32 rows of 64
    words, ours against the reference's (built from its sources for sm_100a; its 8-byte
    k-means indexes past a shared array, so it runs on the 4-byte view only).  The same
    initial centroid rows are used by both (the reference's std::random_shuffle with the
    process's rand() state, restated by ours); the reference's assignment races on ties, so
    the masks are not compared here (the tests pin them on tie-free data)."""
    ref = reference_module()
    if ref is None:
        return None
    small = sorted(arrays, key=lambda a: a.shape[0])[:3]
    views = [torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).pin_memory() for a in small]
    res = {"rows": [int(a.shape[0]) for a in small], "words": 64}
    for name, fn in (("ours_s", lambda t: ibp.preprocess_kmeans(t, 16, None)),
                     ("reference_s", lambda t: ref.preprocess_kmeans(t, 16, None))):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for t in views:
            fn(t)
        torch.cuda.synchronize()
        res[name] = round(time.perf_counter() - t0, 3)
    res["speedup"] = round(res["reference_s"] / max(res["ours_s"], 1e-9), 2)
    return res


def run_batched(args):
    """One batched, graph-replayed launch per step over many tensor sets, against one
    decompress_fetch call per set (the reference's calling pattern).

    embedding_tables: 26 tables of 64 fp32 (int64 [rows, 32]), rows log-uniform in
      [1e4, 4e6], per-table mask preprocess(0.9); a step fetches 2048 Zipf(1.05) rows of every
      table.  decoder_layer: the 9 tensor sets of one 4096-hidden decoder layer (fp16 weights
      and one layer of KV cache, int64 rows of 512 words), sweep masks; a step fetches all
      115,200 rows."""
    import torch
    torch.cuda.set_device(0)
    import invariantbitpacking_b200 as ibp
    from invariantbitpacking_b200 import _capi, synthetic
    from invariantbitpacking_b200.batch import BatchFetcher, SetRegistry
    lib = _capi.lib
    t0 = time.perf_counter()
    if args.config == "embedding_tables":
        arrays = synthetic.embedding_tables()
        thr = 0.9
    else:
        arrays = list(synthetic.decoder_layer().values())
        thr = None
    gen_s = time.perf_counter() - t0
    sets, sizes = [], []
    t0 = time.perf_counter()
    for a in arrays:
        x = torch.from_numpy(a).pin_memory()
        m, b = ibp.preprocess(x, thr)
        sizes.append(ibp.get_compress_size(x, m, b))
        cl = ibp.get_single_compress_len(x, m, b)  # of the uncompressed rows
        bm = ibp.compress_inplace(x, m, b)
        sets.append((x, m, b, bm, cl))
    torch.cuda.synchronize()
    prep_s = time.perf_counter() - t0
    sizes = [sz.numpy().copy() for sz in sizes]
    km = km_vs_ref = None
    if args.config == "embedding_tables":
        t0 = time.perf_counter()
        for a in arrays:
            ibp.preprocess_kmeans(torch.from_numpy(a).pin_memory(), 16, 0.9)
        km = round(time.perf_counter() - t0, 3)
        km_vs_ref = kmeans_vs_reference(torch, ibp, arrays)
    nsets = len(sets)
    v = [s[0].shape[1] for s in sets]
    variants = []
    if args.config == "embedding_tables":
        zs = [synthetic.Zipf(a.shape[0], 1.05, seed=100 + i) for i, a in enumerate(arrays)]
        for _ in range(6):
            variants.append([(i, torch.from_numpy(zs[i].sample(2048)).cuda(), 0, 2048)
                             for i in range(nsets)])
    else:
        variants.append([(i, None, 0, sets[i][0].shape[0]) for i in range(nsets)])
    outs = [[torch.empty((r[3], v[r[0]]), dtype=torch.int64, device="cuda") for r in reqs]
            for reqs in variants]
    step_bytes = [sum(r[3] * v[r[0]] * 8 for r in reqs) for reqs in variants]
    comp_bytes = []
    for reqs in variants:
        cb = 0
        for sid, idx, first, count in reqs:
            sz = sizes[sid]
            cb += int(sz[idx.cpu().numpy()].sum()) if idx is not None else int(sz[first:first + count].sum())
        comp_bytes.append(cb)
    reg = SetRegistry(sets)
    bf = BatchFetcher(reg, max_requests=nsets)
    # correctness of every variant before timing
    for reqs, o in zip(variants, outs):
        bf.fetch(reqs, o)
        torch.cuda.synchronize()
        for (sid, idx, first, count), oo in zip(reqs, o):
            want = arrays[sid][idx.cpu().numpy()] if idx is not None else arrays[sid][first:first + count]
            assert np.array_equal(oo.cpu().numpy(), want), "batched fetch mismatch"
    shape = bf.autotune(variants[0], outs[0])
    bf.capture()
    for k in range(args.warmup):
        bf.fetch(variants[k % len(variants)], outs[k % len(variants)])
    torch.cuda.synchronize()
    # each step replays the captured graph: the request-table copy and one batch kernel
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    with Clocks(torch.cuda.current_device()) as clk:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        tot = cb_tot = 0
        for k in range(args.steps):
            j = k % len(variants)
            evs[k][0].record()
            bf.fetch(variants[j], outs[j])
            evs[k][1].record()
            tot += step_bytes[j]
            cb_tot += comp_bytes[j]
        e1.record()
        e1.synchronize()
    kms = [a.elapsed_time(b) for a, b in evs]
    nk = len(kms)
    launches = args.steps  # one engine kernel per graph replay
    ms = e0.elapsed_time(e1)
    value = tot / ms / 1e6
    # per-call: one decompress_fetch per set, the reference's calling pattern
    for k in range(args.warmup):
        reqs = variants[k % len(variants)]
        for (sid, idx, first, count), oo in zip(reqs, outs[k % len(variants)]):
            x, m, b, bm, cl = sets[sid]
            ibp.decompress_fetch(x, m, b, bm, torch.device("cuda"), cl, idx, output_tensor=oo)
    torch.cuda.synchronize()
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    p0.record()
    ptot = 0
    for k in range(args.steps):
        j = k % len(variants)
        for (sid, idx, first, count), oo in zip(variants[j], outs[j]):
            x, m, b, bm, cl = sets[sid]
            ibp.decompress_fetch(x, m, b, bm, torch.device("cuda"), cl, idx, output_tensor=oo)
        ptot += step_bytes[j]
    p1.record()
    p1.synchronize()
    pms = p0.elapsed_time(p1)
    # de-duplicating batch (ibp_batch_fetch_sorted): rows of each request sorted and each
    # distinct row fetched once; outside the graphs (its shape is set per call)
    for reqs, o in zip(variants, outs):
        bf.fetch(reqs, o, dedup=True)
        torch.cuda.synchronize()
        for (sid, idx, first, count), oo in zip(reqs, o):
            want = arrays[sid][idx.cpu().numpy()] if idx is not None else arrays[sid][first:first + count]
            assert np.array_equal(oo.cpu().numpy(), want), "sorted batched fetch mismatch"
    for k in range(args.warmup):
        bf.fetch(variants[k % len(variants)], outs[k % len(variants)], dedup=True)
    torch.cuda.synchronize()
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0.record()
    stot = 0
    for k in range(args.steps):
        j = k % len(variants)
        bf.fetch(variants[j], outs[j], dedup=True)
        stot += step_bytes[j]
    s1.record()
    s1.synchronize()
    sms = s0.elapsed_time(s1)
    # de-duplicating batch by hash claims inside the fetch (ibp_batch_fetch_hashed)
    for reqs, o in zip(variants, outs):
        bf.fetch(reqs, o, dedup="hash")
        torch.cuda.synchronize()
        for (sid, idx, first, count), oo in zip(reqs, o):
            want = arrays[sid][idx.cpu().numpy()] if idx is not None else arrays[sid][first:first + count]
            assert np.array_equal(oo.cpu().numpy(), want), "hashed batched fetch mismatch"
    for k in range(args.warmup):
        bf.fetch(variants[k % len(variants)], outs[k % len(variants)], dedup="hash")
    torch.cuda.synchronize()
    h0, h1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    h0.record()
    htot = 0
    for k in range(args.steps):
        j = k % len(variants)
        bf.fetch(variants[j], outs[j], dedup="hash")
        htot += step_bytes[j]
    h1.record()
    h1.synchronize()
    hms = h0.elapsed_time(h1)
    ref_steps = min(args.steps, 100)
    try:
        ref_call = reference_per_call(torch, sets, variants, outs, step_bytes, arrays,
                                      args.warmup, ref_steps)
    except Exception as exc:  # reported, not fatal
        ref_call = {"error": repr(exc)[:200]}
    pcie = measured_pcie_h2d(torch)
    kavg = sum(kms) / max(len(kms), 1)
    ach = (sum(comp_bytes[k % len(variants)] for k in range(nk)) / sum(kms) / 1e6) if kms else None
    name = {"embedding_tables": "26 embedding tables x 2048 Zipf(1.05) rows",
            "decoder_layer": "one decoder layer: 9 tensor sets, 115,200 rows of 4 KiB"}[args.config]
    line = {
        "metric": f"batched decompress_fetch delivered GB/s ({name}, host-resident)",
        "value": round(value, 3), "unit": "GB/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
        "data": "synthetic",
        "config": {"workload": args.config, "sets": nsets,
                   "rows_per_set": [int(s[0].shape[0]) for s in sets],
                   "delivered_bytes_per_step": step_bytes[0],
                   "compressed_fraction": round(sum(int(z.sum()) for z in sizes) /
                                                sum(a.nbytes for a in arrays), 4),
                   "launch_shape": shape, "graph": True,
                   "setup_s": {"generate": round(gen_s, 2), "preprocess_compress": round(prep_s, 2),
                               "preprocess_kmeans_all_tables": km},
                   "preprocess_kmeans_vs_reference": km_vs_ref},
        "per_call": {"value": round(ptot / pms / 1e6, 3), "unit": "GB/s",
                     "ms_per_step": round(pms / args.steps, 4),
                     "what": f"{nsets} ibp.decompress_fetch calls per step, one per set"},
        "reference_per_call": ref_call,
        "sorted_batch": {"value": round(stot / sms / 1e6, 3), "unit": "GB/s",
                         "ms_per_step": round(sms / args.steps, 4),
                         "what": "one ibp_batch_fetch_sorted per step (device sort, repeats "
                                 "fetched once; not graph-captured)"},
        "hashed_batch": {"value": round(htot / hms / 1e6, 3), "unit": "GB/s",
                         "ms_per_step": round(hms / args.steps, 4),
                         "what": "one ibp_batch_fetch_hashed per step (hash claims inside the "
                                 "fetch, repeats copied on the device; not graph-captured)"},
        "roofline": {"bound": "pcie", "achieved": None if ach is None else round(ach, 3),
                     "peak": round(pcie, 3), "unit": "GB/s",
                     "frac": None if ach is None else round(ach / pcie, 4), "traffic": None,
                     "what": "batch_fetch_kernel: compressed bytes of the fetched rows / CUDA-"
                             "event time of each graph replay (a 4 KB table copy + the kernel)",
                     "kernel_ms_per_launch": round(kavg, 4),
                     "peak_source": "pinned host->device copy measured in this run"},
        "clocks": clk.summary(),
        "gpu_launches": int(launches),
    }
    print(json.dumps(line), flush=True)


def run_embedding_bag(args):
    """The DLRM caller (ColossalAI CachedEmbeddingBag with IBP, tests/dlrm_comp_merged.py):
    the 26 embedding tables merged into one host-resident table with a GPU cache of 1% of
    its rows; a step looks up 2048 uniformly drawn rows of every table (bags of one row, as
    the reference's harness draws them) through the cached embedding bag, compressed
    (comp=True) against the same bag over the raw table (comp=False, an all-zero bitmask: a
    zero-copy gather), both fetched by this engine."""
    import torch
    torch.cuda.set_device(0)
    from invariantbitpacking_b200 import synthetic, _capi
    from invariantbitpacking_b200.callers import CompressedEmbeddingBag
    lib = _capi.lib
    tables = synthetic.embedding_tables()
    starts = np.concatenate([[0], np.cumsum([t.shape[0] for t in tables])[:-1]])
    merged = torch.from_numpy(np.concatenate(tables).view(np.float32))
    rows, dim = merged.shape
    del tables
    sizes = np.diff(np.concatenate([starts, [rows]]))
    per = 2048
    rng = np.random.default_rng(200)
    batches = []
    for _ in range(64):
        idx = np.concatenate([starts[i] + rng.integers(0, sizes[i], per)
                              for i in range(len(sizes))])
        batches.append(torch.from_numpy(idx).cuda())
    offsets = torch.arange(per * len(sizes), device="cuda")
    res = {}
    for comp in (True, False):
        t0 = time.perf_counter()
        bag = CompressedEmbeddingBag(rows, dim, cache_ratio=0.01, _weight=merged, comp=comp)
        setup = time.perf_counter() - t0
        full_check = merged[batches[0].cpu()].cuda()
        got = bag(batches[0], offsets)
        torch.cuda.synchronize()
        assert torch.equal(got, full_check), "embedding bag mismatch"
        for k in range(args.warmup):
            bag(batches[k % len(batches)], offsets)
        torch.cuda.synchronize()
        for key in bag.stats:
            bag.stats[key] = 0
        l0 = lib.ibp_kernel_launch_count()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for k in range(args.steps):
            bag(batches[k % len(batches)], offsets)
        e1.record()
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        st = dict(bag.stats)
        res[comp] = {"ms_per_step": round(ms / args.steps, 4),
                     "lookups_per_s": round(st["lookups"] / ms * 1e3, 1),
                     "fetched_GBps": round(st["fetched_bytes"] / ms / 1e6, 3),
                     "hit_rate": round(st["hits"] / max(st["lookups"], 1), 4),
                     "setup_s": round(setup, 2),
                     "launches": int(lib.ibp_kernel_launch_count() - l0)}
        if comp:
            res["compressed_fraction"] = round(
                float(bag.comp_len) / bag.words, 4) if bag.comp_len else None
        del bag
        torch.cuda.empty_cache()
    line = {
        "metric": "cached embedding bag over a host-resident table: distinct rows fetched per "
                  "second into the GPU cache (GB/s), compressed vs raw",
        "value": res[True]["fetched_GBps"], "unit": "GB/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": res[True]["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": "embedding_bag: 26 tables merged, "
                               f"{rows} x {dim} fp32 pinned host, GPU cache 1% of rows, "
                               f"{per} uniform lookups per table per step, bags of one row",
                   "compressed_len_fraction": res.get("compressed_fraction")},
        "compressed": res[True], "raw": res[False],
        "gpu_launches": res[True]["launches"],
    }
    print(json.dumps(line), flush=True)


def run_rows(args, where):
    """The reference's whole-set decompression benchmarks: tests/dev_decomp_thput.py
    (where="device": rows in HBM, 256/1024/4096-byte rows, against a clone of the raw rows)
    and tests/decompression_thput.py (where="host": rows in pinned host memory, 256 B-16 KiB
    rows, against a plain host-to-device copy of the raw rows).  100,000 int32 rows, all
    zeros, compressed under random masks that make a target share of the bits invariant
    (12.5% .. 97%), decompressed whole (no index) onto the GPU.  Our decompress_fetch against
    the reference's own (built from its sources for sm_100a, its scripts' launch settings,
    impl 0) and the raw copy; CUDA-event times, every output checked bit for bit."""
    import torch
    torch.cuda.set_device(0)
    import invariantbitpacking_b200 as ibp
    from invariantbitpacking_b200 import _capi
    lib = _capi.lib
    ref = reference_module()
    num = 100_000
    rng = np.random.default_rng(11)
    host = where == "host"
    sizes_b = (256, 1024, 4096, 16384) if host else (256, 1024, 4096)
    reps = max(3, min(args.steps, 5 if host else 20))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    dev = torch.device("cuda")

    def timed(fn):
        for _ in range(max(args.warmup, 1)):
            fn()
        torch.cuda.synchronize()
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        e1.synchronize()
        return e0.elapsed_time(e1) / reps

    def place(t):
        return t.pin_memory() if host else t.to(dev)

    points, launches = [], 0
    with Clocks(torch.cuda.current_device()) as clk:
        for size in sizes_b:
            v = size // 4
            t = place(torch.zeros((num, v), dtype=torch.int32))
            copy_ms = timed((lambda: t.to(dev, non_blocking=True)) if host else (lambda: t.clone()))
            want = torch.zeros((num, v), dtype=torch.int32, device=dev)
            for rate in (0.125, 0.25, 0.5, 0.75, 0.9, 0.95, 0.97):
                # mask bits drawn at random until rate x row bits (+ V + 1) are set; bitval
                # row 0 (zeros), as the reference scripts make them
                bits = 32 * v
                sel = rng.permutation(bits)[:min(bits, int(rate * bits) + v + 1)]
                mw = np.zeros(v, np.uint32)
                np.bitwise_or.at(mw, sel // 32, np.uint32(1) << (sel % 32).astype(np.uint32))
                mask = torch.from_numpy(mw.view(np.int32)).to(dev)
                bitval = torch.zeros(v, dtype=torch.int32, device=dev)
                x = t.clone()
                x = x.pin_memory() if host else x
                szs = ibp.get_compress_size(x, mask, bitval)
                torch.cuda.synchronize()  # host-resident sizes are written asynchronously
                comp_frac = float(szs.sum()) / (num * size)
                cl = ibp.get_single_compress_len(x, mask, bitval)  # before compressing
                bm = ibp.compress_inplace(x, mask, bitval)
                out = torch.empty((num, v), dtype=torch.int32, device=dev)
                l0 = lib.ibp_kernel_launch_count()
                ours = timed(lambda: ibp.decompress_fetch(x, mask, bitval, bm, dev, cl, None,
                                                          output_tensor=out))
                launches += lib.ibp_kernel_launch_count() - l0
                assert torch.equal(out, want), "rows mismatch"
                pt = {"row_bytes": size, "invariant_target": rate,
                      "compressed_fraction": round(comp_frac, 4),
                      "ours_us": round(ours * 1e3, 1), "copy_us": round(copy_ms * 1e3, 1),
                      "ours_GBps": round(num * size / ours / 1e6, 1),
                      "speedup_vs_copy": round(copy_ms / ours, 2)}
                del x
                if ref is not None:
                    xr = t.clone()
                    xr = xr.pin_memory() if host else xr
                    bmr = ref.compress_inplace(xr, mask, bitval, None)
                    holder = {}
                    nb, nt = (None, None) if host else (320, 512)

                    def rcall():
                        holder["o"] = ref.decompress_fetch(xr, mask, bitval, bmr, dev, cl, None,
                                                           nb, nt, 0, None)
                    rt = timed(rcall)
                    pt["ref_us"] = round(rt * 1e3, 1)
                    pt["ref_exact"] = bool(torch.equal(holder["o"], want))
                    pt["speedup_vs_ref"] = round(rt / ours, 2)
                    del xr, holder
                points.append(pt)
                del out
            del t, want
            torch.cuda.empty_cache()
    head = [p for p in points if p["row_bytes"] == 1024 and p["invariant_target"] == 0.5][0]
    sp = [p["speedup_vs_ref"] for p in points if "speedup_vs_ref" in p]
    name = ("device-resident decompress delivered GB/s (100k rows in HBM, no index; reference "
            "dev_decomp_thput pattern)" if not host else
            "host-resident decompress delivered GB/s (100k pinned rows, no index; reference "
            "decompression_thput pattern)")
    line = {
        "metric": name, "value": head["ours_GBps"], "unit": "GB/s", "n_gpus": 1,
        "steps": reps, "warmup": args.warmup, "ms_per_step": round(head["ours_us"] / 1e3, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic",
        "config": {"workload": f"{where}_rows: 100,000 zero int32 rows of "
                               f"{'/'.join(str(z) for z in sizes_b)} B "
                               f"{'pinned on the host' if host else 'in HBM'}, random masks "
                               "at 7 invariant-bit targets; line value = 1024 B rows at 50%",
                   "l2": "sets of 25 MB-1.6 GB; 1024 B rows and up exceed L2"},
        "speedup_vs_ref": {"min": min(sp) if sp else None,
                           "geomean": round(float(np.exp(np.mean(np.log(sp)))), 2)
                           if sp else None, "max": max(sp) if sp else None},
        "points": points,
        "clocks": clk.summary(),
        "gpu_launches": int(launches),
    }
    print(json.dumps(line), flush=True)


def served_sets(torch, ibp):
    """8 host-pinned sets from the plain/graph/embedding generators, rows re-shaped to
    V in {64, 128, 256, 512} int64 words, ~384 MB each."""
    from invariantbitpacking_b200 import synthetic
    plan = [("graph", 64), ("plain", 128), ("embed", 256), ("graph", 512),
            ("plain", 64), ("embed", 128), ("graph", 256), ("plain", 512)]
    target = 384 << 20
    srcs, sets = [], []
    for i, (gen, v) in enumerate(plan):
        rows = target // (v * 8)
        if gen == "graph":
            f = synthetic.graph_features(n=rows * v // 64, seed=40 + i).view(np.float32)
        elif gen == "plain":
            f = synthetic.plain_small(n=rows * v // 128, seed=40 + i)[0].view(np.float32)
        else:
            f = np.concatenate([t.view(np.float32).reshape(-1) for t in synthetic.embedding_tables(
                num_tables=(2 * v + 63) // 64, seed=40 + i, min_rows=rows, max_rows=rows + 1)])
        d = np.ascontiguousarray(f.reshape(-1)[:rows * v * 2]).view(np.int64).reshape(rows, v)
        x = torch.from_numpy(d).pin_memory()
        m, b = ibp.preprocess(x, None)
        cl = ibp.get_single_compress_len(x, m, b)  # of the uncompressed rows
        bm = ibp.compress_inplace(x, m, b)
        srcs.append(d)
        sets.append((x, m, b, bm, cl))
    return srcs, sets


def run_served(args):
    """Poisson request streams over 8 sets; requests of log-uniform [256, 262144] rows with
    uniform row numbers; the continuous-batching server (40 GB output arena) against one
    plain decompress_fetch per request in arrival order, ours and (when its build is present)
    the reference's.  Latency = completion time minus scheduled arrival time."""
    import threading
    import torch
    torch.cuda.set_device(0)
    import invariantbitpacking_b200 as ibp
    from invariantbitpacking_b200.batch import SetRegistry
    from invariantbitpacking_b200.serve import Server
    t0 = time.perf_counter()
    srcs, sets = served_sets(torch, ibp)
    setup_s = time.perf_counter() - t0
    reg = SetRegistry(sets)
    srv = Server(reg, arena_bytes=40 << 30, index_capacity=1 << 26, max_batch=256,
                 max_inflight=args.inflight, batch_bytes=args.batch_mb << 20)
    srv.set_dedup(args.server_dedup)
    ref = reference_module()  # the reference's decompress_fetch as a third arm (or None)
    rates = [float(r) for r in args.rates.split(",")]
    nreq = args.requests
    rng = np.random.default_rng(7)
    # warm-up: every set once through the server and the per-request path (module loads)
    for i, (x, m, b, bm, cl) in enumerate(sets):
        rr = rng.integers(0, srcs[i].shape[0], 4096).astype(np.int64)
        rid = srv.submit(i, rr)
        srv.wait(rid, 600000)
        srv.release(rid)
        ibp.decompress_fetch(x, m, b, bm, torch.device("cuda"), cl,
                             torch.from_numpy(rr).cuda())
    torch.cuda.synchronize()
    results = []
    checked = 0
    for rate in rates:
        gaps = rng.exponential(1.0 / rate, nreq)
        arrive = np.cumsum(gaps)
        sids = rng.integers(0, len(sets), nreq)
        counts = np.exp(rng.uniform(np.log(256), np.log(262144), nreq)).astype(np.int64)
        rows = [rng.integers(0, srcs[s].shape[0], c).astype(np.int64) for s, c in zip(sids, counts)]
        total_bytes = int(sum(c * srcs[s].shape[1] * 8 for s, c in zip(sids, counts)))

        # ---- served: a client thread submits on schedule, the main thread waits/releases
        def served_run(check):
            nonlocal checked
            ids = [None] * nreq
            base = time.monotonic() + 0.05

            def client():
                for j in range(nreq):
                    t = base + arrive[j]
                    while time.monotonic() < t:
                        pass
                    while True:
                        try:
                            ids[j] = srv.submit(int(sids[j]), rows[j])
                            break
                        except RuntimeError:
                            time.sleep(0.0002)

            th = threading.Thread(target=client)
            th.start()
            lat = []
            t_last = 0.0
            kept = {}
            for j in range(nreq):
                while ids[j] is None:
                    time.sleep(0.0001)
                out, tm = srv.wait(ids[j], 600000)
                if check and j % 37 == 0:
                    kept[j] = out.clone()  # checked after the run: no host work while timing
                srv.release(ids[j])
                lat.append(tm[2] / 1e6 - (base + arrive[j]))
                t_last = max(t_last, tm[2] / 1e6)
            th.join()
            for j, out in kept.items():
                assert np.array_equal(out.cpu().numpy(), srcs[sids[j]][rows[j]]), "served mismatch"
                checked += 1
            del kept
            return {"p50_ms": round(float(np.percentile(lat, 50)) * 1e3, 3),
                    "p99_ms": round(float(np.percentile(lat, 99)) * 1e3, 3),
                    "GBps": round(total_bytes / (t_last - base) / 1e9, 3)}

        # ---- per request: one plain decompress_fetch per request, in arrival order (ours,
        # and the reference's own when its build is present)
        rows_pin = [torch.from_numpy(r).pin_memory() for r in rows]

        def per_request(fetch):
            evs = [None] * nreq
            done_t = [0.0] * nreq
            base2 = time.monotonic() + 0.05

            def reaper():
                for j in range(nreq):
                    while evs[j] is None:
                        time.sleep(0.00005)
                    evs[j].synchronize()
                    done_t[j] = time.monotonic()

            rt = threading.Thread(target=reaper)
            rt.start()
            outs = [None] * nreq
            for j in range(nreq):
                t = base2 + arrive[j]
                while time.monotonic() < t:
                    pass
                x, m, b, bm, cl = sets[sids[j]]
                idx = rows_pin[j].to("cuda", non_blocking=True)
                outs[j] = fetch(x, m, b, bm, cl, idx)
                ev = torch.cuda.Event()
                ev.record()
                evs[j] = ev
                if j >= 2:
                    outs[j - 2] = None  # let the caching allocator reuse finished outputs
            rt.join()
            lat2 = [done_t[j] - (base2 + arrive[j]) for j in range(nreq)]
            del outs
            torch.cuda.empty_cache()
            return {"p50_ms": round(float(np.percentile(lat2, 50)) * 1e3, 3),
                    "p99_ms": round(float(np.percentile(lat2, 99)) * 1e3, 3),
                    "GBps": round(total_bytes / (max(done_t) - base2) / 1e9, 3)}

        dev = torch.device("cuda")
        arms = {"served": lambda rep: served_run(rep == 0),
                "per_request": lambda rep: per_request(
                    lambda x, m, b, bm, cl, idx: ibp.decompress_fetch(x, m, b, bm, dev, cl, idx))}
        if ref is not None:
            arms["per_request_reference"] = lambda rep: per_request(
                lambda x, m, b, bm, cl, idx:
                ref.decompress_fetch(x, m, b, bm, dev, cl, idx, None, None, None, None))
        # the arms take turns, `reps` rounds in a rotating order, so a drift of the shared
        # box's host or link speed during the run falls on every arm alike; each metric is
        # the median over the rounds
        names = list(arms)
        runs = {a: [] for a in names}
        for rep in range(args.served_reps):
            order = names[rep % len(names):] + names[:rep % len(names)]
            for a in order:
                runs[a].append(arms[a](rep))
        entry = {"rate_per_s": rate, "requests": nreq,
                 "output_GB": round(total_bytes / 1e9, 2), "rounds": args.served_reps}
        for a in names:
            entry[a] = {k: round(float(np.median([r[k] for r in runs[a]])), 3)
                        for k in ("p50_ms", "p99_ms", "GBps")}
            entry[a]["rounds_GBps"] = [r["GBps"] for r in runs[a]]
        results.append(entry)
    st = srv.stats()
    srv.close()
    head = results[0]
    line = {
        "metric": "served mix: continuous-batching server vs per-request decompress_fetch "
                  "(p50/p99 latency, delivered GB/s)",
        "value": head["served"]["GBps"], "unit": "GB/s", "n_gpus": 1, "steps": nreq,
        "warmup": 0, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "int64", "data": "synthetic",
        "config": {"workload": "served_mix: 8 pinned sets (~384 MB each), V in {64,128,256,512}, "
                               "Poisson arrivals, log-uniform [256, 262144] rows per request",
                   "arena_GB": 40, "max_batch": 256, "max_inflight": args.inflight,
                   "server_dedup": args.server_dedup,
                   "batch_MiB": args.batch_mb,
                   "setup_s": round(setup_s, 1), "batches": st["batches"],
                   "bit_exact_checked_requests": checked},
        "rates": results,
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.config == "served_mix":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the served configuration "
                              "compares against per-request fetches in the same line"}))
            return
        run_served(args)
        return
    if args.config in ("device_rows", "host_rows"):
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the whole-set configurations "
                              "time the reference's GPU build in the same line"}))
            return
        run_rows(args, args.config.split("_")[0])
        return
    if args.config == "device_graph_features":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the device-resident "
                              "configuration times the reference's GPU build in the same line"}))
            return
        run_device_graph(args)
        return
    if args.config == "embedding_bag":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the embedding-bag "
                              "configuration compares compressed and raw tables in one line"}))
            return
        run_embedding_bag(args)
        return
    if args.config != "graph_features":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the batched configurations "
                              "are measured against per-call fetches in the same line"}))
            return
        run_batched(args)
        return
    if args.impl == "reference":
        ws = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        run_reference_arm(args, ws, rank)
        return
    import torch
    ws, rank = dist_setup(args)
    import invariantbitpacking_b200 as ibp
    from invariantbitpacking_b200 import _capi
    lib = _capi.lib

    d, batches = make_workload(args.rows)
    full_rows = [len(bt) for bt in batches]
    shard = args.shard and ws > 1
    if shard:  # this rank's contiguous shard of every batch (rows are independent)
        from invariantbitpacking_b200.shard import shard_bounds
        batches = [bt[slice(*shard_bounds(len(bt), ws, rank))] for bt in batches]
    x = torch.from_numpy(d).pin_memory()
    m, b = ibp.preprocess(x, None)
    comp_len = ibp.get_single_compress_len(x, m, b)
    sizes = ibp.get_compress_size(x, m, b)
    torch.cuda.synchronize()
    sizes_np = sizes.numpy().copy()
    bm = ibp.compress_inplace(x, m, b)
    torch.cuda.synchronize()
    batches_dev = [torch.from_numpy(bt).cuda() for bt in batches]
    batches_host = [torch.from_numpy(bt).pin_memory() for bt in batches]
    uniq_bytes = [int(sizes_np[np.unique(bt)].sum()) for bt in batches]
    uniq_rows = [len(np.unique(bt)) for bt in batches]
    all_bytes = [int(sizes_np[bt].sum()) for bt in batches]
    maxb = max(len(bt) for bt in batches)
    out = torch.empty((maxb, V), dtype=torch.int64, device="cuda")
    wsb = lib.ibp_decompress_fetch_workspace_size(maxb, V, 8, 1)
    wsp = torch.empty(wsb, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()

    def engine_step(k, src=None):
        idx = batches_dev[k % len(batches_dev)]
        _capi.check(lib.ibp_decompress_fetch(
            (src if src is not None else x).data_ptr(), args.rows, V, 8, m.data_ptr(),
            b.data_ptr(), bm.data_ptr(), idx.data_ptr(), idx.shape[0], comp_len,
            out.data_ptr(), -1, -1, -1, wsp.data_ptr(), wsb, stream.cuda_stream))
        return idx.shape[0]

    def kernel_ms(n):
        buf = (ctypes.c_float * n)()
        got = lib.ibp_profile_take(buf, n)
        return [float(buf[i]) for i in range(got)]

    # correctness of the timed configuration before timing it
    for k in range(len(batches)):
        n = engine_step(k)
        torch.cuda.synchronize()
        assert np.array_equal(out[:n].cpu().numpy(), d[batches[k]]), "bench batch mismatch"
    for k in range(args.warmup):
        engine_step(k)
    torch.cuda.synchronize()

    # ---- value: engine call, index resident on the device
    barrier(ws)
    torch.cuda.synchronize()
    l0 = lib.ibp_kernel_launch_count()
    _capi.check(lib.ibp_profile_enable(args.steps))
    with Clocks(torch.cuda.current_device()) as clk:
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record()
        rows = 0
        for k in range(args.steps):
            rows += engine_step(k)
        s1.record()
        s1.synchronize()
    launches = lib.ibp_kernel_launch_count() - l0
    kms = kernel_ms(args.steps)
    ms = max_over_ranks(s0.elapsed_time(s1), ws)
    barrier(ws)
    # the same measurement over a long region (1000 steps), with its own clock samples
    LONG = 1000
    with Clocks(torch.cuda.current_device()) as lclk:
        l0e, l1e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0e.record()
        lrows = 0
        for k in range(LONG):
            lrows += engine_step(k)
        l1e.record()
        l1e.synchronize()
    lms = max_over_ranks(l0e.elapsed_time(l1e), ws)
    barrier(ws)
    long_run = {"steps": LONG, "value": round((lrows * ws if not shard else sum(
                    full_rows[k % len(batches)] for k in range(LONG))) * V * 8 / lms / 1e6, 3),
                "ms_per_step": round(lms / LONG, 4), "clocks": lclk.summary()}
    job_rows = (sum(full_rows[k % len(batches)] for k in range(args.steps)) if shard
                else rows * ws)
    value = job_rows * V * 8 / ms / 1e6  # GB/s, all ranks
    kuniq = [uniq_bytes[k % len(batches)] for k in range(args.steps)]
    kall = [all_bytes[k % len(batches)] for k in range(args.steps)]
    fetch_gbs = sum(kuniq) / sum(kms) / 1e6
    fetch_gbs_dups = sum(kall) / sum(kms) / 1e6
    # host-memory bytes the kernel reads per launch: the ncu capture of this kernel on the
    # 400k-row batch read 714,969 sysmem sectors for its 79,441 distinct rows (9.0 sectors,
    # 288 bytes, per row: the 264-byte rows are read as whole 32-byte sectors)
    traffic = 288.0 * sum(uniq_rows[k % len(batches)] for k in range(args.steps)) / args.steps

    # ---- e2e: public API, index uploaded per step, last row read back per step
    # a loader's pipeline: the next step's index uploads on a copy stream while this step's
    # fetch runs, and the host stays at most AHEAD steps ahead of the GPU (a bounded prefetch
    # queue, which also keeps the allocator from growing a pool of pending index buffers);
    # every upload and every read-back is inside the timed region
    AHEAD = 4
    res_host = torch.empty(V, dtype=torch.int64).pin_memory()
    cur_stream = torch.cuda.current_stream()
    copy_stream = torch.cuda.Stream()

    def upload(k):
        hi = batches_host[k % len(batches)]
        with torch.cuda.stream(copy_stream):
            t = hi.to("cuda", non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(copy_stream)
        return hi, t, ev

    def pipeline(nsteps, start):
        from collections import deque
        done = deque()
        rows_p = nbytes_h2d = nbytes_d2h = 0
        start.record()
        copy_stream.wait_event(start)
        nxt = upload(0)
        for k in range(nsteps):
            hi, idx, ev = nxt
            cur_stream.wait_event(ev)
            idx.record_stream(cur_stream)
            if k + 1 < nsteps:
                nxt = upload(k + 1)
            o = ibp.decompress_fetch(x, m, b, bm, torch.device("cuda"), comp_len, idx)
            res_host.copy_(o[-1], non_blocking=True)
            fin = torch.cuda.Event()
            fin.record(cur_stream)
            done.append(fin)
            if len(done) > AHEAD:
                done.popleft().synchronize()
            rows_p += hi.shape[0]
            nbytes_h2d += hi.numel() * 8
            nbytes_d2h += V * 8
        return rows_p, nbytes_h2d, nbytes_d2h

    pipeline(max(args.warmup, AHEAD + 1), torch.cuda.Event())
    torch.cuda.synchronize()
    barrier(ws)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    rows_e, h2d, d2h = pipeline(args.steps, e0)
    e1.record()
    e1.synchronize()
    ems = max_over_ranks(e0.elapsed_time(e1), ws)
    e2e = job_rows * V * 8 / ems / 1e6

    pcie = measured_pcie_h2d(torch)

    # ---- the ceiling of the fetch kernel's access pattern: the same distinct rows of every
    # batch, in the order the hashed fetch reads them (first occurrence), read as the kernel's
    # first read (the comp_len hint rounded up to 32-byte sectors) and not decoded
    first_bytes = -(-comp_len * 8 // 32) * 32
    heads_dev = []
    for bt in batches:
        _, first = np.unique(bt, return_index=True)
        heads_dev.append(torch.from_numpy(bt[np.sort(first)].astype(np.int64)).cuda())
    for k in range(len(batches)):
        hd = heads_dev[k]
        _capi.check(lib.ibp_read_rows_probe(x.data_ptr(), V * 8, hd.data_ptr(), hd.shape[0],
                                            first_bytes, wsp.data_ptr(), wsb, stream.cuda_stream))
    _capi.check(lib.ibp_profile_enable(len(batches)))
    for k in range(len(batches)):
        hd = heads_dev[k]
        _capi.check(lib.ibp_read_rows_probe(x.data_ptr(), V * 8, hd.data_ptr(), hd.shape[0],
                                            first_bytes, wsp.data_ptr(), wsb, stream.cuda_stream))
    pms = kernel_ms(len(batches))
    pat_gbs = sum(uniq_bytes) / sum(pms) / 1e6
    pattern = {"achieved": round(pat_gbs, 3), "frac_of_copy": round(pat_gbs / pcie, 4),
               "read_bytes_per_row": int(first_bytes),
               "kernel_frac_of_pattern": None,
               "what": "ibp_read_rows_probe: the distinct rows of each batch, in first-occurrence "
                       "order, read as the fetch kernel's first read and not decoded; "
                       "compressed bytes of those rows / probe CUDA-event time"}
    del heads_dev

    # ---- the same fetches of the uncompressed set (impl 2: plain zero-copy gather, same sort
    # and repeat fill): what the batch costs without compression
    raw = torch.from_numpy(d).pin_memory()

    def raw_step(k):
        idx = batches_dev[k % len(batches_dev)]
        _capi.check(lib.ibp_decompress_fetch(
            raw.data_ptr(), args.rows, V, 8, None, None, None, idx.data_ptr(), idx.shape[0],
            -1, out.data_ptr(), -1, -1, 2, wsp.data_ptr(), wsb, stream.cuda_stream))
        return idx.shape[0]

    for k in range(args.warmup):
        raw_step(k)
    torch.cuda.synchronize()
    r0, r1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    r0.record()
    rrows = 0
    for k in range(args.steps):
        rrows += raw_step(k)
    r1.record()
    r1.synchronize()
    raw_gbs = rrows * V * 8 / r0.elapsed_time(r1) / 1e6
    del raw

    # ---- the same fetches from the condensed layout (compress_condensed's rows packed back
    # to back with inclusive byte offsets): each row is read once, at its exact length
    xw = x.numpy()
    cond = torch.from_numpy(xw[np.arange(V)[None, :] < (sizes_np // 8)[:, None]]).pin_memory()
    offs = torch.from_numpy(np.cumsum(sizes_np).astype(np.int64)).cuda()

    def cond_step(k):
        idx = batches_dev[k % len(batches_dev)]
        _capi.check(lib.ibp_decompress_fetch_condensed(
            cond.data_ptr(), cond.numel(), offs.data_ptr(), args.rows, V, 8, m.data_ptr(),
            b.data_ptr(), idx.data_ptr(), idx.shape[0], out.data_ptr(), wsp.data_ptr(), wsb,
            stream.cuda_stream))
        return idx.shape[0]

    for k in range(len(batches)):
        n = cond_step(k)
        torch.cuda.synchronize()
        assert np.array_equal(out[:n].cpu().numpy(), d[batches[k]]), "condensed fetch mismatch"
    for k in range(args.warmup):
        cond_step(k)
    torch.cuda.synchronize()
    _capi.check(lib.ibp_profile_enable(args.steps))
    c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    c0.record()
    crows = 0
    for k in range(args.steps):
        crows += cond_step(k)
    c1.record()
    c1.synchronize()
    ckms = kernel_ms(args.steps)
    cond_gbs = crows * V * 8 / c0.elapsed_time(c1) / 1e6
    cond_fetch = sum(kuniq[:len(ckms)]) / sum(ckms) / 1e6
    condensed = {"value": round(cond_gbs, 3), "unit": "GB/s",
                 "kernel_achieved": round(cond_fetch, 3), "frac": round(cond_fetch / pcie, 4),
                 "kernel_ms_per_launch": round(sum(ckms) / len(ckms), 4),
                 "host_bytes": int(cond.numel() * 8),
                 "what": "same batches from the condensed layout (exact-length row reads; "
                         "ibp_decompress_fetch_condensed); kernel_achieved = compressed bytes "
                         "of the distinct rows / fetch-kernel CUDA-event time"}
    del cond, offs

    # ---- device-resident variant of the same fetch (HBM roofline)
    xd = x.cuda()
    hbm = None
    try:
        peaks = json.load(open(os.path.join(REPO, "MEASURED_PEAKS.json")))
        hbm_peak, hbm_src = float(peaks["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs"
    except Exception:
        hbm_peak, hbm_src = 6650.0, "fallback 6.65 TB/s"
    k400 = [i for i, bt in enumerate(batches) if len(bt) == 400_000][0]
    for r in range(2):
        engine_step(k400, xd)
    _capi.check(lib.ibp_profile_enable(4))
    for r in range(4):
        engine_step(k400, xd)
    dms = kernel_ms(4)
    # the whole call (claim pass, fetch, repeat copies) on the same batch
    torch.cuda.synchronize()
    w0, w1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    w0.record()
    for r in range(10):
        engine_step(k400, xd)
    w1.record()
    w1.synchronize()
    call_ms = w0.elapsed_time(w1) / 10
    nuniq = len(np.unique(batches[k400]))
    hbm_bytes = uniq_bytes[k400] + nuniq * V * 8
    hbm_gbs = hbm_bytes / (sum(dms) / len(dms)) / 1e6
    call_bytes = uniq_bytes[k400] + len(batches[k400]) * V * 8
    hbm = {"bound": "hbm", "achieved": round(hbm_gbs, 1), "peak": hbm_peak, "unit": "GB/s",
           "frac": round(hbm_gbs / hbm_peak, 4), "traffic": None,
           "what": f"row-fetch kernel, device-resident copy of the set, 400k-row batch: "
                   f"compressed bytes read + decoded bytes written of {nuniq} distinct rows",
           "kernel_ms_per_launch": round(sum(dms) / len(dms), 4),
           "peak_source": hbm_src,
           "whole_call": {"ms": round(call_ms, 4),
                          "achieved": round(call_bytes / call_ms / 1e6, 1),
                          "frac": round(call_bytes / call_ms / 1e6 / hbm_peak, 4),
                          "what": "the whole device-resident call (claim pass, fetch, repeat "
                                  "copies): compressed bytes of the distinct rows read + all "
                                  "400k output rows written, per call"}}
    del xd

    line = None
    if rank == 0:
        ref_gpu = None
        if not args.no_reference_gpu:
            try:
                r = reference_gpu(torch, x, m, b, bm, comp_len, batches_dev, args.steps)
                if r is not None:
                    ref_gpu, rout = r
                    torch.cuda.synchronize()
                    ref_gpu["bit_exact_vs_input"] = bool(
                        np.array_equal(rout.cpu().numpy(), d[batches[0]]))
            except Exception as exc:  # reported, not fatal
                ref_gpu = {"error": repr(exc)[:200]}
        setup = None
        if not args.no_reference_gpu:
            try:
                setup = setup_vs_reference(torch, ibp, d, x, m, b, bm, sizes)
            except Exception as exc:  # reported, not fatal
                setup = {"error": repr(exc)[:200]}
        cpu = cpu_baseline(d, m.cpu().numpy(), b.cpu().numpy(), x.numpy(), bm.cpu().numpy(),
                           batches, args.cpu_seconds)
        gather = host_gather_copy_baseline(torch, d, batches)
        sweep = cpu_core_sweep(torch, d, m.cpu().numpy(), b.cpu().numpy(), x.numpy(),
                               bm.cpu().numpy(), batches, args.cpu_seconds)
        if setup and "ours" in setup:
            sweep["gpu_compress_inplace"] = round(
                d.nbytes / setup["ours"]["compress_inplace_ms"] / 1e6, 3)
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "GB/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4),
            "higher_is_better": True, "scaling": "strong" if shard else "weak",
            "vs_baseline": None, "dtype": "int64",
            "data": "synthetic",
            "config": headline_config(args, ws, shard, args.steps, comp_len,
                                      float(sizes_np.sum()) / d.nbytes),
            "e2e": {"value": round(e2e, 3), "unit": "GB/s", "h2d_bytes_per_step": h2d // args.steps,
                    "d2h_bytes_per_step": d2h // args.steps,
                    "what": "public API ibp.decompress_fetch; each step's index uploaded from "
                            "pinned host (on a copy stream, one step ahead) and the last output "
                            "row read back; the host at most 4 steps ahead of the GPU"},
            "roofline": {"bound": "pcie", "achieved": round(fetch_gbs, 3), "peak": round(pcie, 3),
                         "unit": "GB/s", "frac": round(fetch_gbs / pcie, 4),
                         "traffic": int(traffic),
                         "traffic_what": "host-memory (PCIe) bytes read per launch: 288 B per "
                                         "distinct row (ncu sysmem read sectors of the 400k-row "
                                         "batch, 9.0 per row) x distinct rows; algorithmic: "
                                         f"{int(sum(kuniq) / len(kuniq))} B per launch",
                         "what": "fetch_rows_kernel: compressed bytes of the distinct rows of "
                                 "each batch / kernel CUDA-event time",
                         "peak_source": "pinned host->device copy measured in this run "
                                        "(no PCIe figure in MEASURED_PEAKS.json)",
                         "achieved_counting_repeats": round(fetch_gbs_dups, 3),
                         "kernel_ms_per_launch": round(sum(kms) / len(kms), 4),
                         "pattern_ceiling": dict(pattern, kernel_frac_of_pattern=round(
                             fetch_gbs / pat_gbs, 4))},
            "roofline_hbm": hbm,
            "cpu_baseline": cpu,
            "cpu_baseline_uncompressed_gather": gather,
            "cpu_core_sweep": sweep,
            "gpu_uncompressed_gather": {"value": round(raw_gbs, 3), "unit": "GB/s",
                                        "what": "same batches, uncompressed pinned rows, "
                                                "zero-copy gather (impl 2) with the same "
                                                "sort and repeat fill"},
            "condensed": condensed,
            "reference_gpu": ref_gpu,
            "setup_vs_reference": setup,
            "clocks": clk.summary(),
            "gpu_launches": int(launches),
            "value_1000_steps": long_run,
        }
        if not args.no_extras:
            try:
                line["plain_small"] = plain_small_summary(torch, ibp, lib, _capi, pcie,
                                                          max(args.steps, 200), args.warmup)
            except Exception as exc:  # reported, not fatal
                line["plain_small"] = {"error": repr(exc)[:300]}
            line["served_mix"] = served_summary(subconfig_line(
                "served_mix", ["--rates", "1000,2000,20000", "--requests", "150"], 900))
            line["embedding_tables"] = batched_summary(subconfig_line(
                "embedding_tables", ["--steps", "20", "--warmup", "3"], 900))
            line["decoder_layer"] = batched_summary(subconfig_line(
                "decoder_layer", ["--steps", "10", "--warmup", "3"], 900))
        print(json.dumps(line), flush=True)
    barrier(ws)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
