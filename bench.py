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
algorithm on the host cores (the reference implementation has no CPU path of its own).
Under torchrun every rank runs an independent replica on its own GPU (the path has no
exchange step); time is the max over ranks.
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


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--rows", type=int, default=ROWS)
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-reference-gpu", action="store_true")
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
    """nvidia-smi samples during the timed region."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "20"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [q.strip() for q in ln.split(",")]
            if len(p) < 7:
                continue
            try:
                sm.append(float(p[0]))
                mx = max(mx, float(p[1]))
            except ValueError:
                continue
            for nm, val in zip(names, p[3:7]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def make_workload(rows, seed_batches=12):
    from invariantbitpacking_b200 import synthetic
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


def run_reference_arm(args, ws, rank):
    """CPU restatement of the reference algorithm on the host cores, same config/metric."""
    if rank != 0:
        return
    import oracle
    from invariantbitpacking_b200 import synthetic  # noqa: F401
    d, batches = make_workload(args.rows)
    m, b, _ = oracle.preprocess(d[:200_000], None)
    comp, bm = oracle.compress(d, m, b)
    oracle.set_threads(os.cpu_count() or 1)
    for k in range(args.warmup):
        oracle.decompress(comp, m, b, bm, batches[k % len(batches)][:20_000])
    t0 = time.perf_counter()
    rows = 0
    per_step = max(1, int(60_000))
    for k in range(args.steps):
        idx = batches[k % len(batches)][:per_step]
        oracle.decompress(comp, m, b, bm, idx)
        rows += len(idx)
    el = time.perf_counter() - t0
    val = rows * V * 8 / el / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": round(val, 3), "unit": "GB/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(el * 1e3 / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic",
        "config": {"workload": "graph_features 2.4M x 64 int64 (1.2 GB), Zipf(1.1) batches",
                   "rows": args.rows, "sample_rows_per_step": per_step,
                   "mask": "preprocess sweep on the first 200k rows"},
        "cpu_baseline": {"value": round(val, 3), "unit": "GB/s",
                         "cores": oracle.get_threads(), "kind": "port",
                         "sample": f"{args.steps} steps of {per_step} rows of each mini-batch "
                                   "decompressed on the host by the oracle (the reference "
                                   "implements decompress_fetch only as a CUDA kernel)"},
        "e2e": {"value": round(val, 3), "unit": "GB/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def reference_gpu(torch, comp, m, b, bm, comp_len, batches_dev, steps):
    """The reference extension (built from its sources for sm_100a, oracle/_ref) on the same
    compressed rows, through its own positional API; None when it is not built."""
    import glob
    mods = glob.glob(os.path.join(REPO, "oracle", "_ref", "ibp_cuda*.so"))
    if not mods:
        return None
    sys.path.insert(0, os.path.dirname(mods[0]))
    import ibp_cuda as ref
    ref.print_debug(False)
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


def main():
    args = parse()
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
    value = rows * V * 8 * ws / ms / 1e6  # GB/s, all ranks
    kuniq = [uniq_bytes[k % len(batches)] for k in range(args.steps)]
    kall = [all_bytes[k % len(batches)] for k in range(args.steps)]
    fetch_gbs = sum(kuniq) / sum(kms) / 1e6
    fetch_gbs_dups = sum(kall) / sum(kms) / 1e6

    # ---- e2e: public API, index uploaded per step, last row read back per step
    res_host = torch.empty(V, dtype=torch.int64).pin_memory()
    for k in range(args.warmup):
        idx = batches_host[k % len(batches)].to("cuda", non_blocking=True)
        o = ibp.decompress_fetch(x, m, b, bm, torch.device("cuda"), comp_len, idx)
        res_host.copy_(o[-1], non_blocking=True)
    torch.cuda.synchronize()
    barrier(ws)
    h2d = d2h = 0
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    rows_e = 0
    for k in range(args.steps):
        hi = batches_host[k % len(batches)]
        idx = hi.to("cuda", non_blocking=True)
        o = ibp.decompress_fetch(x, m, b, bm, torch.device("cuda"), comp_len, idx)
        res_host.copy_(o[-1], non_blocking=True)
        rows_e += hi.shape[0]
        h2d += hi.numel() * 8
        d2h += V * 8
    e1.record()
    e1.synchronize()
    ems = max_over_ranks(e0.elapsed_time(e1), ws)
    e2e = rows_e * V * 8 * ws / ems / 1e6

    pcie = measured_pcie_h2d(torch)

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
    nuniq = len(np.unique(batches[k400]))
    hbm_bytes = uniq_bytes[k400] + nuniq * V * 8
    hbm_gbs = hbm_bytes / (sum(dms) / len(dms)) / 1e6
    hbm = {"bound": "hbm", "achieved": round(hbm_gbs, 1), "peak": hbm_peak, "unit": "GB/s",
           "frac": round(hbm_gbs / hbm_peak, 4), "traffic": None,
           "what": f"row-fetch kernel, device-resident copy of the set, 400k-row batch: "
                   f"compressed bytes read + decoded bytes written of {nuniq} distinct rows",
           "peak_source": hbm_src}
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
        cpu = cpu_baseline(d, m.cpu().numpy(), b.cpu().numpy(), x.numpy(), bm.cpu().numpy(),
                           batches, args.cpu_seconds)
        gather = host_gather_copy_baseline(torch, d, batches)
        nrows_avg = rows / args.steps
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "GB/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
            "data": "synthetic",
            "config": {"workload": "graph_features: 2.4M x 128 fp32 N(0,0.3^2), 8 mantissa bits, "
                                   "30% zeros -> int64 [2.4M x 64], pinned host (1.2 GB)",
                       "rows": args.rows, "vec_words": V,
                       "batches": "Zipf(1.1) mini-batches cycling 100k/200k/400k rows",
                       "avg_rows_per_step": nrows_avg, "comp_len_words": comp_len,
                       "compressed_fraction": round(float(sizes_np.sum()) / d.nbytes, 4),
                       "l2": "inputs larger than L2 (1.2 GB host set; 51-205 MB outputs)",
                       "parallelism": f"{ws} independent replica(s)"},
            "e2e": {"value": round(e2e, 3), "unit": "GB/s", "h2d_bytes_per_step": h2d // args.steps,
                    "d2h_bytes_per_step": d2h // args.steps,
                    "what": "public API ibp.decompress_fetch; index uploaded from pinned host, "
                            "last output row read back, each step"},
            "roofline": {"bound": "pcie", "achieved": round(fetch_gbs, 3), "peak": round(pcie, 3),
                         "unit": "GB/s", "frac": round(fetch_gbs / pcie, 4), "traffic": None,
                         "what": "fetch_rows_kernel: compressed bytes of the distinct rows of "
                                 "each batch / kernel CUDA-event time",
                         "peak_source": "pinned host->device copy measured in this run "
                                        "(no PCIe figure in MEASURED_PEAKS.json)",
                         "achieved_counting_repeats": round(fetch_gbs_dups, 3),
                         "kernel_ms_per_launch": round(sum(kms) / len(kms), 4)},
            "roofline_hbm": hbm,
            "cpu_baseline": cpu,
            "cpu_baseline_uncompressed_gather": gather,
            "gpu_uncompressed_gather": {"value": round(raw_gbs, 3), "unit": "GB/s",
                                        "what": "same batches, uncompressed pinned rows, "
                                                "zero-copy gather (impl 2) with the same "
                                                "sort and repeat fill"},
            "reference_gpu": ref_gpu,
            "clocks": clk.summary(),
            "gpu_launches": int(launches),
        }
        print(json.dumps(line), flush=True)
    barrier(ws)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
