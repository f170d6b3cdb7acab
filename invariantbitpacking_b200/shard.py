"""Sharded fetch across the GPUs of one node, one process per GPU.

Rows are independent, so a batch's index array is split by position into contiguous shards,
one per rank; each rank fetches its shard from the host-resident set over its own PCIe link
(zero-copy through libibp_b200.so), and nothing crosses NVLink unless every rank needs the
whole batch, in which case `gather=True` all-gathers the shards (NCCL over NVLink/NVSwitch
on GPUs; any torch.distributed backend works).  Each rank should read host memory on its
own NUMA node: `bind_to_gpu_numa` pins the process to the CPUs local to its GPU before the
set is pinned, so first-touch places the pages there.
"""
import os

import torch
import torch.distributed as dist


def shard_bounds(n, world, rank):
    """Positions [lo, hi) of rank's shard of n positions: contiguous, sizes differ by at
    most one, earlier ranks take the extra positions."""
    if world < 1 or not 0 <= rank < world or n < 0:
        raise ValueError(f"bad shard request: n={n} world={world} rank={rank}")
    base, extra = divmod(n, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def parse_cpulist(text):
    """CPU ids of a sysfs cpulist such as '0-3,8,10-11'."""
    cpus = []
    for part in text.strip().split(","):
        if not part:
            continue
        if "-" in part:
            a, b = part.split("-")
            cpus.extend(range(int(a), int(b) + 1))
        else:
            cpus.append(int(part))
    return cpus


def local_cpus_of_bus(bus, sysfs="/sys/bus/pci/devices"):
    """CPUs local to the PCI device `bus` ('0000:1b:00.0'); empty when sysfs does not say."""
    try:
        with open(os.path.join(sysfs, bus, "local_cpulist")) as f:
            return parse_cpulist(f.read())
    except OSError:
        return []


def gpu_local_cpus(device_index, sysfs="/sys/bus/pci/devices"):
    """CPUs on the NUMA node of a CUDA device (empty when the platform does not say)."""
    p = torch.cuda.get_device_properties(device_index)
    bus = f"{p.pci_domain_id:04x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0"
    return local_cpus_of_bus(bus, sysfs)


def bind_to_gpu_numa(device_index):
    """Restrict this process to the CPUs local to its GPU (no-op when unknown); call before
    pinning the host-resident set."""
    cpus = gpu_local_cpus(device_index)
    usable = set(cpus) & os.sched_getaffinity(0)
    if usable:
        os.sched_setaffinity(0, usable)
    return sorted(usable)


class ShardedFetcher:
    """Fetch this rank's shard of each batch; optionally all-gather the whole batch.

    fetch(index) -> rows: defaults to decompress_fetch of the given compressed set onto this
    rank's GPU; any callable with that contract works (the tests use a CPU one)."""

    def __init__(self, comp=None, mask=None, bitval=None, bitmask=None, comp_len=None,
                 group=None, fetch=None, device=None):
        self.group = group
        if fetch is None:
            from . import decompress_fetch
            dev = torch.device(device) if device is not None else \
                torch.device("cuda", torch.cuda.current_device())

            def fetch(index):
                return decompress_fetch(comp, mask, bitval, bitmask, dev, comp_len,
                                        index.to(dev))
        self.fetch = fetch

    def _world(self):
        if not dist.is_available() or not dist.is_initialized():
            return 1, 0
        return dist.get_world_size(self.group), dist.get_rank(self.group)

    def __call__(self, index, gather=False):
        """index: the whole batch (same on every rank).  Returns (rows, (lo, hi)) of this
        rank's shard, or the whole batch's rows when gather=True."""
        world, rank = self._world()
        n = int(index.shape[0])
        lo, hi = shard_bounds(n, world, rank)
        local = self.fetch(index[lo:hi])
        if not gather:
            return local, (lo, hi)
        if world == 1:
            return local
        width = (n + world - 1) // world
        padded = local.new_zeros((width,) + tuple(local.shape[1:]))
        padded[:hi - lo] = local
        if dist.get_backend(self.group) == "nccl":
            flat = padded.new_empty((width * world,) + tuple(local.shape[1:]))
            dist.all_gather_into_tensor(flat, padded, group=self.group)
            parts = list(flat.split(width))
        else:
            parts = [torch.empty_like(padded) for _ in range(world)]
            dist.all_gather(parts, padded, group=self.group)
        out = []
        for r, p in enumerate(parts):
            a, b = shard_bounds(n, world, r)
            out.append(p[:b - a])
        return torch.cat(out)
