"""Batched multi-set fetch: many (tensor set, rows) requests in one launch, CUDA-graph ready.

    reg = SetRegistry([(comp, mask, bitval, bitmask, comp_len), ...])   # once per set group
    bf = BatchFetcher(reg, max_requests=64)
    outs = bf.fetch([(set_id, index_tensor_or_None, first, count), ...])
    bf.capture()     # later fetches replay one CUDA graph: copy of the request table + launch
    outs = bf.fetch(reqs, dedup=True)   # sort + de-duplicate each request's rows first
    outs = bf.fetch(reqs, dedup="hash") # de-duplicate (set, row) by hash claims, no sort

The request table (count + ibp_request records) is written into a pinned host buffer and
copied to the device inside the captured work, so one graph serves any batch of up to
max_requests requests: index arrays and output buffers are just pointers in the table.
Two host/device table pairs alternate so the host can prepare a batch while the previous
one runs.  All computation is libibp_b200.so (include/ibp_b200.h, batched multi-set fetch).
"""
import ctypes

import torch

from . import _capi

_lib = _capi.lib
_HDR = 64  # table header: int32 request count, padded


def _stream():
    return torch.cuda.current_stream().cuda_stream


class SetRegistry:
    """Device-resident descriptors and per-column tables of a group of tensor sets."""

    def __init__(self, sets):
        if not sets:
            raise ValueError("no sets")
        self.sets = []
        descs = (_capi.SetDesc * len(sets))()
        wb = None
        for i, s in enumerate(sets):
            comp, mask, bitval, bitmask = s[:4]
            comp_len = int(s[4]) if len(s) > 4 and s[4] is not None else -1
            if wb is None:
                wb = comp.element_size()
            if comp.element_size() != wb or mask.element_size() != wb:
                raise RuntimeError("all sets of a registry must share one word size")
            if comp.dim() != 2 or not comp.is_contiguous():
                raise RuntimeError("set rows must be a contiguous 2-D tensor")
            if not (comp.device.type == "cuda" or comp.is_pinned()):
                raise RuntimeError("Input tensor must accessible by CUDA device (GPU or pinned memory)")
            d = descs[i]
            d.comp, d.num_vecs, d.vec_size = comp.data_ptr(), comp.shape[0], comp.shape[1]
            d.mask, d.bitval, d.bitmask = mask.data_ptr(), bitval.data_ptr(), bitmask.data_ptr()
            d.comp_len = comp_len
            self.sets.append((comp, mask, bitval, bitmask))
        self.descs = descs
        self.word_bytes = wb
        self.dtype = sets[0][0].dtype
        self.vec_sizes = [s[0].shape[1] for s in self.sets]
        self.num_vecs = [s[0].shape[0] for s in self.sets]
        size = _lib.ibp_sets_registry_size(descs, len(sets), wb)
        self.buf = torch.empty(size, dtype=torch.uint8, device="cuda")
        _capi.check(_lib.ibp_sets_register(descs, len(sets), wb, self.buf.data_ptr(), size,
                                           _stream()))


class BatchFetcher:
    """One batched launch per fetch() over a SetRegistry; optionally graph-captured."""

    def __init__(self, registry, max_requests=256, buffers=2):
        self.reg = registry
        self.max = int(max_requests)
        nbytes = _HDR + ctypes.sizeof(_capi.Request) * self.max
        self.host = [torch.zeros(nbytes, dtype=torch.uint8).pin_memory() for _ in range(buffers)]
        self.dev = [torch.zeros(nbytes, dtype=torch.uint8, device="cuda") for _ in range(buffers)]
        self.done = [None] * buffers
        self.ws = torch.empty(_lib.ibp_batch_fetch_workspace_size(), dtype=torch.uint8,
                              device="cuda")
        self.graphs = None
        self.turn = 0
        self.keep = [None] * buffers
        self.sort_ws = None
        self.last_ws = self.ws

    def _write(self, b, requests, outs):
        if len(requests) > self.max:
            raise ValueError(f"{len(requests)} requests exceed max_requests={self.max}")
        if self.done[b] is not None:
            self.done[b].synchronize()  # the copy that read this host table has finished
        h = self.host[b]
        ctypes.c_int32.from_address(h.data_ptr()).value = len(requests)
        recs = (_capi.Request * self.max).from_address(h.data_ptr() + _HDR)
        keep = []
        for i, (rq, o) in enumerate(zip(requests, outs)):
            sid, idx, first, count = rq
            r = recs[i]
            r.set = int(sid)
            r.index = None if idx is None else idx.data_ptr()
            r.first = int(first)
            r.count = int(count)
            r.out = o.data_ptr()
            keep.append(idx)
        self.keep[b] = (keep, outs)

    def _launch(self, b):
        d = self.dev[b]
        d.copy_(self.host[b], non_blocking=True)
        _capi.check(_lib.ibp_batch_fetch(self.reg.buf.data_ptr(), d.data_ptr() + _HDR,
                                         d.data_ptr(), self.max, self.ws.data_ptr(),
                                         self.ws.numel(), _stream()))

    def outputs_for(self, requests, device="cuda"):
        return [torch.empty((int(rq[3]), self.reg.vec_sizes[int(rq[0])]), dtype=self.reg.dtype,
                            device=device) for rq in requests]

    def _launch_sorted(self, b, nreq, rows):
        need = _lib.ibp_batch_fetch_sorted_workspace_size(rows, nreq)
        if self.sort_ws is None or self.sort_ws.numel() < need:
            self.sort_ws = torch.empty(need, dtype=torch.uint8, device="cuda")
        d = self.dev[b]
        d.copy_(self.host[b], non_blocking=True)
        _capi.check(_lib.ibp_batch_fetch_sorted(self.reg.buf.data_ptr(), d.data_ptr() + _HDR, nreq,
                                                rows, self.sort_ws.data_ptr(),
                                                self.sort_ws.numel(), _stream()))
        self.last_ws = self.sort_ws

    def _launch_hashed(self, b, nreq, rows):
        need = _lib.ibp_batch_fetch_hashed_workspace_size(rows)
        if self.sort_ws is None or self.sort_ws.numel() < need:
            self.sort_ws = torch.empty(need, dtype=torch.uint8, device="cuda")
        d = self.dev[b]
        d.copy_(self.host[b], non_blocking=True)
        _capi.check(_lib.ibp_batch_fetch_hashed(self.reg.buf.data_ptr(), d.data_ptr() + _HDR, nreq,
                                                rows, self.sort_ws.data_ptr(),
                                                self.sort_ws.numel(), _stream()))
        self.last_ws = self.sort_ws

    def fetch(self, requests, outs=None, dedup=False):
        """requests: (set id, int64 CUDA index or None, first row, row count) each.

        dedup=True (or "sort") sorts each request's rows on the device and fetches a repeated
        row once (ibp_batch_fetch_sorted); dedup="hash" claims each (set, row) in a hash table
        inside the fetch instead (ibp_batch_fetch_hashed), which also shares rows between
        requests of one set.  Both run outside the captured graphs, whose table shape is
        fixed at capture."""
        if dedup not in (False, True, "sort", "hash"):
            raise ValueError(f"dedup must be False, True, 'sort' or 'hash', got {dedup!r}")
        requests = [(s, (None if i is None else i.to(torch.int64)), f, c) for s, i, f, c in requests]
        if outs is None:
            outs = self.outputs_for(requests)
        b = self.turn
        self.turn = (self.turn + 1) % len(self.host)
        self._write(b, requests, outs)
        if dedup:
            if requests:
                rows = sum(max(int(r[3]), 0) for r in requests)
                if dedup == "hash":
                    self._launch_hashed(b, len(requests), rows)
                else:
                    self._launch_sorted(b, len(requests), rows)
        elif self.graphs is not None:
            self.last_ws = self.ws
            self.graphs[b].replay()
        else:
            self.last_ws = self.ws
            self._launch(b)
        ev = torch.cuda.Event()
        ev.record()
        self.done[b] = ev
        return outs

    def capture(self):
        """Capture one graph per table buffer (copy of the table + batched launch)."""
        torch.cuda.synchronize()
        graphs = []
        for b in range(len(self.host)):
            ctypes.c_int32.from_address(self.host[b].data_ptr()).value = 0
            self._launch(b)  # warm-up outside capture
            torch.cuda.synchronize()
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                self._launch(b)
            graphs.append(g)
        torch.cuda.synchronize()
        self.graphs = graphs

    def autotune(self, requests, outs=None):
        """Pick the launch shape for this registry from timed runs of `requests`."""
        requests = [(s, (None if i is None else i.to(torch.int64)), f, c) for s, i, f, c in requests]
        if outs is None:
            outs = self.outputs_for(requests)
        b = 0
        self._write(b, requests, outs)
        self.dev[b].copy_(self.host[b], non_blocking=True)
        chosen = (ctypes.c_int32 * 4)()
        d = self.dev[b]
        _capi.check(_lib.ibp_batch_autotune(self.reg.buf.data_ptr(), d.data_ptr() + _HDR,
                                            d.data_ptr(), self.max, self.ws.data_ptr(),
                                            self.ws.numel(), chosen, _stream()))
        return {"threads": chosen[0], "rows_in_flight": chosen[1], "blocks_per_sm": chosen[2]}

    def status(self):
        """Device status word of the last batch (bit 0: a bad row index or set id; bit 1: a
        corrupt row; bit 2: request counts that disagree with a sorted batch's total)."""
        torch.cuda.synchronize()
        return int(self.last_ws[:4].view(torch.int32).item())
