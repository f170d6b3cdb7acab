"""Continuous-batching fetch server (C++ scheduler in libibp_b200.so, ibp_server_*).

    reg = SetRegistry([...])
    srv = Server(reg, arena_bytes=40 << 30)
    rid = srv.submit(set_id, rows=np.array([...], np.int64))   # or first=, count=
    out, times = srv.wait(rid)      # device rows (a view of the arena) + submit/admit/done us
    ... use out ...
    srv.release(rid)                # rows go back to the arena

Requests are admitted in arrival order as their output fits the arena and join the next
batched launch (de-duplicated by hash claims inside the fetch, or by a sort after
set_dedup("sort"); up to the batch limits: 128 MiB of output by default), with up to
`max_inflight` launches on the GPU.
"""
import ctypes

import numpy as np
import torch

from . import _capi

_lib = _capi.lib


class Server:
    def __init__(self, registry, arena_bytes, index_capacity=1 << 25, max_batch=256,
                 max_inflight=2, batch_bytes=None, batch_rows=None):
        self.reg = registry
        self.arena = torch.empty(int(arena_bytes), dtype=torch.uint8, device="cuda")
        self.handle = ctypes.c_void_p()
        _capi.check(_lib.ibp_server_create(
            registry.buf.data_ptr(), registry.descs, len(registry.sets), registry.word_bytes,
            self.arena.data_ptr(), self.arena.numel(), int(index_capacity), int(max_batch),
            int(max_inflight), ctypes.byref(self.handle)))
        self.counts = {}
        if batch_bytes is not None or batch_rows is not None:
            self.set_batch_limits(batch_rows, batch_bytes)

    def set_dedup(self, mode):
        """How later batches find repeated rows: "hash" (claims inside the fetch; default) or
        "sort" (a radix sort of the batch's rows first)."""
        m = {"hash": 0, "sort": 1}.get(mode)
        if m is None:
            raise ValueError(f"set_dedup: mode must be 'hash' or 'sort', got {mode!r}")
        _capi.check(_lib.ibp_server_set_dedup(self.handle, m))

    def set_batch_limits(self, rows=None, nbytes=None):
        """Cap one batch at `rows` rows and `nbytes` output bytes (None: keep)."""
        _capi.check(_lib.ibp_server_set_batch_limits(self.handle, int(rows or 0),
                                                     int(nbytes or 0)))

    def submit(self, set_id, rows=None, first=0, count=None):
        """Queue `rows` (host int64 array) or rows first .. first+count-1 of a set."""
        rid = ctypes.c_int64()
        if rows is not None:
            rows = np.ascontiguousarray(rows, dtype=np.int64)
            count = rows.shape[0]
            ptr = rows.ctypes.data_as(ctypes.c_void_p)
        else:
            ptr = None
        _capi.check(_lib.ibp_server_submit(self.handle, int(set_id), ptr, int(first), int(count),
                                           ctypes.byref(rid)))
        self.counts[rid.value] = (int(set_id), int(count))
        return rid.value

    def wait(self, rid, timeout_ms=-1):
        """(output rows as a CUDA tensor view of the arena, [submit, admit, done] in us)."""
        out = ctypes.c_void_p()
        times = (ctypes.c_double * 3)()
        _capi.check(_lib.ibp_server_wait(self.handle, int(rid), int(timeout_ms),
                                         ctypes.byref(out), times))
        sid, count = self.counts[rid]
        v = self.reg.vec_sizes[sid]
        off = out.value - self.arena.data_ptr()
        nbytes = count * v * self.reg.word_bytes
        rows = self.arena[off:off + nbytes].view(self.reg.dtype).view(count, v)
        return rows, [times[0], times[1], times[2]]

    def cancel(self, rid):
        """Withdraw a request still waiting for admission (RuntimeError once admitted)."""
        _capi.check(_lib.ibp_server_cancel(self.handle, int(rid)))
        self.counts.pop(rid, None)

    def release(self, rid):
        _capi.check(_lib.ibp_server_release(self.handle, int(rid)))
        self.counts.pop(rid, None)

    def stats(self):
        st = (ctypes.c_int64 * 4)()
        _capi.check(_lib.ibp_server_stats(self.handle, st))
        return {"batches": st[0], "rows_done": st[1], "bytes_done": st[2], "pending": st[3]}

    def close(self):
        if self.handle:
            _lib.ibp_server_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
