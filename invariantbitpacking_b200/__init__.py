"""B200-native Invariant Bit Packing: a drop-in for the reference's `ibp` Python API.

Same functions, argument order and defaults as the reference package (ibp/__init__.py:8-41);
the work runs in libibp_b200.so, hand-written sm_100a kernels behind a C ABI
(include/ibp_b200.h).  To switch an existing `import ibp` user over:

    import torch
    import invariantbitpacking_b200 as ibp

The module-level `ibp_cuda` mirrors the reference's extension module of that name, for
callers that use it directly and positionally.
"""
import torch  # noqa: F401  (the reference imports torch first as well)

from . import ibp_cuda
from ._capi import IBPError

ibp_cuda.print_debug(False)

__all__ = ["print_debug", "preprocess", "preprocess_kmeans", "get_compress_size",
           "get_single_compress_len", "compress_inplace", "compress", "compress_condensed",
           "decompress_fetch_condensed",
           "decompress_fetch", "read_shared", "set_fetch_dedup", "set_repeat_wait_limit",
           "ibp_cuda", "IBPError"]


def print_debug(flag):
    ibp_cuda.print_debug(flag)


def preprocess(dataset, threshold=None):
    """Returns mask and bitval tensors."""
    return ibp_cuda.preprocess(dataset, threshold)


def preprocess_kmeans(dataset, centroids, threshold=None, *, seed_rows=None):
    """Returns per-cluster mask and bitval tensors and the cluster of every row."""
    return ibp_cuda.preprocess_kmeans(dataset, centroids, threshold, seed_rows=seed_rows)


def get_compress_size(dataset, mask, bitval, index_arr=None, compress_total=None):
    return ibp_cuda.get_compress_size(dataset, mask, bitval, index_arr, compress_total)


def get_single_compress_len(dataset, mask, bitval, index_arr=None):
    """Average compressed row length in words (ibp/__init__.py:22-29; index_arr unused there
    as well)."""
    comp_sizes = get_compress_size(dataset, mask, bitval)
    torch.cuda.synchronize()
    og_size = dataset.numel() * dataset.element_size()
    comp_size = int(torch.sum(comp_sizes))
    return int(comp_size / og_size * dataset.size(1))


def compress_inplace(dataset, mask, bitval, index_arr=None):
    """Returns the bitmask marking compressed rows."""
    return ibp_cuda.compress_inplace(dataset, mask, bitval, index_arr)


def compress_condensed(dataset, mask, bitval, index_arr=None):
    """Compressed rows packed back to back, and their inclusive byte offsets."""
    return ibp_cuda.compress_condensed(dataset, mask, bitval, index_arr)


def compress(dataset, mask, bitval, index_arr=None):
    """The reference's `compress` calls an extension function that does not exist
    (ibp/__init__.py:35-36); here it returns the condensed form."""
    return ibp_cuda.compress_condensed(dataset, mask, bitval, index_arr)


def decompress_fetch(comp_dataset, mask, bitval, bitmask, device, comp_len=None,
                     index_arr=None, nblks=None, nthds=None, imp=None, output_tensor=None, *,
                     check=False):
    """Decompressed rows (non-blocking).  check=True (keyword only; not in the reference) waits
    for the call and raises RuntimeError when an index was out of range or a row could not be
    decoded, instead of leaving those output rows unwritten."""
    return ibp_cuda.decompress_fetch(comp_dataset, mask, bitval, bitmask, device, comp_len,
                                     index_arr, nblks, nthds, imp, output_tensor, check=check)


def decompress_fetch_condensed(comp, offsets, mask, bitval, vec_size, device, index_arr=None,
                               output_tensor=None, *, check=False):
    """Rows of the condensed layout (compress_condensed's words and byte offsets)."""
    return ibp_cuda.decompress_fetch_condensed(comp, offsets, mask, bitval, vec_size, device,
                                               index_arr, output_tensor, check=check)


def read_shared(filename, shape, dtype):
    return ibp_cuda.read_shared(filename, shape, dtype)


_DEDUP_MODES = {"auto": 0, "sort": 1, "hash": 2}


def set_fetch_dedup(mode):
    """How decompress_fetch finds the repeated rows of an index array, process-wide (no
    counterpart in the reference, which always sorts): "auto" (hash table for compressed rows
    in device memory and for sparse host batches, else sort), "sort", or "hash" (repeats are
    then copied inside the fetch for host rows).  Dense batches whose rows repeat a lot are
    faster with "hash", dense batches with few repeats with "sort".  Also takes 0/1/2."""
    from . import _capi
    m = _DEDUP_MODES.get(mode, mode) if isinstance(mode, str) else mode
    if m not in (0, 1, 2):
        raise ValueError(f"set_fetch_dedup: mode must be one of {sorted(_DEDUP_MODES)} "
                         f"or 0/1/2, got {mode!r}")
    _capi.check(_capi.lib.ibp_set_fetch_dedup(int(m)))


def set_repeat_wait_limit(polls=None):
    """How many polls (~0.25 us apart) a repeated index of a hashed host-row fetch makes for
    its first occurrence's row before decoding its own row from the source, process-wide
    (None: the default, 2^20).  The output is the same whatever the limit; 0 sends every
    such repeat down the decode-from-source path, which tests use to exercise it."""
    from . import _capi
    _capi.check(_capi.lib.ibp_set_repeat_wait_limit(-1 if polls is None else int(polls)))
