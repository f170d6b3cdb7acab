"""Caller shims for the two integrations the reference documents, re-created because their
sources are not part of the reference (empty submodules):

* FlexGen (README.md:101-143): `IBPTensor` carries the `ibp_preprocess` / `ibp_compress`
  additions of FlexGen's TorchTensor, and `general_copy` is FlexGen's host-to-GPU copy with
  the copy replaced by a decompress_fetch into the destination.
* ColossalAI `CachedEmbeddingBag(comp=True, comp_imp=-1)` (tests/dlrm_comp_merged.py:70):
  `CompressedEmbeddingBag` keeps the table in pinned host memory (IBP-compressed, or raw for
  the comp=False baseline), a GPU cache of `cache_ratio` of its rows, and fetches every
  forward's missing rows with one decompress_fetch.

Both go through the package's public functions, so every byte they move is fetched and
decoded by libibp_b200.so.
"""
import torch
import torch.nn.functional as F

from . import decompress_fetch, get_single_compress_len, compress_inplace, preprocess


def _as_words(t):
    """The tensor's rows as int64 words (IBP operates on bits; any dtype works as long as a
    row is a whole number of 8-byte words)."""
    if t.dim() == 1:
        t = t.view(1, -1)
    t2 = t.reshape(t.shape[0], -1)
    if (t2.shape[1] * t2.element_size()) % 8:
        raise ValueError("a row must be a whole number of 8-byte words")
    return t2.view(torch.int64)


class IBPTensor:
    """A host tensor with the IBP state FlexGen's TorchTensor gains (README.md:104-117).

    data: pinned host (or CUDA) tensor, viewed as [rows, row words] int64."""

    def __init__(self, data):
        self.data = data
        self.mask = self.bitval = self.bitmask = None
        self.comp_len = None

    @property
    def compressed(self):
        return self.bitmask is not None

    def ibp_preprocess(self, threshold=None):
        self.mask, self.bitval = preprocess(_as_words(self.data), threshold)

    def ibp_compress(self):
        words = _as_words(self.data)
        self.comp_len = get_single_compress_len(words, self.mask, self.bitval)
        self.bitmask = compress_inplace(words, self.mask, self.bitval)


def _row_range(src_indices, nrows):
    """(first, last) rows when src_indices selects whole rows [first, last), else None."""
    if not src_indices:
        return 0, nrows
    first = src_indices[0]
    rest = src_indices[1:]
    if not isinstance(first, slice) or first.step not in (None, 1):
        return None
    if any(not (isinstance(s, slice) and s == slice(None)) for s in rest):
        return None
    a, b, _ = first.indices(nrows)
    return a, max(a, b)


def general_copy(dst, dst_indices, src, src_indices):
    """FlexGen's general_copy for a compressed source (README.md:128-141): decompress the
    selected rows of `src` (an IBPTensor) straight into `dst[dst_indices]` on the GPU.

    Whole-row selections decompress in one call into the destination (through a temporary
    when the destination view is not contiguous); any other selection decompresses the
    covering rows and copies the slice out.  Uncompressed sources fall back to the plain
    non-blocking copy FlexGen does."""
    dst_tensor = dst[dst_indices] if dst_indices else dst
    if not isinstance(src, IBPTensor) or not src.compressed:
        s = src.data if isinstance(src, IBPTensor) else src
        dst_tensor.copy_(s[src_indices] if src_indices else s, non_blocking=True)
        return dst_tensor
    full = _as_words(src.data)
    rows = src.data.shape[0] if src.data.dim() > 1 else 1
    rr = _row_range(src_indices, rows)
    dev = dst_tensor.device
    if rr is not None:
        a, b = rr
        idx = None if (a, b) == (0, rows) else torch.arange(a, b, device=dev)
        if dst_tensor.is_contiguous() and dst_tensor.dtype == src.data.dtype:
            out = _as_words(dst_tensor)
            decompress_fetch(full, src.mask, src.bitval, src.bitmask, dev, src.comp_len, idx,
                             output_tensor=out)
        else:
            tmp = decompress_fetch(full, src.mask, src.bitval, src.bitmask, dev, src.comp_len,
                                   idx)
            dst_tensor.copy_(tmp.view(src.data.dtype).view((b - a,) + tuple(src.data.shape[1:])))
        return dst_tensor
    first = src_indices[0]
    a, b = (first.indices(rows)[:2] if isinstance(first, slice)
            else (int(first), int(first) + 1))
    idx = torch.arange(a, max(a, b), device=dev)
    tmp = decompress_fetch(full, src.mask, src.bitval, src.bitmask, dev, src.comp_len, idx)
    tmp = tmp.view(src.data.dtype).view((idx.numel(),) + tuple(src.data.shape[1:]))
    sel = (slice(None),) + tuple(src_indices[1:]) if isinstance(first, slice) else \
        (0,) + tuple(src_indices[1:])
    dst_tensor.copy_(tmp[sel])
    return dst_tensor


class CompressedEmbeddingBag(torch.nn.Module):
    """An embedding bag over a host-resident table with a GPU row cache, the shape of
    ColossalAI's CachedEmbeddingBag with IBP (tests/dlrm_comp_merged.py:70-72).

    The table (`_weight`, [num_embeddings, embedding_dim], any dtype whose rows are whole
    8-byte words) is copied to pinned host memory and, with comp=True, preprocessed and
    compressed in place.  A forward looks its distinct rows up in the cache, evicts the
    oldest slots not used by the batch (FIFO), fetches the missing rows with one
    decompress_fetch (comp=False: the same call over the raw rows with an all-zero bitmask,
    i.e. a zero-copy gather), and runs F.embedding_bag over the cached rows."""

    def __init__(self, num_embeddings, embedding_dim, cache_ratio=0.01, _weight=None,
                 comp=True, mode="sum", threshold=None, device="cuda"):
        super().__init__()
        if _weight is None:
            _weight = torch.randn(num_embeddings, embedding_dim)
        if tuple(_weight.shape) != (num_embeddings, embedding_dim):
            raise ValueError("_weight must be [num_embeddings, embedding_dim]")
        self.mode = mode
        self.device = torch.device(device)
        if self.device.type == "cuda" and self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self.host = _weight.detach().to("cpu").contiguous().pin_memory()
        words = _as_words(self.host)
        self.words = words.shape[1]
        dev = self.device
        if comp:
            self.mask, self.bitval = preprocess(words, threshold)
            self.comp_len = get_single_compress_len(words, self.mask, self.bitval)
            self.bitmask = compress_inplace(words, self.mask, self.bitval)
        else:
            self.mask = torch.zeros(self.words, dtype=torch.int64, device=dev)
            self.bitval = torch.zeros(self.words, dtype=torch.int64, device=dev)
            self.bitmask = torch.zeros((num_embeddings + 31) // 32, dtype=torch.int32, device=dev)
            self.comp_len = None
        self.cache_rows = max(1, int(num_embeddings * cache_ratio))
        self.cache = torch.empty((self.cache_rows, embedding_dim), dtype=_weight.dtype, device=dev)
        self.slot_of_row = torch.full((num_embeddings,), -1, dtype=torch.int64, device=dev)
        self.row_of_slot = torch.full((self.cache_rows,), -1, dtype=torch.int64, device=dev)
        self.clock = 0
        self.stats = {"lookups": 0, "hits": 0, "misses": 0, "fetched_bytes": 0}

    def _admit(self, rows):
        """Slots holding `rows` (distinct, device int64), fetching the missing ones."""
        slots = self.slot_of_row[rows]
        miss = slots < 0
        miss_rows = rows[miss]
        nm = int(miss_rows.numel())
        self.stats["lookups"] += int(rows.numel())
        self.stats["misses"] += nm
        self.stats["hits"] += int(rows.numel()) - nm
        if nm == 0:
            return slots
        if rows.numel() > self.cache_rows:
            raise RuntimeError(f"{rows.numel()} distinct rows exceed the cache's "
                               f"{self.cache_rows} slots")
        busy = torch.zeros(self.cache_rows, dtype=torch.bool, device=self.device)
        busy[slots[~miss]] = True
        order = (self.clock + torch.arange(self.cache_rows, device=self.device)) % self.cache_rows
        free = order[~busy[order]][:nm]
        old = self.row_of_slot[free]
        self.slot_of_row[old[old >= 0]] = -1
        got = decompress_fetch(_as_words(self.host), self.mask, self.bitval, self.bitmask,
                               self.device, self.comp_len, miss_rows)
        self.cache.index_copy_(0, free, got.view(self.cache.dtype).view(nm, -1))
        self.slot_of_row[miss_rows] = free
        self.row_of_slot[free] = miss_rows
        self.clock = (self.clock + nm) % self.cache_rows
        self.stats["fetched_bytes"] += nm * self.words * 8
        return self.slot_of_row[rows]

    def forward(self, indices, offsets=None, per_sample_weights=None):
        indices = indices.to(self.device, torch.int64)
        uniq, inv = torch.unique(indices, return_inverse=True)
        slots = self._admit(uniq)
        local = slots[inv]
        return F.embedding_bag(local, self.cache, offsets, mode=self.mode,
                               per_sample_weights=per_sample_weights)
