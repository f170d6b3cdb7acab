"""Drop-in mirror of the reference's compiled extension module `ibp_cuda`.

Same function names, positional signatures, defaults, output placement and argument
checks (with the reference's error messages, raised as RuntimeError like TORCH_CHECK) as
src/ibp_api.cu:20-40 and :124-135; every computation is a call into libibp_b200.so through
its C ABI (invariantbitpacking_b200/_capi.py).  torch provides device memory and the
current stream only.

Behavioural differences from the reference, all deliberate:
  * preprocess and get_compress_size never block the host; decompress_fetch allocates its
    output with torch.empty (every row is written) instead of torch.zeros;
  * compress_inplace blocks only when the dataset is in host memory (the caller may read it
    right away); the reference blocks always (cudaFree);
  * an index array with compress_inplace reads every source row before any row is
    overwritten (the reference races);
  * get_compress_size's counter is updated whatever its dtype's size (the reference writes
    a temporary copy when it is not int64);
  * decompress_fetch rejects impl 3/4 (the reference's upper-bound stand-ins that do not
    decompress) and ignores nblks/nthreads values that do not fit the engine's kernels;
  * decompress_fetch reads an out_device of "cuda" without an index as the current device,
    so an output_tensor there passes the device check (the reference compares the
    unindexed device with the tensor's and refuses);
  * preprocess_kmeans breaks distance ties toward the highest centroid id (the reference
    races) and accepts keyword-only `seed_rows` to fix the centroid seeds.
"""
import numpy as np
import torch

from . import _capi

_lib = _capi.lib
_check = _capi.check

_INT_DTYPE = {1: torch.int8, 2: torch.int16, 4: torch.int32, 8: torch.int64}


def _stream():
    return torch.cuda.current_stream().cuda_stream


# Per-call fast paths (the device index and its current stream as plain integers); the public
# torch.cuda helpers they stand in for cost microseconds of Python per call.
_get_device = getattr(torch._C, "_cuda_getDevice", None) or torch.cuda.current_device
_raw_stream = getattr(torch._C, "_cuda_getCurrentRawStream", None)


def _stream_of(index):
    if _raw_stream is not None:
        return _raw_stream(index)
    return torch.cuda.current_stream(index).cuda_stream


def _ptr(t):
    return None if t is None else t.data_ptr()


def _torch_check(cond, msg):
    if not cond:
        raise RuntimeError(msg)


def _gpu_accessible(t):
    return t.device.type == "cuda" or t.is_pinned()


def _workspace(nbytes, device):
    if nbytes == 0:
        return None, 0
    return torch.empty(int(nbytes), dtype=torch.uint8, device=device), int(nbytes)


def _cuda_device(*tensors):
    for t in tensors:
        if t is not None and t.device.type == "cuda":
            return t.device
    return torch.device("cuda", torch.cuda.current_device())


def _stage_budget(nbytes, device):
    """Stage a host-resident dataset in HBM when it takes at most half the free memory."""
    try:
        free, _ = torch.cuda.mem_get_info(device)
    except Exception:
        return False
    return nbytes <= free // 2


_debug = False


def print_debug(flag):
    """src/ibp_api.cu:9-12"""
    global _debug
    _debug = bool(flag)
    _lib.ibp_set_debug(1 if flag else 0)


def preprocess(dataset, threshold_=None):
    """src/preprocess.cu:17-76 -> (mask, bitval) int tensors of vec_size words on CUDA."""
    _torch_check(dataset.device.type == "cuda" or dataset.is_pinned(),
                 "Input tensor must accessible by CUDA device (GPU or pinned memory)")
    _torch_check(dataset.dim() == 2, "Input tensor must be 2D [num_vecs x vec_size]")
    wb = dataset.element_size()
    _torch_check(wb in (1, 2, 4, 8), "Input tensor must be 1, 2, 4, or 8-byte datatype")
    _torch_check(dataset.is_contiguous(), "Input tensor must be contiguous")
    threshold = -1.0 if threshold_ is None else float(threshold_)
    n, v = dataset.shape
    dev = _cuda_device(dataset)
    with torch.cuda.device(dev):
        mask = torch.empty(v, dtype=_INT_DTYPE[wb], device=dev)
        bitval = torch.empty(v, dtype=_INT_DTYPE[wb], device=dev)
        need = _lib.ibp_preprocess_workspace_size(n, v, wb, threshold)
        if dataset.device.type != "cuda" and _stage_budget(n * v * wb, dev):
            need += (n * v * wb + 255) // 256 * 256
        ws, wsb = _workspace(need, dev)
        _check(_lib.ibp_preprocess(_ptr(dataset), n, v, wb, threshold, _ptr(mask), _ptr(bitval),
                                   _ptr(ws), wsb, _stream()))
    return mask, bitval


def preprocess_kmeans(dataset, num_clusters, threshold_=None, *, seed_rows=None):
    """src/preprocess.cu:88-139 -> (mask[C,V], bitval[C,V] on CUDA, clusters int32 pinned)."""
    _torch_check(dataset.device.type == "cuda" or dataset.is_pinned(),
                 "Input tensor must accessible by CUDA device (GPU or pinned memory)")
    _torch_check(dataset.dim() == 2, "Input tensor must be 2D [num_vecs x vec_size]")
    wb = dataset.element_size()
    _torch_check(wb in (4, 8), "Input tensor must be 4-byte or 8-byte datatype")
    _torch_check(dataset.is_contiguous(), "Input tensor must be contiguous")
    c = int(num_clusters)
    n, v = dataset.shape
    dev = _cuda_device(dataset)
    with torch.cuda.device(dev):
        masks = torch.empty((c, v), dtype=_INT_DTYPE[wb], device=dev)
        bitvals = torch.empty((c, v), dtype=_INT_DTYPE[wb], device=dev)
        clusters = torch.zeros(n, dtype=torch.int32, pin_memory=True)
        need = _lib.ibp_preprocess_kmeans_workspace_size(n, v, wb, c)
        if dataset.device.type != "cuda" and _stage_budget(n * v * wb, dev):
            need += (n * v * wb + 255) // 256 * 256
        ws, wsb = _workspace(need, dev)
        seeds = None
        if seed_rows is not None:
            seeds = np.ascontiguousarray(np.asarray(seed_rows, dtype=np.int64))
        _check(_lib.ibp_preprocess_kmeans(
            _ptr(dataset), n, v, wb, c,
            None if seeds is None else seeds.ctypes.data, _ptr(masks), _ptr(bitvals),
            _ptr(clusters), _ptr(ws), wsb, _stream()))
        # the reference returns after cudaDeviceSynchronize; clusters is a host tensor
        torch.cuda.current_stream().synchronize()
    return masks, bitvals, clusters


def _index_arg(index_array_, what="Index array"):
    if index_array_ is None:
        return None
    idx = index_array_
    _torch_check(idx.device.type == "cuda" or idx.is_pinned(),
                 f"{what} must accessible by CUDA device (GPU or pinned memory)")
    _torch_check(idx.dim() == 1, "Index array should be 1D")
    return idx.to(torch.int64).contiguous()


def _codec_checks(dataset, mask, bitval, codec_only):
    _torch_check(dataset.device.type == "cuda" or dataset.is_pinned(),
                 "Input tensor must accessible by CUDA device (GPU or pinned memory)")
    _torch_check(dataset.dim() in (1, 2),
                 "Input tensor must be 1D [vec_size] or 2D [num_vecs x vec_size]")
    _torch_check(dataset.is_contiguous(), "Input tensor must be contiguous")
    _torch_check(_gpu_accessible(mask),
                 "Mask tensor must accessible by CUDA device (GPU or pinned memory)")
    _torch_check(_gpu_accessible(bitval),
                 "Bitval tensor must accessible by CUDA device (GPU or pinned memory)")
    wb = dataset.element_size()
    if codec_only:
        _torch_check(wb in (4, 8), "Input tensor must be 4-byte or 8-byte datatype")
    else:
        _torch_check(wb in (1, 2, 4, 8), "Input tensor must be 1, 2, 4, or 8-byte datatype")
    _torch_check(mask.element_size() == wb and bitval.element_size() == wb,
                 "Mask and bitval tensors must have the same datatype size (4-byte or 8-byte) "
                 "as input dataset")
    n = 1 if dataset.dim() == 1 else dataset.shape[0]
    v = dataset.shape[0] if dataset.dim() == 1 else dataset.shape[1]
    return n, v, wb


def get_compress_size(dataset, mask, bitval, index_array_=None, compress_ctr_=None):
    """src/compress.cu:25-174 -> int64 compressed bytes per row (non-blocking)."""
    n, v, wb = _codec_checks(dataset, mask, bitval, codec_only=False)
    idx = _index_arg(index_array_)
    nrows = n if idx is None else idx.shape[0]
    ctr = None
    if compress_ctr_ is not None:
        ctr = compress_ctr_
        _torch_check(ctr.device.type == "cuda" or ctr.is_pinned(),
                     "Compress ctr must accessible by CUDA device (GPU or pinned memory)")
        _torch_check(ctr.dim() == 1 and ctr.shape[0] == 1, "Compress ctr should be a single element")
    dev = _cuda_device(dataset, mask, idx)
    with torch.cuda.device(dev):
        if dataset.device.type != "cuda":  # pinned from the start: no pageable copy
            sizes = torch.empty(nrows, dtype=torch.int64, pin_memory=True)
        else:
            sizes = torch.empty(nrows, dtype=torch.int64, device=dataset.device)
        total = None
        if ctr is not None:
            total = ctr if (ctr.device.type == "cuda" and ctr.dtype == torch.int64) else \
                ctr.to(device=dev, dtype=torch.int64, non_blocking=True)
        _check(_lib.ibp_get_compress_size(_ptr(dataset), n, v, wb, _ptr(mask), _ptr(bitval),
                                          _ptr(idx), -1 if idx is None else nrows, _ptr(sizes),
                                          _ptr(total), _stream()))
        if ctr is not None and total is not ctr:
            ctr.copy_(total, non_blocking=True)
    return sizes


def compress_inplace(dataset, mask, bitval, index_array_=None):
    """src/compress.cu:176-236 -> int32 bitmask on CUDA; dataset rows rewritten in place."""
    n, v, wb = _codec_checks(dataset, mask, bitval, codec_only=True)
    idx = _index_arg(index_array_)
    nrows = n if idx is None else idx.shape[0]
    dev = _cuda_device(dataset, mask, idx)
    with torch.cuda.device(dev):
        bitmask = torch.zeros((nrows + 31) // 32, dtype=torch.int32, device=dev)
        need = _lib.ibp_compress_inplace_workspace_size(nrows, v, wb, 0 if idx is None else 1)
        ws, wsb = _workspace(need, dev)
        _check(_lib.ibp_compress_inplace(_ptr(dataset), n, v, wb, _ptr(mask), _ptr(bitval),
                                         _ptr(idx), -1 if idx is None else nrows,
                                         _ptr(bitmask), _ptr(ws), wsb, _stream()))
        if dataset.device.type != "cuda":
            torch.cuda.current_stream().synchronize()
    return bitmask


def compress_condensed(dataset, mask, bitval, index_array_=None):
    """src/compress.cu:238-313 -> (condensed words, inclusive byte offsets int64)."""
    n, v, wb = _codec_checks(dataset, mask, bitval, codec_only=True)
    idx = _index_arg(index_array_)
    nrows = n if idx is None else idx.shape[0]
    dev = _cuda_device(dataset, mask, idx)
    with torch.cuda.device(dev):
        offs = torch.empty(nrows, dtype=torch.int64, device=dev)
        total = torch.zeros(1, dtype=torch.int64, device=dev)
        _check(_lib.ibp_get_compress_size(_ptr(dataset), n, v, wb, _ptr(mask), _ptr(bitval),
                                          _ptr(idx), -1 if idx is None else nrows, _ptr(offs),
                                          None, _stream()))
        ws, wsb = _workspace(_lib.ibp_condensed_offsets_workspace_size(nrows), dev)
        _check(_lib.ibp_condensed_offsets(_ptr(offs), nrows, _ptr(total), _ptr(ws), wsb,
                                          _stream()))
        nbytes = int(total.item())  # synchronises, as the reference does
        if dataset.device.type != "cuda":
            comp = torch.zeros(nbytes // wb, dtype=dataset.dtype, pin_memory=True)
        else:
            comp = torch.zeros(nbytes // wb, dtype=dataset.dtype, device=dataset.device)
        ws2, wsb2 = _workspace(_lib.ibp_compress_condensed_workspace_size(v, wb), dev)
        _check(_lib.ibp_compress_condensed(_ptr(dataset), n, v, wb, _ptr(mask), _ptr(bitval),
                                           _ptr(idx), -1 if idx is None else nrows, _ptr(offs),
                                           _ptr(comp), _ptr(ws2), wsb2, _stream()))
        if dataset.device.type != "cuda":
            offs = offs.to("cpu").pin_memory()
            torch.cuda.current_stream().synchronize()
    return comp, offs


def _raise_on_status(ws, what):
    """check=True: read the call's device status word (blocking) and raise for the rows the
    call could not produce (an out-of-range index, a row whose bitmap does not fit its
    mask); bit 3 (a repeat decoded its own row after waiting) leaves the output correct."""
    if ws is None:
        return
    import ctypes
    st = torch.zeros(1, dtype=torch.int32)
    _check(_lib.ibp_read_status(_ptr(ws), ctypes.c_void_p(st.data_ptr()), _stream()))
    bits = int(st[0])
    problems = []
    if bits & 1:
        problems.append("an index was out of range (its output rows were not written)")
    if bits & 2:
        problems.append("a row marked compressed has a bitmap that does not fit the mask "
                        "(the bitmask/mask do not belong to the data; its output row was not "
                        "written)")
    if problems:
        raise RuntimeError(f"{what}: " + "; ".join(problems))


def decompress_fetch(comp_dataset, mask, bitval, bitmask, out_device, comp_len_=None,
                     index_array_=None, nblks_=None, nthreads_=None, impl_=None,
                     output_tensor=None, *, check=False):
    """src/decompress.cu:10-156 -> decompressed rows (non-blocking).

    check=True (keyword only; no counterpart in the reference) waits for the call and raises
    RuntimeError when an index was out of range or a row could not be decoded; the default
    leaves those rows unwritten without a host synchronisation (print_debug(True) prints a
    message instead)."""
    _torch_check(comp_dataset.is_cuda or comp_dataset.is_pinned(),
                 "Input tensor must accessible by CUDA device (GPU or pinned memory)")
    dim = comp_dataset.dim()
    _torch_check(dim in (1, 2),
                 "Input tensor must be 1D [vec_size] or 2D [num_vecs x vec_size] got "
                 f"{dim}")
    _torch_check(comp_dataset.is_contiguous(), "Input tensor must be contiguous")
    _torch_check(mask.is_cuda or mask.is_pinned(),
                 "Mask tensor must accessible by CUDA device (GPU or pinned memory)")
    _torch_check(bitval.is_cuda or bitval.is_pinned(),
                 "Bitval tensor must accessible by CUDA device (GPU or pinned memory)")
    wb = comp_dataset.element_size()
    _torch_check(wb in (4, 8), "Input tensor must be 4-byte or 8-byte datatype")
    _torch_check(mask.element_size() == wb and bitval.element_size() == wb,
                 "Mask and bitval tensors must have the same datatype size (4-byte or 8-byte) "
                 "as input dataset")
    if bitmask.dtype != torch.int32:
        raise RuntimeError(f"expected scalar type Int but found {bitmask.dtype}")
    shape = comp_dataset.shape
    n, v = (1, shape[0]) if dim == 1 else (shape[0], shape[1])
    if not isinstance(out_device, torch.device):
        out_device = torch.device(out_device)
    if out_device.type == "cuda" and out_device.index is None:
        out_device = torch.device("cuda", _get_device())
    idx = None
    if index_array_ is not None:
        _torch_check(index_array_.is_cuda,
                     "Index array must accessible by CUDA device (GPU or pinned memory)")
        _torch_check(index_array_.dim() == 1, "Index array should be 1D")
        idx = index_array_
        if idx.dtype != torch.int64:
            idx = idx.to(torch.int64)
        if not idx.is_contiguous():
            idx = idx.contiguous()
    nrows = n if idx is None else idx.shape[0]
    impl = -1 if impl_ is None else int(impl_)
    comp_len = v
    if comp_len_ is not None and int(comp_len_) > 0:
        comp_len = int(comp_len_)
    if output_tensor is not None:
        _torch_check(output_tensor.device == out_device,
                     "Output tensor device does not match specified output device")
        _torch_check(output_tensor.dtype == comp_dataset.dtype,
                     "Output tensor dtype does not match input dataset dtype")
        _torch_check(output_tensor.shape[0] == nrows and output_tensor.shape[1] == v,
                     "Output tensor shape does not match expected decompressed shape")
        out = output_tensor
    else:
        out = torch.empty((nrows, v), dtype=comp_dataset.dtype, device=out_device,
                          pin_memory=out_device.type != "cuda")
    if out_device.type != "cuda" and not out.is_pinned():
        out = out.pin_memory()
    dev = _cuda_device(comp_dataset, mask, idx, out)
    cur = _get_device()
    if dev.index is not None and dev.index != cur:
        with torch.cuda.device(dev):
            return _fetch_call(comp_dataset, n, v, wb, mask, bitval, bitmask, idx, nrows,
                               comp_len, out, nblks_, nthreads_, impl, dev, dev.index, check)
    return _fetch_call(comp_dataset, n, v, wb, mask, bitval, bitmask, idx, nrows, comp_len,
                       out, nblks_, nthreads_, impl, dev, cur, check)


def _fetch_call(comp_dataset, n, v, wb, mask, bitval, bitmask, idx, nrows, comp_len, out,
                nblks_, nthreads_, impl, dev, dev_index, check):
    need = _lib.ibp_decompress_fetch_workspace_size(nrows, v, wb, 0 if idx is None else 1)
    ws, wsb = _workspace(need, dev)
    stream = _stream_of(dev_index)
    _check(_lib.ibp_decompress_fetch(
        comp_dataset.data_ptr(), n, v, wb, mask.data_ptr(), bitval.data_ptr(),
        bitmask.data_ptr(), None if idx is None else idx.data_ptr(),
        -1 if idx is None else nrows, comp_len, out.data_ptr(),
        -1 if nblks_ is None else int(nblks_),
        -1 if nthreads_ is None else int(nthreads_), impl,
        None if ws is None else ws.data_ptr(), wsb, stream))
    if check:
        _raise_on_status(ws, "decompress_fetch")
    elif _debug and ws is not None:
        st = torch.zeros(1, dtype=torch.int32)
        import ctypes
        _check(_lib.ibp_read_status(_ptr(ws), ctypes.c_void_p(st.data_ptr()), stream))
        if int(st[0]) & 1:
            print("[ibp] decompress_fetch: an index was out of range; its rows were skipped")
    return out


def decompress_fetch_condensed(comp, offsets, mask, bitval, vec_size, out_device,
                               index_array_=None, output_tensor=None, *, check=False):
    """Rows of the condensed layout written by compress_condensed (no reference
    counterpart: the reference writes this layout but cannot read it back on the GPU).

    comp: the condensed words (1-D, device or pinned host); offsets: the inclusive byte
    offsets compress_condensed returned (int64, one per row; device, or pinned host).
    Returns [len(index) or num_rows, vec_size] decompressed rows (non-blocking; check=True
    waits and raises for out-of-range indices and rows that cannot be decoded)."""
    _torch_check(comp.device.type == "cuda" or comp.is_pinned(),
                 "Input tensor must accessible by CUDA device (GPU or pinned memory)")
    _torch_check(comp.is_contiguous(), "Input tensor must be contiguous")
    _torch_check(_gpu_accessible(offsets),
                 "Offsets tensor must accessible by CUDA device (GPU or pinned memory)")
    _torch_check(offsets.dtype == torch.int64 and offsets.dim() == 1 and offsets.is_contiguous(),
                 "Offsets tensor must be a contiguous 1D int64 tensor")
    _torch_check(_gpu_accessible(mask),
                 "Mask tensor must accessible by CUDA device (GPU or pinned memory)")
    _torch_check(_gpu_accessible(bitval),
                 "Bitval tensor must accessible by CUDA device (GPU or pinned memory)")
    wb = comp.element_size()
    _torch_check(wb in (4, 8), "Input tensor must be 4-byte or 8-byte datatype")
    _torch_check(mask.element_size() == wb and bitval.element_size() == wb,
                 "Mask and bitval tensors must have the same datatype size (4-byte or 8-byte) "
                 "as input dataset")
    v = int(vec_size)
    _torch_check(mask.numel() >= v and bitval.numel() >= v,
                 "Mask and bitval tensors must hold vec_size words")
    n = offsets.shape[0]
    out_device = torch.device(out_device)
    if out_device.type == "cuda" and out_device.index is None:
        out_device = torch.device("cuda", torch.cuda.current_device())
    idx = None
    if index_array_ is not None:
        _torch_check(index_array_.device.type == "cuda",
                     "Index array must accessible by CUDA device (GPU or pinned memory)")
        _torch_check(index_array_.dim() == 1, "Index array should be 1D")
        idx = index_array_.to(torch.int64).contiguous()
    nrows = n if idx is None else idx.shape[0]
    if output_tensor is not None:
        _torch_check(output_tensor.device == out_device,
                     "Output tensor device does not match specified output device")
        _torch_check(output_tensor.dtype == comp.dtype,
                     "Output tensor dtype does not match input dataset dtype")
        _torch_check(output_tensor.shape[0] == nrows and output_tensor.shape[1] == v,
                     "Output tensor shape does not match expected decompressed shape")
        out = output_tensor
    else:
        out = torch.empty((nrows, v), dtype=comp.dtype, device=out_device,
                          pin_memory=out_device.type != "cuda")
    if out_device.type != "cuda" and not out.is_pinned():
        out = out.pin_memory()
    dev = _cuda_device(comp, mask, idx, out)
    with torch.cuda.device(dev):
        need = _lib.ibp_decompress_fetch_workspace_size(nrows, v, wb, 0 if idx is None else 1)
        ws, wsb = _workspace(need, dev)
        _check(_lib.ibp_decompress_fetch_condensed(
            _ptr(comp), comp.numel(), _ptr(offsets), n, v, wb, _ptr(mask), _ptr(bitval), _ptr(idx),
            -1 if idx is None else nrows, _ptr(out), _ptr(ws), wsb, _stream()))
        if check:
            _raise_on_status(ws, "decompress_fetch_condensed")
        elif _debug and ws is not None:
            st = torch.zeros(1, dtype=torch.int32)
            import ctypes
            _check(_lib.ibp_read_status(_ptr(ws), ctypes.c_void_p(st.data_ptr()), _stream()))
            if int(st[0]) & 3:
                print("[ibp] decompress_fetch_condensed: bad index or corrupt row; skipped")
    return out


def read_shared(filename, shape, dtype):
    """src/ibp_api.cu:52-122: file contents in a new shared-memory CPU tensor."""
    t = torch.empty(list(shape), dtype=dtype).share_memory_()
    nbytes = t.numel() * t.element_size()
    buf = t.reshape(-1).view(torch.uint8).numpy() if nbytes else None
    with open(filename, "rb") as f:
        off = 0
        chunk = 1 << 30
        while off < nbytes:
            got = f.readinto(memoryview(buf[off:off + chunk]))
            if not got:
                break
            off += got
    return t
