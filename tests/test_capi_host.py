"""Host-side checks that need no GPU: the C-ABI library loads and exports every symbol the
public header declares, argument errors come back as status codes with messages (never a
crash or exit), and the drop-in layer rejects bad tensors with the reference's messages."""
import os
import re

import numpy as np
import pytest
import torch

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(REPO, "include", "ibp_b200.h")


def header_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(ibp_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_header_symbol():
    from invariantbitpacking_b200 import _capi
    declared = header_functions()
    assert len(declared) >= 17
    for name in declared:
        assert hasattr(_capi.lib, name), name
    assert sorted(_capi.SIGNATURES) == declared


def test_abi_version():
    from invariantbitpacking_b200 import _capi
    assert _capi.lib.ibp_abi_version() == 1


def test_argument_errors_are_status_codes():
    from invariantbitpacking_b200 import _capi
    lib = _capi.lib
    st = lib.ibp_preprocess(None, 10, 10, 3, 0.9, None, None, None, 0, None)
    assert st == _capi.IBP_ERR_ARGUMENT
    assert b"1, 2, 4, or 8-byte" in lib.ibp_last_error()
    st = lib.ibp_decompress_fetch(None, 0, 0, 8, None, None, None, None, -1, -1, None, -1, -1, 3,
                                  None, 0, None)
    assert st == _capi.IBP_ERR_UNSUPPORTED
    assert b"impl 3" in lib.ibp_last_error()
    st = lib.ibp_compress_inplace(None, 4, 4, 2, None, None, None, -1, None, None, 0, None)
    assert st == _capi.IBP_ERR_ARGUMENT
    assert b"4-byte or 8-byte" in lib.ibp_last_error()
    st = lib.ibp_preprocess_kmeans(None, 5, 4, 8, 0, None, None, None, None, None, 0, None)
    assert st == _capi.IBP_ERR_ARGUMENT
    with pytest.raises(RuntimeError, match="4-byte or 8-byte"):
        _capi.check(lib.ibp_compress_inplace(None, 4, 4, 2, None, None, None, -1, None, None, 0,
                                             None))


def test_workspace_size_queries_are_host_arithmetic():
    from invariantbitpacking_b200 import _capi
    lib = _capi.lib
    a = lib.ibp_preprocess_workspace_size(1000, 64, 8, -1.0)
    b = lib.ibp_preprocess_workspace_size(1000, 64, 8, 0.9)
    assert a > b > 64 * 64 * 4  # counts + 7 vs 1 mask/bitval pairs
    assert lib.ibp_preprocess_kmeans_workspace_size(1000, 32, 8, 16) >= 16 * 32 * 64 * 4
    c0 = lib.ibp_compress_inplace_workspace_size(100, 64, 8, 0)
    c1 = lib.ibp_compress_inplace_workspace_size(100, 64, 8, 1)
    assert c1 - c0 >= 100 * 64 * 8


def test_sweep_thresholds_match_reference_float_loop():
    """The sweep visits the float32 sequence of the reference's `threshold += 0.05` loop."""
    t, seq = np.float32(0.7), []
    while t <= np.float32(1.0):
        seq.append(t)
        t = np.float32(np.float64(t) + 0.05)
    assert len(seq) == 7 and seq[-1] == np.float32(1.0)
    assert seq[4] == np.float32(0.90000004)


def test_dropin_rejects_unpinned_host_tensors_with_reference_messages():
    import invariantbitpacking_b200 as ibp
    x = torch.zeros((4, 8), dtype=torch.int64)  # pageable host memory
    m = torch.zeros(8, dtype=torch.int64)
    with pytest.raises(RuntimeError, match="Input tensor must accessible by CUDA device"):
        ibp.preprocess(x)
    with pytest.raises(RuntimeError, match="Input tensor must accessible by CUDA device"):
        ibp.get_compress_size(x, m, m)
    with pytest.raises(RuntimeError, match="Input tensor must accessible by CUDA device"):
        ibp.compress_inplace(x, m, m)
    with pytest.raises(RuntimeError, match="Input tensor must accessible by CUDA device"):
        ibp.decompress_fetch(x, m, m, torch.zeros(1, dtype=torch.int32), "cuda")


# Positional parameters of every export of the reference's extension module ibp_cuda
# (src/ibp_api.cu:20-40 declarations, :124-135 bindings; pybind11 gives none a default).
REF_EXTENSION_ARITY = {"print_debug": 1, "preprocess": 2, "preprocess_kmeans": 3,
                       "get_compress_size": 5, "compress_inplace": 4, "compress_condensed": 4,
                       "decompress_fetch": 11, "read_shared": 3}
# Positional parameters of the reference's `ibp` package (ibp/__init__.py:8-41).
REF_PACKAGE_PARAMS = {
    "preprocess": ["dataset", "threshold"],
    "preprocess_kmeans": ["dataset", "centroids", "threshold"],
    "get_compress_size": ["dataset", "mask", "bitval", "index_arr", "compress_total"],
    "get_single_compress_len": ["dataset", "mask", "bitval", "index_arr"],
    "compress_inplace": ["dataset", "mask", "bitval", "index_arr"],
    "compress": ["dataset", "mask", "bitval", "index_arr"],
    "decompress_fetch": ["comp_dataset", "mask", "bitval", "bitmask", "device", "comp_len",
                         "index_arr", "nblks", "nthds", "imp", "output_tensor"],
}


def _positional(fn):
    import inspect
    sig = inspect.signature(fn)
    return sig, [p for p in sig.parameters.values()
                 if p.kind in (p.POSITIONAL_ONLY, p.POSITIONAL_OR_KEYWORD)]


def _check_extension_arity(mod):
    for fn, n in REF_EXTENSION_ARITY.items():
        sig, pos = _positional(getattr(mod, fn))
        assert len(pos) == n, (fn, len(pos))
        sig.bind(*range(n))  # the reference's full positional call binds


def test_dropin_signatures_match_reference():
    """The package mirrors ibp/__init__.py's positional signatures, and its ibp_cuda mirrors
    the extension's: every export takes exactly the reference's positional arguments."""
    import invariantbitpacking_b200 as ibp
    for fn, params in REF_PACKAGE_PARAMS.items():
        _, pos = _positional(getattr(ibp, fn))
        assert [p.name for p in pos] == params, fn
    _check_extension_arity(ibp.ibp_cuda)


def test_dropin_directory_imports_as_ibp_and_ibp_cuda():
    """With dropin/ on sys.path, `import ibp` and `import ibp_cuda` (the reference's import
    lines) resolve to the engine, with the reference's signatures; checked in a fresh
    interpreter whose sys.path holds dropin/ but not the repository root."""
    import json
    import subprocess
    import sys
    code = r"""
import json, sys, inspect
import torch
import ibp
import ibp_cuda
import invariantbitpacking_b200.ibp_cuda as mirror
out = {"ibp_file": ibp.__file__, "ibp_cuda_file": ibp_cuda.__file__,
       "same": ibp_cuda.decompress_fetch is mirror.decompress_fetch,
       "pkg": {fn: [p.name for p in inspect.signature(getattr(ibp, fn)).parameters.values()]
               for fn in ("preprocess", "preprocess_kmeans", "get_compress_size",
                          "get_single_compress_len", "compress_inplace", "compress",
                          "decompress_fetch")},
       "ext": {fn: len([p for p in inspect.signature(getattr(ibp_cuda, fn)).parameters.values()
                        if p.kind in (p.POSITIONAL_ONLY, p.POSITIONAL_OR_KEYWORD)])
               for fn in ("print_debug", "preprocess", "preprocess_kmeans", "get_compress_size",
                          "compress_inplace", "compress_condensed", "decompress_fetch",
                          "read_shared")}}
print(json.dumps(out))
"""
    env = dict(os.environ, PYTHONPATH=os.path.join(REPO, "dropin"))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env,
                       cwd="/", timeout=300)
    assert r.returncode == 0, r.stderr[-3000:]
    got = json.loads(r.stdout.strip().splitlines()[-1])
    assert got["ibp_file"] == os.path.join(REPO, "dropin", "ibp", "__init__.py")
    assert got["ibp_cuda_file"] == os.path.join(REPO, "dropin", "ibp_cuda.py")
    assert got["same"]
    assert got["pkg"] == REF_PACKAGE_PARAMS
    assert got["ext"] == REF_EXTENSION_ARITY


def test_read_shared_round_trip(tmp_path):
    import invariantbitpacking_b200 as ibp
    a = np.arange(3 * 5, dtype=np.float32).reshape(3, 5)
    f = tmp_path / "t.bin"
    a.tofile(f)
    t = ibp.read_shared(str(f), [3, 5], torch.float32)
    assert t.is_shared() and np.array_equal(t.numpy(), a)


def test_set_fetch_dedup_modes():
    """The dedup knob is a host-side setting: names and numbers are accepted, anything else
    is refused by the Python layer and by the C ABI, and auto is restored."""
    import invariantbitpacking_b200 as ibp
    from invariantbitpacking_b200 import _capi
    try:
        for m in ("sort", "hash", "auto", 1, 2, 0):
            ibp.set_fetch_dedup(m)
        for bad in ("fast", 3, -1):
            with pytest.raises(ValueError):
                ibp.set_fetch_dedup(bad)
        with pytest.raises(_capi.IBPError):
            _capi.check(_capi.lib.ibp_set_fetch_dedup(7))
    finally:
        ibp.set_fetch_dedup("auto")


def test_noalloc_limit_constant_matches_header():
    from invariantbitpacking_b200 import _capi
    m = re.search(r"#define\s+IBP_NOALLOC_SCRATCH_BYTES\s+(\d+)", open(HEADER).read())
    assert m and int(m.group(1)) == _capi.NOALLOC_SCRATCH_BYTES == 4 << 20
    # the documented fit test: the workspace query of the regular entry point
    assert _capi.lib.ibp_decompress_fetch_workspace_size(80_000, 64, 8, 1) <= 4 << 20
    assert _capi.lib.ibp_decompress_fetch_workspace_size(120_000, 64, 8, 1) > 4 << 20
