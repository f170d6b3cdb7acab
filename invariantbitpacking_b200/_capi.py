"""ctypes binding of libibp_b200.so (the C ABI declared in include/ibp_b200.h).

The shared library is the product: every computation runs in its CUDA kernels.  If the
library is missing this module raises at import -- there is no CPU fallback.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libibp_b200.so")

IBP_OK = 0
IBP_ERR_ARGUMENT = 1
IBP_ERR_WORKSPACE = 2
IBP_ERR_CUDA = 3
IBP_ERR_UNSUPPORTED = 4

_P = ctypes.c_void_p
_I64 = ctypes.c_int64
_I32 = ctypes.c_int32
_INT = ctypes.c_int
_SZ = ctypes.c_size_t
_F = ctypes.c_float

# name -> (restype, argtypes); mirrors include/ibp_b200.h
SIGNATURES = {
    "ibp_last_error": (ctypes.c_char_p, []),
    "ibp_abi_version": (_INT, []),
    "ibp_set_debug": (None, [_INT]),
    "ibp_read_status": (_INT, [_P, _P, _P]),
    "ibp_set_fetch_dedup": (_INT, [_I32]),
    "ibp_set_repeat_wait_limit": (_INT, [_I32]),
    "ibp_profile_enable": (_INT, [_I32]),
    "ibp_profile_take": (_I32, [_P, _I32]),
    "ibp_kernel_launch_count": (ctypes.c_ulonglong, []),
    "ibp_preprocess_workspace_size": (_SZ, [_I64, _I64, _INT, _F]),
    "ibp_preprocess": (_INT, [_P, _I64, _I64, _INT, _F, _P, _P, _P, _SZ, _P]),
    "ibp_preprocess_kmeans_workspace_size": (_SZ, [_I64, _I64, _INT, _I32]),
    "ibp_preprocess_kmeans": (_INT, [_P, _I64, _I64, _INT, _I32, _P, _P, _P, _P, _P, _SZ, _P]),
    "ibp_get_compress_size": (_INT, [_P, _I64, _I64, _INT, _P, _P, _P, _I64, _P, _P, _P]),
    "ibp_compress_inplace_workspace_size": (_SZ, [_I64, _I64, _INT, _INT]),
    "ibp_compress_inplace": (_INT, [_P, _I64, _I64, _INT, _P, _P, _P, _I64, _P, _P, _SZ, _P]),
    "ibp_condensed_offsets_workspace_size": (_SZ, [_I64]),
    "ibp_condensed_offsets": (_INT, [_P, _I64, _P, _P, _SZ, _P]),
    "ibp_compress_condensed_workspace_size": (_SZ, [_I64, _INT]),
    "ibp_compress_condensed": (_INT, [_P, _I64, _I64, _INT, _P, _P, _P, _I64, _P, _P, _P, _SZ,
                                      _P]),
    "ibp_decompress_fetch_workspace_size": (_SZ, [_I64, _I64, _INT, _INT]),
    "ibp_decompress_fetch": (_INT, [_P, _I64, _I64, _INT, _P, _P, _P, _P, _I64, _I32, _P, _I32,
                                    _I32, _I32, _P, _SZ, _P]),
    "ibp_sets_registry_size": (_SZ, [_P, _I32, _INT]),
    "ibp_sets_register": (_INT, [_P, _I32, _INT, _P, _SZ, _P]),
    "ibp_batch_fetch_workspace_size": (_SZ, []),
    "ibp_batch_fetch": (_INT, [_P, _P, _P, _I32, _P, _SZ, _P]),
    "ibp_batch_autotune": (_INT, [_P, _P, _P, _I32, _P, _SZ, _P, _P]),
    "ibp_read_rows_probe": (_INT, [_P, _I64, _P, _I64, _I32, _P, _SZ, _P]),
    "ibp_decompress_fetch_condensed": (_INT, [_P, _I64, _P, _I64, _I64, _INT, _P, _P, _P, _I64,
                                               _P, _P, _SZ, _P]),
    "ibp_batch_fetch_sorted_workspace_size": (_SZ, [_I64, _I32]),
    "ibp_batch_fetch_sorted": (_INT, [_P, _P, _I32, _I64, _P, _SZ, _P]),
    "ibp_batch_fetch_hashed_workspace_size": (_SZ, [_I64]),
    "ibp_batch_fetch_hashed": (_INT, [_P, _P, _I32, _I64, _P, _SZ, _P]),
    "ibp_server_create": (_INT, [_P, _P, _I32, _INT, _P, _SZ, _I64, _I32, _I32, _P]),
    "ibp_server_submit": (_INT, [_P, _I32, _P, _I64, _I64, _P]),
    "ibp_server_wait": (_INT, [_P, _I64, _I32, _P, _P]),
    "ibp_server_release": (_INT, [_P, _I64]),
    "ibp_server_cancel": (_INT, [_P, _I64]),
    "ibp_server_set_batch_limits": (_INT, [_P, _I64, _I64]),
    "ibp_server_set_dedup": (_INT, [_P, _I32]),
    "ibp_server_stats": (_INT, [_P, _P]),
    "ibp_server_destroy": (_INT, [_P]),
    "ibp_decompress_fetch_noalloc": (_INT, [_P, _I64, _I64, _INT, _P, _P, _P, _P, _I64, _I32,
                                            _P, _P]),
    "ibp_decompress_fetch_noalloc_status": (_INT, [_P, _P]),
}

# Bytes of the static scratch behind ibp_decompress_fetch_noalloc (IBP_NOALLOC_SCRATCH_BYTES)
NOALLOC_SCRATCH_BYTES = 4194304


class SetDesc(ctypes.Structure):
    """ibp_set_desc"""
    _fields_ = [("comp", _P), ("num_vecs", _I64), ("vec_size", _I64), ("mask", _P),
                ("bitval", _P), ("bitmask", _P), ("comp_len", _I32), ("reserved", _I32)]


class Request(ctypes.Structure):
    """ibp_request (48 bytes, the layout the batch kernel reads from device memory)"""
    _fields_ = [("set", _I32), ("reserved", _I32), ("index", _P), ("first", _I64),
                ("count", _I64), ("out", _P)]


class IBPError(RuntimeError):
    """An engine call failed; the message is the engine's own (ibp_last_error)."""

    def __init__(self, status, msg):
        super().__init__(msg)
        self.status = status


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python invariantbitpacking_b200/build.py` "
            "(the engine has no CPU fallback)")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


lib = _load()


def check(status):
    """Raise IBPError (a RuntimeError) for a failing status."""
    if status != IBP_OK:
        msg = lib.ibp_last_error().decode(errors="replace")
        raise IBPError(status, msg or f"ibp error {status}")


def exported_symbols():
    return sorted(SIGNATURES)
