"""Drop-in `ibp` package: the reference's Python front end (ibp/__init__.py:1-41), served by
the B200 engine.

Put the `dropin/` directory of this repository on sys.path (PYTHONPATH) ahead of any other
`ibp`, and existing code that does `import torch; import ibp` runs unmodified on the engine:
the same functions, argument order and defaults, each forwarding to the package
invariantbitpacking_b200 (whose work runs in libibp_b200.so).  The repository root is added
to sys.path when the engine package is not importable on its own.
"""
import os
import sys

import torch  # noqa: F401  (the reference imports torch before its extension as well)

try:
    import invariantbitpacking_b200 as _engine
except ImportError:
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))
    import invariantbitpacking_b200 as _engine

import ibp_cuda  # noqa: E402  (dropin/ibp_cuda.py: the engine's mirror of the extension)

ibp_cuda.print_debug(False)


def print_debug(flag):
    _engine.print_debug(flag)


def preprocess(dataset, threshold=None):
    """Returns mask and bitval tensors."""
    return _engine.preprocess(dataset, threshold)


def preprocess_kmeans(dataset, centroids, threshold=None):
    """Returns per-cluster mask and bitval tensors and each row's cluster."""
    return _engine.preprocess_kmeans(dataset, centroids, threshold)


def get_compress_size(dataset, mask, bitval, index_arr=None, compress_total=None):
    return _engine.get_compress_size(dataset, mask, bitval, index_arr, compress_total)


def get_single_compress_len(dataset, mask, bitval, index_arr=None):
    return _engine.get_single_compress_len(dataset, mask, bitval, index_arr)


def compress_inplace(dataset, mask, bitval, index_arr=None):
    """Returns the bitmask marking compressed rows."""
    return _engine.compress_inplace(dataset, mask, bitval, index_arr)


def compress(dataset, mask, bitval, index_arr=None):
    return _engine.compress(dataset, mask, bitval, index_arr)


def decompress_fetch(comp_dataset, mask, bitval, bitmask, device, comp_len=None,
                     index_arr=None, nblks=None, nthds=None, imp=None, output_tensor=None):
    return _engine.decompress_fetch(comp_dataset, mask, bitval, bitmask, device, comp_len,
                                    index_arr, nblks, nthds, imp, output_tensor)
