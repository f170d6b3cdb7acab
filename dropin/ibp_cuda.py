"""Drop-in `ibp_cuda` module: the reference's compiled extension (src/ibp_api.cu:124-135),
served by the B200 engine.

With the `dropin/` directory of this repository on sys.path, `import ibp_cuda` (and the
`import ibp_cuda as ibp` of the reference's throughput scripts) gets the engine's mirror of
the extension: the same eight functions with the same positional signatures, output
placement and argument checks (invariantbitpacking_b200.ibp_cuda).
"""
import os
import sys

try:
    from invariantbitpacking_b200 import ibp_cuda as _mirror
except ImportError:
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from invariantbitpacking_b200 import ibp_cuda as _mirror

print_debug = _mirror.print_debug
preprocess = _mirror.preprocess
preprocess_kmeans = _mirror.preprocess_kmeans
get_compress_size = _mirror.get_compress_size
compress_inplace = _mirror.compress_inplace
compress_condensed = _mirror.compress_condensed
decompress_fetch = _mirror.decompress_fetch
read_shared = _mirror.read_shared

__all__ = ["print_debug", "preprocess", "preprocess_kmeans", "get_compress_size",
           "compress_inplace", "compress_condensed", "decompress_fetch", "read_shared"]
