"""Build the reference IBP extension (``ibp_cuda``) for sm_100a, from its own sources.

Test infrastructure only.  This compiles the four translation units of the
reference PyTorch extension (src/ibp_api.cu, src/preprocess.cu, src/compress.cu,
src/decompress.cu with the header-only kernels under include/) exactly where
they lie under the read-only reference checkout, with the flags of the
reference's setup.py (-O3 -std=c++17 --use_fast_math -lineinfo) but for
sm_100a instead of sm_70/sm_80.  Objects and the linked module go to
``oracle/_ref/`` only (git-ignored; it travels with the repository snapshot to
a GPU box, where tests/golden/make_golden.py runs it to dump golden vectors).

Nothing in the product imports this module or its output.

Usage: python oracle/build_ref.py --ref <reference checkout> [--jobs 4]
       (or set IBP_REFERENCE_DIR to the checkout and omit --ref)
"""
import argparse
import concurrent.futures as cf
import os
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
SOURCES = ["src/ibp_api.cu", "src/preprocess.cu", "src/compress.cu", "src/decompress.cu"]
INCLUDES = ["include", "include/preproc", "include/misc", "include/compress"]


def module_path():
    return os.path.join(OUT, "ibp_cuda" + sysconfig.get_config_var("EXT_SUFFIX"))


def _flags():
    import torch
    import torch.utils.cpp_extension as ce
    incs = ce.include_paths(device_type="cuda") + [sysconfig.get_paths()["include"]]
    abi = int(torch._C._GLIBCXX_USE_CXX11_ABI)
    return incs, abi


def reference_dir():
    """The reference checkout named by IBP_REFERENCE_DIR, or None."""
    ref = os.environ.get("IBP_REFERENCE_DIR")
    return ref if ref and os.path.isdir(os.path.join(ref, "src")) else None


def build(ref=None, jobs=4, quiet=False):
    ref = ref or reference_dir()
    if not ref:
        raise FileNotFoundError("no reference checkout: pass --ref or set IBP_REFERENCE_DIR")
    if not os.path.isdir(os.path.join(ref, "src")):
        raise FileNotFoundError(f"reference sources not found under {ref}")
    os.makedirs(os.path.join(OUT, "obj"), exist_ok=True)
    target = module_path()
    srcs = [os.path.join(ref, s) for s in SOURCES]
    newest_src = max(os.path.getmtime(s) for s in srcs)
    if os.path.exists(target) and os.path.getmtime(target) > newest_src:
        return target
    incs, abi = _flags()
    nvcc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    base = [nvcc, "-O3", "-std=c++17", "--use_fast_math", "-lineinfo",
            "-gencode", "arch=compute_100a,code=sm_100a",
            "-Xcompiler", "-fPIC", f"-D_GLIBCXX_USE_CXX11_ABI={abi}",
            "-DTORCH_EXTENSION_NAME=ibp_cuda", "-DTORCH_API_INCLUDE_EXTENSION_H",
            "-w"]
    base += [f"-I{os.path.join(ref, i)}" for i in INCLUDES]
    base += [f"-I{i}" for i in incs]

    def one(src):
        obj = os.path.join(OUT, "obj", os.path.basename(src) + ".o")
        cmd = base + ["-c", src, "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{r.stderr[-4000:]}")
        return obj

    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(one, srcs))
    import torch.utils.cpp_extension as ce
    libdirs = ce.library_paths(device_type="cuda")
    cmd = ["g++", "-shared", "-o", target] + objs
    cmd += [f"-L{d}" for d in libdirs] + [f"-Wl,-rpath,{d}" for d in libdirs]
    cmd += ["-lc10", "-ltorch", "-ltorch_cpu", "-ltorch_python", "-lc10_cuda", "-ltorch_cuda", "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stderr[-4000:]}")
    if not quiet:
        print("built", target)
    return target


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=None,
                    help="reference checkout (default: $IBP_REFERENCE_DIR)")
    ap.add_argument("--jobs", type=int, default=4)
    a = ap.parse_args()
    build(a.ref, a.jobs)
    sys.exit(0)
