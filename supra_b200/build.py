"""Builds libsupra_b200.so (all CUDA kernels + the C ABI) in-tree for sm_100a.

    python -m supra_b200.build [--verbose]

Objects go to supra_b200/_build/, the library to supra_b200/lib/libsupra_b200.so.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libsupra_b200.so")

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
HOST_CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off", "-ccbin", HOST_CXX,
          f"-I{os.path.join(REPO, 'include')}", f"-I{CSRC}", "--expt-relaxed-constexpr"]


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def _compile(src: str, verbose: bool) -> str:
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    deps = [src] + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    deps.append(os.path.join(REPO, "include", "supra_b200.h"))
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(d) for d in deps):
        return obj
    cmd = [NVCC] + ARCH + COMMON + ["-c", src, "-o", obj]
    if src.endswith(".cpp"):
        cmd = [NVCC, "-x", "c++"] + COMMON + ["-c", src, "-o", obj]
    elif verbose:
        cmd += ["-Xptxas", "-v"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{res.stdout}\n{res.stderr}")
    if verbose and res.stderr:
        print(res.stderr)
    return obj


def build(verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    srcs = sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 2)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(o) for o in objs):
        return LIB
    cmd = [NVCC] + ARCH + ["-shared", "-Xcompiler", "-fPIC", "-ccbin", HOST_CXX, "-o", LIB + ".tmp"] + objs + ["-lcuda"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    os.replace(LIB + ".tmp", LIB)
    return LIB


TORCH_EXT_SRC = os.path.join(HERE, "torch_ext", "autograd_ops.cpp")
TORCH_EXT = os.path.join(LIBDIR, "supra_b200_torch_ops.so")


def build_torch_ops() -> str:
    """Builds the libtorch autograd operators (torch.ops.supra_b200.*) in-tree, linked to the library
    by rpath. Needs torch's C++ headers; no device code, so it builds without a GPU."""
    import torch.utils.cpp_extension as ext

    lib = build()
    if os.path.exists(TORCH_EXT) and os.path.getmtime(TORCH_EXT) >= max(os.path.getmtime(TORCH_EXT_SRC),
                                                                         os.path.getmtime(lib)):
        return TORCH_EXT
    bdir = os.path.join(BUILD, "torch_ops")
    os.makedirs(bdir, exist_ok=True)
    ext.load(name="supra_b200_torch_ops", sources=[TORCH_EXT_SRC], build_directory=bdir, with_cuda=True,
             extra_include_paths=[os.path.join(REPO, "include")],
             extra_ldflags=[f"-L{LIBDIR}", "-lsupra_b200", f"-Wl,-rpath,{LIBDIR}", "-Wl,-rpath,$ORIGIN"],
             is_python_module=False, verbose=False)
    shutil.copy2(os.path.join(bdir, "supra_b200_torch_ops.so"), TORCH_EXT)
    return TORCH_EXT


if __name__ == "__main__":
    print(build(verbose="--verbose" in sys.argv))
    if "--torch-ops" in sys.argv:
        print(build_torch_ops())
