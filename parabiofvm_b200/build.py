"""Build the CUDA library ``parabiofvm_b200/_lib/libbfvm_cuda.so`` in-tree with nvcc for sm_100a,
and the C++20 host API over it, ``parabiofvm_b200/_lib/libbiofvm_b200.so`` (``host/``).

Each translation unit is compiled to an object in ``parabiofvm_b200/_build`` (in parallel, only when
its sources changed) and linked into one shared library that exports the C ABI of
``include/bfvm.h``.  Host code is compiled without floating-point contraction so the coefficient
precompute rounds exactly like the reference's.
"""

from __future__ import annotations

import concurrent.futures
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIBDIR = os.path.join(PKG, "_lib")
LIB = os.path.join(LIBDIR, "libbfvm_cuda.so")
HOST = os.path.join(PKG, "host")
HOST_LIB = os.path.join(LIBDIR, "libbiofvm_b200.so")
HOST_INCLUDE = os.path.join(HOST, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC,-ffp-contract=off",
              "-Xptxas", "-warn-spills", "-I" + os.path.join(ROOT, "include")]


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs.append(os.path.join(ROOT, "include", "bfvm.h"))
    return hs


def _compile(src, verbose):
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    newest_dep = max(os.path.getmtime(p) for p in [src] + _headers())
    if os.path.exists(obj) and os.path.getmtime(obj) >= newest_dep:
        return obj, ""
    cmd = [_nvcc(), *ARCH, *NVCC_FLAGS, "-c", src, "-o", obj]
    if src.endswith(".cpp"):
        cmd.insert(1, "-x")
        cmd.insert(2, "cu")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj, (r.stdout + r.stderr) if verbose else ""


def build(verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    srcs = sources()
    with concurrent.futures.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        results = list(ex.map(lambda s: _compile(s, verbose), srcs))
    objs = [o for o, _ in results]
    for _, log in results:
        if log:
            print(log, file=sys.stderr)
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [_nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    build_host()
    return LIB


def _cxx():
    for cand in (os.environ.get("HOST_CXX"), "g++", shutil.which("g++")):
        if cand and shutil.which(cand):
            return cand
    raise RuntimeError("g++ not found")


def build_host() -> str:
    """The C++20 host API (include/BioFVM/*.h) as one shared library linked to the CUDA library."""
    srcs = sorted(os.path.join(HOST, "src", f) for f in os.listdir(os.path.join(HOST, "src")) if f.endswith(".cpp"))
    deps = srcs + [os.path.join(HOST_INCLUDE, "BioFVM", f) for f in os.listdir(os.path.join(HOST_INCLUDE, "BioFVM"))]
    deps += [LIB, os.path.join(ROOT, "include", "bfvm.h")]
    if os.path.exists(HOST_LIB) and os.path.getmtime(HOST_LIB) >= max(os.path.getmtime(p) for p in deps):
        return HOST_LIB
    cmd = [_cxx(), "-std=c++20", "-O2", "-fPIC", "-shared", "-Wall", "-Wextra", "-I" + HOST_INCLUDE,
           "-o", HOST_LIB, *srcs, "-L" + LIBDIR, "-lbfvm_cuda", "-Wl,-rpath,$ORIGIN"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"host library build failed:\n{r.stdout}\n{r.stderr}")
    return HOST_LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
