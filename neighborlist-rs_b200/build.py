"""Build the CUDA library in-tree: neighborlist_rs/_lib/libnlb200.so (sm_100a).

    python neighborlist-rs_b200/build.py [--force]

Every .cu/.cpp under csrc/ is compiled to an object in _build/ (skipped when
up to date) and linked into one shared library exporting the C ABI declared
in include/neighborlist_b200.h.  nvcc cross-compiles for sm_100a without a
GPU.  Floating-point flags: -fmad=false for device code and
-ffp-contract=off for host code, so no multiply-add is ever fused (the
reference's f64 arithmetic never fuses either).
"""

from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
OUT_DIR = os.path.join(HERE, "neighborlist_rs", "_lib")
OUT = os.path.join(OUT_DIR, "libnlb200.so")
INCLUDE = os.path.join(ROOT, "include")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = shutil.which("nvcc") or os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "-fmad=false", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-O2", "-I" + INCLUDE, "-I" + CSRC,
]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-Wall",
             "-I" + os.path.join(CUDA_HOME, "include"), "-I" + INCLUDE, "-I" + CSRC]


def _sources():
    out = []
    for name in sorted(os.listdir(CSRC)):
        if name.endswith((".cu", ".cpp")):
            out.append(os.path.join(CSRC, name))
    return out


def _headers_mtime():
    m = 0.0
    for d in (CSRC, INCLUDE):
        for name in os.listdir(d):
            if name.endswith((".h", ".cuh")):
                m = max(m, os.path.getmtime(os.path.join(d, name)))
    return m


def _compile(src, force, hdr_mtime):
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    if (not force and os.path.exists(obj)
            and os.path.getmtime(obj) >= max(os.path.getmtime(src), hdr_mtime)):
        return obj, None
    if src.endswith(".cu"):
        cmd = [NVCC] + NVCC_FLAGS + ["-c", src, "-o", obj]
    else:
        cmd = ["g++"] + CXX_FLAGS + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return obj, f"{' '.join(cmd)}\n{r.stdout}\n{r.stderr}"
    return obj, None


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(OUT_DIR, exist_ok=True)
    hdr = _headers_mtime()
    srcs = _sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 2)) as ex:
        results = list(ex.map(lambda s: _compile(s, force, hdr), srcs))
    errs = [e for _, e in results if e]
    if errs:
        raise RuntimeError("CUDA library build failed:\n" + "\n".join(errs))
    objs = [o for o, _ in results]
    newest = max(os.path.getmtime(o) for o in objs)
    if force or not os.path.exists(OUT) or os.path.getmtime(OUT) < newest:
        cmd = [NVCC] + ARCH + ["-shared", "-o", OUT] + objs + ["-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if verbose:
        print("built", OUT)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
