"""Builds libmsplat_cuda.so in-tree for sm_100a with nvcc.

Every translation unit is compiled with ``-fmad=false``: the splatting kernels
reproduce the reference backend's float32 decisions (tile rectangles, depth keys,
alpha and transmittance cut-offs) bit for bit, which needs every multiply and add
rounded separately in the reference's order. The CUDA runtime is linked statically
so the library does not depend on which libcudart the host process loaded first.

    python -m msplat_street_b200.build [--force]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libmsplat_cuda.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CFLAGS = ["-O3", "-std=c++17", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC,-O2", "-Xptxas", "-O3",
          "-I", os.path.join(ROOT, "include"), "-I", CSRC]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libmsplat_cuda.so")


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    inc = os.path.join(ROOT, "include")
    hs += [os.path.join(inc, f) for f in os.listdir(inc) if f.endswith(".h")]
    return hs


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    nv = nvcc()
    hdrs = headers()
    objs = []
    jobs = []
    for src in sources():
        obj = os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + hdrs):
            jobs.append([nv, *ARCH, *CFLAGS, "-c", src, "-o", obj])

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {cmd[-3]}:\n{r.stdout}\n{r.stderr}")
        return r.stderr

    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        for warn in ex.map(run, jobs):
            if warn and verbose:
                print(warn, file=sys.stderr)
    if force or jobs or _stale(LIB, objs):
        run([nv, *ARCH, "-shared", "-cudart", "static", "-o", LIB, *objs])
    return LIB


GRADCHECK = os.path.join(BUILD, "gradcheck_cuda")


def build_reference_gradcheck(ref_root: str, force: bool = False) -> str:
    """Links the reference's own gradient check (tests/gradcheck.cpp, read where the
    reference sources lie) against this library through integration/bindings_cuda.cpp,
    the bindings.h implementation over the C-ABI. Needs g++ and the reference tree;
    the result runs without either."""
    src = os.path.join(ref_root, "tests", "gradcheck.cpp")
    shim = os.path.join(PKG, "integration", "bindings_cuda.cpp")
    lib = build(force)
    deps = [src, shim, lib, os.path.join(ROOT, "include", "msplat_cuda.h")]
    if force or _stale(GRADCHECK, deps):
        cmd = ["g++", "-O2", "-std=c++17", "-I", os.path.join(ref_root, "core", "metal"), "-I",
               os.path.join(ref_root, "core", "include"), "-I", os.path.join(ROOT, "include"), "-o", GRADCHECK, src,
               shim, "-L", PKG, "-lmsplat_cuda", "-Wl,-rpath,$ORIGIN/.."]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"gradcheck build failed:\n{r.stdout}\n{r.stderr}")
    return GRADCHECK


TRAIN_BINDINGS = os.path.join(BUILD, "train_bindings")


def build_bindings_bench(ref_root: str, force: bool = False) -> str:
    """Builds integration/train_bindings.cpp (training-step throughput through
    bindings.h with host tensors, as the reference's own callers hold them) against the
    reference's headers and integration/bindings_cuda.cpp. Needs g++ and the reference
    tree; the result runs without either."""
    src = os.path.join(PKG, "integration", "train_bindings.cpp")
    shim = os.path.join(PKG, "integration", "bindings_cuda.cpp")
    lib = build(force)
    deps = [src, shim, lib, os.path.join(ROOT, "include", "msplat_cuda.h")]
    if force or _stale(TRAIN_BINDINGS, deps):
        cmd = ["g++", "-O2", "-std=c++17", "-I", os.path.join(ref_root, "core", "metal"), "-I",
               os.path.join(ref_root, "core", "include"), "-I", os.path.join(ROOT, "include"), "-o", TRAIN_BINDINGS,
               src, shim, "-L", PKG, "-lmsplat_cuda", "-Wl,-rpath,$ORIGIN/.."]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"train_bindings build failed:\n{r.stdout}\n{r.stderr}")
    return TRAIN_BINDINGS


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    args = ap.parse_args(argv)
    print(build(args.force, args.verbose))


if __name__ == "__main__":
    main()
