"""Build recipe for the sm_100a library ``dare_b200/libdare_gpu.so``.

Each translation unit is compiled with nvcc for ``-gencode
arch=compute_100a,code=sm_100a`` and linked into one shared library that
exports the C ABI declared in ``include/dare_gpu.h``.  The library is built
in-tree so it travels with the repository.

    python -m dare_b200.build            # incremental
    python -m dare_b200.build --force    # rebuild everything
"""
from __future__ import annotations

import argparse
import concurrent.futures
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libdare_gpu.so")
NVCC = os.environ.get("DARE_NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
          "-I", os.path.join(ROOT, "include"), "--expt-relaxed-constexpr"]

# translation unit -> extra flags.  The 1-D / 2-D assembly kernel reproduces
# the CPU path's separately rounded products and sums, so FMA contraction is
# off there; the 3-D assembly (dare_assembly3.cu) works to 1e-13 relative.
SOURCES = {
    "dare_core.cu": [],
    "dare_assembly.cu": ["--fmad=false"],
    "dare_assembly3.cu": [],
    "dare_slabs.cu": [],
    "dare_bicgstab2.cu": [],
    "dare_mixed.cu": [],
    "dare_step.cu": [],
    "dare_noalloc.cu": [],
    "dare_batched.cu": [],
    "dare_unet.cu": [],
    "dare_learned.cu": [],
    "dare_vtk.cu": [],
}


def _stale(obj: str, deps: list[str]) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(ROOT, "include", "dare_gpu.h"))
    objs, cmds = [], []
    for src, extra in SOURCES.items():
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(obj)
        if force or _stale(obj, [path] + headers):
            cmds.append([NVCC, *ARCH, *COMMON, *extra, "-c", path, "-o", obj])
    # translation units compile independently: one nvcc per host core
    with concurrent.futures.ThreadPoolExecutor(max_workers=max(1, os.cpu_count() or 1)) as pool:
        for cmd in cmds:
            if verbose:
                print(" ".join(cmd))
        for f in [pool.submit(subprocess.run, cmd, check=True) for cmd in cmds]:
            f.result()
    if force or _stale(LIB, objs):
        cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcuda"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    build_examples(force, verbose)
    return LIB


EXAMPLES = {"example_diffusion": os.path.join(HERE, "cxx", "example_diffusion.cpp"),
            "example_counter_diffusion": os.path.join(HERE, "cxx", "example_counter_diffusion.cpp")}
BIN = os.path.join(HERE, "bin")


def build_examples(force: bool = False, verbose: bool = False) -> None:
    """C++ programs written against include/dare_gpu.hpp, linked to the library."""
    os.makedirs(BIN, exist_ok=True)
    hdrs = [os.path.join(ROOT, "include", "dare_gpu.hpp"), os.path.join(ROOT, "include", "dare_gpu.h"), LIB]
    for name, src in EXAMPLES.items():
        exe = os.path.join(BIN, name)
        if force or _stale(exe, [src] + hdrs):
            cmd = ["g++", "-O2", "-std=c++17", "-Wall", "-I", os.path.join(ROOT, "include"), src, "-L", HERE,
                   "-ldare_gpu", "-Wl,-rpath,$ORIGIN/..", "-o", exe]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    args = ap.parse_args(argv)
    print(build(force=args.force, verbose=args.verbose))
    return 0


if __name__ == "__main__":
    sys.exit(main())
