"""Build the batchfit B200 CUDA library in-tree: batchfit_b200/libbatchfit_cuda.so.

    python -m batchfit_b200.build [--force]

nvcc cross-compiles for sm_100a only (``-gencode arch=compute_100a,code=sm_100a``);
no GPU is needed to build.  The CUDA runtime is linked statically so the library
depends only on the driver.
"""

from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libbatchfit_cuda.so")
OBJ = os.path.join(HERE, "_build")
SOURCES = ["bf_kernels.cu", "bf_long.cu", "bf_capi.cu", "bf_noalloc.cu", "bf_batch.cu", "bf_batch_kernels.cu", "bf_batch_guess.cu",
           "bf_server.cu", "bf_npy.cu", "bf_coords.cu"]
HEADERS = ["bf_args.h", "bf_batch.h", "bf_batch.cuh", "bf_context.h", "bf_device.cuh", "bf_guess.cuh", "bf_kernels.h",
           "bf_lm.cuh", "bf_models.cuh", "bf_xgrid.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
         "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "include")]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False, csrc: str = CSRC, lib: str = LIB, obj: str = OBJ,
          defines: tuple = ()) -> str:
    deps = [os.path.join(csrc, f) for f in SOURCES + HEADERS] + [os.path.join(ROOT, "include", "batchfit_cuda.h")]
    if not force and not _stale(lib, deps):
        return lib
    os.makedirs(obj, exist_ok=True)
    cc = nvcc()

    headers = [os.path.join(csrc, f) for f in HEADERS] + [os.path.join(ROOT, "include", "batchfit_cuda.h")]
    # Objects are reused only when built with the same flags (recorded beside them).
    stamp = os.path.join(obj, "flags.txt")
    flags = " ".join([*ARCH, *FLAGS, *[f"-D{d}" for d in defines]])
    same_flags = os.path.exists(stamp) and open(stamp).read() == flags
    with open(stamp, "w") as fh:
        fh.write(flags)

    def compile_one(src: str) -> str:
        target = os.path.join(obj, src.replace(".cu", ".o"))
        if not force and same_flags and not _stale(target, [os.path.join(csrc, src), *headers]):
            return target  # every header is shared: an object is current only if newer than all of them
        cmd = [cc, *ARCH, *FLAGS, *[f"-D{d}" for d in defines], "-c", os.path.join(csrc, src), "-o", target]
        if verbose:
            print(" ".join(cmd))
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{res.stderr}")
        return target

    with ThreadPoolExecutor(max_workers=len(SOURCES)) as pool:
        objs = list(pool.map(compile_one, SOURCES))
    tmp = lib + ".tmp"
    cmd = [cc, *ARCH, "-shared", "-cudart=static", "-o", tmp, *objs, "-lpthread", "-ldl", "-lrt"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"link failed:\n{res.stderr}")
    os.replace(tmp, lib)
    return lib


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    args = ap.parse_args(argv)
    print(build(force=args.force, verbose=args.verbose))
    return 0


if __name__ == "__main__":
    sys.exit(main())
