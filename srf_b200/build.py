"""Build the in-tree CUDA library ``srf_b200/libsrf_b200.so`` for sm_100a.

Each ``csrc/*.cu`` file is compiled separately (in parallel) with nvcc and linked into
one shared library with the CUDA runtime linked statically, so the library depends on
nothing but the driver. ``python -m srf_b200.build [--force] [--ptxas-verbose]``.
"""

import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJDIR = os.path.join(HERE, "_build")
LIBPATH = os.path.join(HERE, "libsrf_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I", INCLUDE,
              "--expt-relaxed-constexpr"]


def nvcc():
    exe = shutil.which("nvcc")
    if exe:
        return exe
    cand = "/usr/local/cuda/bin/nvcc"
    if os.path.exists(cand):
        return cand
    raise RuntimeError("nvcc not found: the srf_b200 CUDA library cannot be built")


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _deps():
    return sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + [
        os.path.join(INCLUDE, "srf_b200.h"), os.path.abspath(__file__)]


def up_to_date():
    if not os.path.exists(LIBPATH):
        return False
    t = os.path.getmtime(LIBPATH)
    return all(os.path.getmtime(d) <= t for d in _deps())


def _compile(src, verbose_ptxas):
    obj = os.path.join(OBJDIR, os.path.basename(src)[:-3] + ".o")
    cmd = [nvcc()] + ARCH + NVCC_FLAGS + (["-Xptxas", "-v"] if verbose_ptxas else []) + [
        "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(force=False, verbose_ptxas=False, quiet=True):
    """Compile every CUDA source and link libsrf_b200.so. Returns the library path."""
    if not force and not verbose_ptxas and up_to_date():
        return LIBPATH
    os.makedirs(OBJDIR, exist_ok=True)
    srcs = sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        results = list(ex.map(lambda s: _compile(s, verbose_ptxas), srcs))
    objs = [o for o, _ in results]
    if verbose_ptxas:
        for (_, log), s in zip(results, srcs):
            print(f"== {os.path.basename(s)}\n{log}")
    tmp = LIBPATH + ".tmp"
    cmd = [nvcc()] + ARCH + ["-shared", "-cudart", "static", "-o", tmp] + objs
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIBPATH)
    if not quiet:
        print("built", LIBPATH)
    return LIBPATH


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas-verbose", action="store_true")
    a = ap.parse_args(argv)
    build(force=a.force, verbose_ptxas=a.ptxas_verbose, quiet=False)


if __name__ == "__main__":
    sys.exit(main())
