"""Build libexa_aderdg.so for sm_100a (in-tree, next to this file).

    python exahype-engine_b200/build.py

nvcc cross-compiles on a machine without a GPU. The library is rebuilt only when a source is
newer than it (or when force=True).
"""
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libexa_aderdg.so")
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "-Xcompiler", "-fPIC", "-shared", "--expt-relaxed-constexpr"]


def _nvcc():
    for c in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")) + glob.glob(os.path.join(HERE, "csrc", "*.cuh")) +
                  [os.path.join(REPO, "include", "exa_aderdg.h")])


def build_user_pde(src, out, force=False, verbose=False):
    """Compile an application's PDE functor (a .cu file using include/exa_aderdg_user.cuh) into a
    shared library linked against libexa_aderdg.so (built first); loading it registers the
    functor's instantiations with the library."""
    lib = build(verbose=verbose)
    deps = [src] + sources() + [os.path.join(REPO, "include", "exa_aderdg_user.cuh")]
    if not force and os.path.exists(out) and os.path.getmtime(out) >= max(os.path.getmtime(s) for s in deps):
        return out
    cmd = [_nvcc()] + NVCC_FLAGS + (["-Xptxas", "-v"] if verbose else []) + \
        ["-I", os.path.join(REPO, "include"), "-o", out + ".tmp", src, "-L", HERE, "-lexa_aderdg",
         "-Xlinker", "-rpath=$ORIGIN/" + os.path.relpath(HERE, os.path.dirname(os.path.abspath(out)))]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed on %s" % src)
    os.replace(out + ".tmp", out)
    assert os.path.exists(lib)
    return out


def build(force=False, verbose=False):
    srcs = sources()
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(s) for s in srcs):
        return LIB
    # the soname lets an application's PDE library (build_user_pde) bind to the copy already loaded
    cmd = [_nvcc()] + NVCC_FLAGS + (["-Xptxas", "-v"] if verbose else []) + \
        ["-Xlinker", "-soname=libexa_aderdg.so", "-o", LIB + ".tmp", os.path.join(HERE, "csrc", "exa_aderdg.cu")]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed")
    if verbose:
        sys.stderr.write(r.stderr)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
