"""Builds libgofft_b200.so in-tree for sm_100a.

Each CUDA translation unit under csrc/ is compiled in parallel with
``nvcc -gencode arch=compute_100a,code=sm_100a`` and linked into one shared
library with the CUDA runtime linked statically, so the library loads without
torch and only needs the NVIDIA driver.  Objects go to csrc/_build/ and are
rebuilt when the source or a project header it includes is newer.

    python -m fft_b200.build [--force] [--verbose]
"""
import argparse
import concurrent.futures
import glob
import os
import re
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(CSRC, "_build")
LIB = os.path.join(HERE, "libgofft_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
         "--expt-relaxed-constexpr", "-I", CSRC, "-I", INCLUDE]


def nvcc():
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(exe):
        raise RuntimeError("nvcc not found")
    return exe


_INC = re.compile(r'^\s*#\s*include\s+"([^"]+)"', re.M)


def _local_deps(path, seen=None):
    """The project headers `path` includes, directly or through other
    project headers (quoted includes resolved against the including file's
    folder, csrc/ and include/)."""
    seen = set() if seen is None else seen
    try:
        text = open(path).read()
    except OSError:
        return seen
    for name in _INC.findall(text):
        for base in (os.path.dirname(path), CSRC, INCLUDE):
            h = os.path.normpath(os.path.join(base, name))
            if os.path.exists(h):
                if h not in seen:
                    seen.add(h)
                    _local_deps(h, seen)
                break
    return seen


def _compile(src, force, verbose):
    obj = os.path.join(OBJ, os.path.basename(src).replace(".cu", ".o"))
    if not force and os.path.exists(obj):
        t = os.path.getmtime(obj)
        newest = max([os.path.getmtime(src)] + [os.path.getmtime(h) for h in _local_deps(src)])
        if t >= newest:
            return obj, ""
    cmd = [nvcc()] + ARCH + FLAGS + (["-Xptxas", "-v"] if verbose else []) + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s" % (src, r.stderr[-6000:]))
    return obj, r.stderr


def build(force=False, verbose=False):
    os.makedirs(OBJ, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    with concurrent.futures.ThreadPoolExecutor(max_workers=max(1, len(srcs))) as ex:
        results = list(ex.map(lambda s: _compile(s, force, verbose), srcs))
    objs = [o for o, _ in results]
    if verbose:
        for _, log in results:
            sys.stderr.write(log)
    newest = max(os.path.getmtime(o) for o in objs)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [nvcc()] + ARCH + ["-shared", "-Xcompiler", "-fPIC", "-o", LIB] + objs + ["-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stderr[-4000:])
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))
