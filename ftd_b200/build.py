"""Build recipe for the correlator's native library (``ftd_b200/libftdx.so``).

Compiles every ``csrc/*.cu`` for sm_100a with nvcc and links them, together
with the C++ drop-in shims under ``csrc/shim/``, into one shared library in
the package directory (in-tree, so that it travels with the source tree).
Rebuilds only when a source or header is newer than the library.

Usage: ``python -m ftd_b200.build [--force]``.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libftdx.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
           "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "include"), "-I", CSRC]


def _sources():
    cu = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    cpp = sorted(glob.glob(os.path.join(CSRC, "shim", "*.cpp")))
    return cu, cpp


def _deps():
    return (glob.glob(os.path.join(CSRC, "**", "*"), recursive=True)
            + glob.glob(os.path.join(ROOT, "include", "*.h")) + [os.path.abspath(__file__)])


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.isfile(d))


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {os.path.basename(cmd[-1])}")
    return r


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile the library if needed and return its path."""
    cu, cpp = _sources()
    if not force and not _stale(LIB, _deps()):
        return LIB
    os.makedirs(OBJ, exist_ok=True)
    objs = []
    for src in cu:
        obj = os.path.join(OBJ, os.path.basename(src) + ".o")
        cmd = [NVCC, *ARCH, *NVFLAGS, "-Xptxas", "-v", "-c", src, "-o", obj]
        r = _run(cmd)
        if verbose:
            sys.stderr.write(r.stderr)
        objs.append(obj)
    for src in cpp:
        obj = os.path.join(OBJ, "shim_" + os.path.basename(src) + ".o")
        cmd = [NVCC, *NVFLAGS, "-x", "c++", "-c", src, "-o", obj]
        _run(cmd)
        objs.append(obj)
    tmp = LIB + ".tmp"
    _run([NVCC, *ARCH, "-shared", "-o", tmp, *objs, "-lcufft", "-Xlinker",
          "-rpath=/usr/local/cuda/lib64"])
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
