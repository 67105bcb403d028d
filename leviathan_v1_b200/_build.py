"""Build recipe of the in-tree CUDA library ``libleviathan_b200.so``.

The library is compiled with nvcc for sm_100a only and written next to the
Python package (``leviathan_v1_b200/lib/``) so that it travels with the source
tree.  No fast-math: the step keeps IEEE division and square root like the
reference build (CMakeLists.txt:19-26).
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
REPO_DIR = os.path.dirname(PKG_DIR)
CSRC = os.path.join(PKG_DIR, "csrc")
LIB_DIR = os.path.join(PKG_DIR, "lib")
LIB_NAME = "libleviathan_b200.so"
LIB_PATH = os.path.join(LIB_DIR, LIB_NAME)

SOURCES = ["lev_engine.cu"]
HEADERS = sorted(f for f in os.listdir(CSRC) if f.endswith(".cuh"))

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3",
    "-std=c++17",
    "-lineinfo",
    "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC",
    "-Xcompiler", "-fvisibility=default",
    "-shared",
    "-Xlinker", "-Bsymbolic",
]


def nvcc_path() -> str:
    cand = shutil.which("nvcc")
    if cand:
        return cand
    cand = "/usr/local/cuda/bin/nvcc"
    if os.path.exists(cand):
        return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build")


def _inputs():
    files = [os.path.join(CSRC, s) for s in SOURCES + HEADERS]
    files.append(os.path.join(REPO_DIR, "include", "leviathan_b200.h"))
    files.append(os.path.abspath(__file__))
    return files


def needs_build() -> bool:
    if not os.path.exists(LIB_PATH):
        return True
    t = os.path.getmtime(LIB_PATH)
    return any(os.path.getmtime(f) > t for f in _inputs() if os.path.exists(f))


def build(force: bool = False, verbose: bool = False, ptxas_v: bool = False) -> str:
    """Compile the library (if stale) and return its path."""
    if not force and not needs_build():
        return LIB_PATH
    os.makedirs(LIB_DIR, exist_ok=True)
    tmp = LIB_PATH + ".tmp"
    cmd = [nvcc_path(), *ARCH_FLAGS, *NVCC_FLAGS,
           "-I", os.path.join(REPO_DIR, "include"), "-I", CSRC]
    if ptxas_v:
        cmd += ["-Xptxas", "-v"]
    cmd += [os.path.join(CSRC, s) for s in SOURCES]
    cmd += ["-o", tmp, "-lcudart"]
    if verbose:
        print(" ".join(cmd), flush=True)
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + proc.stdout + proc.stderr)
    if verbose or ptxas_v:
        sys.stdout.write(proc.stdout + proc.stderr)
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_v="-v" in sys.argv)
