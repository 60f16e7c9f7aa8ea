"""Build the sm_100a shared library ``maddening_b200/liblbm_b200.so`` in-tree.

    python -m maddening_b200.build [--verbose]

The library is a plain C ABI (``include/lbm_b200.h``) compiled by nvcc with
the CUDA runtime linked statically, so it loads next to any torch build.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "liblbm_b200.so"
SOURCES = ["lbm_abi.cu"]
HEADERS = ["lbm_kernels.cuh", "lbm_lattice.cuh", "lbm_adjoint.cuh", "lbm_staged.cuh",
           "lbm_pair.cuh", "lbm_pipe.cuh", "lbm_multiphase.cuh", "lbm_pack.cuh"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
         "-Xcompiler", "-fPIC,-O3", "-shared", "-cudart", "static",
         "--split-compile=0"]


def nvcc() -> str:
    cand = os.environ.get("NVCC") or shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found (set NVCC or put CUDA on PATH)")
    return cand


def _inputs():
    files = [CSRC / s for s in SOURCES] + [CSRC / h for h in HEADERS]
    files.append(ROOT / "include" / "lbm_b200.h")
    files.append(Path(__file__))
    return files


def up_to_date() -> bool:
    if not LIB.exists():
        return False
    t = LIB.stat().st_mtime
    return all(f.stat().st_mtime <= t for f in _inputs())


def build(verbose: bool = False, force: bool = False) -> Path:
    if up_to_date() and not force:
        return LIB
    cmd = [nvcc(), *ARCH, *FLAGS, "-I", str(ROOT / "include"),
           *(str(CSRC / s) for s in SOURCES), "-o", str(LIB) + ".tmp"]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError(f"nvcc failed ({res.returncode})")
    if verbose:
        sys.stdout.write(res.stdout + res.stderr)
    os.replace(str(LIB) + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(verbose="--verbose" in sys.argv, force=True)
    print(LIB)
