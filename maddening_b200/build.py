"""Build the sm_100a shared library ``maddening_b200/liblbm_b200.so`` in-tree.

    python -m maddening_b200.build [--verbose]

The library is a plain C ABI (``include/lbm_b200.h``) compiled by nvcc with
the CUDA runtime linked statically, so it loads next to any torch build.  Its
translation units compile in parallel, then link into the one library.  A
build is skipped only when the library's recorded input digest (sources,
headers, flags, nvcc version) equals the current one, so a library built from
other sources is always rebuilt, whatever its timestamps.
"""

from __future__ import annotations

import hashlib
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "liblbm_b200.so"
DIGEST = PKG / "liblbm_b200.so.sha256"
SOURCES = ["lbm_abi.cu", "lbm_tiled.cu"]
HEADERS = ["lbm_host.h", "lbm_kernels.cuh", "lbm_lattice.cuh", "lbm_adjoint.cuh",
           "lbm_staged.cuh", "lbm_tiled.cuh", "lbm_pair.cuh", "lbm_pipe.cuh",
           "lbm_multiphase.cuh", "lbm_pack.cuh"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CFLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
          "-Xcompiler", "-fPIC,-O3", "--split-compile=0"]
LFLAGS = ["-shared", "-cudart", "static"]


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


def input_digest() -> str:
    h = hashlib.sha256()
    for f in _inputs():
        h.update(f.name.encode())
        h.update(f.read_bytes())
    h.update(" ".join(ARCH + CFLAGS + LFLAGS).encode())
    try:
        h.update(subprocess.run([nvcc(), "--version"], capture_output=True,
                                text=True).stdout.encode())
    except (RuntimeError, OSError):
        pass
    return h.hexdigest()


def up_to_date() -> bool:
    return LIB.exists() and DIGEST.exists() and DIGEST.read_text().strip() == input_digest()


def build(verbose: bool = False, force: bool = False) -> Path:
    if not force and up_to_date():
        return LIB
    digest = input_digest()
    objdir = PKG / "_build"
    objdir.mkdir(exist_ok=True)
    procs = []
    for src in SOURCES:
        obj = objdir / (Path(src).stem + ".o")
        cmd = [nvcc(), *ARCH, *CFLAGS, "-I", str(ROOT / "include"), "-c", str(CSRC / src),
               "-o", str(obj)]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
            print(" ".join(cmd), flush=True)
        procs.append((obj, subprocess.Popen(cmd, stdout=subprocess.PIPE,
                                            stderr=subprocess.STDOUT, text=True)))
    failed = False
    for _obj, pr in procs:
        out, _ = pr.communicate()
        if verbose or pr.returncode != 0:
            sys.stdout.write(out)
        failed |= pr.returncode != 0
    if failed:
        raise RuntimeError("nvcc failed")
    cmd = [nvcc(), *ARCH, *LFLAGS, *(str(o) for o, _ in procs), "-o", str(LIB) + ".tmp"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError(f"nvcc link failed ({res.returncode})")
    os.replace(str(LIB) + ".tmp", LIB)
    DIGEST.write_text(digest + "\n")
    return LIB


if __name__ == "__main__":
    build(verbose="--verbose" in sys.argv, force=True)
    print(LIB)
