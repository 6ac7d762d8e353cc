"""Builds libsaruman_b200.so in-tree with nvcc for sm_100a.

    python -m saruman_b200.build [--force]

The library is one shared object holding the kernels, the C ABI
(include/saruman_b200.h) and the host writer.  The CUDA runtime is linked
statically, so the reference's host C can link against it without further
libraries.
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
LIB = PKG / "libsaruman_b200.so"
SOURCES = ["kernels.cu", "gather.cu", "filter.cu", "abi.cu", "writer.cpp", "server.cpp", "compact.cpp", "sam.cpp",
           "costmodel.cu", "probe.cu", "input.cpp"]
HEADERS = ["kernels.cuh", "saru_core.cuh", "band_tile.cuh", "writer.h", "server_internal.h",
           "filter_core.cuh", "filter_calls.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler",
              "-fPIC,-O3,-Wall", "-Xptxas", "-v"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _stale() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = [CSRC / s for s in SOURCES + HEADERS] + [ROOT / "include" / "saruman_b200.h",
                                                    Path(__file__)]
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and not _stale():
        return LIB
    out_dir = PKG / "_build"
    out_dir.mkdir(exist_ok=True)
    objs = []
    log = []
    for src in SOURCES:
        obj = out_dir / (src + ".o")
        cmd = [nvcc(), *ARCH, *NVCC_FLAGS, "-I", str(ROOT / "include"), "-c", str(CSRC / src),
               "-o", str(obj)]
        if src.endswith(".cpp"):
            cmd = [nvcc(), "-x", "c++", "-O3", "-std=c++17", "-Xcompiler", "-fPIC,-O3,-Wall",
                   "-c", str(CSRC / src), "-o", str(obj)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        log.append(r.stdout + r.stderr)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
        objs.append(str(obj))
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc(), *ARCH, "-shared", "-o", str(tmp), *objs, "-Xlinker", "--no-undefined",
           "-lpthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    (out_dir / "ptxas.log").write_text("\n".join(log))
    if verbose:
        print("\n".join(log))
    return LIB


if __name__ == "__main__":
    p = build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(p)
