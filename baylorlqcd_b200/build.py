"""Build libqqcd_gpu.so in-tree with nvcc for sm_100a.

Compiles every baylorlqcd_b200/csrc/*.cu into baylorlqcd_b200/_build/ in parallel and
links the shared library next to this file.  Objects are rebuilt only when a source
or header is newer.  Run as ``python -m baylorlqcd_b200.build``.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
BUILD = HERE / "_build"
LIB = HERE / "libqqcd_gpu.so"
INCLUDE = HERE.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
              "--expt-relaxed-constexpr", "-I", str(INCLUDE)]
# Host-code flags of single sources.  The eigen-iteration's dense Schur step on the host
# takes nearly all of an eigenmode solve's time; with AVX2 (x86-64-v3, present on the
# B200 hosts' CPUs) and the plain complex multiply and divide formulas
# (its values are finite and of modest size: no NaN recovery or range reduction needed)
# it runs about twice as fast.  Contraction stays off.
HOST_FLAGS = {"qq_eigen.cu": ["-Xcompiler", "-march=x86-64-v3", "-Xcompiler", "-fcx-limited-range",
                              "-Xcompiler", "-ffp-contract=off"]}


def _nvcc() -> str:
    cand = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    return cand if Path(cand).exists() else "nvcc"


def _newest_header() -> float:
    hs = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list(INCLUDE.glob("*.h"))
    return max(p.stat().st_mtime for p in hs)


def _compile(src: Path, hdr_time: float) -> Path:
    obj = BUILD / (src.stem + ".o")
    if obj.exists() and obj.stat().st_mtime >= max(src.stat().st_mtime, hdr_time):
        return obj
    cmd = [_nvcc(), *ARCH, *NVCC_FLAGS, *HOST_FLAGS.get(src.name, []), "-c", str(src), "-o", str(obj)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{res.stderr}")
    return obj


def build(verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    srcs = sorted(CSRC.glob("*.cu"))
    hdr = _newest_header()
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, hdr), srcs))
    if not LIB.exists() or LIB.stat().st_mtime < max(o.stat().st_mtime for o in objs):
        tmp = LIB.with_suffix(".so.tmp")
        cmd = [_nvcc(), *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-lcudart"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stderr}")
        os.replace(tmp, LIB)
    if verbose:
        print(f"built {LIB}")
    return LIB


if __name__ == "__main__":
    build(verbose=True)
    sys.exit(0)
