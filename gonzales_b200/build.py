"""Builds libgzg.so in-tree with nvcc for sm_100a (B200).

Sources: gonzales_b200/csrc/*.cu and *.cpp.  Host C++ is compiled by nvcc's
host compiler; the CUDA runtime is linked statically.  Rebuilds only when a
source or header is newer than the library.
"""
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
OUT = PKG / "libgzg.so"
BUILD = PKG / "_build"
INCLUDE = PKG.parent / "include"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC,-fvisibility=hidden", "-I", str(INCLUDE)]
CUDA_FLAGS = ARCH + ["-lineinfo", "-Xptxas", "-warn-spills" + (",-v" if os.environ.get("GZG_PTXAS_VERBOSE") else "")]


def _sources():
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))


def _stale():
    if not OUT.exists():
        return True
    t = OUT.stat().st_mtime
    deps = list(CSRC.glob("*")) + list(INCLUDE.glob("*.h")) + [Path(__file__)]
    return any(p.stat().st_mtime > t for p in deps)


def build(force=False, verbose=False):
    if not force and not _stale():
        return OUT
    BUILD.mkdir(exist_ok=True)
    objs = []
    headers = [p for p in CSRC.glob("*") if p.suffix in (".h", ".cuh")] + list(INCLUDE.glob("*.h")) + [Path(__file__)]
    newest_header = max(p.stat().st_mtime for p in headers)
    for src in _sources():
        obj = BUILD / (src.name + ".o")
        objs.append(str(obj))
        if not force and obj.exists() and obj.stat().st_mtime > max(src.stat().st_mtime, newest_header):
            continue  # up to date
        cmd = [NVCC, "-c", str(src), "-o", str(obj)] + COMMON
        if src.suffix == ".cu":
            cmd += CUDA_FLAGS
        else:
            cmd += ["-x", "c++", "-Wno-deprecated-gpu-targets",
                    "-DGZG_SOBOL_PATH=" + str(PKG / "data" / "sobol_1024x52.bin")]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    tmp = OUT.with_suffix(".so.tmp")
    link = [NVCC, "-shared", "-o", str(tmp)] + ARCH + [*objs, "-lpthread"]
    if verbose:
        print(" ".join(link))
    subprocess.run(link, check=True)
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(OUT)
