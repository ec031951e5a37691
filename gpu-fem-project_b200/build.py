"""Build recipe for libfemb200.so (CUDA sm_100a + host C++), written next to this file.

nvcc cross-compiles for sm_100a without a GPU; the shared library is built
in-tree so that it travels with the repository to the GPU machine.
"""
from __future__ import annotations

import concurrent.futures
import os
import pathlib
import subprocess
import sys

PKG = pathlib.Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
LIB = PKG / "libfemb200.so"

SOURCES = ["fem_kernels.cu", "fem_nonlinear.cu", "fem_rows.cu", "fem_batch.cu", "fem_server.cu", "fem_static.cu",
           "fem_frag.cu", "fem_host.cpp"]
PROBE_SOURCES = ["fem_probe.cu"]  # libfemprobe.so: arithmetic-peak calibration, not part of the assembly ABI
PROBE_LIB = PKG / "libfemprobe.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    cand = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    return cand if os.path.exists(cand) else "nvcc"


def _stale(target: pathlib.Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> pathlib.Path:
    _build_lib(LIB, SOURCES, force, verbose)
    _build_lib(PROBE_LIB, PROBE_SOURCES, force, verbose)
    return LIB


def _build_lib(lib: pathlib.Path, sources, force: bool, verbose: bool) -> None:
    srcs = [CSRC / s for s in sources if (CSRC / s).exists()]
    deps = srcs + list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))
    if not force and not _stale(lib, deps):
        return
    obj_dir = PKG / "_build"
    obj_dir.mkdir(exist_ok=True)
    common = [f"-I{INCLUDE}", f"-I{CSRC}", "-O3", "-std=c++17"]
    cmds, objs = [], []
    for src in srcs:
        obj = obj_dir / (src.name + ".o")
        if src.suffix == ".cu":
            cmd = [_nvcc(), *ARCH, "-lineinfo", "-Xcompiler", "-fPIC,-fopenmp", *common, "-c", str(src), "-o", str(obj)]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
        else:
            cmd = ["g++", "-fPIC", "-fopenmp", *common, "-c", str(src), "-o", str(obj)]
        cmds.append(cmd)
        objs.append(str(obj))
    with concurrent.futures.ThreadPoolExecutor(max_workers=len(cmds)) as ex:
        list(ex.map(_run, cmds))
    _run([_nvcc(), *ARCH, "-shared", "-Xcompiler", "-fopenmp", "-o", str(lib), *objs, "-lgomp"])


def _run(cmd):
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("build step failed: " + " ".join(cmd))
    if res.stderr.strip() and os.environ.get("FEM_BUILD_VERBOSE"):
        sys.stderr.write(res.stderr)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
