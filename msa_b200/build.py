"""Builds libmsa_b200.so in-tree (sm_100a only) with nvcc.

    python -m msa_b200.build            # rebuild if any source is newer
    python -m msa_b200.build --force
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
INCLUDE = PKG.parent / "include"
LIB = PKG / "libmsa_b200.so"
BUILD_DIR = PKG / "_build"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = ["tables.cpp", "abi.cpp", "partition.cpp", "nw_kernels.cu", "nj_kernel.cu", "probe.cu", "noalloc.cu",
           "serve.cpp", "facade.cu", "fasta.cpp"]
# The command line (museqa), linked against the library.
CLI = PKG / "museqa"
CLI_SOURCE = "cli.cpp"
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
              "--expt-relaxed-constexpr", "-I", str(INCLUDE)]


def _nvcc() -> str:
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    cand = Path(cuda) / "bin" / "nvcc"
    return str(cand) if cand.exists() else "nvcc"


def _stale() -> bool:
    if not LIB.exists() or not CLI.exists():
        return True
    t = min(LIB.stat().st_mtime, CLI.stat().st_mtime)
    deps = [CSRC / s for s in SOURCES] + [CSRC / CLI_SOURCE] + list(CSRC.glob("*.hpp")) + list(CSRC.glob("*.cuh")) \
        + list(CSRC.glob("*.inc")) + list(INCLUDE.glob("*.h")) + list(INCLUDE.glob("*.hpp")) + [Path(__file__)]
    return any(p.exists() and p.stat().st_mtime > t for p in deps)


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None) -> Path:
    if not force and not _stale():
        return LIB
    BUILD_DIR.mkdir(exist_ok=True)
    nvcc = _nvcc()
    objs = []
    for src in SOURCES:
        obj = BUILD_DIR / (src + ".o")
        lang = [] if src.endswith(".cu") else ["-x", "cu"] if src.endswith(".cpp") and "kernel" in src else []
        cmd = [nvcc, *ARCH, *NVCC_FLAGS, *(extra or []), *lang, "-c", str(CSRC / src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        objs.append(str(obj))
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc, *ARCH, "-shared", "-o", str(tmp), *objs, "-lcudart", "-lpthread"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    cli_tmp = CLI.with_suffix(".tmp")
    cmd = [nvcc, *ARCH, *NVCC_FLAGS, "-x", "cu", str(CSRC / CLI_SOURCE), "-o", str(cli_tmp), "-L", str(PKG),
           "-lmsa_b200", "-Xlinker", "-rpath,$ORIGIN"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(cli_tmp, CLI)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
