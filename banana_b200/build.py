"""Build recipe for libbanana_b200.so (CUDA, sm_100a) and the host C++ driver.

Everything is compiled in-tree so the built shared objects travel with the source tree.
Kernels are compiled with -fmad=false and IEEE division / square root: every float
operation rounds once in source order, which the bit-exact parity tests rely on.
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
HOST = PKG / "host"
INCLUDE = ROOT / "include"
LIB = PKG / "libbanana_b200.so"
BUILD_DIR = PKG / "_build"

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
    "--expt-relaxed-constexpr",
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _run(cmd: list[str]) -> None:
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("command failed: " + " ".join(cmd))


def _stale(target: Path, sources: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(s.stat().st_mtime > t for s in sources)


def build_cuda(force: bool = False, verbose: bool = False) -> Path:
    """Compile every csrc/*.cu for sm_100a and link libbanana_b200.so."""
    nvcc = _nvcc()
    BUILD_DIR.mkdir(exist_ok=True)
    headers = sorted(CSRC.glob("*.cuh")) + [INCLUDE / "banana_b200.h"]
    objs = []
    for cu in sorted(CSRC.glob("*.cu")):
        obj = BUILD_DIR / (cu.stem + ".o")
        if force or _stale(obj, [cu] + headers):
            cmd = [nvcc, *NVCC_FLAGS, "-I", str(INCLUDE), "-I", str(CSRC), "-c", str(cu), "-o", str(obj)]
            if verbose:
                cmd += ["-Xptxas", "-v"]
                print(" ".join(cmd))
            _run(cmd)
        objs.append(obj)
    if force or _stale(LIB, objs):
        _run([nvcc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", *map(str, objs), "-o", str(LIB),
              "-lcudart"])
    return LIB


def build_host(force: bool = False) -> Path | None:
    """Compile the host C++ solver driver (plugin-API mirror) against the C ABI."""
    srcs = sorted(HOST.glob("*.cpp"))
    if not srcs:
        return None
    exe = PKG / "bnn_flip_run"
    deps = srcs + sorted(HOST.glob("*.h")) + [INCLUDE / "banana_b200.h", LIB]
    if force or _stale(exe, deps):
        cmd = ["g++", "-O2", "-std=c++17", "-I", str(INCLUDE), "-I", str(HOST), *map(str, srcs), "-o", str(exe),
               "-L", str(PKG), "-lbanana_b200", f"-Wl,-rpath,{PKG}", "-Wl,-rpath,$ORIGIN"]
        _run(cmd)
    return exe


def build(force: bool = False, verbose: bool = False) -> None:
    build_cuda(force=force, verbose=verbose)
    build_host(force=force)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
