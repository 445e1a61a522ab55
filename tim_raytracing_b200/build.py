"""Builds the in-tree shared library ``libtim_rt.so`` (CUDA kernels for sm_100a
plus the C-ABI host runtime) with nvcc. Run ``python -m tim_raytracing_b200.build``.

Floating-point flags are part of the product's contract: ``--fmad=false``,
``-prec-div=true``, ``-prec-sqrt=true`` and ``-ftz=false`` keep the
intersection arithmetic IEEE round-to-nearest, operation by operation, which
is what makes hit ids and t bit-identical to the reference's arithmetic.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libtim_rt.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17",
    "--fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
    "-Xcompiler", "-fPIC,-O2,-ffp-contract=off,-fno-fast-math",
    "-I" + str(CSRC), "-I" + str(ROOT / "include"),
]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libtim_rt.so")
    return cand


def sources() -> list[Path]:
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def _stale(obj: Path, src: Path) -> bool:
    if not obj.exists():
        return True
    deps = [src] + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list((ROOT / "include").glob("*.h"))
    t = obj.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps) or Path(__file__).stat().st_mtime > t


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compiles every CUDA/C++ source of the package and links libtim_rt.so."""
    nvcc = _nvcc()
    BUILD.mkdir(exist_ok=True)
    srcs = sources()
    objs = [BUILD / (s.name + ".o") for s in srcs]
    todo = [(s, o) for s, o in zip(srcs, objs) if force or _stale(o, s)]

    def compile_one(so):
        s, o = so
        cmd = [nvcc] + NVCC_FLAGS + ["-c", str(s), "-o", str(o)]
        if verbose:
            cmd += ["-Xptxas", "-v"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {s.name}:\n{r.stdout}\n{r.stderr}")
        return r.stderr

    if todo:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(todo))) as ex:
            for log in ex.map(compile_one, todo):
                if verbose and log:
                    print(log, file=sys.stderr)
    if force or todo or not LIB.exists():
        cmd = [nvcc] + ARCH + ["-shared", "-o", str(LIB)] + [str(o) for o in objs] + ["-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
