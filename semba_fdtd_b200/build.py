"""Build recipe for libsemba_gpu.so (sm_100a) and its FMA variant.

Two libraries are built from the same sources:

* ``libsemba_gpu.so`` -- ``-fmad=false``: every multiply and add rounds on its
  own, so the kernels reproduce the reference FP32 build bit for bit.  This is
  the default library.
* ``libsemba_gpu_fast.so`` -- ``-fmad=true``: the compiler may contract
  multiply-adds into FMAs (results within 1e-5 relative L2 of the exact build).

Host code is compiled with ``-ffp-contract=off`` and without ``-march`` so the
set-up arithmetic also rounds where the reference rounds.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
OUT = HERE / "_build"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = ["kernels.cu", "batch.cu", "host_setup.cpp", "transfer.cu", "resume.cu", "farfield.cu", "paint.cu"]
LIBS = {"libsemba_gpu.so": ["-fmad=false"], "libsemba_gpu_fast.so": ["-fmad=true"]}


def _nvcc() -> str:
    cand = os.environ.get("CUDA_HOME", "/usr/local/cuda") + "/bin/nvcc"
    return cand if os.path.exists(cand) else "nvcc"


def _stale(target: Path) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    deps = [CSRC / s for s in SOURCES] + list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + [HERE.parent / "include" / "semba_gpu.h", Path(__file__)]
    return any(d.stat().st_mtime > t for d in deps if d.exists())


def build(force: bool = False, verbose: bool = False) -> dict:
    """Compile both libraries into semba_fdtd_b200/_build; returns their paths."""
    OUT.mkdir(parents=True, exist_ok=True)
    paths = {}
    for lib, flags in LIBS.items():
        target = OUT / lib
        paths[lib] = str(target)
        if not force and not _stale(target):
            continue
        objs = []
        for src in SOURCES:
            obj = OUT / (Path(src).stem + ("_fast" if "fast" in lib else "") + ".o")
            cmd = [_nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", *flags,
                   "-Xcompiler", "-fPIC,-ffp-contract=off,-O2", "-I", str(HERE.parent / "include"),
                   "-c", str(CSRC / src), "-o", str(obj)]
            if verbose:
                print(" ".join(cmd), file=sys.stderr)
            subprocess.run(cmd, check=True)
            objs.append(str(obj))
        cmd = [_nvcc(), *ARCH, "-shared", "--cudart", "static", "-o", str(target), *objs]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
    return paths


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
