"""Build the CUDA library in-tree: clothcraft_b200/_lib/libclothcraft_b200.so.

sm_100a only. detect.cu is compiled with --fmad=false so that the FP64
narrow phase rounds every multiply and add separately (bit-identical contact
decisions to the CPU path); the other units keep FMA contraction.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRC = HERE / "csrc"
OUT_DIR = HERE / "_lib"
LIB = OUT_DIR / "libclothcraft_b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
UNITS = {
    "detect.cu": ["--fmad=false"],
    "sweep.cu": [],
    "sweep32.cu": [],
    "radix.cu": [],
    "newton.cu": [],
    "color.cu": [],
    "learned.cu": [],
    "mlp_tc.cu": [],
    "solver.cu": [],
}
NVCC = os.environ.get("NVCC", "nvcc")


def _flags():
    return ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fno-fast-math",
                   "--expt-relaxed-constexpr", "-I", str(SRC), "-I", str(HERE.parent / "include")]


def build(force: bool = False, verbose: bool = False) -> Path:
    OUT_DIR.mkdir(parents=True, exist_ok=True)
    sources = [SRC / u for u in UNITS]
    deps = list(SRC.glob("*.cu")) + list(SRC.glob("*.cuh")) + [HERE.parent / "include" / "clothcraft.h",
                                                              Path(__file__)]
    if LIB.exists() and not force and LIB.stat().st_mtime >= max(p.stat().st_mtime for p in deps):
        return LIB
    objs = []

    def compile_one(unit):
        src = SRC / unit
        obj = OUT_DIR / (src.stem + ".o")
        cmd = [NVCC, "-c", str(src), "-o", str(obj)] + _flags() + UNITS[unit]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed for %s:\n%s%s" % (unit, r.stdout, r.stderr))
        if verbose and (r.stdout or r.stderr):
            print(r.stdout + r.stderr, file=sys.stderr)
        return obj

    with ThreadPoolExecutor(max_workers=len(UNITS)) as ex:
        objs = list(ex.map(compile_one, list(UNITS)))
    tmp = LIB.with_suffix(".so.tmp%d" % os.getpid())
    cmd = [NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", str(tmp)] + [str(o) for o in objs] + ["-lrt", "-ldl", "-lpthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n%s%s" % (r.stdout, r.stderr))
    os.replace(tmp, LIB)
    for o in objs:
        o.unlink(missing_ok=True)
    return LIB


if __name__ == "__main__":
    print(build(force=True, verbose="-v" in sys.argv))
