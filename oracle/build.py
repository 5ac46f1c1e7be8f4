"""Build recipe of the oracle (test infrastructure only).

Compiles the FP64 C++ restatement of ClothCraft's CPU path into
``oracle/_build/liboracle.so``. ``-ffp-contract=off`` keeps every multiply and
add separately rounded, as Rust's f64 arithmetic is, so detection decisions
and contact keys can be compared bit for bit.
"""
from __future__ import annotations

import os
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
SOURCES = ["oracle_ogc.cpp", "oracle_vbd.cpp", "oracle_capi.cpp", "oracle_newton.cpp", "oracle_learned.cpp"]
OUT = HERE / "_build" / "liboracle.so"


def build(force: bool = False) -> Path:
    srcs = [HERE / s for s in SOURCES if (HERE / s).exists()]
    headers = list(HERE.glob("*.hpp")) + [HERE.parent / "include" / "clothcraft.h"]
    if OUT.exists() and not force:
        newest = max(p.stat().st_mtime for p in srcs + headers)
        if OUT.stat().st_mtime >= newest:
            return OUT
    OUT.parent.mkdir(parents=True, exist_ok=True)
    tmp = OUT.with_suffix(".so.tmp%d" % os.getpid())
    cmd = [
        "g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off",
        "-fno-fast-math", "-Wall", "-Wno-unknown-pragmas", "-o", str(tmp),
    ] + [str(s) for s in srcs]
    subprocess.run(cmd, check=True)
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    print(build(force=True))
