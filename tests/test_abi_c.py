"""The drop-in boundary is plain C: a C99 translation unit that includes
include/clothcraft.h compiles warning-free, links against the library and sees
the struct sizes the Python mirror uses (a Rust, Go or C caller binds the same
layout). Runs without a GPU: only the version entry point is called."""
import ctypes as C
import os
import shutil
import subprocess

import pytest

from clothcraft_b200 import abi, native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROGRAM = r"""
#include <stdio.h>
#include "clothcraft.h"
int main(void) {
    printf("%d %lu %lu %lu %lu %lu %lu\n", (int)cc_abi_version(), (unsigned long)sizeof(cc_vbd_settings),
           (unsigned long)sizeof(cc_metrics), (unsigned long)sizeof(cc_grab), (unsigned long)sizeof(cc_material),
           (unsigned long)sizeof(cc_ogc_settings), (unsigned long)sizeof(cc_contacts));
    return 0;
}
"""


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_header_compiles_as_c99_and_links(tmp_path):
    lib = native.load()._name
    src = tmp_path / "probe.c"
    src.write_text(PROGRAM)
    exe = tmp_path / "probe"
    libdir = os.path.dirname(lib)
    cmd = ["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"), str(src), "-o",
           str(exe), "-L", libdir, "-l:" + os.path.basename(lib), "-Wl,-rpath," + libdir]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    version, *sizes = [int(t) for t in out.stdout.split()]
    assert version == 3
    assert sizes == [C.sizeof(abi.cc_vbd_settings), C.sizeof(abi.cc_metrics), C.sizeof(abi.cc_grab),
                     C.sizeof(abi.cc_material), C.sizeof(abi.cc_ogc_settings), C.sizeof(abi.cc_contacts)]
