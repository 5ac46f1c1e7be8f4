"""The C-ABI library loads without a GPU and exports every entry point that
include/clothcraft.h declares (no compute calls here)."""
import ctypes as C
import re
from pathlib import Path

from clothcraft_b200 import abi, native

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    text = (ROOT / "include" / "clothcraft.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(cc_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_entry_point():
    L = native.load()
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    # every declared function has a ctypes signature in the binding
    assert set(names) <= set(native.SIGNATURES), set(names) - set(native.SIGNATURES)


def test_abi_version_and_no_device_is_reported_not_faked():
    L = native.load()
    assert L.cc_abi_version() == 3
    count = C.c_int()
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if not has_gpu:
        assert L.cc_set_device(0) == abi.CC_ERR_CUDA


def test_struct_layouts_match_header_sizes():
    # field order/size mirrors include/clothcraft.h (LP64)
    assert C.sizeof(abi.cc_material) == 80
    assert C.sizeof(abi.cc_vbd_settings) == 8 + 8 + 8 + 24 + 32 + 16 + 8 + 8
    assert C.sizeof(abi.cc_grab) == 16 + 24 + 24 + 8
    assert C.sizeof(abi.cc_mesh) == 21 * 8
