"""The Rust binding written out in INTEGRATION.md must lay its #[repr(C)]
structs out field for field as the header does (the Python ctypes mirror is
checked against the header's sizes in test_abi_c.py): a binding struct with
fewer fields than the library writes would be overrun by every call."""
import os
import re

from clothcraft_b200 import abi

DOC = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "INTEGRATION.md")


def rust_fields(name):
    text = open(DOC).read()
    m = re.search(r"pub struct %s \{(.*?)\}" % name, text, re.S)
    assert m, name
    body = re.sub(r"/\*.*?\*/", "", m.group(1), flags=re.S)
    return re.findall(r"pub (\w+):", body)


def test_rust_structs_match_the_ctypes_mirror():
    for name in ("cc_vbd_settings", "cc_metrics", "cc_grab", "cc_ogc_settings", "cc_newton_report"):
        mirror = [f for f, _ in getattr(abi, name)._fields_]
        assert rust_fields(name) == mirror, name
