"""The Rust binding (bindings/rust, not compiled here: no Rust toolchain)
against the C header: its #[repr(C)] structs list the header's fields in
the header's order, and every function it declares exists in the header
and in the built library."""
import os
import re

from rtrace_b200 import _capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
RS = open(os.path.join(ROOT, "bindings", "rust", "src", "lib.rs")).read()
HEADER = open(os.path.join(ROOT, "include", "rtrace_gpu.h")).read()


def rust_fields(name):
    m = re.search(r"pub struct %s \{(.*?)\n    \}" % name, RS, re.S)
    assert m, name
    return re.findall(r"pub (\w+):", m.group(1))


def test_structs_follow_the_header():
    for rs, ct in (("RtOutlineConfig", _capi.rt_outline_config), ("RtRenderParams", _capi.rt_render_params),
                   ("RtStats", _capi.rt_stats)):
        assert rust_fields(rs) == [f[0] for f in ct._fields_], rs


def test_declared_functions_exist():
    names = re.findall(r"pub fn (rt_\w+)\(", RS)
    assert len(names) >= 10
    for n in names:
        assert re.search(r"\b%s\(" % n, HEADER), n
