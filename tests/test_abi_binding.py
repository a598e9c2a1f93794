"""The documented Rust binding against the C header.

Every `#[repr(C)] pub struct` block of INTEGRATION.md must list the fields of
the matching `typedef struct` of include/opendynamo.h with the same names,
order and C-equivalent types; its C layout size (natural alignment, as
`#[repr(C)]` lays it out on x86-64 and aarch64) must equal the ctypes mirror
the package uses and, for od_params, the library's own sizeof
(od_params_size). A binding that stops early would make od_default_params /
od_create read and write past a Rust-owned struct.
"""

from __future__ import annotations

import ctypes
import os
import re

import pytest

from opendynamo_b200 import _native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "opendynamo.h")
DOC = os.path.join(ROOT, "INTEGRATION.md")

# C type -> (Rust type, size, alignment) on LP64
C2RUST = {"int": ("i32", 4), "double": ("f64", 8), "float": ("f32", 4), "long long": ("i64", 8),
          "unsigned long long": ("u64", 8), "const char*": ("*const c_char", 8), "size_t": ("usize", 8)}
RUST_SIZE = {r: n for r, n in C2RUST.values()}
PAIRS = {"OdParams": ("od_params", N.OdParams), "OdRunOpts": ("od_run_opts", N.OdRunOpts),
         "OdRunResult": ("od_run_result", N.OdRunResult), "OdBox": ("od_box", N.OdBox),
         "OdIcParams": ("od_ic_params", N.OdIcParams)}


def _strip_comments(src: str) -> str:
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return re.sub(r"//[^\n]*", "", src)


def header_structs() -> dict:
    src = _strip_comments(open(HEADER).read())
    out = {}
    for m in re.finditer(r"typedef\s+struct\s+(\w+)\s*\{(.*?)\}\s*(\w+)\s*;", src, flags=re.S):
        fields = []
        for decl in m.group(2).split(";"):
            decl = " ".join(decl.split())
            if not decl:
                continue
            dm = re.match(r"((?:const\s+)?(?:unsigned\s+)?(?:long\s+long|int|double|float|char|size_t)\s*\*?)\s*(.*)",
                          decl)
            assert dm, decl
            ctype = dm.group(1).replace(" *", "*").strip()
            for name in dm.group(2).split(","):
                name = name.strip()
                if name.startswith("*"):
                    ctype, name = ctype + "*", name[1:].strip()
                fields.append((name, ctype))
        out[m.group(3)] = fields
    return out


def doc_structs() -> dict:
    text = open(DOC).read()
    out = {}
    for m in re.finditer(r"#\[repr\(C\)\]\s*pub struct (\w+)\s*\{(.*?)\}", text, flags=re.S):
        body = m.group(2)
        fields = re.findall(r"pub\s+(\w+)\s*:\s*([^,\n]+?)\s*(?:,|\n)", body)
        out[m.group(1)] = [(n, t.strip()) for n, t in fields]
    return out


def c_layout_size(types) -> int:
    off, align = 0, 1
    for t in types:
        n = RUST_SIZE[t]
        off = (off + n - 1) // n * n + n
        align = max(align, n)
    return (off + align - 1) // align * align


def test_every_header_struct_the_doc_binds_is_parsed():
    h = header_structs()
    for c_name, _ in PAIRS.values():
        assert c_name in h, c_name
    d = doc_structs()
    for rust in PAIRS:
        assert rust in d, f"INTEGRATION.md has no #[repr(C)] pub struct {rust}"


@pytest.mark.parametrize("rust", sorted(PAIRS))
def test_doc_struct_mirrors_header(rust):
    c_name, ct = PAIRS[rust]
    hf = header_structs()[c_name]
    df = doc_structs()[rust]
    assert [n for n, _ in df] == [n for n, _ in hf], (rust, df, hf)
    for (n, rt), (_, ctype) in zip(df, hf):
        assert C2RUST[ctype][0] == rt, (rust, n, rt, ctype)
    # ctypes mirror used by the package: same names and order, same size
    assert [f[0] for f in ct._fields_] == [n for n, _ in hf]
    assert c_layout_size([t for _, t in df]) == ctypes.sizeof(ct), rust


def test_params_size_matches_library():
    lib = N.lib()
    assert lib.od_params_size() == ctypes.sizeof(N.OdParams)
    rust = [t for _, t in doc_structs()["OdParams"]]
    assert c_layout_size(rust) == lib.od_params_size() == 120


def test_abi_version_matches_header_and_doc():
    src = open(HEADER).read()
    v = int(re.search(r"#define OD_ABI_VERSION (\d+)", src).group(1))
    assert N.lib().od_abi_version() == v
    doc = open(DOC).read()
    assert f"pub const OD_ABI_VERSION: i32 = {v};" in doc


def test_default_params_stay_inside_the_struct():
    """od_default_params writes exactly sizeof(od_params) bytes: a guard
    region after a ctypes OdParams is left untouched."""
    class Guarded(ctypes.Structure):
        _fields_ = [("p", N.OdParams), ("guard", ctypes.c_ubyte * 64)]
    g = Guarded()
    ctypes.memset(ctypes.byref(g.guard), 0xA5, 64)
    N.lib().od_default_params(ctypes.byref(g.p))
    assert bytes(g.guard) == b"\xa5" * 64
    assert g.p.viscosity_model == 0 and g.p.t_ref == 273.15 and g.p.s_suth == 110.4
