"""The Rust crate (llr-reco_b200/rust) is checked here without a Rust toolchain: every function
its extern block declares exists in include/llr_b200.h with the same parameter count and is
exported by the built library, and its llr_config mirrors the C struct field by field."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CRATE = os.path.join(ROOT, "llr-reco_b200", "rust")
HEADER = os.path.join(ROOT, "include", "llr_b200.h")
LIB = os.path.join(ROOT, "llr-reco_b200", "libllr_b200.so")


def _strip_c_comments(s):
    return re.sub(r"/\*.*?\*/", "", s, flags=re.S)


def _c_decls():
    txt = _strip_c_comments(open(HEADER).read())
    out = {}
    for m in re.finditer(r"\b(?:int|const char\*|cudaError_t)\s+(\w+)\s*\(([^;{]*?)\)\s*;", txt, flags=re.S):
        args = m.group(2).strip()
        out[m.group(1)] = 0 if args in ("", "void") else args.count(",") + 1
    return out


def _rust_decls():
    txt = open(os.path.join(CRATE, "src", "ffi.rs")).read()
    block = txt[txt.index('extern "C" {'):]
    out = {}
    for m in re.finditer(r"pub fn (\w+)\s*\(([^)]*)\)", block, flags=re.S):
        args = re.sub(r"//[^\n]*", "", m.group(2)).strip().rstrip(",")
        out[m.group(1)] = 0 if not args else args.count(",") + 1
    return out


def test_crate_files_exist():
    for f in ("Cargo.toml", "build.rs", "src/lib.rs", "src/ffi.rs", "tests/recon.rs"):
        assert os.path.isfile(os.path.join(CRATE, f)), f


def test_extern_block_matches_header_and_library():
    c = _c_decls()
    r = _rust_decls()
    assert len(r) > 50
    lib = ctypes.CDLL(LIB) if os.path.exists(LIB) else None
    for name, n in r.items():
        assert name in c, f"{name} is not declared in llr_b200.h"
        assert c[name] == n, f"{name}: {n} parameters in Rust, {c[name]} in C"
        if lib is not None:
            assert hasattr(lib, name), f"{name} is not exported"


def test_config_struct_mirrors_c():
    txt = _strip_c_comments(open(HEADER).read())
    body = txt[txt.index("typedef struct llr_config {"):txt.index("} llr_config;")]
    c_fields = re.findall(r"\b(?:int32_t|float|uint64_t)\s+(\w+)(?:\[3\])?\s*;", body)
    rs = open(os.path.join(CRATE, "src", "ffi.rs")).read()
    rbody = rs[rs.index("pub struct llr_config {"):]
    rbody = rbody[:rbody.index("}")]
    r_fields = re.findall(r"pub (\w+):", rbody)
    assert r_fields == c_fields
    if os.path.exists(LIB):
        import llr_b200._lib as L
        assert ctypes.sizeof(L.llr_config) == 120
