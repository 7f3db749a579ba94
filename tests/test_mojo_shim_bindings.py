"""Static check of the Mojo FFI shims (mojoblas_b200/mojo/*.mojo) against the C ABI.

Mojo is not installed where these tests run, so the shims cannot be compiled
here; what can break silently is the binding itself.  Every
`lib.get_function[fn (...) -> R]("mbg_...")` in the shims must name a function
that include/mojoblas_gpu.h declares and the library exports, with the same
number of arguments and, position by position, the Mojo type that carries the
C type: Int8 for char, Int32 for int, Int64 for int64_t, Float32 for float,
Float64 for double, OpaquePointer for any pointer.
"""
import re
from pathlib import Path

import pytest

from mojoblas_b200 import _lib as L

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "mojoblas_gpu.h"
SHIMS = sorted((ROOT / "mojoblas_b200" / "mojo").glob("*.mojo"))


def c_kind(decl: str) -> str:
    decl = decl.strip()
    if "*" in decl:
        return "ptr"
    words = decl.replace("const", "").split()
    base = words[0] if words else ""
    return {"char": "i8", "int": "i32", "int64_t": "i64", "float": "f32", "double": "f64"}[base]


MOJO_KIND = {"Int8": "i8", "Int32": "i32", "Int64": "i64", "Float32": "f32", "Float64": "f64",
             "OpaquePointer": "ptr"}


def header_signatures():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    sigs = {}
    for ret, name, args in re.findall(r"([\w\s\*]+?)\b(mbg_\w+)\s*\(([^)]*)\)\s*;", text):
        args = args.strip()
        kinds = [] if args in ("", "void") else [c_kind(a) for a in args.split(",")]
        ret = ret.strip()
        sigs[name] = ("ptr" if ret.endswith("*") else c_kind(ret.split()[-1]), kinds)
    return sigs


def shim_bindings():
    out = []
    for path in SHIMS:
        text = path.read_text()
        for params, ret, name in re.findall(
                r"get_function\[\s*fn\s*\((.*?)\)\s*->\s*(\w+)\s*\]\(\"(mbg_\w+)\"\)", text, flags=re.S):
            kinds = [MOJO_KIND[t.strip()] for t in params.split(",") if t.strip()]
            out.append((path.name, name, MOJO_KIND[ret], kinds))
    return out


def test_shims_bind_something():
    names = {b[1] for b in shim_bindings()}
    # host shims: the twelve level-3 routines and four level-2 ones; device shim: the _ex forms and the runtime
    for sym in ("mbg_sgemm", "mbg_dtrsm", "mbg_dsyr2k", "mbg_strmm", "mbg_sgemv", "mbg_dtrsv", "mbg_dgemm_ex",
                "mbg_dsymm_ex", "mbg_set_stream", "mbg_synchronize"):
        assert sym in names, sym


@pytest.mark.parametrize("binding", shim_bindings(), ids=lambda b: f"{b[0]}:{b[1]}")
def test_binding_matches_header(binding):
    shim, name, ret, kinds = binding
    sigs = header_signatures()
    assert name in sigs, f"{shim} binds {name}, which the header does not declare"
    c_ret, c_kinds = sigs[name]
    assert ret == c_ret, (name, ret, c_ret)
    assert kinds == c_kinds, (name, kinds, c_kinds)


def test_bound_symbols_are_exported():
    lib = L.load()
    missing = sorted({b[1] for b in shim_bindings() if not hasattr(lib, b[1])})
    assert not missing, missing
