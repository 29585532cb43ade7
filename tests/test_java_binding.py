"""The Java Panama FFM binding (gpjson_b200/java/.../GpjNative.java) against
the C header: no JDK exists here, so its downcall handles are checked as
text — every entry point the header declares is bound under its name, with
a FunctionDescriptor whose layouts follow the C declaration (int / unsigned /
int32_t -> JAVA_INT, int64_t / uint64_t / size_t -> JAVA_LONG, pointers ->
ADDRESS, void -> ofVoid), and the gpj_server_config offsets it writes match
the C struct's (through the ctypes mirror of it)."""

from __future__ import annotations

import ctypes
import re

from gpjson_b200 import _lib
from tests.conftest import ROOT

JAVA = ROOT / "gpjson_b200" / "java" / "com" / "koenv" / "gpjson" / "gpu" / "GpjNative.java"
HEADER = ROOT / "include" / "gpjson_b200.h"


def c_layout(decl: str) -> str:
    decl = decl.strip()
    if "*" in decl:
        return "ADDRESS"
    words = decl.replace("const", "").split()
    base = words[0] if len(words) == 1 else " ".join(words[:-1]) if words[-1].isidentifier() and len(words) > 1 else words[0]
    base = base.strip()
    if base in ("int", "unsigned", "int32_t", "uint32_t"):
        return "JAVA_INT"
    if base in ("int64_t", "uint64_t", "size_t"):
        return "JAVA_LONG"
    if base == "void":
        return "VOID"
    raise AssertionError(f"no layout for C type {decl!r}")


def header_signatures() -> dict[str, list[str]]:
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    out = {}
    for m in re.finditer(r"([A-Za-z_][\w \t\*]*?)\b(gpj_\w+)\s*\(([^)]*)\)\s*;", text):
        ret, name, args = m.group(1), m.group(2), m.group(3)
        params = [a for a in (x.strip() for x in args.split(",")) if a and a != "void"]
        # drop the parameter names
        types = []
        for p in params:
            p = re.sub(r"\b[a-z_][a-z0-9_]*$", "", p.strip()) if not p.strip().endswith("*") else p
            types.append(c_layout(p if p.strip() else "int"))
        out[name] = [c_layout(ret)] + types
    return out


def java_signatures() -> dict[str, list[str]]:
    text = JAVA.read_text()
    out = {}
    for m in re.finditer(r'fn\("(gpj_\w+)",\s*FunctionDescriptor\.(ofVoid|of)\(([^;]*?)\)\);', text, flags=re.S):
        name, kind, args = m.group(1), m.group(2), m.group(3)
        layouts = [a.strip() for a in args.split(",") if a.strip()]
        out[name] = (["VOID"] + layouts) if kind == "ofVoid" else layouts
    return out


def test_java_binding_binds_every_entry_point_with_its_c_signature():
    want, got = header_signatures(), java_signatures()
    assert len(want) > 60
    assert set(got) == set(want), (set(want) - set(got), set(got) - set(want))
    for name, layouts in want.items():
        assert got[name] == layouts, (name, got[name], layouts)
    # the Python binding exports the same set
    assert set(got) == set(_lib.SIGNATURES)


def test_java_server_config_offsets_match_the_c_struct():
    text = JAVA.read_text()
    sets = re.findall(r"cfg\.set\((JAVA_INT|JAVA_LONG), (\d+), (\w+)\)", text)
    by_name = {"device": "device", "numLevels": "num_levels", "budgetBytes": "budget_bytes", "maxBatch": "max_batch",
               "workers": "workers"}
    assert len(sets) == 5
    for layout, off, var in sets:
        field = getattr(_lib.ServerConfig, by_name[var])
        assert field.offset == int(off), var
        assert field.size == (8 if layout == "JAVA_LONG" else 4), var
    assert ctypes.sizeof(_lib.ServerConfig) == 24
