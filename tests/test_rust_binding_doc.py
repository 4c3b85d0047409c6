"""The Rust binding given in INTEGRATION.md against the C ABI it binds.

Rust is not installed here, so the binding cannot be compiled; this checks by
parsing instead: every `#[repr(C)]` struct of the snippet has the same field
names, in the same order, as the typedef of the same name in
include/simlab_lbm.h, with matching element counts for arrays, and every
function the snippet declares exists in the header with the same number of
parameters.
"""
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
HDR = (ROOT / "include" / "simlab_lbm.h").read_text()
DOC = (ROOT / "INTEGRATION.md").read_text()


def c_structs():
    out = {}
    for body, name in re.findall(r"typedef struct \{(.*?)\}\s*(\w+);", HDR, re.S):
        fields = []
        body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
        for decl in body.split(";"):
            decl = decl.strip()
            if not decl:
                continue
            parts = decl.split(",")  # "uint64_t t0, t1": one type, several names
            m = re.match(r"(?:const\s+)?[\w\s]+?\s*\**\s*(\w+)((?:\[\d+\])*)$", parts[0].strip())
            assert m, decl
            names = [(m.group(1), m.group(2))] + [re.match(r"\**\s*(\w+)((?:\[\d+\])*)$", q.strip()).groups() for q in parts[1:]]
            for nm, arr in names:
                fields.append((nm, [int(d) for d in re.findall(r"\[(\d+)\]", arr)]))
        out[name] = fields
    return out


def rust_block():
    m = re.search(r"```rust\n(// crates/cfd/src/b200/ffi\.rs.*?)```", DOC, re.S)
    assert m, "the ffi block of INTEGRATION.md"
    return m.group(1)


def rust_structs(code):
    out = {}
    for name, body in re.findall(r"#\[repr\(C\)\](?:\s*#\[derive\([^)]*\)\])?\s*pub struct (\w+)\s*\{(.*?)\}", code, re.S):
        fields = []
        for f in re.findall(r"pub (\w+):\s*([^,]+?)\s*(?:,|$)", body.strip()):
            ty = f[1].strip()
            dims = [int(d) for d in re.findall(r";\s*(\d+)\]", ty)][::-1]
            fields.append((f[0], dims))
        out[name] = fields
    return out


def test_rust_structs_match_the_header():
    c = c_structs()
    r = rust_structs(rust_block())
    assert len(r) >= 11
    for name, fields in r.items():
        assert name in c, name
        assert fields == c[name], (name, fields, c[name])


def test_rust_functions_exist_in_the_header():
    code = rust_block()
    fns = re.findall(r"pub fn (lbm_\w+)\((.*?)\)", code, re.S)
    assert len(fns) >= 30
    for name, args in fns:
        m = re.search(r"\b" + name + r"\(([^;]*?)\);", HDR, re.S)
        assert m, name
        nc = 0 if m.group(1).strip() in ("", "void") else m.group(1).count(",") + 1
        nr = 0 if not args.strip() else args.count(",") + 1
        assert nc == nr, (name, nc, nr)
