"""The Rust binding in INTEGRATION.md against the C header, without a Rust
toolchain: every `#[repr(C)]` struct it declares has the C struct's size and
field offsets (computed with repr(C)'s layout rules, compared with what the
C compiler gives the header's struct for the fields of the same names), and
every `extern "C"` function it declares exists in the header with the same
number of parameters and matching parameter and return types (pointer
depth, constness of the pointee, and the width of scalars and pointees)."""
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "eschalign_b200.h")
DOC = os.path.join(ROOT, "INTEGRATION.md")

SCALAR = {"i8": (1, "i"), "u8": (1, "u"), "c_char": (1, "c"), "i32": (4, "i"), "u32": (4, "u"),
          "i64": (8, "i"), "u64": (8, "u"), "usize": (8, "u"), "c_void": (0, "v")}
C_SCALAR = {"int8_t": "i8", "uint8_t": "u8", "char": "c_char", "int32_t": "i32",
            "uint32_t": "u32", "int64_t": "i64", "uint64_t": "u64", "size_t": "usize",
            "int": "i32", "void": "c_void", "esg_status": "i32"}


def rust_code():
    text = open(DOC).read()
    return "\n".join(re.findall(r"```rust\n(.*?)```", text, flags=re.S))


def rust_structs():
    code = re.sub(r"/\*.*?\*/", "", rust_code(), flags=re.S)
    out = {}
    for name, body in re.findall(
            r"#\[repr\(C\)\](?:\s*#\[derive\([^)]*\)\])?\s*pub struct (\w+)\s*\{(.*?)\}", code,
            flags=re.S):
        fields = []
        for part in body.split(","):
            part = part.strip()
            if not part:
                continue
            m = re.match(r"pub (\w+)\s*:\s*(.+)$", part, flags=re.S)
            assert m, (name, part)
            fields.append((m.group(1), " ".join(m.group(2).split())))
        out[name] = fields
    return out


def c_name(rust):
    return "esg_" + re.sub(r"(?<!^)(?=[A-Z])", "_", rust[3:]).lower()


def layout(ty, structs):
    """(size, align) of a Rust type under repr(C)."""
    ty = ty.strip()
    if ty.startswith("*"):
        return 8, 8
    m = re.match(r"\[(.+);\s*(\d+)\]$", ty)
    if m:
        s, a = layout(m.group(1), structs)
        return s * int(m.group(2)), a
    if ty in SCALAR:
        return SCALAR[ty][0], SCALAR[ty][0]
    fields = structs[ty]
    off, align = 0, 1
    for _, fty in fields:
        s, a = layout(fty, structs)
        off = (off + a - 1) // a * a + s
        align = max(align, a)
    return (off + align - 1) // align * align, align


def offsets(name, structs):
    off, out = 0, []
    for fname, fty in structs[name]:
        s, a = layout(fty, structs)
        off = (off + a - 1) // a * a
        out.append((fname, off))
        off += s
    return out


def test_repr_c_structs_match_the_header(tmp_path):
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    structs = rust_structs()
    assert len(structs) >= 10, sorted(structs)
    lines = ["#include <stddef.h>", "#include <stdio.h>", f'#include "{HEADER}"',
             "int main(void) {"]
    for name in structs:
        cn = c_name(name)
        lines.append(f'printf("{name} size %zu\\n", sizeof({cn}));')
        for fname, _ in structs[name]:
            lines.append(f'printf("{name} {fname} %zu\\n", offsetof({cn}, {fname}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run([cc, "-o", str(exe), str(src)], check=True)
    got = {}
    for line in subprocess.run([str(exe)], check=True, capture_output=True,
                               text=True).stdout.splitlines():
        name, what, val = line.split()
        got[(name, what)] = int(val)
    for name in structs:
        assert got[(name, "size")] == layout(name, structs)[0], name
        for fname, off in offsets(name, structs):
            assert got[(name, fname)] == off, (name, fname)


def _c_param(p):
    """A C parameter or return type as (depth, pointee-or-scalar, const of
    the innermost pointee)."""
    p = re.sub(r"\b(esg_\w+|uint\w+|int\w+|char|void|size_t)\s+\w+$", r"\1", p.strip())
    p = re.sub(r"\s*\*\s*\w+$", "*", p)  # a named pointer parameter
    depth = p.count("*")
    base = p.replace("*", " ").replace("const", " ").split()
    base = base[-1] if base else ""
    inner_const = bool(re.match(r"\s*const\b", p)) and depth > 0
    base = C_SCALAR.get(base, base)
    if base.startswith("esg_") and base != "esg_status":
        base = "Esg" + "".join(w.capitalize() for w in base[4:].split("_"))
    return depth, base, inner_const


def _rust_param(t):
    t = " ".join(t.split())
    depth = 0
    consts = []
    while t.startswith("*"):
        m = re.match(r"\*(const|mut)\s+(.*)$", t)
        consts.append(m.group(1) == "const")
        t = m.group(2)
        depth += 1
    base = t.split("::")[-1]
    return depth, base, (consts[-1] if consts else False)


def header_functions():
    src = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    src = re.sub(r"#.*", "", src)
    out = {}
    for ret, name, params in re.findall(r"([\w\s\*]+?)\b(esg_\w+)\s*\(([^)]*)\)\s*;", src):
        ps = [] if params.strip() in ("", "void") else [x for x in params.split(",")]
        out[name] = (_c_param(ret.strip().split("\n")[-1]), [_c_param(x) for x in ps])
    return out


def test_extern_functions_match_the_header():
    hdr = header_functions()
    code = re.sub(r"//.*", "", rust_code())
    code = re.sub(r"/\*.*?\*/", "", code, flags=re.S)
    fns = re.findall(r"fn (esg_\w+)\((.*?)\)\s*(?:->\s*([^;]+?))?\s*;", code, flags=re.S)
    assert len(fns) >= 30, len(fns)
    for name, params, ret in fns:
        assert name in hdr, name
        c_ret, c_params = hdr[name]
        ps = [x for x in (p.strip() for p in params.split(",")) if x]
        r_params = [_rust_param(p.split(":", 1)[1]) for p in ps]
        assert len(r_params) == len(c_params), (name, len(r_params), len(c_params))
        for k, (rp, cp) in enumerate(zip(r_params, c_params)):
            assert rp[0] == cp[0], (name, k, "pointer depth", rp, cp)
            rb, cb = rp[1], cp[1]
            if rp[0] and cb in SCALAR and rb in SCALAR:
                assert SCALAR[rb][0] == SCALAR[cb][0], (name, k, rp, cp)
            else:
                assert rb == cb, (name, k, rp, cp)
            if rp[0]:
                assert rp[2] == cp[2], (name, k, "constness", rp, cp)
        r_ret = _rust_param(ret) if ret else (0, "c_void", False)
        assert r_ret[0] == c_ret[0] and (r_ret[1] == c_ret[1] or (
            r_ret[1] in SCALAR and c_ret[1] in SCALAR
            and SCALAR[r_ret[1]][0] == SCALAR[c_ret[1]][0])), (name, "return", r_ret, c_ret)
