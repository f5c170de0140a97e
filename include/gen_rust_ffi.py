"""Generates umap_b200_ffi.rs, the Rust `extern "C"` declarations of every entry point, enum
constant and type in umap_b200.h, for a Rust crate that binds the library (the crate's
`src/ffi.rs`, which its build.rs links against libumap_b200.so and its safe wrappers call).

    python include/gen_rust_ffi.py            # rewrites include/umap_b200_ffi.rs
    python include/gen_rust_ffi.py --check    # exit 1 if the committed file is stale

The translation is mechanical (C99 fixed-width integers and floats to their Rust names,
`const T*` to `*const T`, `T*` to `*mut T`, opaque handles to zero-sized `#[repr(C)]`
structs), so the header stays the single source of truth.
"""
from __future__ import annotations

import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
HEADER = os.path.join(HERE, "umap_b200.h")
OUT = os.path.join(HERE, "umap_b200_ffi.rs")

BASE = {"uint64_t": "u64", "uint32_t": "u32", "int32_t": "i32", "uint8_t": "u8", "int": "c_int",
        "float": "f32", "double": "f64", "void": "c_void", "char": "c_char", "size_t": "usize"}


def _strip_comments(s: str) -> str:
    s = re.sub(r"/\*.*?\*/", " ", s, flags=re.S)
    return re.sub(r"//[^\n]*", " ", s)


def rust_type(ctype: str) -> str:
    t = " ".join(ctype.replace("*", " * ").split())
    stars = t.count("*")
    toks = [x for x in t.split() if x != "*"]
    const = toks[0] == "const"
    base = toks[-1]
    r = BASE.get(base, base)
    if stars == 0:
        return r
    inner = ("*const " if const else "*mut ") + r
    for _ in range(stars - 1):
        inner = "*mut " + inner
    return inner


def parse(header: str):
    src = _strip_comments(header)
    enums = []
    for body in re.findall(r"enum\s+\w+\s*\{(.*?)\}", src, re.S):
        for item in body.split(","):
            m = re.match(r"\s*(\w+)\s*=\s*(-?\d+)\s*$", item)
            if m:
                enums.append((m.group(1), int(m.group(2))))
    m = re.search(r"typedef\s+struct\s+umap_config\s*\{(.*?)\}\s*umap_config\s*;", src, re.S)
    fields = []
    for decl in m.group(1).split(";"):
        decl = " ".join(decl.split())
        if decl:
            typ, name = decl.rsplit(" ", 1)
            fields.append((name, rust_type(typ)))
    opaque = re.findall(r"typedef\s+struct\s+(\w+)\s+\1\s*;", src)
    funcs = []
    for ret, name, args in re.findall(r"^\s*(int|const char\s*\*)\s*(umap_\w+)\s*\(([^;]*?)\)\s*;", src, re.M | re.S):
        params = []
        args = " ".join(args.split())
        if args and args != "void":
            for a in args.split(","):
                a = a.strip()
                mm = re.match(r"(.*?)(\w+)$", a)
                params.append((mm.group(2), rust_type(mm.group(1))))
        funcs.append((name, rust_type(ret), params))
    ver = re.search(r"#define\s+UMAP_B200_ABI_VERSION\s+(\d+)", src).group(1)
    # other numeric #defines: layout flag bits (u32) and counts such as the warm start's phases
    defines = [(n, "u32" if u else "usize", v) for n, v, u in
               re.findall(r"^#define\s+(UMAP_\w+)\s+(\d+)(u?)\b", src, re.M) if n != "UMAP_B200_ABI_VERSION"]
    return ver, enums, fields, opaque, funcs, defines


def render(header: str) -> str:
    ver, enums, fields, opaque, funcs, defines = parse(header)
    out = ["// Generated from include/umap_b200.h by include/gen_rust_ffi.py; do not edit by hand.",
           "// Every entry point of the B200 UMAP library, for a Rust crate's src/ffi.rs.",
           "#![allow(non_camel_case_types, dead_code)]",
           "use std::os::raw::{c_char, c_int, c_void};",
           "",
           f"pub const UMAP_B200_ABI_VERSION: c_int = {ver};"]
    out += [f"pub const {n}: c_int = {v};" for n, v in enums]
    out += [f"pub const {n}: {t} = {v};" for n, t, v in defines]
    out += ["", "#[repr(C)]", "#[derive(Clone, Copy, Debug, Default)]", "pub struct umap_config {"]
    out += [f"    pub {n}: {t}," for n, t in fields]
    out += ["}", ""]
    for o in opaque:
        out += ["#[repr(C)]", f"pub struct {o} {{", "    _opaque: [u8; 0],", "}"]
    out += ["", "extern \"C\" {"]
    for name, ret, params in funcs:
        ps = ", ".join(f"{n}: {t}" for n, t in params)
        out.append(f"    pub fn {name}({ps}) -> {ret};")
    out += ["}", ""]
    return "\n".join(out)


def main() -> int:
    text = render(open(HEADER).read())
    if "--check" in sys.argv:
        ok = os.path.exists(OUT) and open(OUT).read() == text
        if not ok:
            print("include/umap_b200_ffi.rs is stale: run python include/gen_rust_ffi.py", file=sys.stderr)
        return 0 if ok else 1
    with open(OUT, "w") as f:
        f.write(text)
    return 0


if __name__ == "__main__":
    sys.exit(main())
