"""Generate src/lib.rs, the raw Rust declarations of include/scrs_gpu.h.

    python rust/scrs-b200-sys/gen_bindings.py            # rewrite src/lib.rs
    python rust/scrs-b200-sys/gen_bindings.py --check    # exit 1 when it is stale

The header is plain C with one declaration per SCRS_API line group, so a small
parser suffices: status and enum constants become `pub const`, structs with a
body become `#[repr(C)]` structs, opaque handles zero-sized `#[repr(C)]`
structs, and every entry point one `extern "C"` declaration.
"""
import re
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
HEADER = HERE.parents[1] / "include" / "scrs_gpu.h"
OUT = HERE / "src" / "lib.rs"

SCALARS = {"int32_t": "i32", "uint32_t": "u32", "uint64_t": "u64", "uint16_t": "u16", "uint8_t": "u8",
           "int64_t": "i64", "float": "f32", "double": "f64", "char": "c_char", "void": "c_void",
           "size_t": "usize"}


RUST_KEYWORDS = {"as", "break", "const", "continue", "crate", "else", "enum", "extern", "false", "fn", "for", "if",
                 "impl", "in", "let", "loop", "match", "mod", "move", "mut", "pub", "ref", "return", "self", "static",
                 "struct", "super", "trait", "true", "type", "unsafe", "use", "where", "while", "async", "await",
                 "dyn"}


def ident(name: str) -> str:
    return f"r#{name}" if name in RUST_KEYWORDS else name


def strip_comments(text: str) -> str:
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    return re.sub(r"//[^\n]*", " ", text)


def rust_type(ctype: str, structs: set) -> str:
    """C type (possibly const-qualified pointers) -> Rust FFI type."""
    t = ctype.replace("*", " * ").split()
    base_const = False
    base = None
    ptrs = []  # constness of each pointer level, innermost first
    for tok in t:
        if tok == "const":
            if base is None:
                base_const = True
            elif ptrs:
                ptrs[-1] = True
        elif tok == "*":
            ptrs.append(False)
        elif base is None:
            base = tok
        else:
            raise ValueError(f"unparsed type: {ctype}")
    if base in SCALARS:
        r = SCALARS[base]
    elif base in structs:
        r = base
    else:
        raise ValueError(f"unknown type {base} in {ctype}")
    if not ptrs:
        return "()" if r == "c_void" else r
    # the first pointer points at the (possibly const) base; later ones at pointers
    consts = [base_const] + ptrs[:-1]
    for c in consts:
        r = ("*const " if c else "*mut ") + r
    return r


def split_decl(decl: str):
    """'const uint8_t* const* name' -> (type, name)."""
    m = re.match(r"(.*?)([A-Za-z_][A-Za-z0-9_]*)\s*$", decl.strip())
    return m.group(1).strip(), m.group(2)


def parse(text: str):
    code = strip_comments(text)
    consts = re.findall(r"\b(SCRS_[A-Z0-9_]+)\s*=\s*(-?\d+)", code)
    opaque = re.findall(r"typedef\s+struct\s+(\w+)\s+\1\s*;", code)
    bodies = re.findall(r"typedef\s+struct\s+(\w+)\s*\{(.*?)\}\s*\1\s*;", code, flags=re.S)
    structs = set(opaque) | {n for n, _ in bodies}
    out_structs = []
    for name, body in bodies:
        fields = []
        for stmt in body.split(";"):
            stmt = " ".join(stmt.split())
            if not stmt:
                continue
            first, *rest = [s.strip() for s in stmt.split(",")]
            ctype, fname = split_decl(first)
            fields.append((fname, rust_type(ctype, structs)))
            for extra in rest:  # 'uint64_t k, m, symbol_len'
                stars = extra.count("*")
                fields.append((extra.replace("*", "").strip(), rust_type(ctype + "*" * stars, structs)))
        out_structs.append((name, fields))
    funcs = []
    for m in re.finditer(r"^SCRS_API\s+([^;(]*?)\b(scrs_\w+)\s*\(([^;]*?)\)\s*;", code, flags=re.M):
        ret = " ".join(m.group(1).split())
        args = []
        params = " ".join(m.group(3).split())
        if params and params != "void":
            for p in params.split(","):
                ctype, pname = split_decl(p)
                args.append((pname, rust_type(ctype, structs)))
        funcs.append((m.group(2), rust_type(ret, structs), args))
    return consts, opaque, out_structs, funcs


def render(consts, opaque, structs, funcs) -> str:
    lines = ["//! Raw declarations of `include/scrs_gpu.h` (the B200 erasure-coding engines' C ABI).",
             "//! Generated by gen_bindings.py from the header; do not edit.",
             "#![allow(non_camel_case_types)]",
             "",
             "use core::ffi::{c_char, c_void};",
             ""]
    for name, value in consts:
        lines.append(f"pub const {name}: i32 = {value};")
    lines.append("")
    for name in opaque:
        lines += [f"#[repr(C)]", f"pub struct {name} {{", "    _private: [u8; 0],", "}", ""]
    for name, fields in structs:
        lines += ["#[repr(C)]", "#[derive(Clone, Copy, Debug)]", f"pub struct {name} {{"]
        lines += [f"    pub {ident(f)}: {t}," for f, t in fields]
        lines += ["}", ""]
    lines.append('extern "C" {')
    for name, ret, args in funcs:
        a = ", ".join(f"{ident(n)}: {t}" for n, t in args)
        r = "" if ret == "()" else f" -> {ret}"
        lines.append(f"    pub fn {name}({a}){r};")
    lines.append("}")
    return "\n".join(lines) + "\n"


def main():
    text = render(*parse(HEADER.read_text()))
    if "--check" in sys.argv:
        ok = OUT.exists() and OUT.read_text() == text
        print("up to date" if ok else "stale")
        sys.exit(0 if ok else 1)
    OUT.parent.mkdir(parents=True, exist_ok=True)
    OUT.write_text(text)
    print(OUT)


if __name__ == "__main__":
    main()
