"""Extract the reference's known-answer tests into tests/golden/reference_kats.json.

Run in a container that has the SCRS reference sources:

    python tests/golden/make_kats.py /path/to/reference

The reference crate cannot be compiled here (no Rust toolchain), so its
known-answer assertions are read as text from its test modules:

* scrs/src/algebra/gf256.rs   known_small_products, inv_known_values,
                              known_powers_of_generator (EXP/LOG cycle)
* scrs/src/algebra/gf65536.rs known_answers_pin_basis_and_wire_order
* scrs/src/lib.rs             engine selection boundaries
* scrs/src/selector.rs        recommended_picks_engine_by_geometry,
                              resolve_rejects_bad_geometry
* scrs/src/batch/codec.rs     capacity boundaries, error-detail cases
* scrs/proptest-regressions/afft/differential.txt  regression seeds

The JSON also records the file:line of every extracted assertion.
"""
import json
import re
import sys
from pathlib import Path


def lines_of(root, rel):
    return (root / rel).read_text().splitlines()


def find(pattern, lines, rel):
    out = []
    rx = re.compile(pattern)
    for no, line in enumerate(lines, 1):
        m = rx.search(line)
        if m:
            out.append((no, m))
    if not out:
        raise SystemExit(f"pattern {pattern!r} not found in {rel}")
    return out


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_kats.py <path to the SCRS reference checkout>")
    root = Path(sys.argv[1])
    kats = {"source": "SCRS reference test modules (read as text)"}

    rel = "scrs/src/algebra/gf256.rs"
    L = lines_of(root, rel)
    kats["gf256_mul"] = [
        {"a": int(m.group(1), 16), "b": int(m.group(2), 16), "product": int(m.group(3), 16),
         "at": f"{rel}:{no}"}
        for no, m in find(r"GfElem\(0x([0-9A-Fa-f]+)\)\.mul\(GfElem\(0x([0-9A-Fa-f]+)\)\),\s*GfElem\(0x([0-9A-Fa-f]+)\)", L, rel)
    ]
    kats["gf256_inv"] = [
        {"a": int(m.group(1), 16), "inverse": int(m.group(2), 16), "at": f"{rel}:{no}"}
        for no, m in find(r"GfElem\(0x([0-9A-Fa-f]+)\)\.inv\(\),\s*GfElem\(0x([0-9A-Fa-f]+)\)", L, rel)
    ]
    (no, m), = find(r"pub const REDUCTION_POLY: u16 = 0x([0-9A-Fa-f]+);", L, rel)
    kats["gf256_poly"] = {"value": int(m.group(1), 16), "at": f"{rel}:{no}"}
    (no, m), = find(r"pub const GENERATOR: u8 = 0x([0-9A-Fa-f]+);", L, rel)
    kats["gf256_generator"] = {"value": int(m.group(1), 16), "at": f"{rel}:{no}"}

    rel = "scrs/src/algebra/gf65536.rs"
    L = lines_of(root, rel)
    kats["gf65536_mul"] = [
        {"a": int(m.group(1), 16), "b": int(m.group(2), 16), "product": int(m.group(3), 16), "at": f"{rel}:{no}"}
        for no, m in find(r"GfElem\(0x([0-9a-f]+)\)\.mul\(GfElem\(0x([0-9a-f]+)\)\),\s*GfElem\(0x([0-9a-f]+)\)", L, rel)
    ]
    kats["gf65536_square"] = [
        {"a": int(m.group(1), 16), "square": int(m.group(2), 16), "at": f"{rel}:{no}"}
        for no, m in find(r"GfElem\(0x([0-9a-f]+)\)\.square\(\),\s*GfElem\(0x([0-9a-f]+)\)", L, rel)
    ]
    kats["gf65536_inv"] = [
        {"a": int(m.group(1), 16), "inverse": int(m.group(2), 16), "at": f"{rel}:{no}"}
        for no, m in find(r"GfElem\(0x([0-9a-f]+)\)\.inv\(\),\s*GfElem\(0x([0-9a-f]+)\)", L, rel)
    ]
    kats["gf65536_to_bytes"] = [
        {"a": int(m.group(1), 16), "bytes": [int(m.group(2), 16), int(m.group(3), 16)], "at": f"{rel}:{no}"}
        for no, m in find(r"GfElem\(0x([0-9a-f]+)\)\.to_bytes\(\),\s*\[0x([0-9a-f]+),\s*0x([0-9a-f]+)\]", L, rel)
    ]
    (no, m), = find(r"pub const DELTA: BaseElem = BaseElem\(0x([0-9A-Fa-f]+)\);", L, rel)
    kats["gf65536_delta"] = {"value": int(m.group(1), 16), "at": f"{rel}:{no}"}
    (no, m), = find(r"pub const GENERATOR: GfElem = GfElem\(0x([0-9A-Fa-f]+)\);", L, rel)
    kats["gf65536_generator"] = {"value": int(m.group(1), 16), "at": f"{rel}:{no}"}

    rel = "scrs/src/lib.rs"
    L = lines_of(root, rel)
    kats["recommended_gf16_engine"] = [
        {"k": int(m.group(1)), "m": int(m.group(2)), "engine": m.group(3), "at": f"{rel}:{no}"}
        for no, m in find(r"recommended_gf16_engine\((\d+),\s*(\d+)\),\s*Gf16Engine::(\w+)", L, rel)
    ]

    rel = "scrs/src/selector.rs"
    L = lines_of(root, rel)
    text = "\n".join(L)
    rec = []
    for m in re.finditer(r"Profile::recommended\(Field::(\w+),\s*(\d+),\s*(\d+),\s*(\d+)\)\s*\.unwrap\(\)\s*\.engine\(\),\s*Engine::(\w+)", text):
        no = text[: m.start()].count("\n") + 1
        rec.append({"field": m.group(1), "k": int(m.group(2)), "m": int(m.group(3)),
                    "symbol_len": int(m.group(4)), "engine": m.group(5), "at": f"{rel}:{no}"})
    kats["profile_recommended"] = rec
    res = []
    for m in re.finditer(r"Profile::resolve\(Engine::(\w+),\s*(\d+),\s*(\d+),\s*(\d+)\),\s*Err\(ConfigError::(\w+)(?: \{ cap: (\d+) \})?\)", text):
        no = text[: m.start()].count("\n") + 1
        res.append({"engine": m.group(1), "k": int(m.group(2)), "m": int(m.group(3)),
                    "symbol_len": int(m.group(4)), "error": m.group(5),
                    "cap": int(m.group(6)) if m.group(6) else None, "at": f"{rel}:{no}"})
    kats["profile_resolve_errors"] = res

    rel = "scrs/src/batch/codec.rs"
    L = lines_of(root, rel)
    caps = []
    for no, m in find(r"crate::batch::(\w+)BatchCodec::new\((\d+),\s*(\d+),\s*(\d+)\)\.is_(ok|err)\(\)", L, rel):
        caps.append({"engine": m.group(1), "k": int(m.group(2)), "m": int(m.group(3)),
                     "symbol_len": int(m.group(4)), "ok": m.group(5) == "ok", "at": f"{rel}:{no}"})
    kats["batch_capacity"] = caps
    enc_cases = []
    for no, m in find(r"^\s*\((\d+usize|\d+),\s*(\d+usize|\d+),\s*(\d+usize|\d+)\),\s*$", L, rel):
        enc_cases.append([int(re.sub(r"usize", "", g)) for g in m.groups()] + [f"{rel}:{no}"])
    kats["batch_fast_vs_reference_cases"] = enc_cases

    rel = "scrs/proptest-regressions/afft/differential.txt"
    L = lines_of(root, rel)
    regs = []
    for no, line in enumerate(L, 1):
        m = re.search(r"k = (\d+), m = (\d+), field_elements = (\d+), data_source = \[([0-9, ]+)\], ordering = \[([0-9, ]+)\]", line)
        if m:
            regs.append({"k": int(m.group(1)), "m": int(m.group(2)), "field_elements": int(m.group(3)),
                         "data_source": [int(x) for x in m.group(4).split(",")],
                         "ordering": [int(x) for x in m.group(5).split(",")], "at": f"{rel}:{no}"})
    kats["afft_differential_regressions"] = regs

    out = Path(__file__).with_name("reference_kats.json")
    out.write_text(json.dumps(kats, indent=1) + "\n")
    print(f"wrote {out} ({sum(len(v) for v in kats.values() if isinstance(v, list))} entries)")


if __name__ == "__main__":
    main()
