"""The ctypes mirrors of the C ABI's structs (scrs_b200/*.py) against
include/scrs_gpu.h: same fields, in the same order, with the same sizes, so
that adding a field on one side without the other fails here and not as
garbage on a GPU box.  The header is parsed with the Rust raw-bindings
generator's parser (rust/scrs-b200-sys/gen_bindings.py)."""
import ctypes as C
import importlib.util
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]

# Rust FFI type (as the generator renders it) -> byte size on x86-64
SIZES = {"i32": 4, "u32": 4, "u16": 2, "u8": 1, "i64": 8, "u64": 8, "f32": 4, "f64": 8, "usize": 8}


def header_structs():
    spec = importlib.util.spec_from_file_location("gen_bindings", ROOT / "rust" / "scrs-b200-sys" / "gen_bindings.py")
    gb = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(gb)
    _, _, structs, _ = gb.parse((ROOT / "include" / "scrs_gpu.h").read_text())
    return {name: fields for name, fields in structs}


def mirrors():
    from scrs_b200 import api, batch, serving, tune

    return {"scrs_profile": api._Profile, "scrs_error": api._Error, "scrs_push_outcome": api._Push,
            "scrs_stripe_desc": batch._Desc, "scrs_tune_key": tune._Key, "scrs_tune_params": tune._Params,
            "scrs_request": serving._Request, "scrs_completion": serving._Completion,
            "scrs_server_stats": serving._Stats}


def field_size(rust_type: str) -> int:
    return 8 if rust_type.startswith("*") else SIZES[rust_type]


def test_every_header_struct_has_a_mirror():
    assert set(header_structs()) == set(mirrors())


@pytest.mark.parametrize("name", sorted(header_structs()))
def test_mirror_matches_header(name):
    fields = header_structs()[name]
    mirror = mirrors()[name]
    got = [(f[0].rstrip("_"), C.sizeof(f[1])) for f in mirror._fields_]
    want = [(n, field_size(t)) for n, t in fields]
    assert got == want, (name, got, want)
    # natural alignment on both sides: the offsets then agree as well
    off = 0
    for (n, t), f in zip(fields, mirror._fields_):
        size = field_size(t)
        off = (off + size - 1) // size * size
        assert getattr(mirror, f[0]).offset == off, (name, n)
        off += size
