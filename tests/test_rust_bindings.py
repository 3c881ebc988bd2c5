"""The Rust raw bindings (rust/scrs-b200-sys/src/lib.rs) are generated from
include/scrs_gpu.h: they are current, declare every entry point of the
header, and give each #[repr(C)] struct the header's fields in order.  (No
Rust toolchain here: the crate is checked as text.)"""
import re
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
GEN = ROOT / "rust" / "scrs-b200-sys" / "gen_bindings.py"
LIB = ROOT / "rust" / "scrs-b200-sys" / "src" / "lib.rs"


def test_bindings_are_current():
    r = subprocess.run([sys.executable, str(GEN), "--check"], capture_output=True, text=True)
    assert r.returncode == 0, "rust bindings are stale: run " + str(GEN)


def test_every_entry_point_is_declared():
    header = (ROOT / "include" / "scrs_gpu.h").read_text()
    declared = set(re.findall(r"^SCRS_API [^()]*?\b(scrs_[a-z0-9_]+)\(", header, flags=re.M))
    bound = set(re.findall(r"pub fn (scrs_[a-z0-9_]+)\(", LIB.read_text()))
    assert declared and declared == bound


def test_struct_fields_follow_the_header():
    rs = LIB.read_text()
    fields = dict(re.findall(r"pub struct (scrs_\w+) \{\n((?:    pub [^\n]*\n)*)\}", rs))
    assert [l.split(":")[0].split()[-1] for l in fields["scrs_stripe_desc"].splitlines()] == \
        ["op", "engine", "k", "m", "symbol_len", "r#in", "out", "indices"]
    assert "pub r#in: *const u8" in fields["scrs_request"]
    assert [l.split(":")[0].split()[-1] for l in fields["scrs_error"].splitlines()] == ["code", "reserved", "a", "b"]
