"""The Rust trait-impl crate (rust/scrs-b200) over the C ABI: every status
code the header defines maps to exactly one variant of the reference's error
enums (or, for the runtime codes, to RuntimeFailure) in its error module, and
the crate implements each trait of the reference's surface with the methods
the trait declares.  (No Rust toolchain here: the crate is checked as text.)"""
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
HEADER = (ROOT / "include" / "scrs_gpu.h").read_text()
ERR = (ROOT / "rust" / "scrs-b200" / "src" / "error.rs").read_text()
LIB = (ROOT / "rust" / "scrs-b200" / "src" / "lib.rs").read_text()


def header_status_codes():
    block = HEADER[HEADER.index("/* ---- status codes"):HEADER.index("/* PushOutcome")]
    return dict((n, int(v)) for n, v in re.findall(r"(SCRS_(?:OK|CONFIG_\w+|ENCODE_\w+|DECODE_\w+|ERR_\w+))\s*=\s*(\d+)",
                                                    block))


def check_arms():
    body = ERR[ERR.index("pub fn check("):ERR.index("pub(crate) fn config(")]
    arms = {}
    for names, target in re.findall(r"((?:sys::SCRS_\w+\s*\|?\s*)+)=>\s*(return Ok\(\(\)\)|Failure::\w+\((?:\w+::\w+)?)",
                                    body):
        for n in re.findall(r"sys::(SCRS_\w+)", names):
            assert n not in arms, f"{n} has two arms"
            arms[n] = target
    return arms


def test_every_status_maps_to_exactly_one_variant():
    codes = header_status_codes()
    arms = check_arms()
    assert set(arms) == set(codes), set(codes) ^ set(arms)
    variants = [arms[n] for n in codes if not n.startswith("SCRS_ERR") and n != "SCRS_OK"]
    assert len(variants) == len(set(variants)), "two codes map to one reference variant"
    for name in codes:
        target = arms[name]
        if name == "SCRS_OK":
            assert target.startswith("return Ok")
        elif name.startswith("SCRS_CONFIG_"):
            assert target.startswith("Failure::Config(ConfigError::")
        elif name.startswith("SCRS_ENCODE_"):
            assert target.startswith("Failure::Encode(EncodeError::")
        elif name.startswith("SCRS_DECODE_"):
            assert target.startswith("Failure::Decode(DecodeError::")
        else:
            assert target.startswith("Failure::Runtime(")


def test_variant_names_follow_the_python_mirror():
    """The Rust mapping and scrs_b200/api.py's status table name the same
    reference variant for every code."""
    from scrs_b200.api import _STATUS

    codes = header_status_codes()
    arms = check_arms()
    for name, code in codes.items():
        if code == 0 or code >= 900:
            continue
        cls, variant, _ = _STATUS[code]
        assert arms[name] == f"Failure::{cls[:-5]}({cls}::{variant}", (name, arms[name], cls, variant)


def test_trait_impls_cover_the_reference_surface():
    want = {
        "BatchEncoder for GpuBatchEncoder": ["fn scratch(", "fn encode_into(", "fn encode_into_with("],
        "BatchDecoder for GpuBatchDecoder": ["fn scratch(", "fn decode_into(", "fn decode_into_with("],
        "IncrementalEncoder for GpuIncrementalEncoder": ["fn feed(", "fn repair(", "fn fed_count(", "fn reset("],
        "SymbolSink for GpuDecoder": ["fn push(", "fn is_complete(", "fn finalize("],
        "Decoder for GpuDecoder": ["fn scratch(", "fn rank(", "fn received(", "fn reset(", "fn finalize_into(",
                                   "fn finalize_into_with("],
    }
    for head, fns in want.items():
        i = LIB.index("impl " + head + " {")
        body = LIB[i:LIB.index("\n}\n", i)]
        for f in fns:
            assert f in body, (head, f)
    for fac in ("pub fn batch_encoder(", "pub fn batch_decoder(", "pub fn incremental_encoder(", "pub fn decoder("):
        assert fac in LIB
    # every raw call the crate makes is declared by the raw bindings
    sys_rs = (ROOT / "rust" / "scrs-b200-sys" / "src" / "lib.rs").read_text()
    for fn in set(re.findall(r"sys::(scrs_\w+)\(", LIB + ERR)):
        assert f"pub fn {fn}(" in sys_rs, fn
