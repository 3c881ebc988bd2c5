"""Pin the oracle's field arithmetic to the reference's known answers
(tests/golden/reference_kats.json, extracted from scrs/src/algebra/*.rs)."""
import ctypes as C
import json
from pathlib import Path

import numpy as np
import pytest

import gfpy

KATS = json.loads((Path(__file__).parent / "golden" / "reference_kats.json").read_text())


@pytest.fixture(scope="module")
def raw(oracle_raw):
    for n in ("oracle_gf256_mul", "oracle_gf256_mul_xtime"):
        getattr(oracle_raw, n).restype = C.c_uint8
        getattr(oracle_raw, n).argtypes = [C.c_uint8, C.c_uint8]
    for n in ("oracle_gf256_inv", "oracle_gf256_inv_xtime"):
        getattr(oracle_raw, n).restype = C.c_uint8
        getattr(oracle_raw, n).argtypes = [C.c_uint8]
    oracle_raw.oracle_gf256_exp.restype = C.c_uint8
    oracle_raw.oracle_gf256_exp.argtypes = [C.c_uint32]
    oracle_raw.oracle_gf65536_mul.restype = C.c_uint16
    oracle_raw.oracle_gf65536_mul.argtypes = [C.c_uint16, C.c_uint16]
    for n in ("oracle_gf65536_square", "oracle_gf65536_inv"):
        getattr(oracle_raw, n).restype = C.c_uint16
        getattr(oracle_raw, n).argtypes = [C.c_uint16]
    oracle_raw.oracle_gf65536_pow.restype = C.c_uint16
    oracle_raw.oracle_gf65536_pow.argtypes = [C.c_uint16, C.c_uint32]
    return oracle_raw


def test_gf256_constants_match_reference():
    assert KATS["gf256_poly"]["value"] == 0x11B
    assert KATS["gf256_generator"]["value"] == gfpy.GEN
    assert KATS["gf65536_delta"]["value"] == gfpy.DELTA
    assert KATS["gf65536_generator"]["value"] == gfpy.GEN16


@pytest.mark.parametrize("case", KATS["gf256_mul"], ids=lambda c: c["at"])
def test_gf256_known_products(raw, case):  # gf256.rs:430-441
    assert raw.oracle_gf256_mul(case["a"], case["b"]) == case["product"]
    assert gfpy.mul(case["a"], case["b"]) == case["product"]


@pytest.mark.parametrize("case", KATS["gf256_inv"], ids=lambda c: c["at"])
def test_gf256_known_inverses(raw, case):  # gf256.rs:443-451
    assert raw.oracle_gf256_inv(case["a"]) == case["inverse"]
    assert raw.oracle_gf256_inv(1) == 1 and raw.oracle_gf256_inv(0) == 0


def test_gf256_table_mul_matches_xtime_exhaustively(raw):  # gf256.rs:397-401
    for a in range(256):
        for b in range(0, 256, 7):
            assert raw.oracle_gf256_mul(a, b) == raw.oracle_gf256_mul_xtime(a, b) == gfpy.mul_xtime(a, b)
    for a in range(1, 256):
        assert raw.oracle_gf256_inv(a) == raw.oracle_gf256_inv_xtime(a)
        assert raw.oracle_gf256_mul(a, raw.oracle_gf256_inv(a)) == 1


def test_gf256_generator_cycles_all_nonzero(raw):  # gf256.rs:413-426, :459-465
    seen = {raw.oracle_gf256_exp(i) for i in range(255)}
    assert seen == set(range(1, 256))
    assert raw.oracle_gf256_exp(255) == 1


@pytest.mark.parametrize("case", KATS["gf65536_mul"], ids=lambda c: c["at"])
def test_gf65536_known_products(raw, case):  # gf65536.rs:223
    assert raw.oracle_gf65536_mul(case["a"], case["b"]) == case["product"]
    assert gfpy.mul16(case["a"], case["b"]) == case["product"]


def test_gf65536_known_square_inverse_bytes(raw):  # gf65536.rs:224-227
    for c in KATS["gf65536_square"]:
        assert raw.oracle_gf65536_square(c["a"]) == c["square"]
    for c in KATS["gf65536_inv"]:
        assert raw.oracle_gf65536_inv(c["a"]) == c["inverse"]
        assert gfpy.inv16(c["a"]) == c["inverse"]
    for c in KATS["gf65536_to_bytes"]:
        assert list(c["a"].to_bytes(2, "little")) == c["bytes"]


def test_gf65536_generator_is_primitive(raw):  # gf65536.rs:231-236
    for p in (3, 5, 17, 257):
        assert raw.oracle_gf65536_pow(gfpy.GEN16, 65535 // p) != 1
    assert raw.oracle_gf65536_pow(gfpy.GEN16, 65535) == 1


def test_gf65536_field_axioms_and_schoolbook(raw):  # gf65536.rs:238-261
    rng = np.random.default_rng(7)
    for a, b, c in rng.integers(0, 65536, size=(300, 3)):
        a, b, c = int(a), int(b), int(c)
        ab = raw.oracle_gf65536_mul(a, b)
        assert ab == gfpy.mul16(a, b) == raw.oracle_gf65536_mul(b, a)
        assert raw.oracle_gf65536_mul(ab, c) == raw.oracle_gf65536_mul(a, raw.oracle_gf65536_mul(b, c))
        assert raw.oracle_gf65536_mul(a, b ^ c) == ab ^ raw.oracle_gf65536_mul(a, c)
        if a:
            assert raw.oracle_gf65536_mul(a, raw.oracle_gf65536_inv(a)) == 1
