"""Pin the GF(65536) oracle engines (Tower, additive FFT) to the reference's
definitional tests: tower/encoder.rs:194-217, tower/decoder.rs:600-673,
afft/transform.rs:565-689, afft/encoder.rs:283-382, afft/decoder.rs:807-960,
afft/differential.rs (+ proptest-regressions/afft/differential.txt)."""
import ctypes as C
import json
from pathlib import Path

import numpy as np
import pytest

from scrs_b200.api import DEPENDENT, Engine, PushOutcome

import gfpy
from scenarios import encode_word, k_subsets, lazy_decode, lcg_permutations

KATS = json.loads((Path(__file__).parent / "golden" / "reference_kats.json").read_text())


def tower_data(k, L):  # tower/decoder.rs:560-567
    return np.array([((r * 37) ^ (b * 19) ^ 0x5A) & 0xFF for r in range(k) for b in range(L)], dtype=np.uint8)


def afft_data(k, L):  # afft/decoder.rs:774-778
    out = []
    for i in range(k * L):
        rot = ((i << 3) | (i >> 61)) & ((1 << 64) - 1)
        out.append(((i * 37) ^ rot ^ 0x5A) & 0xFF)
    return np.array(out, dtype=np.uint8)


def tower_coeff(k, m, i, j):
    x = gfpy.pow16(gfpy.GEN16, i)
    y = gfpy.pow16(gfpy.GEN16, k + j)
    return gfpy.inv16(x ^ y)


def test_tower_coefficients_and_incremental_sum(oracle, oracle_raw):  # tower/cauchy.rs, tower/encoder.rs:194
    k, m, L = 4, 3, 10
    out = (C.c_uint16 * (k * m))()
    assert oracle_raw.oracle_tower_coefficient_matrix(k, m, out) == 0
    for i in range(k):
        for j in range(m):
            assert out[i * m + j] == tower_coeff(k, m, i, j)
    p = oracle.resolve(Engine.TOWER, k, m, L)
    data = np.array([(r * 31 + b * 7) & 0xFF for r in range(k) for b in range(L)], dtype=np.uint8)
    word = encode_word(oracle, p, data)
    for j in range(m):
        exp = np.zeros(L, dtype=np.uint8)
        for i in range(k):
            exp ^= gfpy.scale16_bytes(data[i * L:(i + 1) * L], tower_coeff(k, m, i, j))
        assert np.array_equal(word[k + j], exp)




@pytest.mark.parametrize("k,m,L", [(4, 3, 18)])
def test_tower_exhaustive_small(oracle, k, m, L):  # tower/decoder.rs:600-614
    p = oracle.resolve(Engine.TOWER, k, m, L)
    data = tower_data(k, L)
    word = encode_word(oracle, p, data)
    for subset in k_subsets(k + m, k):
        assert np.array_equal(lazy_decode(oracle, p, word, subset), data)


def test_tower_beyond_gf256_capacity(oracle):  # tower/decoder.rs:616-633
    k, m, L = 256, 3, 4
    p = oracle.resolve(Engine.TOWER, k, m, L)
    data = tower_data(k, L)
    word = encode_word(oracle, p, data)
    order = [i for i in range(k + m) if i not in (17, 255, k + 2)]
    dec = oracle.decoder(p)
    for i in order:
        dec.push(i, word[i])
        if dec.is_complete():
            break
    assert dec.finalize() == data.tobytes()


def test_tower_random_patterns(oracle):  # tower/decoder.rs:635-656
    k, m, L = 64, 32, 66
    p = oracle.resolve(Engine.TOWER, k, m, L)
    data = tower_data(k, L)
    word = encode_word(oracle, p, data)
    for perm in lcg_permutations(k + m, 20):
        assert np.array_equal(lazy_decode(oracle, p, word, perm[:k]), data)


def test_push_bookkeeping_large_index(oracle):  # tower/decoder.rs:658-673, afft/decoder.rs:892-907
    for engine in (Engine.TOWER, Engine.AFFT):
        dec = oracle.decoder(oracle.resolve(engine, 300, 2, 2))
        assert dec.push(299, bytes([1, 2])) == PushOutcome.advanced(1, 1)
        assert dec.push(299, bytes([3, 4])) == DEPENDENT
        assert dec.rank() == 1


# ---- additive FFT -------------------------------------------------------

def subspace_polys(count):  # transform.rs:246-269
    coeffs = [1]
    out = []
    for dim in range(count):
        basis = 1 << dim
        norm = lin_eval(coeffs, basis)
        out.append((list(coeffs), gfpy.inv16(norm)))
        nxt = [0] * (len(coeffs) + 1)
        for i, c in enumerate(coeffs):
            nxt[i] ^= gfpy.mul16(norm, c)
            nxt[i + 1] ^= gfpy.mul16(c, c)
        coeffs = nxt
    return out


def lin_eval(coeffs, v):
    p, r = v, 0
    for c in coeffs:
        r ^= gfpy.mul16(c, p)
        p = gfpy.mul16(p, p)
    return r


def direct_evaluate(coefficients, point):  # transform.rs:565-582
    polys = subspace_polys(len(coefficients).bit_length() - 1)
    normalized = [gfpy.mul16(lin_eval(c, point), ni) for c, ni in polys]
    res = 0
    for idx, coef in enumerate(coefficients):
        bv = 1
        for bit, val in enumerate(normalized):
            if idx & (1 << bit):
                bv = gfpy.mul16(bv, val)
        res ^= gfpy.mul16(coef, bv)
    return res


def afft_forward(raw, vals):
    arr = (C.c_uint16 * len(vals))(*vals)
    assert raw.oracle_afft_forward(len(vals), arr) == 0
    return list(arr)


def test_transform_matches_direct_novel_basis(oracle_raw):  # transform.rs:599-615
    for size in [1, 2, 4, 8, 16, 32]:
        coefs = [((i * 0x2917) + 0x1357) & 0xFFFF for i in range(size)]
        expected = [direct_evaluate(coefs, pt) for pt in range(size)]
        assert afft_forward(oracle_raw, coefs) == expected


def test_forward_inverse_roundtrip(oracle_raw):  # transform.rs:617-633
    state = 0x12345678
    for size in [1, 2, 4, 8, 16, 64, 256, 1024]:
        vals = []
        for _ in range(size):
            state = (state * 1664525 + 1013904223) & 0xFFFFFFFF
            vals.append(state & 0xFFFF)
        arr = (C.c_uint16 * size)(*vals)
        oracle_raw.oracle_afft_forward(size, arr)
        oracle_raw.oracle_afft_inverse(size, arr)
        assert list(arr) == vals


def test_truncated_inverse_and_trunc_range(oracle_raw):  # transform.rs:634-689
    for size in [2, 4, 8, 16, 32]:
        for active in range(1, size + 1):
            coefs = [((i * 0x1F31) + 0x2345) & 0xFFFF if i < active else 0 for i in range(size)]
            evals = afft_forward(oracle_raw, coefs)
            rows = np.zeros(size * 2, dtype=np.uint8)
            for r in range(active):
                rows[2 * r:2 * r + 2] = [evals[r] & 0xFF, evals[r] >> 8]
            oracle_raw.oracle_afft_inverse_truncated_bytes(size, rows.ctypes.data_as(C.c_void_p), 2, active)
            got = [int(rows[2 * r]) | (int(rows[2 * r + 1]) << 8) for r in range(size)]
            assert got == coefs
    for size in [2, 4, 8, 16]:
        for active in range(1, size + 1):
            src = np.zeros(size * 2, dtype=np.uint8)
            for r in range(active):
                v = ((r * 0x2917) + 0x1357) & 0xFFFF
                src[2 * r:2 * r + 2] = [v & 0xFF, v >> 8]
            full = src.copy()
            oracle_raw.oracle_afft_forward_bytes(size, full.ctypes.data_as(C.c_void_p), 2)
            for start in range(size):
                for end in range(start + 1, size + 1):
                    ranged = src.copy()
                    oracle_raw.oracle_afft_forward_bytes_trunc_range(size, ranged.ctypes.data_as(C.c_void_p), 2,
                                                                     active, start, end)
                    assert np.array_equal(ranged[2 * start:2 * end], full[2 * start:2 * end])


def lagrange_repairs(data, k, m, L):
    """Repair j = the degree<k interpolant of data at points 0..k-1, evaluated
    at point k+j (afft/encoder.rs:346-382)."""
    out = np.zeros((m, L), dtype=np.uint8)
    for j in range(m):
        ev = k + j
        basis = []
        for d in range(k):
            num = den = 1
            for o in range(k):
                if o == d:
                    continue
                num = gfpy.mul16(num, ev ^ o)
                den = gfpy.mul16(den, d ^ o)
            basis.append(gfpy.mul16(num, gfpy.inv16(den)))
        for d in range(k):
            out[j] ^= gfpy.scale16_bytes(data[d * L:(d + 1) * L], basis[d])
    return out.reshape(-1)


@pytest.mark.parametrize("k,m,L", [(5, 3, 6), (8, 8, 4), (13, 3, 4), (4, 9, 2), (16, 16, 2)])
def test_afft_encode_is_lagrange_interpolation(oracle, k, m, L):  # afft/encoder.rs:346-382
    data = np.array([((i * 29) ^ 0xA5) & 0xFF for i in range(k * L)], dtype=np.uint8)
    word = encode_word(oracle, oracle.resolve(Engine.AFFT, k, m, L), data)
    assert np.array_equal(np.concatenate(word[k:]), lagrange_repairs(data, k, m, L))


def test_afft_strip_blocking_and_fusion(oracle_raw):  # afft/encoder.rs:294-344
    for (k, m, L, fused) in [(5, 3, 64, 0), (100, 20, 64, 0), (17, 7, 130, 0), (512, 128, 40, 0),
                             (4, 2, 64, 1), (16, 4, 40, 1), (256, 64, 48, 1), (512, 128, 40, 1)]:
        data = np.array([(i * (149 if fused else 137) + (3 if fused else 11)) & 0xFF for i in range(k * L)],
                        dtype=np.uint8)
        ref = np.zeros(m * L, dtype=np.uint8)
        oracle_raw.oracle_afft_encode_blocked(k, m, L, data.ctypes.data_as(C.c_void_p),
                                              ref.ctypes.data_as(C.c_void_p), L, 0)
        for width, fz in [(2, 0), (L, fused), (2, fused)]:
            got = np.zeros(m * L, dtype=np.uint8)
            oracle_raw.oracle_afft_encode_blocked(k, m, L, data.ctypes.data_as(C.c_void_p),
                                                  got.ctypes.data_as(C.c_void_p), width, fz)
            assert np.array_equal(got, ref), (k, m, L, width, fz)


def test_walsh_locator_matches_direct_products(oracle_raw):  # afft/decoder.rs:807-845
    for size in [2, 4, 8, 16, 64, 256]:
        known = np.array([(p % 3 == 0) or (p % 7 == 1) for p in range(size)], dtype=np.uint8)
        erased = [p for p in range(size) if not known[p]]
        vals = (C.c_uint16 * size)()
        ders = (C.c_uint16 * size)()
        oracle_raw.oracle_afft_locator(known.ctypes.data_as(C.c_void_p), size, vals, ders)
        for p in range(size):
            if known[p]:
                exp = 1
                for e in erased:
                    exp = gfpy.mul16(exp, p ^ e)
                assert vals[p] == exp and ders[p] == 0
            else:
                exp = 1
                for e in erased:
                    if e != p:
                        exp = gfpy.mul16(exp, p ^ e)
                assert ders[p] == exp and vals[p] == 0


@pytest.mark.parametrize("k,m,L", [(4, 4, 10), (5, 3, 6)])
def test_afft_exhaustive_recovery(oracle, k, m, L):  # afft/decoder.rs:848-876
    p = oracle.resolve(Engine.AFFT, k, m, L)
    data = afft_data(k, L)
    word = encode_word(oracle, p, data)
    for subset in k_subsets(k + m, k):
        assert np.array_equal(lazy_decode(oracle, p, word, subset), data)


def test_afft_random_patterns(oracle):  # afft/decoder.rs:878-890, :909-960
    for k, m, L in [(32, 16, 34), (16, 8, 64)]:
        p = oracle.resolve(Engine.AFFT, k, m, L)
        data = afft_data(k, L)
        word = encode_word(oracle, p, data)
        for perm in lcg_permutations(k + m, 20):
            assert np.array_equal(lazy_decode(oracle, p, word, perm[:k]), data)


def differential_case(oracle, k, m, fe, data_source, ordering):
    L = fe * 2
    data = np.array(data_source[:k * L], dtype=np.uint8)
    tw = encode_word(oracle, oracle.resolve(Engine.TOWER, k, m, L), data)
    af = encode_word(oracle, oracle.resolve(Engine.AFFT, k, m, L), data)
    idx = sorted(range(k + m), key=lambda i: (ordering[i], i))[:k]
    t = lazy_decode(oracle, oracle.resolve(Engine.TOWER, k, m, L), tw, idx)
    a = lazy_decode(oracle, oracle.resolve(Engine.AFFT, k, m, L), af, idx)
    assert np.array_equal(t, data) and np.array_equal(a, data)


@pytest.mark.parametrize("case", KATS["afft_differential_regressions"], ids=lambda c: c["at"])
def test_differential_regression_seeds(oracle, case):  # proptest-regressions/afft/differential.txt
    differential_case(oracle, case["k"], case["m"], case["field_elements"], case["data_source"], case["ordering"])


def test_differential_fuzz_against_tower(oracle):  # afft/differential.rs:27-55
    rng = np.random.default_rng(2024)
    for _ in range(64):
        k, m, fe = int(rng.integers(1, 13)), int(rng.integers(1, 13)), int(rng.integers(1, 9))
        differential_case(oracle, k, m, fe, list(rng.integers(0, 256, 12 * 16)),
                          list(rng.integers(0, 65536, 24)))
