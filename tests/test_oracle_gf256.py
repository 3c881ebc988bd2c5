"""Pin the GF(256) oracle engines to the reference's definitional tests
(scrs/src/batch/codec.rs, encoder/streaming.rs, decoder/streaming.rs,
matrices/{cauchy,good_cauchy}.rs)."""
import ctypes as C
import json
from pathlib import Path

import numpy as np
import pytest

from scrs_b200.api import COMPLETE, DEPENDENT, DecodeError, EncodeError, Engine, PushOutcome

import gfpy
from scenarios import (batch_decode, data_for, deterministic_subsets, direct_gf256_repairs,
                       encode_word, k_subsets, lazy_decode)

KATS = json.loads((Path(__file__).parent / "golden" / "reference_kats.json").read_text())
GF256 = [Engine.STANDARD_CAUCHY, Engine.GOOD_CAUCHY]


def coeffs(raw, engine, k, m):
    out = (C.c_uint8 * (k * m))()
    raw.oracle_gf256_coefficient_matrix(int(engine), k, m, out)
    return np.frombuffer(bytes(out), dtype=np.uint8)


def test_coefficients_are_cauchy(oracle_raw):  # cauchy.rs:38-101, good_cauchy.rs:90-144
    for k, m in [(3, 2), (10, 4), (64, 16), (200, 55), (1, 254), (254, 1)]:
        std = coeffs(oracle_raw, Engine.STANDARD_CAUCHY, k, m)
        for i in range(k):
            for j in range(m):
                assert std[i * m + j] == gfpy.inv(i ^ (k + j))
        if k + m <= 255:
            good = coeffs(oracle_raw, Engine.GOOD_CAUCHY, k, m)
            for i in range(k):
                for j in range(m):
                    # get(i,j) = inv(g^i + g^(k+j)) equals the diagonal factorization
                    assert good[i * m + j] == gfpy.inv(gfpy.EXP[i % 255] ^ gfpy.EXP[(k + j) % 255])
                    assert good[i * m + j] != 0


@pytest.mark.parametrize("engine", GF256)
@pytest.mark.parametrize("k,m,L", [(1, 1, 2), (4, 2, 16), (8, 4, 64), (16, 8, 1024), (32, 16, 1024),
                                   (128, 64, 1024), (200, 50, 256), (1, 254, 64), (254, 1, 64), (3, 5, 7)])
def test_encode_matches_direct_sum(oracle, oracle_raw, engine, k, m, L):
    # optimized_encode_matches_reference (codec.rs:1072-1107) and
    # prop_encode_repair_correctness (codec.rs:913-933)
    if engine == Engine.GOOD_CAUCHY and k + m > 255:
        pytest.skip("Good Cauchy capacity is 255")
    p = oracle.resolve(engine, k, m, L)
    data = np.array([(x * 131 + 7) & 0xFF for x in range(k * L)], dtype=np.uint8)
    out = np.zeros(m * L, dtype=np.uint8)
    enc = oracle.batch_encoder(p)
    enc.encode_into_with(data, out, enc.scratch())
    assert np.array_equal(out, direct_gf256_repairs(coeffs(oracle_raw, engine, k, m), data, k, m, L))


@pytest.mark.parametrize("engine", GF256)
@pytest.mark.parametrize("k,m,L", [(3, 2, 4), (4, 3, 8), (3, 3, 4)])
def test_roundtrip_all_subsets(oracle, engine, k, m, L):  # codec.rs:706-799
    p = oracle.resolve(engine, k, m, L)
    data = np.array([((i * 7) & 0xFF) for i in range(k * L)], dtype=np.uint8)
    word = encode_word(oracle, p, data)
    for subset in k_subsets(k + m, k):
        assert np.array_equal(batch_decode(oracle, p, word, subset), data), subset
        assert np.array_equal(lazy_decode(oracle, p, word, subset[::-1]), data), subset


@pytest.mark.parametrize("k,m,L", [(1, 1, 2), (4, 2, 16), (8, 4, 64), (6, 6, 33), (16, 8, 100), (32, 16, 64)])
def test_decode_matches_rref_reference(oracle, oracle_raw, k, m, L):
    # optimized_decode_matches_reference (codec.rs:936-1014)
    oracle_raw.oracle_gf256_rref_decode.restype = C.c_size_t
    data = np.array([(x * 131 + 7) & 0xFF for x in range(k * L)], dtype=np.uint8)
    for engine in GF256:
        p = oracle.resolve(engine, k, m, L)
        word = encode_word(oracle, p, data)
        for subset in deterministic_subsets(k, m):
            fast = batch_decode(oracle, p, word, subset)
            idx = (C.c_uint64 * k)(*subset)
            ptrs = (C.c_void_p * k)(*[word[i].ctypes.data for i in subset])
            ref = np.zeros(k * L, dtype=np.uint8)
            rank = oracle_raw.oracle_gf256_rref_decode(int(engine), k, m, L, idx, ptrs, ref.ctypes.data_as(C.c_void_p))
            assert rank == k
            assert np.array_equal(fast, ref) and np.array_equal(fast, data)
            lazy = lazy_decode(oracle, p, word, subset)
            assert np.array_equal(lazy, data)


def test_decode_error_details(oracle):  # codec.rs:803-870, :1016-1047
    p = oracle.resolve(Engine.STANDARD_CAUCHY, 3, 2, 4)
    dec = oracle.batch_decoder(p)
    word = encode_word(oracle, p, np.zeros(12, dtype=np.uint8))
    out = np.zeros(12, dtype=np.uint8)
    s = dec.scratch()
    with pytest.raises(DecodeError) as e:
        dec.decode_into_with([(0, word[0]), (1, word[1])], out, s)
    assert e.value.variant == "WrongCount" and e.value.fields == {"expected": 3, "got": 2}
    with pytest.raises(DecodeError) as e:
        dec.decode_into_with([(0, word[0]), (1, word[1]), (5, np.zeros(4, np.uint8))], out, s)
    assert e.value.variant == "IndexOutOfRange" and e.value.fields == {"index": 5, "n": 5}
    with pytest.raises(DecodeError) as e:
        dec.decode_into_with([(0, word[0]), (1, word[1]), (0, word[0])], out, s)
    assert e.value.variant == "DuplicateIndex" and e.value.fields == {"index": 0}
    with pytest.raises(DecodeError) as e:
        dec.decode_into_with([(0, word[0]), (1, word[1]), (2, np.zeros(3, np.uint8))], out, s)
    assert e.value.variant == "WrongPayloadLen" and e.value.fields == {"expected": 4, "got": 3}
    with pytest.raises(DecodeError) as e:
        dec.decode_into_with([(0, word[0]), (1, word[1]), (2, word[2])], np.zeros(11, np.uint8), s)
    assert e.value.fields == {"expected": 12, "got": 11}
    other = oracle.batch_decoder(oracle.resolve(Engine.STANDARD_CAUCHY, 4, 2, 4))
    with pytest.raises(DecodeError) as e:
        dec.decode_into_with([(0, word[0]), (1, word[1]), (2, word[2])], out, other.scratch())
    assert e.value.variant == "ScratchMismatch"


def test_encode_error_details(oracle):  # codec.rs:682-692
    enc = oracle.batch_encoder(oracle.resolve(Engine.STANDARD_CAUCHY, 3, 2, 4))
    with pytest.raises(EncodeError) as e:
        enc.encode_into(np.zeros(11, np.uint8), np.zeros(8, np.uint8))
    assert e.value.variant == "WrongInputLen" and e.value.fields == {"expected": 12, "got": 11}
    with pytest.raises(EncodeError) as e:
        enc.encode_into(np.zeros(12, np.uint8), np.zeros(9, np.uint8))
    assert e.value.variant == "WrongOutputLen" and e.value.fields == {"expected": 8, "got": 9}


def test_decode_overwrites_garbage_output(oracle):  # codec.rs:1049-1069
    p = oracle.resolve(Engine.STANDARD_CAUCHY, 4, 3, 17)
    data = np.array([((x * 29) & 0xFF) ^ 0x5C for x in range(4 * 17)], dtype=np.uint8)
    word = encode_word(oracle, p, data)
    assert np.array_equal(batch_decode(oracle, p, word, [0, 2, 4, 5]), data)


def test_streaming_encoder_matches_batch(oracle):  # good_cauchy.rs:276-307, encoder/streaming.rs
    for k, m, L in [(4, 3, 8), (10, 4, 64), (60, 16, 33)]:
        p = oracle.resolve(Engine.GOOD_CAUCHY, k, m, L)
        data = data_for(k, L, 11)
        word = encode_word(oracle, p, data)
        inc = oracle.incremental_encoder(p)
        for i in reversed(range(k)):
            inc.feed(i, data[i * L:(i + 1) * L])
        assert inc.fed_count() == k
        for j in range(m):
            assert inc.repair(j) == word[k + j].tobytes()
        with pytest.raises(EncodeError) as e:
            inc.feed(0, data[:L])
        assert e.value.variant == "DuplicateData" and e.value.fields == {"index": 0}
        with pytest.raises(EncodeError) as e:
            inc.feed(k, data[:L])
        assert e.value.fields == {"index": k, "n": k + m}
        with pytest.raises(EncodeError) as e:
            inc.feed(1, data[:L - 1])
        assert e.value.variant == "WrongPayloadLen"
        with pytest.raises(EncodeError) as e:
            inc.repair(m)
        assert e.value.variant == "IndexOutOfRange" and e.value.fields == {"index": m, "n": k + m}
        inc.reset()
        assert inc.fed_count() == 0 and inc.repair(0) == bytes(L)


def test_lazy_decoder_push_contract(oracle):  # decoder/streaming.rs:388-438
    k, m, L = 4, 3, 8
    p = oracle.resolve(Engine.STANDARD_CAUCHY, k, m, L)
    data = data_for(k, L, 3)
    word = encode_word(oracle, p, data)
    dec = oracle.decoder(p)
    assert dec.push(k, word[k]) == PushOutcome.advanced(1, 1)
    assert dec.push(k, word[k]) == DEPENDENT
    assert dec.push(1, word[1]) == PushOutcome.advanced(2, 3)
    assert dec.push(2, word[2]) == PushOutcome.advanced(3, 4)
    with pytest.raises(DecodeError) as e:
        dec.finalize_into(np.zeros(k * L, np.uint8))
    assert e.value.variant == "InsufficientRank" and e.value.fields == {"rank": 3, "k": 4}
    assert dec.push(k + 1, word[k + 1]) == COMPLETE
    assert dec.is_complete() and dec.rank() == 4 and dec.received() == 5
    assert dec.push(0, word[0]) == DEPENDENT
    assert dec.push(3, word[3]) == DEPENDENT
    with pytest.raises(DecodeError) as e:
        dec.push(3, word[3])
    assert e.value.variant == "TooManySymbols" and e.value.fields == {"cap": 7, "received": 7}
    with pytest.raises(DecodeError) as e:
        dec.finalize_into(np.zeros(k * L - 1, np.uint8))
    assert e.value.variant == "WrongOutputLen"
    assert dec.finalize() == data.tobytes()
    dec.reset()
    assert dec.rank() == 0 and dec.received() == 0 and not dec.is_complete()


def test_any_round_trips(oracle):  # selector.rs:605-662
    for engine, k, m, L in [(Engine.STANDARD_CAUCHY, 10, 4, 64), (Engine.GOOD_CAUCHY, 10, 4, 64),
                            (Engine.AFFT, 8, 4, 64), (Engine.TOWER, 32, 4, 64)]:
        p = oracle.resolve(engine, k, m, L)
        data = np.array([(i * 7 + 1) & 0xFF for i in range(k * L)], dtype=np.uint8)
        word = encode_word(oracle, p, data)
        order = [k + j for j in range(m)] + list(range(1, k))
        dec = oracle.decoder(p)
        for i in order:
            dec.push(i, word[i])
            if dec.is_complete():
                break
        out = np.zeros(k * L, dtype=np.uint8)
        dec.finalize_into_with(out, dec.scratch())
        assert np.array_equal(out, data)
