"""Seeded restatements of the reference's property tests, run on the GPU.

* ``prop_roundtrip_all_subsets`` (scrs/src/batch/codec.rs:889-910): random
  k, m in 1..=4 and symbol_len in 1..=8; every k-subset of the codeword
  decodes to the data.  Here for both GF(256) engines, with the repairs also
  compared to the oracle's.
* ``differential_fuzz_against_tower_cauchy`` (scrs/src/afft/differential.rs:23-58):
  256 cases of k, m in 1..=12 and 1..=8 field elements per symbol; the tower
  and the additive-FFT codewords each decode from the same k symbols, chosen
  by a random ordering, to the data and to each other.  Here each codeword
  is also compared to the oracle's.

The cases come from a seeded generator instead of proptest's shrinking
search, so a failure names its case and replays exactly.
"""
import numpy as np
import pytest

from scrs_b200.api import Engine

from scenarios import batch_decode, encode_word, k_subsets, lazy_decode

pytestmark = pytest.mark.gpu


def roundtrip_cases(n_cases, seed):
    rng = np.random.default_rng(seed)
    for c in range(n_cases):
        k, m = int(rng.integers(1, 5)), int(rng.integers(1, 5))
        L = int(rng.integers(1, 9))
        data = rng.integers(0, 256, k * L, dtype=np.uint8)
        yield c, k, m, L, data


@pytest.mark.parametrize("engine", [Engine.STANDARD_CAUCHY, Engine.GOOD_CAUCHY])
def test_roundtrip_all_subsets(gpu, oracle, engine):
    for c, k, m, L, data in roundtrip_cases(48, 0x9A0 + int(engine)):
        p, po = gpu.resolve(engine, k, m, L), oracle.resolve(engine, k, m, L)
        word = encode_word(gpu, p, data)
        exp = encode_word(oracle, po, data)
        assert all(np.array_equal(a, b) for a, b in zip(word, exp)), (c, k, m, L)
        for subset in k_subsets(k + m, k):
            assert np.array_equal(batch_decode(gpu, p, word, subset), data), (c, k, m, L, subset)


def test_differential_tower_against_afft(gpu, oracle):
    rng = np.random.default_rng(0xD1FF)
    for c in range(256):
        k, m = int(rng.integers(1, 13)), int(rng.integers(1, 13))
        L = 2 * int(rng.integers(1, 9))
        data = rng.integers(0, 256, k * L, dtype=np.uint8)
        ordering = rng.integers(0, 1 << 16, k + m)
        # the reference sorts the indices by (ordering[index], index) and keeps k
        order = sorted(range(k + m), key=lambda i: (int(ordering[i]), i))[:k]
        outs = []
        for engine in (Engine.TOWER, Engine.AFFT):
            p = gpu.resolve(engine, k, m, L)
            word = encode_word(gpu, p, data)
            exp = encode_word(oracle, oracle.resolve(engine, k, m, L), data)
            assert all(np.array_equal(a, b) for a, b in zip(word, exp)), (c, engine, k, m, L)
            out = lazy_decode(gpu, p, word, order)
            assert np.array_equal(out, data), (c, engine, k, m, L, order)
            outs.append(out)
        assert np.array_equal(outs[0], outs[1]), (c, k, m, L)
