"""Scenario helpers shared by the oracle-pinning tests and the GPU parity
tests.  Every helper takes an ``Api`` so the same scenario runs on the CUDA
library and on the oracle."""
import itertools

import numpy as np

from scrs_b200.api import Engine

import gfpy


def data_for(k, L, seed):
    return gfpy.rng_bytes(k * L, seed)


def encode_word(api, profile, data):
    """Return the full codeword (list of n symbols as uint8 arrays)."""
    k, m, L = profile.k, profile.m, profile.symbol_len
    rows = [data[i * L:(i + 1) * L].copy() for i in range(k)]
    if profile.engine == Engine.TOWER:
        enc = api.incremental_encoder(profile)
        for i in range(k):
            enc.feed(i, rows[i])
        reps = [np.frombuffer(enc.repair(j), dtype=np.uint8).copy() for j in range(m)]
    else:
        enc = api.batch_encoder(profile)
        out = np.zeros(m * L, dtype=np.uint8)
        enc.encode_into_with(data, out, enc.scratch())
        reps = [out[j * L:(j + 1) * L].copy() for j in range(m)]
    return rows + reps


def batch_decode(api, profile, word, subset):
    dec = api.batch_decoder(profile)
    out = np.full(profile.k * profile.symbol_len, 0xAB, dtype=np.uint8)
    dec.decode_into_with([(i, word[i]) for i in subset], out, dec.scratch())
    return out


def lazy_decode(api, profile, word, order):
    dec = api.decoder(profile)
    for i in order:
        dec.push(i, word[i])
    out = np.full(profile.k * profile.symbol_len, 0x5C, dtype=np.uint8)
    dec.finalize_into_with(out, dec.scratch())
    return out


def k_subsets(n, k):
    return [list(c) for c in itertools.combinations(range(n), k)]


def deterministic_subsets(k, m):
    """The reference's erasure sampler (scrs/src/batch/codec.rs:950-975)."""
    n = k + m
    subsets = [list(range(k))]
    for erase_count in range(1, min(m, k) + 1):
        for shift in range(max(k, 1)):
            if len(subsets) >= 64:
                break
            erased = sorted(set((shift + t * 3) % k for t in range(erase_count)))
            subset = [i for i in range(k) if i not in erased]
            subset += [k + (shift + t) % m for t in range(len(erased))]
            subset.sort()
            if subset not in subsets:
                subsets.append(subset)
    if m >= k:
        subsets.append(list(range(k, n)))
    return subsets


def lcg_permutations(n, count, state=0x123456789ABCDEF0):
    """Fisher-Yates with the reference's LCG (tower/decoder.rs:640-644)."""
    mask = (1 << 64) - 1
    out = []
    for _ in range(count):
        idx = list(range(n))
        for pos in range(n - 1, 0, -1):
            state = (state * 6364136223846793005 + 1) & mask
            j = state % (pos + 1)
            idx[pos], idx[j] = idx[j], idx[pos]
        out.append(idx)
    return out


def direct_gf256_repairs(engine_coeffs, data, k, m, L):
    """Byte-wise sum C[i][j] * data[i] (scrs/src/batch/codec.rs:913-933)."""
    out = np.zeros((m, L), dtype=np.uint8)
    rows = data.reshape(k, L)
    for j in range(m):
        for i in range(k):
            out[j] ^= gfpy.scale_bytes(rows[i], engine_coeffs[i * m + j])
    return out.reshape(-1)


def device_stripes(torch, oracle, specs, rng):
    """Device buffers for (op, engine, k, m, L) specs: encode stripes of random
    data, decode stripes of k received rows (random erasures, shuffled order).
    Returns (stripes, output tensors, expected bytes, tensors to keep alive)."""
    from scrs_b200.batch import OP_ENCODE, Stripe

    stripes, expect, outs, keep = [], [], [], []
    for op, engine, k, m, L in specs:
        p = oracle.resolve(engine, k, m, L)
        data = rng.integers(0, 256, k * L, dtype=np.uint8)
        if op == OP_ENCODE:
            exp = np.concatenate(encode_word(oracle, p, data)[k:])  # tower: k in-order feeds
            d_in = torch.from_numpy(data).cuda()
            d_out = torch.zeros(m * L, dtype=torch.uint8, device="cuda")
            stripes.append(Stripe(op, engine, k, m, L, d_in.data_ptr(), d_out.data_ptr()))
            expect.append(exp)
        else:
            word = encode_word(oracle, p, data)
            e = int(rng.integers(0, min(k, m) + 1))
            erased = rng.choice(k, e, replace=False).tolist()
            repairs = rng.choice(m, e, replace=False).tolist()
            idx = [i for i in range(k) if i not in erased] + [k + j for j in repairs]
            idx = rng.permutation(idx).tolist()
            d_in = torch.from_numpy(np.concatenate([word[i] for i in idx])).cuda()
            d_out = torch.zeros(k * L, dtype=torch.uint8, device="cuda")
            stripes.append(Stripe(op, engine, k, m, L, d_in.data_ptr(), d_out.data_ptr(), idx))
            expect.append(data)
        keep.append(d_in)
        outs.append(d_out)
    return stripes, outs, expect, keep


def make_mixed_batch(torch, n_stripes, seed, lens=(1024, 4096, 65536), kmax=64, mmax=16):
    """(op, engine, k, m, L) specs of a mixed GF(256) stripe batch: k ~ U[4, kmax],
    m ~ U[1, mmax], L from `lens`, Standard or Good Cauchy, encode and decode
    alternating.  Returns (specs, the generator for the stripes' contents)."""
    from scrs_b200.batch import OP_DECODE, OP_ENCODE

    rng = np.random.default_rng(seed)
    specs = []
    for s in range(n_stripes):
        k = int(rng.integers(4, kmax + 1))
        m = int(rng.integers(1, mmax + 1))
        L = int(rng.choice(lens))
        engine = Engine.STANDARD_CAUCHY if rng.integers(0, 2) else Engine.GOOD_CAUCHY
        op = OP_ENCODE if s % 2 == 0 else OP_DECODE
        specs.append((op, engine, k, m, L))
    return specs, rng
