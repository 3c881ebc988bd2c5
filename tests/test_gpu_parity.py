"""Parity of the sm_100a engines with the CPU oracle (bit-exact: every output
is integer/byte work).  Each scenario runs through the C ABI of the CUDA
library and through the oracle's identical ABI on the same seeded inputs."""
import numpy as np
import pytest

from scrs_b200.api import DEPENDENT, ConfigError, DecodeError, EncodeError, Engine, PushOutcome

import gfpy
from scenarios import (batch_decode, deterministic_subsets, device_stripes, encode_word, k_subsets, lazy_decode,
                       lcg_permutations, make_mixed_batch)

pytestmark = pytest.mark.gpu

GF256 = [Engine.STANDARD_CAUCHY, Engine.GOOD_CAUCHY]


def words_equal(a, b):
    return all(np.array_equal(x, y) for x, y in zip(a, b))


# ---------------------------------------------------------------- GF(256)

@pytest.mark.parametrize("engine", GF256)
@pytest.mark.parametrize("k,m,L", [(1, 1, 2), (4, 2, 16), (8, 4, 64), (10, 4, 4096), (16, 8, 1024),
                                   (32, 16, 1024), (64, 16, 4096), (128, 64, 1024), (200, 50, 256),
                                   (1, 254, 64), (254, 1, 64), (3, 5, 7), (6, 6, 33), (16, 8, 100),
                                   (10, 4, 1000), (40, 16, 65536), (33, 3, 1025), (200, 56, 256)])
def test_gf256_encode_matches_oracle(gpu, oracle, engine, k, m, L):
    if engine == Engine.GOOD_CAUCHY and k + m > 255:
        # Good Cauchy holds at most 255 symbols: both sides refuse the profile alike
        with pytest.raises(ConfigError) as got_err:
            gpu.resolve(engine, k, m, L)
        with pytest.raises(ConfigError) as exp_err:
            oracle.resolve(engine, k, m, L)
        assert got_err.value.code == 102 and got_err.value == exp_err.value
        return
    p = gpu.resolve(engine, k, m, L)
    data = gfpy.rng_bytes(k * L, k * 1000 + m)
    got = np.zeros(m * L, np.uint8)
    exp = np.zeros(m * L, np.uint8)
    enc = gpu.batch_encoder(p)
    s = enc.scratch()
    enc.encode_into_with(data, got, s)
    oracle.batch_encoder(p).encode_into(data, exp)
    assert np.array_equal(got, exp)
    enc.encode_into_with(data, got, s)  # scratch reuse
    assert np.array_equal(got, exp)


@pytest.mark.parametrize("engine", GF256)
@pytest.mark.parametrize("k,m,L", [(3, 2, 4), (4, 3, 8), (3, 3, 4), (5, 4, 31)])
def test_gf256_all_subsets(gpu, oracle, engine, k, m, L):
    p = gpu.resolve(engine, k, m, L)
    data = gfpy.rng_bytes(k * L, 99)
    word = encode_word(gpu, p, data)
    assert words_equal(word, encode_word(oracle, p, data))
    for subset in k_subsets(k + m, k):
        assert np.array_equal(batch_decode(gpu, p, word, subset), data), subset
        assert np.array_equal(lazy_decode(gpu, p, word, subset[::-1]), data), subset


@pytest.mark.parametrize("k,m,L", [(1, 1, 2), (4, 2, 16), (8, 4, 64), (6, 6, 33), (16, 8, 100), (32, 16, 64),
                                   (10, 4, 4096), (64, 16, 1024), (128, 127, 96), (128, 128, 96)])
def test_gf256_decode_sampled_patterns(gpu, k, m, L):
    for engine in GF256:
        if engine == Engine.GOOD_CAUCHY and k + m > 255:
            continue
        p = gpu.resolve(engine, k, m, L)
        data = gfpy.rng_bytes(k * L, 7 + k)
        word = encode_word(gpu, p, data)
        for subset in deterministic_subsets(k, m)[:24]:
            assert np.array_equal(batch_decode(gpu, p, word, subset), data), subset
            assert np.array_equal(lazy_decode(gpu, p, word, subset), data), subset


def test_gf256_incremental_encoder(gpu, oracle):
    for k, m, L in [(4, 3, 8), (10, 4, 4096), (60, 16, 33), (100, 100, 2048)]:
        p = gpu.resolve(Engine.GOOD_CAUCHY, k, m, L)
        data = gfpy.rng_bytes(k * L, 5 * k)
        inc, inc_o = gpu.incremental_encoder(p), oracle.incremental_encoder(p)
        order = list(range(k))[::-1]
        for t, i in enumerate(order):
            inc.feed(i, data[i * L:(i + 1) * L])
            inc_o.feed(i, data[i * L:(i + 1) * L])
            if t in (0, k // 2):  # partial sums are readable mid-stream
                assert inc.repair(m - 1) == inc_o.repair(m - 1)
        assert inc.fed_count() == k
        assert all(inc.repair(j) == inc_o.repair(j) for j in range(m))
        with pytest.raises(EncodeError) as e:
            inc.feed(0, data[:L])
        assert e.value.variant == "DuplicateData"
        inc.reset()
        assert inc.fed_count() == 0 and inc.repair(0) == bytes(L)


def error_of(fn):
    try:
        fn()
    except (EncodeError, DecodeError) as e:
        return e
    return None


def test_gf256_error_parity(gpu, oracle):
    p = gpu.resolve(Engine.STANDARD_CAUCHY, 3, 2, 4)
    word = encode_word(oracle, p, np.zeros(12, np.uint8))
    cases = [
        [(0, word[0]), (1, word[1])],
        [(0, word[0]), (1, word[1]), (5, np.zeros(4, np.uint8))],
        [(0, word[0]), (1, word[1]), (0, word[0])],
        [(0, word[0]), (1, word[1]), (2, np.zeros(3, np.uint8))],
    ]
    for syms in cases:
        for out_len in (12, 11):
            eg = error_of(lambda: gpu.batch_decoder(p).decode_into(syms, np.zeros(out_len, np.uint8)))
            eo = error_of(lambda: oracle.batch_decoder(p).decode_into(syms, np.zeros(out_len, np.uint8)))
            assert eg == eo and eg is not None
    enc = gpu.batch_encoder(p)
    enc_o = oracle.batch_encoder(p)
    for dl, rl in [(11, 8), (12, 9)]:
        assert error_of(lambda: enc.encode_into(np.zeros(dl, np.uint8), np.zeros(rl, np.uint8))) == \
            error_of(lambda: enc_o.encode_into(np.zeros(dl, np.uint8), np.zeros(rl, np.uint8)))
    other = gpu.batch_decoder(gpu.resolve(Engine.STANDARD_CAUCHY, 4, 2, 4))
    e = error_of(lambda: gpu.batch_decoder(p).decode_into_with([(0, word[0]), (1, word[1]), (2, word[2])],
                                                               np.zeros(12, np.uint8), other.scratch()))
    assert e.variant == "ScratchMismatch"


def test_lazy_decoder_push_contract_matches_oracle(gpu, oracle):
    for engine, k, m, L in [(Engine.GOOD_CAUCHY, 4, 3, 8), (Engine.TOWER, 4, 3, 8), (Engine.AFFT, 4, 3, 8)]:
        p = gpu.resolve(engine, k, m, L)
        word = encode_word(oracle, p, gfpy.rng_bytes(k * L, 1))
        dg, do = gpu.decoder(p), oracle.decoder(p)
        seq = [k, k, 1, 2, k + 1, 0, 3, 3]
        for i in seq:
            rg = error_of(lambda: dg.push(i, word[i])) or dg.received()
            ro = error_of(lambda: do.push(i, word[i])) or do.received()
            assert rg == ro
        assert dg.rank() == do.rank() and dg.is_complete() == do.is_complete()
        assert dg.finalize() == do.finalize()


# ---------------------------------------------------------------- tower

@pytest.mark.parametrize("k,m,L", [(4, 3, 10), (4, 3, 18), (32, 8, 65536), (64, 32, 66), (256, 3, 4),
                                   (300, 20, 130), (2, 1, 4), (2048, 512, 16)])
def test_tower_encode_matches_oracle(gpu, oracle, k, m, L):
    p = gpu.resolve(Engine.TOWER, k, m, L)
    data = gfpy.rng_bytes(k * L, 11 * k + m)
    assert words_equal(encode_word(gpu, p, data), encode_word(oracle, p, data))


def test_tower_recovery(gpu, oracle):
    k, m, L = 4, 3, 18
    p = gpu.resolve(Engine.TOWER, k, m, L)
    data = gfpy.rng_bytes(k * L, 3)
    word = encode_word(gpu, p, data)
    for subset in k_subsets(k + m, k):
        assert np.array_equal(lazy_decode(gpu, p, word, subset), data)
        assert np.array_equal(batch_decode(gpu, p, word, subset), data)
    k, m, L = 64, 32, 66
    p = gpu.resolve(Engine.TOWER, k, m, L)
    data = gfpy.rng_bytes(k * L, 4)
    word = encode_word(gpu, p, data)
    for perm in lcg_permutations(k + m, 8):
        assert np.array_equal(lazy_decode(gpu, p, word, perm[:k]), data)


def test_tower_cfg2_shape(gpu, oracle):
    """k=32, m=8, L=65536 with 8 data symbols erased (random permutation)."""
    k, m, L = 32, 8, 65536
    p = gpu.resolve(Engine.TOWER, k, m, L)
    data = gfpy.rng_bytes(k * L, 0x5C250002)
    word = encode_word(gpu, p, data)
    rng = np.random.default_rng(2)
    erased = set(rng.choice(k, 8, replace=False).tolist())
    order = [i for i in rng.permutation(k + m).tolist() if i not in erased][:k]
    assert np.array_equal(lazy_decode(gpu, p, word, order), data)
    assert np.array_equal(lazy_decode(oracle, p, word, order), data)


# ---------------------------------------------------------------- AFFT

@pytest.mark.parametrize("k,m,L", [(5, 3, 6), (8, 4, 64), (3, 2, 2), (100, 20, 64), (17, 7, 130), (4, 2, 64),
                                   (16, 4, 40), (256, 64, 48), (512, 128, 40), (1, 1, 2), (8, 8, 4),
                                   (4096, 4096, 1024), (32768, 32768, 4), (40000, 25536, 2),
                                   (32768, 16384, 256)])
def test_afft_encode_matches_oracle(gpu, oracle, k, m, L):
    p = gpu.resolve(Engine.AFFT, k, m, L)
    data = gfpy.rng_bytes(k * L, 17 * k + m)
    got = np.zeros(m * L, np.uint8)
    exp = np.zeros(m * L, np.uint8)
    enc = gpu.batch_encoder(p)
    enc.encode_into_with(data, got, enc.scratch())
    oracle.batch_encoder(p).encode_into(data, exp)
    assert np.array_equal(got, exp)


@pytest.mark.parametrize("k,m,L", [(4, 4, 10), (5, 3, 6)])
def test_afft_exhaustive_recovery(gpu, k, m, L):
    p = gpu.resolve(Engine.AFFT, k, m, L)
    data = gfpy.rng_bytes(k * L, 8)
    word = encode_word(gpu, p, data)
    for subset in k_subsets(k + m, k):
        assert np.array_equal(lazy_decode(gpu, p, word, subset), data), subset
        assert np.array_equal(batch_decode(gpu, p, word, subset), data), subset


def test_afft_random_and_large_patterns(gpu, oracle):
    for k, m, L in [(32, 16, 34), (16, 8, 64), (300, 2, 2)]:
        p = gpu.resolve(Engine.AFFT, k, m, L)
        data = gfpy.rng_bytes(k * L, k)
        word = encode_word(gpu, p, data)
        for perm in lcg_permutations(k + m, 6):
            assert np.array_equal(lazy_decode(gpu, p, word, perm[:k]), data)
    # the config-3a shape: decode from a random half of 8192 points
    k, m, L = 4096, 4096, 1024
    p = gpu.resolve(Engine.AFFT, k, m, L)
    data = gfpy.rng_bytes(k * L, 0x5C250003)
    word = encode_word(gpu, p, data)
    sel = np.random.default_rng(3).permutation(k + m)[:k].tolist()
    assert np.array_equal(lazy_decode(gpu, p, word, sel), data)


def test_afft_cfg3b_shape(gpu, oracle):
    """The config-3b shape (k=32768, m=16384, L=256): repairs equal the
    oracle's, and the data comes back from a random 32768 of the 49152
    symbols (full path) and from all but 3 data symbols (targeted path),
    through the batch and the lazy decoders."""
    k, m, L = 32768, 16384, 256
    p = gpu.resolve(Engine.AFFT, k, m, L)
    data = gfpy.rng_bytes(k * L, 0x5C25003B)
    word = encode_word(gpu, p, data)
    exp = np.zeros(m * L, np.uint8)
    oracle.batch_encoder(p).encode_into(data, exp)
    assert np.array_equal(np.concatenate(word[k:]), exp)
    rng = np.random.default_rng(0x3B)
    sel = rng.permutation(k + m)[:k].tolist()
    assert np.array_equal(batch_decode(gpu, p, word, sel), data)
    assert np.array_equal(lazy_decode(gpu, p, word, sel), data)
    few = rng.permutation([i for i in range(k) if i not in (5, 777, 32767)] + [k + 1, k + 9000, k + m - 1]).tolist()
    assert np.array_equal(batch_decode(gpu, p, word, few), data)



@pytest.mark.parametrize("k,m,L", [(1500, 700, 130), (1200, 300, 96), (10000, 3000, 64), (8192, 100, 64),
                                   (16384, 16384, 32), (2000, 48, 4096)])
def test_afft_mid_size_shapes(gpu, oracle, k, m, L):
    """Transforms of 2^11 to 2^15 points: the power-of-two encode (k = 8192,
    16384), the general-k encode and the full decode at each transform size,
    with odd symbol lengths and up to 64 column groups: repairs equal the
    oracle's and a random k of the n symbols give the data back."""
    p = gpu.resolve(Engine.AFFT, k, m, L)
    data = gfpy.rng_bytes(k * L, 0xC1 + k + m)
    word = encode_word(gpu, p, data)
    exp = np.zeros(m * L, np.uint8)
    oracle.batch_encoder(p).encode_into(data, exp)
    assert np.array_equal(np.concatenate(word[k:]), exp)
    sel = np.random.default_rng(k + m).permutation(k + m)[:k].tolist()
    assert np.array_equal(batch_decode(gpu, p, word, sel), data)
    assert np.array_equal(lazy_decode(gpu, p, word, sel), data)

@pytest.mark.parametrize("k,m,L", [(4096, 64, 1024), (1000, 24, 258), (37, 11, 6), (2048, 8, 4096)])
def test_afft_targeted_few_erasures(gpu, oracle, k, m, L):
    """r <= 5 missing data symbols take the targeted path (one coefficient
    table + multiply-XOR over all k inputs); r = 6 the full transforms.  Both
    must recover the data exactly, through the lazy and the batch decoders,
    for aligned and odd symbol lengths."""
    p = gpu.resolve(Engine.AFFT, k, m, L)
    data = gfpy.rng_bytes(k * L, k + L)
    word = encode_word(oracle, p, data)
    rng = np.random.default_rng(k)
    for r in (1, 2, 3, 4, 5, 6):
        if r > m:
            continue
        erased = set(rng.choice(k, r, replace=False).tolist())
        reps = (k + rng.choice(m, r, replace=False)).tolist()
        sub = [i for i in range(k) if i not in erased] + reps
        order = rng.permutation(sub).tolist()
        assert np.array_equal(batch_decode(gpu, p, word, order), data), r
        assert np.array_equal(lazy_decode(gpu, p, word, order), data), r


# ---------------------------------------------------------------- device-pointer forms

def test_device_pointer_entry_points(gpu, oracle):
    torch = pytest.importorskip("torch")
    k, m, L = 10, 4, 4096
    p = gpu.resolve(Engine.GOOD_CAUCHY, k, m, L)
    data = gfpy.rng_bytes(k * L, 42)
    exp = np.zeros(m * L, np.uint8)
    oracle.batch_encoder(p).encode_into(data, exp)
    d_data = torch.from_numpy(data).cuda()
    d_rep = torch.zeros(m * L, dtype=torch.uint8, device="cuda")
    enc = gpu.batch_encoder(p)
    enc.encode_into_with(d_data, d_rep, enc.scratch())
    torch.cuda.synchronize()
    assert np.array_equal(d_rep.cpu().numpy(), exp)
    word = [data[i * L:(i + 1) * L] for i in range(k)] + [exp[j * L:(j + 1) * L] for j in range(m)]
    idx = [0, 2, 3, 4, 6, 8, 10, 11, 12, 13]
    rows = torch.from_numpy(np.concatenate([word[i] for i in idx])).cuda()
    out = torch.zeros(k * L, dtype=torch.uint8, device="cuda")
    dec = gpu.batch_decoder(p)
    dec.decode_into_with((idx, rows), out, dec.scratch())
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), data)
    # lazy decoder with device pushes and device finalize
    ld = gpu.decoder(p)
    for i in idx:
        ld.push(i, torch.from_numpy(word[i]).cuda())
    out2 = torch.zeros(k * L, dtype=torch.uint8, device="cuda")
    ld.finalize_into_with(out2, ld.scratch())
    torch.cuda.synchronize()
    assert np.array_equal(out2.cpu().numpy(), data)


# ---------------------------------------------------------------- batched stripes

def test_stripe_batch_matches_oracle(gpu, oracle):
    torch = pytest.importorskip("torch")
    from scrs_b200.batch import StripeBatch

    specs, rng = make_mixed_batch(torch, 96, 4, lens=(1024, 4096, 1000, 64))
    stripes, outs, expect, keep = device_stripes(torch, oracle, specs, rng)
    b = StripeBatch(gpu.lib, len(stripes))
    b.set(stripes)
    for mode in ("persistent", "graph", "plain", "graph"):
        for o in outs:
            o.zero_()
        if mode == "plain":
            b.run_plain()
        else:
            b.run(graph=(mode == "graph"))
        torch.cuda.synchronize()
        b.check()
        for o, exp in zip(outs, expect):
            assert np.array_equal(o.cpu().numpy(), exp), mode
    assert b.last_launches == 2  # plan + persistent drain


def test_stripe_batch_with_tower_stripes(gpu, oracle):
    """Tower stripes in the same batch as GF(256) stripes (each field through
    its own plan launch and persistent drain): encodes equal the oracle's k
    in-order feeds, decodes the data, in persistent, graph and plain modes;
    tower stripes of more inputs than one staged segment (16 rows), odd
    group counts and zero erasures among them.  Host-buffer batches refuse
    tower stripes."""
    torch = pytest.importorskip("torch")
    from scrs_b200.api import RuntimeFailure
    from scrs_b200.batch import OP_DECODE, OP_ENCODE, StripeBatch

    specs, rng = make_mixed_batch(torch, 24, 21, lens=(1024, 4096, 1000, 64), kmax=40, mmax=12)
    tower = [(32, 8, 4096), (8, 4, 1000), (300, 20, 130), (64, 32, 66), (17, 3, 2048), (2, 1, 4)]
    for q, (k, m, L) in enumerate(tower):
        specs.insert(3 * q + 1, (OP_ENCODE, Engine.TOWER, k, m, L))
        specs.insert(3 * q + 2, (OP_DECODE, Engine.TOWER, k, m, L))
    stripes, outs, expect, keep = device_stripes(torch, oracle, specs, rng)
    b = StripeBatch(gpu.lib, len(stripes))
    b.set(stripes)
    for mode in ("persistent", "graph", "plain", "graph"):
        for o in outs:
            o.zero_()
        if mode == "plain":
            b.run_plain()
        else:
            b.run(graph=(mode == "graph"))
        torch.cuda.synchronize()
        b.check()
        for q, (o, exp) in enumerate(zip(outs, expect)):
            assert np.array_equal(o.cpu().numpy(), exp), (mode, specs[q])
    assert b.last_launches == 4  # a plan launch and a persistent drain per field
    h = torch.zeros(64, dtype=torch.uint8).pin_memory()
    with pytest.raises(RuntimeFailure):
        b.set_arrays(np.array([OP_ENCODE]), np.array([int(Engine.TOWER)]), np.array([2]), np.array([1]),
                     np.array([32]), np.array([h.data_ptr()], dtype=np.uint64),
                     np.array([h.data_ptr() + 32], dtype=np.uint64), host=True)


def test_stripe_batch_host_buffers_pipelined(gpu, oracle):
    """Host-buffer batches run in up to 64 pieces whose copies overlap the
    compute; a decode stripe's present rows are copied on the host and only
    its missing rows come back from the device.  Results must equal the
    oracle's, run after run, pipelined and one launch per stripe, with decode
    stripes that lost no data symbol among them."""
    torch = pytest.importorskip("torch")
    from scrs_b200.batch import OP_DECODE, OP_ENCODE, StripeBatch

    specs, rng = make_mixed_batch(torch, 40, 9, lens=(1024, 4096, 1000, 64), kmax=24, mmax=8)
    n = len(specs)
    ops, engines, ks, ms, Ls, ins, outs, expect, keep = [], [], [], [], [], [], [], [], []
    kmax = max(s[2] for s in specs)
    indices = np.zeros((n, kmax), np.uint16)
    for s, (op, engine, k, m, L) in enumerate(specs):
        p = oracle.resolve(engine, k, m, L)
        data = rng.integers(0, 256, k * L, dtype=np.uint8)
        if op == OP_ENCODE:
            exp = np.zeros(m * L, np.uint8)
            oracle.batch_encoder(p).encode_into(data, exp)
            h_in = torch.from_numpy(data).pin_memory()
        else:
            word = encode_word(oracle, p, data)
            e = int(rng.integers(0, min(k, m) + 1))
            erased = rng.choice(k, e, replace=False).tolist()
            idx = [i for i in range(k) if i not in erased] + [k + j for j in rng.choice(m, e, replace=False).tolist()]
            idx = rng.permutation(idx).tolist()
            indices[s, :k] = idx
            h_in = torch.from_numpy(np.concatenate([word[i] for i in idx])).pin_memory()
            exp = data
        h_out = torch.zeros(len(exp), dtype=torch.uint8).pin_memory()
        ops.append(op), engines.append(int(engine)), ks.append(k), ms.append(m), Ls.append(L)
        ins.append(h_in.data_ptr()), outs.append(h_out.data_ptr())
        expect.append(exp), keep.append((h_in, h_out))
    b = StripeBatch(gpu.lib, n)
    b.set_arrays(np.array(ops), np.array(engines), np.array(ks), np.array(ms), np.array(Ls),
                 np.array(ins, dtype=np.uint64), np.array(outs, dtype=np.uint64), indices=indices, host=True)
    assert any(s[0] == OP_DECODE and not any(i >= s[2] for i in indices[q, :s[2]]) for q, s in enumerate(specs))
    for mode in ("pipelined", "pipelined", "plain"):
        for _, h_out in keep:
            h_out.zero_()
        if mode == "plain":
            b.run_plain()
        else:
            b.run()
        torch.cuda.synchronize()
        b.check()
        for (_, h_out), exp in zip(keep, expect):
            assert np.array_equal(h_out.numpy(), exp), mode


@pytest.mark.parametrize("engine,k,m,L", [(Engine.GOOD_CAUCHY, 10, 4, 4096), (Engine.STANDARD_CAUCHY, 6, 3, 100),
                                          (Engine.TOWER, 8, 4, 1024)])
def test_recipe_cache_repeated_patterns(gpu, oracle, engine, k, m, L):
    """Repeated erasure patterns reuse the device-resident recipe (LRU of 32);
    every decode stays exact through hits, misses and evictions."""
    p = gpu.resolve(engine, k, m, L)
    data = gfpy.rng_bytes(k * L, 77)
    word = encode_word(oracle, p, data)
    pats = [s for s in k_subsets(k + m, k) if any(i >= k for i in s)][:40]
    assert len(pats) == 40
    dec = gpu.batch_decoder(p)
    s = dec.scratch()
    seq = pats + [pats[39], pats[10], pats[0]]
    for q, sub in enumerate(seq):
        out = np.full(k * L, 0xAB, np.uint8)
        dec.decode_into_with([(i, word[i]) for i in sub], out, s)
        assert np.array_equal(out, data), q
    assert s.recipe_hits == 2  # pats[39] and pats[10]; pats[0] was evicted
    lazy = gpu.decoder(p)
    ls = lazy.scratch()
    for sub in (pats[5], pats[5], pats[6], pats[5]):
        lazy.reset()
        for i in sub:
            lazy.push(i, word[i])
        out = np.zeros(k * L, np.uint8)
        lazy.finalize_into_with(out, ls)
        assert np.array_equal(out, data)
    assert ls.recipe_hits == 2


def test_bounded_wait_reports_timeout_and_context_survives(gpu, oracle):
    """A device wait that nothing completes gives up after its limit and reports
    SCRS_ERR_DEVICE_TIMEOUT; the context keeps working afterwards."""
    import ctypes as C
    import time

    from scrs_b200.api import _Error

    lib = gpu.lib.lib
    lib.scrs_selftest_wait_timeout.restype = C.c_int32
    lib.scrs_selftest_wait_timeout.argtypes = [C.c_uint64, C.POINTER(_Error)]
    for _ in range(2):
        err = _Error()
        t0 = time.monotonic()
        rc = lib.scrs_selftest_wait_timeout(2_000_000, C.byref(err))
        assert rc == 906 and err.code == 906
        assert time.monotonic() - t0 < 5.0
    err = _Error()
    assert lib.scrs_selftest_wait_timeout(0, C.byref(err)) == 907
    p = gpu.resolve(Engine.GOOD_CAUCHY, 10, 4, 4096)  # the context is still usable
    data = gfpy.rng_bytes(10 * 4096, 5)
    got, exp = np.zeros(4 * 4096, np.uint8), np.zeros(4 * 4096, np.uint8)
    gpu.batch_encoder(p).encode_into(data, got)
    oracle.batch_encoder(p).encode_into(data, exp)
    assert np.array_equal(got, exp)
