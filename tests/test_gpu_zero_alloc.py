"""Steady-state calls allocate nothing, as the reference's allocation contract
for its reusable facades (scrs/tests/zero_alloc.rs:48-155): after the
handles, their scratches and one warm-up call exist, the *_with encodes and
decodes, incremental feeds and repair reads, pushes and finalizes of every
engine make no device or pinned-host allocation (the library's own count,
scrs_alloc_count, stays flat and the device's free memory is unchanged).
The GPU library goes further than the reference on one point: a new erasure
pattern (a recipe-cache miss) allocates nothing either, since every cache
entry is sized for the largest erasure count when the scratch is made."""
import numpy as np
import pytest

from scrs_b200.api import Engine

pytestmark = pytest.mark.gpu

# (engine, k, m, symbol_len, missing) as the reference's cases, plus the
# headline GF(256) geometry and a targeted / full-path AFFT pair
CASES = [(Engine.STANDARD_CAUCHY, 8, 4, 64, 2), (Engine.GOOD_CAUCHY, 8, 4, 64, 2), (Engine.TOWER, 8, 4, 64, 2),
         (Engine.AFFT, 8, 4, 64, 2), (Engine.AFFT, 16, 8, 64, 6), (Engine.GOOD_CAUCHY, 10, 4, 4096, 4),
         (Engine.TOWER, 32, 8, 1024, 8)]


def _patterns(k, m, missing, rng, count):
    """`count` received index lists with `missing` data symbols erased (the
    first one is the reference's (missing..k) + (k..k+missing))."""
    out = [list(range(missing, k)) + list(range(k, k + missing))]
    while len(out) < count:
        erased = set(rng.choice(k, missing, replace=False).tolist())
        reps = rng.choice(m, missing, replace=False).tolist()
        out.append(rng.permutation([i for i in range(k) if i not in erased] + [k + j for j in reps]).tolist())
    return out


@pytest.mark.parametrize("engine,k,m,L,missing", CASES, ids=lambda v: getattr(v, "name", str(v)))
def test_steady_state_calls_allocate_nothing(gpu, engine, k, m, L, missing):
    torch = pytest.importorskip("torch")
    lib = gpu.lib
    p = gpu.resolve(engine, k, m, L)
    data = ((np.arange(k * L, dtype=np.uint64) * 131 + 7) & 0xFF).astype(np.uint8)
    d_data = torch.from_numpy(data).cuda()
    repairs = np.zeros(m * L, np.uint8)
    d_rep = torch.zeros(m * L, dtype=torch.uint8, device="cuda")
    block = gpu.batch_encoder(p) if engine != Engine.TOWER else None
    block_s = block.scratch() if block else None
    inc = gpu.incremental_encoder(p) if engine in (Engine.GOOD_CAUCHY, Engine.TOWER) else None
    if block:
        block.encode_into_with(data, repairs, block_s)
    else:
        for i in range(k):
            inc.feed(i, data[i * L:(i + 1) * L])
        repairs = np.frombuffer(b"".join(inc.repair(j) for j in range(m)), np.uint8).copy()
    word = np.concatenate([data, repairs]).reshape(k + m, L)
    d_word = torch.from_numpy(word).cuda()
    pats = _patterns(k, m, missing, np.random.default_rng(7 + k), 3)
    rows = [np.ascontiguousarray(word[pt]).reshape(-1) for pt in pats]
    d_rows = [d_word[torch.tensor(pt, device="cuda")].reshape(-1).contiguous() for pt in pats]
    stream_dec = gpu.decoder(p)
    stream_s = stream_dec.scratch()
    batch_dec = gpu.batch_decoder(p)
    batch_s = batch_dec.scratch()
    out = np.zeros(k * L, np.uint8)
    d_out = torch.zeros(k * L, dtype=torch.uint8, device="cuda")
    d_rowviews = [[d_word[i] for i in pt] for pt in pats]

    def steady(pattern_ids):
        if block:
            block.encode_into_with(data, repairs, block_s)
            block.encode_into_with(d_data, d_rep, block_s)
        if inc:
            inc.reset()
            for i in range(k):
                inc.feed(i, data[i * L:(i + 1) * L] if i % 2 else d_data[i * L:(i + 1) * L])
            inc.repair(0)
        for q in pattern_ids:
            stream_dec.reset()
            for i in pats[q]:
                stream_dec.push(i, word[i])
            stream_dec.finalize_into_with(out, stream_s)
            assert np.array_equal(out, data)
            stream_dec.reset()
            for i, row in zip(pats[q], d_rowviews[q]):
                stream_dec.push(i, row)
            stream_dec.finalize_into_with(d_out, stream_s)
            batch_dec.decode_into_with([(i, rows[q][t * L:(t + 1) * L]) for t, i in enumerate(pats[q])], out,
                                       batch_s)
            assert np.array_equal(out, data)
            batch_dec.decode_into_with((pats[q], d_rows[q]), d_out, batch_s)
        torch.cuda.synchronize()

    steady([0])  # warm-up: the one call per path the reference makes before counting
    before, free_before = lib.alloc_count(), torch.cuda.mem_get_info()[0]
    steady([0, 0])  # the same pattern again
    steady([1, 2, 1])  # new erasure patterns: recipe-cache misses, then a hit
    assert lib.alloc_count() == before, engine
    assert torch.cuda.mem_get_info()[0] == free_before, engine
    assert torch.equal(d_out.cpu(), torch.from_numpy(data))


def test_warm_server_allocates_nothing(gpu, oracle):
    """A serving loop that has run a request mix once runs it again without
    allocating (one slot, so the coalesced groups repeat exactly)."""
    torch = pytest.importorskip("torch")
    from scrs_b200.serving import OP_DECODE, OP_ENCODE, Server

    rng = np.random.default_rng(0x5A)
    shapes = [(Engine.GOOD_CAUCHY, 10, 4, 4096), (Engine.STANDARD_CAUCHY, 20, 6, 1024), (Engine.TOWER, 16, 4, 1024),
              (Engine.AFFT, 64, 32, 512)]
    reqs = []
    for engine, k, m, L in shapes:
        p = gpu.resolve(engine, k, m, L)
        data = torch.from_numpy(rng.integers(0, 256, k * L, dtype=np.uint8)).cuda()
        rep = torch.zeros(m * L, dtype=torch.uint8, device="cuda")
        if engine == Engine.TOWER:
            inc = gpu.incremental_encoder(p)
            for i in range(k):
                inc.feed(i, data[i * L:(i + 1) * L])
            rep.copy_(torch.frombuffer(bytearray(b"".join(inc.repair(j) for j in range(m))), dtype=torch.uint8))
        else:
            gpu.batch_encoder(p).encode_into_with(data, rep, gpu.batch_encoder(p).scratch())
        word = torch.cat([data.view(k, L), rep.view(m, L)])
        idx = list(range(2, k)) + [k, k + 1]
        rows = word[torch.tensor(idx, device="cuda")].reshape(-1).contiguous()
        reqs.append((OP_ENCODE, engine, k, m, L, data, torch.zeros(m * L, dtype=torch.uint8, device="cuda"), None))
        reqs.append((OP_DECODE, engine, k, m, L, rows, torch.zeros(k * L, dtype=torch.uint8, device="cuda"), idx))
    srv = Server(gpu.lib, 1 << 30, slots=1)
    for op, engine, k, m, L, *_ in reqs:
        if engine in (Engine.TOWER, Engine.AFFT):
            srv.reserve(op, engine, k, m, L)

    def one_pass():
        for t, (op, engine, k, m, L, d_in, d_out, idx) in enumerate(reqs):
            srv.submit(op, engine, k, m, L, d_in.data_ptr(), d_out.data_ptr(), idx, tag=t)
        done = srv.drain()
        assert len(done) == len(reqs) and all(c.status == 0 for c in done)
        torch.cuda.synchronize()

    one_pass()
    before, free_before = gpu.lib.alloc_count(), torch.cuda.mem_get_info()[0]
    one_pass()
    one_pass()
    assert gpu.lib.alloc_count() == before
    assert torch.cuda.mem_get_info()[0] == free_before
    for op, engine, k, m, L, d_in, d_out, idx in reqs:
        if op == OP_DECODE:
            assert torch.equal(d_out, reqs[[r[1] for r in reqs].index(engine)][5]), engine
    srv.close()
