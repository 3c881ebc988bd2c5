"""The serving loop (scrs_server_*): every request's result is identical when
it runs alone and when it runs in a mix of overlapping requests of all four
engines, and equals the oracle's result; admission waits for memory under a
small budget; a request larger than the budget is refused at submit."""
import numpy as np
import pytest

from scrs_b200.api import ConfigError, DecodeError, Engine, RuntimeFailure

from scenarios import encode_word

pytestmark = pytest.mark.gpu

OP_ENCODE, OP_DECODE = 0, 1


def make_requests(torch, oracle, seed=11):
    """(op, engine, k, m, L, input tensor, indices, expected bytes) for a mix
    of engines, sizes and erasure patterns."""
    rng = np.random.default_rng(seed)
    shapes = [(Engine.GOOD_CAUCHY, 10, 4, 4096), (Engine.STANDARD_CAUCHY, 6, 3, 1000),
              (Engine.GOOD_CAUCHY, 40, 16, 2048), (Engine.STANDARD_CAUCHY, 3, 2, 64),
              (Engine.TOWER, 8, 4, 1024), (Engine.TOWER, 32, 8, 4096),
              (Engine.AFFT, 64, 64, 256), (Engine.AFFT, 100, 28, 512),
              (Engine.AFFT, 16384, 16384, 256), (Engine.AFFT, 3000, 500, 2048)]
    reqs = []
    for rep in range(3):
        for engine, k, m, L in shapes:
            p = oracle.resolve(engine, k, m, L)
            data = rng.integers(0, 256, k * L, dtype=np.uint8)
            word = encode_word(oracle, p, data)
            if (rep + k) % 2 == 0:
                reqs.append((OP_ENCODE, engine, k, m, L, torch.from_numpy(data).cuda(), None,
                             np.concatenate(word[k:])))
            else:
                e = int(rng.integers(0, min(k, m) + 1))
                erased = set(rng.choice(k, e, replace=False).tolist())
                extra = rng.choice(m, e, replace=False).tolist()
                idx = [i for i in range(k) if i not in erased] + [k + j for j in extra]
                idx = rng.permutation(idx).tolist()
                rows = torch.from_numpy(np.concatenate([word[i] for i in idx])).cuda()
                reqs.append((OP_DECODE, engine, k, m, L, rows, idx, data))
    return reqs


def run(server, torch, reqs, order):
    outs = [None] * len(reqs)
    for q in order:
        op, engine, k, m, L, d_in, idx, exp = reqs[q]
        outs[q] = torch.full((len(exp),), 0xAB, dtype=torch.uint8, device="cuda")
        server.submit(op, engine, k, m, L, d_in.data_ptr(), outs[q].data_ptr(), idx, tag=q)
    done = server.drain()
    assert sorted(c.tag for c in done) == sorted(order)
    assert all(c.status == 0 for c in done), [c.status for c in done]
    assert all(c.done_ns >= c.submit_ns for c in done)
    torch.cuda.synchronize()
    return outs


def test_results_alone_and_in_mix_match(gpu, oracle):
    torch = pytest.importorskip("torch")
    from scrs_b200.serving import Server

    reqs = make_requests(torch, oracle)
    srv = Server(gpu.lib, 1 << 30, slots=4)
    alone = []
    for q in range(len(reqs)):  # each request alone: submit, then wait for it
        alone.append(run(srv, torch, reqs, [q])[q])
    order = np.random.default_rng(3).permutation(len(reqs)).tolist()
    mixed = run(srv, torch, reqs, order)  # all at once: admitted as slots free up
    for q, r in enumerate(reqs):
        exp = r[-1]
        assert np.array_equal(alone[q].cpu().numpy(), exp), q
        assert np.array_equal(mixed[q].cpu().numpy(), exp), q
    st = srv.stats()
    assert st["completed"] == 2 * len(reqs) and st["failed"] == 0
    assert st["batches"] >= 1
    srv.close()


def test_prepared_requests_and_array_completions(gpu, oracle):
    """Requests built once (Server.prepare) and submitted twice give the same
    bytes as the oracle, and progress_arrays reports every completion once
    with its tag, a zero status and ordered timestamps."""
    torch = pytest.importorskip("torch")
    from scrs_b200.serving import Server

    reqs = make_requests(torch, oracle, seed=23)[:12]
    srv = Server(gpu.lib, 1 << 30, slots=4)
    outs = [torch.full((len(r[-1]),), 0xAB, dtype=torch.uint8, device="cuda") for r in reqs]
    prepared = [srv.prepare(op, engine, k, m, L, d_in.data_ptr(), outs[q].data_ptr(), idx, tag=q)
                for q, (op, engine, k, m, L, d_in, idx, _) in enumerate(reqs)]
    for round_ in range(2):
        for p in prepared:
            srv.submit_prepared(p)
        tags, status, sub_ns, done_ns = [], [], [], []
        while srv.pending:
            t, st, a, b = srv.progress_arrays()
            tags.extend(t.tolist())
            status.extend(st.tolist())
            sub_ns.extend(a.tolist())
            done_ns.extend(b.tolist())
        assert sorted(tags) == list(range(len(reqs)))
        assert all(v == 0 for v in status)
        assert all(b >= a for a, b in zip(sub_ns, done_ns))
        torch.cuda.synchronize()
        for q, r in enumerate(reqs):
            assert np.array_equal(outs[q].cpu().numpy(), r[-1]), (round_, q)
    srv.close()


def test_small_budget_queues_and_completes(gpu, oracle):
    torch = pytest.importorskip("torch")
    from scrs_b200.serving import Server

    reqs = [r for r in make_requests(torch, oracle, seed=5) if r[1] in (Engine.GOOD_CAUCHY, Engine.STANDARD_CAUCHY,
                                                                        Engine.TOWER)]
    biggest = max(r[2] * r[4] + (r[3] if r[0] == OP_ENCODE else r[2]) * r[4] for r in reqs)
    srv = Server(gpu.lib, 3 * biggest, slots=8)  # a few requests' worth of memory
    outs = run(srv, torch, reqs, list(range(len(reqs))))
    for o, r in zip(outs, reqs):
        assert np.array_equal(o.cpu().numpy(), r[-1])
    srv.close()


def test_submit_errors(gpu):
    torch = pytest.importorskip("torch")
    from scrs_b200.serving import Server

    srv = Server(gpu.lib, 1 << 20, slots=2)
    buf = torch.zeros(1 << 21, dtype=torch.uint8, device="cuda")
    p = buf.data_ptr()
    with pytest.raises(RuntimeFailure):  # 2 MiB request under a 1 MiB budget
        srv.submit(OP_ENCODE, Engine.GOOD_CAUCHY, 16, 16, 65536, p, p)
    with pytest.raises(ConfigError):
        srv.submit(OP_ENCODE, Engine.GOOD_CAUCHY, 0, 4, 64, p, p)
    with pytest.raises(DecodeError):  # duplicate index
        srv.submit(OP_DECODE, Engine.GOOD_CAUCHY, 3, 2, 64, p, p, [0, 0, 1])
    with pytest.raises(DecodeError):  # index out of range
        srv.submit(OP_DECODE, Engine.GOOD_CAUCHY, 3, 2, 64, p, p, [0, 1, 9])
    assert srv.pending == 0
    srv.close()


def test_inputs_written_on_held_back_streams(gpu, oracle):
    """Inputs produced on side streams that are held back (torch.cuda._sleep)
    and submitted at once with those streams: every request's work must wait
    for its producer, including requests coalesced into one GF(256) batch from
    different streams."""
    torch = pytest.importorskip("torch")
    from scrs_b200.serving import Server

    reqs = make_requests(torch, oracle, seed=17)
    streams = [torch.cuda.Stream() for _ in range(3)]
    staged = [torch.zeros_like(r[5]) for r in reqs]
    outs = [torch.full((len(r[-1]),), 0xAB, dtype=torch.uint8, device="cuda") for r in reqs]
    torch.cuda.synchronize()
    srv = Server(gpu.lib, 1 << 30, slots=4)
    for st in streams:
        with torch.cuda.stream(st):
            torch.cuda._sleep(40_000_000)  # about 20 ms
    for q, (op, engine, k, m, L, d_in, idx, exp) in enumerate(reqs):
        st = streams[q % len(streams)]
        with torch.cuda.stream(st):
            staged[q].copy_(d_in)  # lands after the hold
        srv.submit(op, engine, k, m, L, staged[q].data_ptr(), outs[q].data_ptr(), idx, tag=q, stream=st)
    done = srv.drain()
    assert all(c.status == 0 for c in done), [c.status for c in done]
    torch.cuda.synchronize()
    for q, r in enumerate(reqs):
        assert np.array_equal(outs[q].cpu().numpy(), r[-1]), q
    srv.close()


def test_reserve_builds_resident_engines_at_start_up(gpu, oracle):
    torch = pytest.importorskip("torch")
    from scrs_b200.serving import Server

    srv = Server(gpu.lib, 1 << 30, slots=3)
    assert srv.stats()["resident_bytes"] == 0
    srv.reserve(OP_DECODE, Engine.AFFT, 64, 64, 256)
    srv.reserve(OP_ENCODE, Engine.TOWER, 8, 4, 1024)
    one = srv.stats()["resident_bytes"]
    assert one > 0
    srv.reserve(OP_DECODE, Engine.AFFT, 64, 64, 256)  # already resident: nothing new
    assert srv.stats()["resident_bytes"] == one
    with pytest.raises(RuntimeFailure):  # GF(256) stripe batches need no resident engines
        srv.reserve(OP_ENCODE, Engine.GOOD_CAUCHY, 10, 4, 4096)
    with pytest.raises(ConfigError):
        srv.reserve(OP_ENCODE, Engine.TOWER, 0, 4, 64)
    # requests of reserved profiles: correct results
    reqs = [r for r in make_requests(torch, oracle, seed=23) if (r[1], r[2], r[3], r[4]) in
            ((Engine.AFFT, 64, 64, 256), (Engine.TOWER, 8, 4, 1024))]
    assert reqs
    outs = run(srv, torch, reqs, list(range(len(reqs))))
    for o, r in zip(outs, reqs):
        assert np.array_equal(o.cpu().numpy(), r[-1])
    # not while a slot runs requests: hold the producer stream so the slot stays busy
    held = torch.cuda.Stream()
    op, engine, k, m, L, d_in, idx, exp = reqs[0]
    out = torch.zeros(len(exp), dtype=torch.uint8, device="cuda")
    with torch.cuda.stream(held):
        torch.cuda._sleep(40_000_000)
    srv.submit(op, engine, k, m, L, d_in.data_ptr(), out.data_ptr(), idx, tag=1, stream=held)
    with pytest.raises(RuntimeFailure):
        srv.reserve(OP_ENCODE, Engine.TOWER, 16, 4, 1024)
    done = srv.drain()
    assert [c.status for c in done] == [0]
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), exp)
    srv.close()
