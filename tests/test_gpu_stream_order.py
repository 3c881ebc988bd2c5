"""Stream order of the per-symbol device entry points.

A device feed or push copies the caller's buffer on the caller's stream, so
the copy runs after the work that produced the buffer there and before the
work the caller enqueues there next.  A device finalize returns without
waiting; the next pushes into the same decoder (after a reset) wait on the
device for that decode's reads of the payload buffer.

Each test makes the hazard real with ``torch.cuda._sleep``: the stream that
produces (or reads) a buffer is held back for tens of milliseconds, so a copy
or decode that were not ordered after it would see the wrong bytes.  Expected
bytes come from the oracle.
"""
import numpy as np
import pytest

from scrs_b200.api import Engine

from scenarios import data_for, encode_word

pytestmark = pytest.mark.gpu

HOLD_CYCLES = 60_000_000  # about 30 ms at the B200's SM clock


def _torch():
    return pytest.importorskip("torch")


@pytest.mark.parametrize("engine,k,m,L", [(Engine.GOOD_CAUCHY, 10, 4, 4096), (Engine.TOWER, 8, 4, 2048)])
def test_device_feed_follows_the_producing_stream(gpu, oracle, engine, k, m, L):
    torch = _torch()
    p = gpu.resolve(engine, k, m, L)
    data = data_for(k, L, 71)
    word = encode_word(oracle, oracle.resolve(engine, k, m, L), data)
    src = torch.from_numpy(data).cuda().view(k, L)
    buf = torch.zeros((k, L), dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    inc = gpu.incremental_encoder(p)
    side = torch.cuda.Stream()
    with torch.cuda.stream(side):
        torch.cuda._sleep(HOLD_CYCLES)
        buf.copy_(src)  # the feeds must see these bytes, not the zeros
        for i in range(k):
            inc.feed(i, buf[i])
        buf.fill_(0x5A)  # and not these: the caller reuses its buffer
    for j in range(m):
        assert np.array_equal(np.frombuffer(inc.repair(j), dtype=np.uint8), word[k + j]), j
    torch.cuda.synchronize()


@pytest.mark.parametrize("engine,k,m,L", [(Engine.GOOD_CAUCHY, 10, 4, 4096), (Engine.TOWER, 8, 4, 2048),
                                          (Engine.AFFT, 16, 16, 256)])
def test_device_push_follows_the_producing_stream(gpu, oracle, engine, k, m, L):
    torch = _torch()
    p = gpu.resolve(engine, k, m, L)
    data = data_for(k, L, 72)
    word = encode_word(oracle, oracle.resolve(engine, k, m, L), data)
    order = list(range(m, k + m))[:k]  # the first m data symbols lost
    src = torch.from_numpy(np.stack([word[i] for i in order])).cuda()
    buf = torch.zeros_like(src)
    torch.cuda.synchronize()
    dec = gpu.decoder(p)
    side = torch.cuda.Stream()
    with torch.cuda.stream(side):
        torch.cuda._sleep(HOLD_CYCLES)
        buf.copy_(src)
        for q, i in enumerate(order):
            dec.push(i, buf[q])
        buf.fill_(0xA5)
    out = np.zeros(k * L, np.uint8)
    dec.finalize_into_with(out, dec.scratch())
    assert np.array_equal(out, data)
    torch.cuda.synchronize()


@pytest.mark.parametrize("engine,k,m,L", [(Engine.GOOD_CAUCHY, 10, 4, 4096), (Engine.TOWER, 8, 4, 2048),
                                          (Engine.AFFT, 16, 16, 256)])
@pytest.mark.parametrize("second", ["device", "host"])
def test_refill_waits_for_the_last_device_finalize(gpu, oracle, engine, k, m, L, second):
    """Finalize on a held-back stream, reset, refill with another word (device
    pushes on another stream, or host pushes uploaded by the next finalize)
    and finalize again: both outputs must be their own words' data."""
    torch = _torch()
    p = gpu.resolve(engine, k, m, L)
    po = oracle.resolve(engine, k, m, L)
    data1, data2 = data_for(k, L, 73), data_for(k, L, 74)
    word1, word2 = encode_word(oracle, po, data1), encode_word(oracle, po, data2)
    order = list(range(m // 2, m // 2 + k))  # data symbols 0 .. m/2-1 lost
    rows1 = [torch.from_numpy(word1[i]).cuda() for i in order]
    rows2 = [torch.from_numpy(word2[i]).cuda() for i in order]
    out1 = torch.zeros(k * L, dtype=torch.uint8, device="cuda")
    out2 = torch.zeros_like(out1)
    torch.cuda.synchronize()
    dec = gpu.decoder(p)
    s1, s2 = dec.scratch(), dec.scratch()
    for q, i in enumerate(order):
        dec.push(i, rows1[q])
    held, other = torch.cuda.Stream(), torch.cuda.Stream()
    with torch.cuda.stream(held):
        torch.cuda._sleep(HOLD_CYCLES)
        dec.finalize_into_with(out1, s1)  # reads the payload rows ~30 ms from now
    dec.reset()
    with torch.cuda.stream(other):
        for q, i in enumerate(order):
            if second == "device":
                dec.push(i, rows2[q])
            else:
                dec.push(i, word2[i])
        dec.finalize_into_with(out2, s2)
    torch.cuda.synchronize()
    assert np.array_equal(out1.cpu().numpy(), data1)
    assert np.array_equal(out2.cpu().numpy(), data2)


def test_legacy_stream_entry_points_order_with_the_default_stream(gpu, oracle):
    """scrs_inc_feed_device / scrs_dec_push_device copy on the legacy default
    stream, which orders them with torch's default stream."""
    torch = _torch()
    import ctypes as C

    from scrs_b200.api import _Error, _Push

    k, m, L = 10, 4, 4096
    p = gpu.resolve(Engine.GOOD_CAUCHY, k, m, L)
    data = data_for(k, L, 75)
    word = encode_word(oracle, oracle.resolve(Engine.GOOD_CAUCHY, k, m, L), data)
    src = torch.from_numpy(data).cuda().view(k, L)
    buf = torch.zeros_like(src)
    torch.cuda.synchronize()
    inc = gpu.incremental_encoder(p)
    err = _Error()
    torch.cuda._sleep(HOLD_CYCLES)  # on the default stream
    buf.copy_(src)
    for i in range(k):
        assert gpu.lib.inc_feed_device(inc._ptr, i, buf[i].data_ptr(), L, C.byref(err)) == 0
    buf.fill_(0x33)
    for j in range(m):
        assert np.array_equal(np.frombuffer(inc.repair(j), dtype=np.uint8), word[k + j]), j
    dec = gpu.decoder(p)
    rows = torch.from_numpy(np.stack([word[i] for i in range(m, k + m)])).cuda()
    torch.cuda.synchronize()
    o = _Push()
    torch.cuda._sleep(HOLD_CYCLES)
    buf2 = rows.clone()  # produced on the default stream after the hold
    for q, i in enumerate(range(m, k + m)):
        assert gpu.lib.dec_push_device(dec._ptr, i, buf2[q].data_ptr(), L, C.byref(o), C.byref(err)) == 0
    buf2.fill_(0x44)
    out = np.zeros(k * L, np.uint8)
    dec.finalize_into_with(out, dec.scratch())
    assert np.array_equal(out, data)
    torch.cuda.synchronize()


@pytest.mark.parametrize("graph", [False, True])
def test_stripe_batch_set_waits_for_the_last_run(gpu, oracle, graph):
    """Run a batch on a held-back stream, then set the same batch object to
    other stripes at once and run them on another stream: the first run must
    still compute its own stripes (the set waits for it before rewriting the
    device descriptors)."""
    torch = _torch()
    from scrs_b200.batch import StripeBatch

    from scenarios import device_stripes, make_mixed_batch

    specs1, rng1 = make_mixed_batch(torch, 48, 31, lens=(1024, 4096))
    specs2, rng2 = make_mixed_batch(torch, 48, 32, lens=(1024, 4096))
    st1, outs1, exp1, keep1 = device_stripes(torch, oracle, specs1, rng1)
    st2, outs2, exp2, keep2 = device_stripes(torch, oracle, specs2, rng2)
    torch.cuda.synchronize()
    b = StripeBatch(gpu.lib, 64)
    held, other = torch.cuda.Stream(), torch.cuda.Stream()
    b.set(st1)
    with torch.cuda.stream(held):
        torch.cuda._sleep(HOLD_CYCLES)
        b.run(graph=graph)
    b.set(st2)
    with torch.cuda.stream(other):
        b.run(graph=graph)
    torch.cuda.synchronize()
    b.check()
    for o, e in zip(outs1, exp1):
        assert np.array_equal(o.cpu().numpy(), e)
    for o, e in zip(outs2, exp2):
        assert np.array_equal(o.cpu().numpy(), e)
