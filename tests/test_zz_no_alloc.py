"""The allocation-free GF(256) decode entry point (scrs_gf256_decode_static),
called through the C ABI, must return the same bytes as the regular device
decode (scrs_batch_decode_into_with_device) on two calls in a row.

Callers that cannot allocate device memory (cudaMalloc may synchronise the
device, and a process that reserved its memory pool at start-up has no
headroom) use this entry point; its recipe scratch is one fixed device array
shared by all calls.  Once the first call on the device has done its set-up,
calls must leave the library's allocation count and the device's free memory
unchanged, and report no device timeout through the caller's status word.
This file is collected last so a failure here never hides the other tests'
results."""
import ctypes as C

import numpy as np
import pytest

from scrs_b200.api import Engine, _Error

pytestmark = pytest.mark.gpu

LIMIT = 16384  # bytes of the fixed recipe array


def static_decode(lib, engine, k, m, L, indices, d_rows, d_out, d_status=None):
    fn = lib.lib.scrs_gf256_decode_static
    fn.restype = C.c_int32
    fn.argtypes = [C.c_int32, C.c_uint64, C.c_uint64, C.c_uint64, C.POINTER(C.c_uint64), C.c_void_p,
                   C.c_uint64, C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p, C.POINTER(_Error)]
    idx = (C.c_uint64 * len(indices))(*indices)
    err = _Error()
    st = fn(int(engine), k, m, L, idx, d_rows.data_ptr(), len(indices), d_out.data_ptr(), d_out.numel(), None,
            None if d_status is None else d_status.data_ptr(), C.byref(err))
    return st, err


def recipe_bytes(k, r):
    return ((2 * (3 * k + 3 * r) + 15) & ~15) + k * max(r, 1)


def make_case(gpu, torch, engine, k, m, L, sel, rng):
    """(selection, received rows, expected data) of a fresh random stripe,
    its expected output decoded by the regular device entry point."""
    p = gpu.resolve(engine, k, m, L)
    enc = gpu.batch_encoder(p)
    data = torch.from_numpy(rng.integers(0, 256, k * L, dtype=np.uint8)).cuda()
    rep = torch.zeros(m * L, dtype=torch.uint8, device="cuda")
    enc.encode_into_with(data, rep, enc.scratch())
    word = torch.cat([data.view(k, L), rep.view(m, L)])
    rows = word[torch.tensor(sel, device="cuda")].reshape(-1).contiguous()
    dec = gpu.batch_decoder(p)
    expect = torch.zeros(k * L, dtype=torch.uint8, device="cuda")
    dec.decode_into_with((sel, rows), expect, dec.scratch())
    torch.cuda.synchronize()
    assert torch.equal(expect, data)
    return sel, rows, expect


def test_static_decode_matches_regular_decode_twice(gpu):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(0x5C25)
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    # k = 128, r = 116 needs 16320 bytes, just under the limit
    at_limit = list(range(116, 128)) + list(range(128, 128 + 116))
    assert recipe_bytes(128, 116) <= LIMIT < recipe_bytes(128, 117)
    cases = [(Engine.GOOD_CAUCHY, 10, 4, 4096, None),  # random pattern
             (Engine.STANDARD_CAUCHY, 32, 8, 1000, None),  # ragged length, two input segments
             (Engine.GOOD_CAUCHY, 12, 4, 512, list(range(12))),  # r = 0: every data symbol received
             (Engine.STANDARD_CAUCHY, 128, 128, 64, at_limit)]
    built = []
    for engine, k, m, L, sel in cases:
        for call in range(2):  # two calls in a row: the shared array must not leak state
            s = sel if sel is not None else rng.permutation(k + m)[:k].tolist()
            built.append((engine, k, m, L) + make_case(gpu, torch, engine, k, m, L, s, rng))

    def run_all():
        for engine, k, m, L, s, rows, expect in built:
            got = torch.full((k * L,), 0xA5, dtype=torch.uint8, device="cuda")
            st, err = static_decode(gpu.lib, engine, k, m, L, s, rows, got, status)
            torch.cuda.synchronize()
            assert st == 0, (st, err.code, err.a, err.b)
            assert torch.equal(got, expect), (engine, k, m, L)

    run_all()  # the first calls on the device do the one-time set-up
    outs = [torch.empty(k * L, dtype=torch.uint8, device="cuda") for _, k, _, L, *_ in built]
    torch.cuda.synchronize()
    before, free_before = gpu.lib.alloc_count(), torch.cuda.mem_get_info()[0]
    for (engine, k, m, L, s, rows, expect), got in zip(built, outs):
        st, err = static_decode(gpu.lib, engine, k, m, L, s, rows, got, status)
        assert st == 0, (st, err.code, err.a, err.b)
    torch.cuda.synchronize()
    assert gpu.lib.alloc_count() == before
    assert torch.cuda.mem_get_info()[0] == free_before
    assert int(status.item()) == 0
    for (engine, k, m, L, s, rows, expect), got in zip(built, outs):
        assert torch.equal(got, expect), (engine, k, m, L)


def test_static_decode_rejects_oversized_recipe(gpu):
    torch = pytest.importorskip("torch")
    k, m, L = 128, 128, 64
    rows = torch.zeros(k * L, dtype=torch.uint8, device="cuda")
    out = torch.zeros(k * L, dtype=torch.uint8, device="cuda")
    for r in (117, 128):  # one erasure past the limit, and every data symbol erased
        sel = list(range(r, k)) + list(range(k, k + r))
        st, err = static_decode(gpu.lib, Engine.STANDARD_CAUCHY, k, m, L, sel, rows, out)
        assert st == 905 and err.b == LIMIT and err.a == recipe_bytes(k, r) > LIMIT
