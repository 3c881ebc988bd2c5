"""The allocation-free GF(256) decode entry point (scrs_gf256_decode_static),
called through the C ABI, must return the same bytes as the regular device
decode (scrs_batch_decode_into_with_device) on two calls in a row.

Callers that cannot allocate device memory (cudaMalloc may synchronise the
device, and a process that reserved its memory pool at start-up has no
headroom) use this entry point; its recipe scratch is one fixed device array
shared by all calls.  This file is collected last so a failure here never
hides the other tests' results."""
import ctypes as C

import numpy as np
import pytest

from scrs_b200.api import Engine, _Error

pytestmark = pytest.mark.gpu


def static_decode(lib, engine, k, m, L, indices, d_rows, d_out):
    fn = lib.lib.scrs_gf256_decode_static
    fn.restype = C.c_int32
    fn.argtypes = [C.c_int32, C.c_uint64, C.c_uint64, C.c_uint64, C.POINTER(C.c_uint64), C.c_void_p,
                   C.c_uint64, C.c_void_p, C.c_uint64, C.c_void_p, C.POINTER(_Error)]
    idx = (C.c_uint64 * len(indices))(*indices)
    err = _Error()
    st = fn(int(engine), k, m, L, idx, d_rows.data_ptr(), len(indices), d_out.data_ptr(), d_out.numel(), None,
            C.byref(err))
    return st, err


def test_static_decode_matches_regular_decode_twice(gpu):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(0x5C25)
    cases = [(Engine.GOOD_CAUCHY, 10, 4, 4096), (Engine.STANDARD_CAUCHY, 32, 8, 1000)]
    for engine, k, m, L in cases:
        p = gpu.resolve(engine, k, m, L)
        enc = gpu.batch_encoder(p)
        dec = gpu.batch_decoder(p)
        ds = dec.scratch()
        for call in range(2):  # two calls in a row: the shared array must not leak state
            data = torch.from_numpy(rng.integers(0, 256, k * L, dtype=np.uint8)).cuda()
            rep = torch.zeros(m * L, dtype=torch.uint8, device="cuda")
            enc.encode_into_with(data, rep, enc.scratch())
            word = torch.cat([data.view(k, L), rep.view(m, L)])
            sel = rng.permutation(k + m)[:k].tolist()
            rows = word[torch.tensor(sel, device="cuda")].reshape(-1).contiguous()
            expect = torch.zeros(k * L, dtype=torch.uint8, device="cuda")
            dec.decode_into_with((sel, rows), expect, ds)
            got = torch.full((k * L,), 0xA5, dtype=torch.uint8, device="cuda")
            st, err = static_decode(gpu.lib, engine, k, m, L, sel, rows, got)
            torch.cuda.synchronize()
            assert st == 0, (st, err.code, err.a, err.b)
            assert torch.equal(got, expect), (engine, k, m, L, call)
            assert torch.equal(got, data)


def test_static_decode_rejects_oversized_recipe(gpu):
    torch = pytest.importorskip("torch")
    k, m, L = 128, 128, 64  # recipe 2*(3*128+3*128) + 128*128 bytes > 16 KiB
    rows = torch.zeros(k * L, dtype=torch.uint8, device="cuda")
    out = torch.zeros(k * L, dtype=torch.uint8, device="cuda")
    sel = list(range(k, 2 * k))  # every data symbol erased: r = 128
    st, err = static_decode(gpu.lib, Engine.STANDARD_CAUCHY, k, m, L, sel, rows, out)
    assert st == 905 and err.b == 16384 and err.a > 16384
