"""Handles used from several threads at once.

Engines are not shared between threads (as in the reference, each is used by
one thread at a time), but independent handles may run concurrently, and the
first launches of a kernel on a device set its shared-memory attributes.  A
fresh process starts 8 threads behind a barrier, each building its own
engines and running GF(256), tower and additive-FFT work whose kernels need
more than 48 KiB of dynamic shared memory; every thread's bytes must equal
the oracle's.
"""
import subprocess
import sys
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]

CHILD = r'''
import sys, threading
import numpy as np
sys.path.insert(0, sys.argv[1]); sys.path.insert(0, sys.argv[1] + "/tests")
import torch
import scrs_b200
from scrs_b200.api import Api, Engine, Library
from scenarios import data_for, encode_word
from conftest import build_oracle

oracle = Api(Library(build_oracle(), prefix="oracle_", device=False))
gpu = scrs_b200.api_default()
cases = [(Engine.GOOD_CAUCHY, 40, 16, 4096), (Engine.TOWER, 32, 8, 4096), (Engine.AFFT, 512, 512, 1024)]
expect = {}
for engine, k, m, L in cases:
    data = data_for(k, L, 90 + k)
    expect[engine] = (data, encode_word(oracle, oracle.resolve(engine, k, m, L), data))
N = 8
gate = threading.Barrier(N)
errors = []

def work(t):
    try:
        torch.cuda.set_device(0)
        gate.wait()
        for engine, k, m, L in cases:
            data, word = expect[engine]
            p = gpu.resolve(engine, k, m, L)
            if engine == Engine.TOWER:
                inc = gpu.incremental_encoder(p)
                for i in range(k):
                    inc.feed(i, data[i * L:(i + 1) * L])
                reps = [np.frombuffer(inc.repair(j), dtype=np.uint8) for j in range(m)]
            else:
                enc = gpu.batch_encoder(p)
                out = np.zeros(m * L, np.uint8)
                enc.encode_into_with(data, out, enc.scratch())
                reps = [out[j * L:(j + 1) * L] for j in range(m)]
            assert all(np.array_equal(a, b) for a, b in zip(reps, word[k:])), (t, engine, "encode")
            idx = list(range(m // 2, m // 2 + k))
            dec = gpu.batch_decoder(p)
            out = np.zeros(k * L, np.uint8)
            dec.decode_into_with([(i, word[i]) for i in idx], out, dec.scratch())
            assert np.array_equal(out, data), (t, engine, "decode")
    except BaseException as e:  # reported by the parent
        errors.append(repr(e))

threads = [threading.Thread(target=work, args=(t,)) for t in range(N)]
for th in threads: th.start()
for th in threads: th.join()
print("errors:", errors)
sys.exit(1 if errors else 0)
'''


def test_independent_handles_on_many_threads_from_first_use():
    r = subprocess.run([sys.executable, "-c", CHILD, str(ROOT)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, (r.stdout[-3000:], r.stderr[-3000:])
