"""Autotuner table and geometry key (host logic of include/scrs_gpu.h
scrs_tune_*; no device needed): key buckets follow their definition, entries
round-trip through the table and through a JSON file, bad entries are refused."""
import math

import numpy as np
import pytest

from scrs_b200.api import RuntimeFailure


@pytest.fixture
def lib():
    from scrs_b200.api import Library
    from scrs_b200.build import build
    from scrs_b200 import tune

    L = Library(build(), prefix="scrs_", device=True)
    tune.clear(L)
    yield L
    tune.clear(L)


def descs(rows):
    """rows: (op, k, m, L, indices or None) -> DESC_DTYPE records (null buffers)."""
    from scrs_b200.batch import DESC_DTYPE

    d = np.zeros(len(rows), dtype=DESC_DTYPE)
    keep = []
    for s, (op, k, m, L, idx) in enumerate(rows):
        d[s]["op"], d[s]["engine"], d[s]["k"], d[s]["m"], d[s]["symbol_len"] = op, 1, k, m, L
        if idx is not None:
            a = np.asarray(idx, dtype=np.uint16)
            keep.append(a)
            d[s]["indices"] = a.ctypes.data
    return d, keep


def expected_key(rows):
    """The key's definition: ceil(log2(max k)), ceil(log2(mean outputs)), floor(log2(mean L))."""
    outs = []
    for op, k, m, L, idx in rows:
        outs.append(m if op == 0 else k - sum(1 for i in idx if i < k))
    mean_out = -(-sum(outs) // len(rows))
    mean_l = sum(r[3] for r in rows) // len(rows)
    k_max = max(r[1] for r in rows)
    return (0, math.ceil(math.log2(k_max)) if k_max > 1 else 0,
            math.ceil(math.log2(mean_out)) if mean_out > 1 else 0, int(math.floor(math.log2(mean_l))))


@pytest.mark.parametrize("rows", [
    [(0, 10, 4, 4096, None), (1, 10, 4, 4096, [0, 1, 2, 3, 4, 5, 10, 11, 12, 13])],
    [(0, 64, 16, 65536, None)],
    [(1, 1, 1, 1024, [0]), (1, 3, 2, 1000, [4, 3, 2])],
    [(0, 33, 1, 1024, None), (0, 4, 9, 4096, None), (1, 20, 5, 16384, [19, 18, 17] + list(range(20, 25)) + list(range(12)))],
])
def test_key_buckets(lib, rows):
    from scrs_b200 import tune

    d, keep = descs(rows)
    k = tune.key_of(lib, d)
    assert (k.field, k.k_bucket, k.m_bucket, k.l_bucket) == expected_key(rows)


def test_table_round_trip_and_json(lib, tmp_path):
    from scrs_b200 import tune
    from scrs_b200.tune import TuneKey, TuneParams

    assert tune.entries(lib) == []
    a, b = TuneKey(0, 4, 2, 12), TuneKey(0, 6, 3, 14)
    tune.set_entry(lib, a, TuneParams(10, 8, 2.5))
    tune.set_entry(lib, b, TuneParams(24, 4, 7.25))
    tune.set_entry(lib, a, TuneParams(8, 6, 2.0))  # replaces
    got = dict(tune.entries(lib))
    assert got == {a: TuneParams(8, 6, 2.0), b: TuneParams(24, 4, 7.25)}
    path = tmp_path / "tune.json"
    assert tune.save(lib, path) == 2
    tune.clear(lib)
    assert tune.entries(lib) == []
    assert tune.load(lib, path) == 2
    assert dict(tune.entries(lib)) == got
    (tmp_path / "bad.json").write_text('{"format": "other", "entries": []}')
    with pytest.raises(ValueError):
        tune.load(lib, tmp_path / "bad.json")


@pytest.mark.parametrize("params", [(0, 4), (33, 4), (16, 0), (16, 33)])
def test_table_refuses_bad_params(lib, params):
    from scrs_b200 import tune
    from scrs_b200.tune import TuneKey, TuneParams

    with pytest.raises(RuntimeFailure):
        tune.set_entry(lib, TuneKey(0, 4, 2, 12), TuneParams(*params))
    with pytest.raises(RuntimeFailure):  # only GF(256) stripe batches are tuned
        tune.set_entry(lib, TuneKey(1, 4, 2, 12), TuneParams(16, 4))
    assert tune.entries(lib) == []
