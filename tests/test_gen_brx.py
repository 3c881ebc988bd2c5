"""The generated jump-table XOR networks (scrs_b200/csrc/gen_brx.py) compute
c*x over GF(256): the common-subexpression pass keeps every output plane's
XOR set, and the planes reassemble to the table product."""
import importlib.util
from pathlib import Path

import numpy as np

import gfpy

_spec = importlib.util.spec_from_file_location(
    "gen_brx", Path(__file__).resolve().parents[1] / "scrs_b200" / "csrc" / "gen_brx.py")
gen = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(gen)


def expand(term, pairs):
    if term < 8:
        return {term}
    a, b = pairs[term - 8]
    return expand(a, pairs) ^ expand(b, pairs)


def test_cse_keeps_xor_sets():
    for c in range(256):
        rows = gen.rows_of(c)
        pairs, new_rows = gen.cse_rows(rows)
        assert len(pairs) <= gen.MAX_TEMPS
        for r in range(8):
            acc = set()
            for t in new_rows[r]:
                acc ^= expand(t, pairs)
            assert acc == set(rows[r]), (c, r)


def test_planes_give_products():
    x = np.arange(256, dtype=np.uint8)
    for c in range(256):
        rows = gen.rows_of(c)
        got = np.zeros(256, np.uint8)
        for r in range(8):
            bit = np.zeros(256, np.uint8)
            for s in rows[r]:
                bit ^= (x >> s) & 1
            got |= bit << r
        exp = np.array([gfpy.mul(c, int(v)) for v in x], np.uint8)
        assert np.array_equal(got, exp), c
