"""Stripe batches whose encode stripes run through kernels specialised to
their coefficient matrix (jit.cu): bit-exact with the oracle for both engines,
aligned, unaligned and partial-chunk lengths, next to decode stripes of the
generic drain; the same bytes with specialisation off; small groups stay on
the generic drain."""
import numpy as np
import pytest

from scrs_b200.api import Engine

from scenarios import device_stripes

pytestmark = pytest.mark.gpu

OP_ENCODE, OP_DECODE = 0, 1


def run_and_check(torch, b, outs, expect, graph):
    for o in outs:
        o.zero_()
    b.run(graph=graph)
    torch.cuda.synchronize()
    b.check()
    for q, (o, exp) in enumerate(zip(outs, expect)):
        assert np.array_equal(o.cpu().numpy(), exp), q


def test_specialised_encode_groups_match_oracle(gpu, oracle):
    torch = pytest.importorskip("torch")
    from scrs_b200.batch import StripeBatch

    rng = np.random.default_rng(31)
    # three eligible groups with at least one persistent grid of items each,
    # a small eligible group (stays generic) and decode stripes (generic)
    specs = [(OP_ENCODE, Engine.GOOD_CAUCHY, 10, 4, 4096)] * 600
    specs += [(OP_ENCODE, Engine.STANDARD_CAUCHY, 6, 3, 1000)] * 1200   # unaligned, one partial chunk
    specs += [(OP_ENCODE, Engine.GOOD_CAUCHY, 3, 5, 2050)] * 600        # two chunks, the second ragged
    specs += [(OP_ENCODE, Engine.GOOD_CAUCHY, 12, 4, 4096)] * 8         # too few items
    specs += [(OP_DECODE, Engine.GOOD_CAUCHY, 10, 4, 4096)] * 64
    order = rng.permutation(len(specs))
    specs = [specs[i] for i in order]
    stripes, outs, expect, keep = device_stripes(torch, oracle, specs, rng)
    b = StripeBatch(gpu.lib, len(stripes))
    b.set(stripes)
    assert b.jit_stripes == 600 + 1200 + 600
    run_and_check(torch, b, outs, expect, graph=False)
    run_and_check(torch, b, outs, expect, graph=True)
    assert b.last_launches == 5  # plan, three specialised drains, generic drain
    plan_ms, spec_ms, gen_ms = b.run_timed_drains()
    assert spec_ms > 0 and gen_ms > 0
    b.set_jit(False)
    b.set(stripes)
    assert b.jit_stripes == 0
    run_and_check(torch, b, outs, expect, graph=False)


def test_specialised_cfg1_geometry_with_decodes(gpu, oracle):
    """The benchmark's shape at a small count: Good Cauchy k=10 m=4 L=4096,
    encode stripes specialised, decode stripes on the generic drain."""
    torch = pytest.importorskip("torch")
    from scrs_b200.batch import StripeBatch, jit_prepare

    assert jit_prepare(gpu.lib, Engine.GOOD_CAUCHY, 10, 4) > 0
    rng = np.random.default_rng(37)
    specs = [(OP_ENCODE if s % 2 == 0 else OP_DECODE, Engine.GOOD_CAUCHY, 10, 4, 4096) for s in range(1400)]
    stripes, outs, expect, keep = device_stripes(torch, oracle, specs, rng)
    b = StripeBatch(gpu.lib, len(stripes))
    b.set(stripes)
    assert b.jit_stripes == 700
    run_and_check(torch, b, outs, expect, graph=True)


def test_specialised_widest_geometries(gpu, oracle):
    """The largest staged row count (k = 32) and the largest product count
    (k * m = 64) a specialised kernel takes."""
    torch = pytest.importorskip("torch")
    from scrs_b200.batch import StripeBatch

    rng = np.random.default_rng(41)
    specs = [(OP_ENCODE, Engine.GOOD_CAUCHY, 32, 2, 4096)] * 600
    specs += [(OP_ENCODE, Engine.STANDARD_CAUCHY, 16, 4, 2048)] * 1200
    stripes, outs, expect, keep = device_stripes(torch, oracle, specs, rng)
    b = StripeBatch(gpu.lib, len(stripes))
    b.set(stripes)
    assert b.jit_stripes == 1800
    run_and_check(torch, b, outs, expect, graph=False)



def test_more_groups_than_specialised_runs(gpu, oracle):
    """Five eligible encode groups, each large enough: four get specialised
    kernels, the fifth runs on the generic drain; every output is exact."""
    torch = pytest.importorskip("torch")
    from scrs_b200.batch import StripeBatch

    rng = np.random.default_rng(43)
    geoms = [(Engine.GOOD_CAUCHY, 3, 2), (Engine.GOOD_CAUCHY, 4, 3), (Engine.STANDARD_CAUCHY, 5, 2),
             (Engine.STANDARD_CAUCHY, 2, 4), (Engine.GOOD_CAUCHY, 6, 1)]
    specs = [(OP_ENCODE, e, k, m, 4096) for e, k, m in geoms for _ in range(600)]
    specs = [specs[i] for i in rng.permutation(len(specs))]
    stripes, outs, expect, keep = device_stripes(torch, oracle, specs, rng)
    b = StripeBatch(gpu.lib, len(stripes))
    b.set(stripes)
    assert b.jit_stripes == 4 * 600
    run_and_check(torch, b, outs, expect, graph=True)
    assert b.last_launches == 5  # four specialised drains and the generic drain (no decodes, no plan)
