"""Autotuner of the persistent drain (scrs_stripe_batch_autotune): every
launch configuration it may pick gives the oracle's bytes, the pick is one of
its candidates and is used by later runs (graph runs re-captured), and a
host-buffer batch tunes on its staged inputs."""
import numpy as np
import pytest

from scenarios import device_stripes, make_mixed_batch

pytestmark = pytest.mark.gpu


@pytest.fixture
def clean_table(gpu):
    from scrs_b200 import tune

    tune.clear(gpu.lib)
    yield
    tune.clear(gpu.lib)


def check(torch, b, outs, expect, graph):
    for o in outs:
        o.zero_()
    b.run(graph=graph)
    torch.cuda.synchronize()
    b.check()
    for o, exp in zip(outs, expect):
        assert np.array_equal(o.cpu().numpy(), exp)


@pytest.mark.parametrize("seg_rows,ctas", [(1, 2), (7, 8), (8, 4), (16, 6), (24, 3), (32, 3), (32, 1)])
def test_every_launch_configuration_is_exact(gpu, oracle, clean_table, seg_rows, ctas):
    """Stripes with up to 64 inputs (several segments at every seg_rows),
    ragged and unaligned symbol lengths."""
    torch = pytest.importorskip("torch")
    from scrs_b200 import tune
    from scrs_b200.batch import StripeBatch

    specs, rng = make_mixed_batch(torch, 24, 17, lens=(1024, 4096, 1000, 64, 2050))
    stripes, outs, expect, keep = device_stripes(torch, oracle, specs, rng)
    b = StripeBatch(gpu.lib, len(stripes))
    b.set(stripes)
    tune.set_entry(gpu.lib, b.tune_key, tune.TuneParams(seg_rows, ctas))
    lp = b.launch_params
    assert lp.seg_rows == min(seg_rows, max(s[2] for s in specs))
    assert 1 <= lp.ctas_per_sm <= ctas
    check(torch, b, outs, expect, graph=False)
    check(torch, b, outs, expect, graph=True)


def test_autotune_picks_a_candidate_and_runs_use_it(gpu, oracle, clean_table):
    torch = pytest.importorskip("torch")
    from scrs_b200 import tune
    from scrs_b200.batch import StripeBatch

    specs, rng = make_mixed_batch(torch, 64, 23, lens=(1024, 4096, 1000))
    stripes, outs, expect, keep = device_stripes(torch, oracle, specs, rng)
    b = StripeBatch(gpu.lib, len(stripes))
    b.set(stripes)
    default = b.launch_params
    assert default.seg_rows == min(16, max(s[2] for s in specs))
    check(torch, b, outs, expect, graph=True)  # graph captured under the default
    chosen = b.autotune(reps=3)
    k_max = max(s[2] for s in specs)
    assert chosen.seg_rows in {min(c, k_max) for c in (8, 12, 16, 24, 32, k_max)}
    assert chosen.drain_ms > 0
    lp = b.launch_params
    assert (lp.seg_rows, lp.ctas_per_sm) == (chosen.seg_rows, chosen.ctas_per_sm)
    assert dict(tune.entries(gpu.lib))[b.tune_key].seg_rows == chosen.seg_rows
    check(torch, b, outs, expect, graph=True)  # re-captured with the tuned parameters
    check(torch, b, outs, expect, graph=False)
    # a second batch of the same geometry finds the entry
    b2 = StripeBatch(gpu.lib, len(stripes))
    b2.set(stripes)
    assert b2.tune_key == b.tune_key
    assert (b2.launch_params.seg_rows, b2.launch_params.ctas_per_sm) == (chosen.seg_rows, chosen.ctas_per_sm)


def test_autotune_host_buffer_batch(gpu, oracle, clean_table):
    torch = pytest.importorskip("torch")
    from scrs_b200.batch import StripeBatch

    specs, rng = make_mixed_batch(torch, 16, 29, lens=(1024, 4096), kmax=40, mmax=8)
    stripes, outs, expect, keep = device_stripes(torch, oracle, specs, rng)
    n = len(specs)
    kmax = max(s[2] for s in specs)
    indices = np.zeros((n, kmax), np.uint16)
    host_in, host_out = [], []
    for s, st in enumerate(stripes):
        host_in.append(keep[s].cpu().pin_memory())
        host_out.append(torch.zeros(outs[s].numel(), dtype=torch.uint8).pin_memory())
        if st.indices is not None:
            indices[s, :st.k] = st.indices
    b = StripeBatch(gpu.lib, n)
    b.set_arrays(np.array([s.op for s in stripes]), np.array([int(s.engine) for s in stripes]),
                 np.array([s.k for s in stripes]), np.array([s.m for s in stripes]),
                 np.array([s.symbol_len for s in stripes]), np.array([h.data_ptr() for h in host_in], dtype=np.uint64),
                 np.array([h.data_ptr() for h in host_out], dtype=np.uint64), indices=indices, host=True)
    chosen = b.autotune(reps=2)
    assert chosen.seg_rows >= 1
    for h in host_out:
        h.zero_()
    b.run()
    torch.cuda.synchronize()
    b.check()
    for h, exp in zip(host_out, expect):
        assert np.array_equal(h.numpy(), exp)
