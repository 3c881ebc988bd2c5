"""Encode kernels specialised to one coefficient matrix (include/scrs_gpu.h
scrs_jit_prepare): the generated source compiles for sm_100a with NVRTC for
both GF(256) engines across the eligible geometries, and ineligible requests
are refused.  Compile only: no device needed."""
import pytest

from scrs_b200.api import Engine, RuntimeFailure


@pytest.fixture(scope="module")
def lib():
    from scrs_b200.api import Library
    from scrs_b200.build import build

    return Library(build(), prefix="scrs_", device=True)


@pytest.mark.parametrize("engine,k,m", [(Engine.GOOD_CAUCHY, 10, 4), (Engine.STANDARD_CAUCHY, 10, 4),
                                        (Engine.GOOD_CAUCHY, 1, 1), (Engine.STANDARD_CAUCHY, 3, 5),
                                        (Engine.GOOD_CAUCHY, 32, 2), (Engine.STANDARD_CAUCHY, 16, 4),
                                        (Engine.GOOD_CAUCHY, 7, 9)])
def test_specialised_kernel_compiles(lib, engine, k, m):
    from scrs_b200.batch import jit_prepare

    assert jit_prepare(lib, engine, k, m, load=False) > 0


@pytest.mark.parametrize("engine,k,m", [(Engine.GOOD_CAUCHY, 33, 1), (Engine.GOOD_CAUCHY, 16, 5),
                                        (Engine.TOWER, 4, 2), (Engine.GOOD_CAUCHY, 0, 4)])
def test_ineligible_requests_are_refused(lib, engine, k, m):
    from scrs_b200.batch import jit_prepare

    with pytest.raises(RuntimeFailure) as e:
        jit_prepare(lib, engine, k, m, load=False)
    assert e.value.variant == "BadArgument"
