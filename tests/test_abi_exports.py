"""The CUDA library loads and exports exactly the entry points that
include/scrs_gpu.h declares (no compute; runs without a GPU)."""
import ctypes as C
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared():
    text = (ROOT / "include" / "scrs_gpu.h").read_text()
    return sorted(set(re.findall(r"^SCRS_API [^()]*?\b(scrs_[a-z0-9_]+)\(", text, flags=re.M)))


@pytest.fixture(scope="module")
def lib_path():
    from scrs_b200.build import build

    return build()


def test_header_declares_the_trait_surface():
    names = declared()
    for n in ["scrs_profile_resolve", "scrs_profile_recommended", "scrs_batch_encode_into_with",
              "scrs_batch_decode_into_with", "scrs_inc_feed", "scrs_inc_repair", "scrs_dec_push",
              "scrs_dec_finalize_into_with", "scrs_stripe_batch_run"]:
        assert n in names


def test_library_exports_every_declared_symbol(lib_path):
    lib = C.CDLL(str(lib_path))
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_resolves_all_signatures(lib_path):
    from scrs_b200.api import Library
    from scrs_b200.batch import _bind

    lib = Library(lib_path, prefix="scrs_", device=True)
    _bind(lib)
    assert lib.abi_version() == 0x00010000


def test_profile_logic_without_device(lib_path):
    """Profile resolution is host logic; it needs no GPU."""
    from scrs_b200.api import Api, ConfigError, Engine, Library

    api = Api(Library(lib_path))
    assert api.resolve(Engine.TOWER, 32, 8, 64).engine == Engine.TOWER
    assert api.recommended_gf16_engine(32, 8) == Engine.TOWER
    with pytest.raises(ConfigError) as e:
        api.resolve(Engine.GOOD_CAUCHY, 200, 100, 64)
    assert e.value.fields == {"cap": 255}
