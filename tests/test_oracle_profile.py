"""Profile selection and constructor validation against the reference's own
assertions (scrs/src/selector.rs tests, scrs/src/lib.rs tests)."""
import json
from pathlib import Path

import pytest

from scrs_b200.api import ConfigError, Engine, Field

KATS = json.loads((Path(__file__).parent / "golden" / "reference_kats.json").read_text())
ENG = {"StandardCauchy": Engine.STANDARD_CAUCHY, "GoodCauchy": Engine.GOOD_CAUCHY,
       "Tower": Engine.TOWER, "Afft": Engine.AFFT}


@pytest.mark.parametrize("case", KATS["recommended_gf16_engine"], ids=lambda c: c["at"])
def test_recommended_gf16_engine(oracle, case):  # lib.rs:99-130
    assert oracle.recommended_gf16_engine(case["k"], case["m"]) == ENG[case["engine"]]


@pytest.mark.parametrize("case", KATS["profile_recommended"], ids=lambda c: c["at"])
def test_profile_recommended(oracle, case):  # selector.rs:540-565
    field = Field.GF256 if case["field"] == "Gf256" else Field.GF65536
    assert oracle.recommended(field, case["k"], case["m"], case["symbol_len"]).engine == ENG[case["engine"]]


@pytest.mark.parametrize("case", KATS["profile_resolve_errors"], ids=lambda c: c["at"])
def test_profile_resolve_errors(oracle, case):  # selector.rs:567-585
    with pytest.raises(ConfigError) as ei:
        oracle.resolve(ENG[case["engine"]], case["k"], case["m"], case["symbol_len"])
    assert ei.value.variant == case["error"]
    if case["cap"] is not None:
        assert ei.value.fields["cap"] == case["cap"]


@pytest.mark.parametrize("case", KATS["batch_capacity"], ids=lambda c: c["at"])
def test_batch_capacity_boundaries(oracle, case):  # batch/codec.rs:698-704
    eng = ENG[case["engine"]]
    if case["ok"]:
        oracle.batch_encoder(oracle.resolve(eng, case["k"], case["m"], case["symbol_len"]))
    else:
        with pytest.raises(ConfigError):
            oracle.resolve(eng, case["k"], case["m"], case["symbol_len"])


def test_unsupported_modes(oracle):  # selector.rs:587-603
    afft = oracle.resolve(Engine.AFFT, 8, 4, 64)
    with pytest.raises(ConfigError) as ei:
        oracle.incremental_encoder(afft)
    assert ei.value.variant == "UnsupportedMode" and ei.value.fields["engine"] == Engine.AFFT
    tower = oracle.resolve(Engine.TOWER, 32, 4, 64)
    with pytest.raises(ConfigError) as ei:
        oracle.batch_encoder(tower)
    assert ei.value.fields["engine"] == Engine.TOWER
    std = oracle.resolve(Engine.STANDARD_CAUCHY, 8, 4, 64)
    with pytest.raises(ConfigError):
        oracle.incremental_encoder(std)


def test_engine_capacities(oracle):  # selector.rs:24-32, tower/encoder.rs:190, afft/encoder.rs:284-288
    oracle.resolve(Engine.STANDARD_CAUCHY, 255, 1, 1)
    with pytest.raises(ConfigError):
        oracle.resolve(Engine.GOOD_CAUCHY, 255, 1, 1)
    oracle.resolve(Engine.TOWER, 256, 2, 64)
    with pytest.raises(ConfigError):
        oracle.resolve(Engine.TOWER, 32768, 32768, 2)
    oracle.resolve(Engine.AFFT, 32769, 1, 2)
    with pytest.raises(ConfigError) as ei:
        oracle.resolve(Engine.AFFT, 65535, 2, 2)
    assert ei.value.fields["cap"] == 65536
    with pytest.raises(ConfigError) as ei:
        oracle.resolve(Engine.AFFT, 1, 1, 3)
    assert ei.value.variant == "OddSymbolLen"
