"""B200 (sm_100a) erasure-coding engines with the SCRS trait surface.

The compute path is the CUDA library ``scrs_b200/_lib/libscrs_b200.so``
(hand-written sm_100a kernels behind the C ABI in include/scrs_gpu.h).  Import
fails loudly if that library has not been built; there is no CPU fallback.
"""
from pathlib import Path

from .api import (COMPLETE, DEPENDENT, Api, BatchDecoder, BatchEncoder, ConfigError, DecodeError,
                  Decoder, EncodeError, Engine, Field, IncrementalEncoder, Library, Profile,
                  PushOutcome, PushOutcomeKind, RuntimeFailure, ScrsError)

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libscrs_b200.so"

_default = None


def load_library() -> Library:
    if not LIB_PATH.exists():
        raise ImportError(
            f"CUDA library {LIB_PATH} is missing; build it with `python -m scrs_b200.build` "
            "(there is no CPU fallback)")
    return Library(LIB_PATH, prefix="scrs_", device=True)


def api_default() -> Api:
    global _default
    if _default is None:
        _default = Api(load_library())
    return _default


def resolve(engine, k, m, symbol_len) -> Profile:
    return api_default().resolve(engine, k, m, symbol_len)


def recommended(field, k, m, symbol_len) -> Profile:
    return api_default().recommended(field, k, m, symbol_len)


def batch_encoder(profile):
    return api_default().batch_encoder(profile)


def batch_decoder(profile):
    return api_default().batch_decoder(profile)


def incremental_encoder(profile):
    return api_default().incremental_encoder(profile)


def decoder(profile):
    return api_default().decoder(profile)
