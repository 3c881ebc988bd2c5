"""Autotuner of the persistent stripe-batch drain (include/scrs_gpu.h
scrs_tune_* and scrs_stripe_batch_autotune).

Two launch parameters are tuned per batch geometry: ``seg_rows`` (input rows
staged in shared memory per segment, 1..32) and ``ctas_per_sm`` (the
persistent grid, hence stripes per CTA).  ``StripeBatch.autotune`` times the
candidates on a batch's own stripes and stores the winner in the library's
process-wide table; every later run of a batch with the same geometry key uses
it.  ``save`` / ``load`` keep the table in a JSON file between processes."""
from __future__ import annotations

import ctypes as C
import json
from dataclasses import asdict, dataclass
from pathlib import Path
from typing import List, Tuple

from .api import Library, _Error

FORMAT = "scrs-b200-tune/1"


class _Key(C.Structure):
    _fields_ = [("field", C.c_uint32), ("k_bucket", C.c_uint32), ("m_bucket", C.c_uint32), ("l_bucket", C.c_uint32)]


class _Params(C.Structure):
    _fields_ = [("seg_rows", C.c_uint32), ("ctas_per_sm", C.c_uint32), ("drain_ms", C.c_float),
                ("reserved", C.c_uint32)]


@dataclass(frozen=True)
class TuneKey:
    field: int
    k_bucket: int
    m_bucket: int
    l_bucket: int


@dataclass(frozen=True)
class TuneParams:
    seg_rows: int
    ctas_per_sm: int
    drain_ms: float = 0.0


def _key(k: _Key) -> TuneKey:
    return TuneKey(k.field, k.k_bucket, k.m_bucket, k.l_bucket)


def _params(p: _Params) -> TuneParams:
    return TuneParams(p.seg_rows, p.ctas_per_sm, round(float(p.drain_ms), 6))


def bind(lib: Library):
    L = lib.lib
    if getattr(lib, "_tune_bound", False):
        return
    E = C.POINTER(_Error)
    L.scrs_tune_key_of.restype = C.c_int32
    L.scrs_tune_key_of.argtypes = [C.c_void_p, C.c_uint64, C.POINTER(_Key), E]
    L.scrs_stripe_batch_tune_key.restype = C.c_int32
    L.scrs_stripe_batch_tune_key.argtypes = [C.c_void_p, C.POINTER(_Key), E]
    L.scrs_stripe_batch_launch_params.restype = C.c_int32
    L.scrs_stripe_batch_launch_params.argtypes = [C.c_void_p, C.POINTER(_Params), E]
    L.scrs_stripe_batch_autotune.restype = C.c_int32
    L.scrs_stripe_batch_autotune.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.POINTER(_Params), E]
    L.scrs_tune_table_size.restype = C.c_uint64
    L.scrs_tune_table_size.argtypes = []
    L.scrs_tune_table_entry.restype = C.c_int32
    L.scrs_tune_table_entry.argtypes = [C.c_uint64, C.POINTER(_Key), C.POINTER(_Params), E]
    L.scrs_tune_table_set.restype = C.c_int32
    L.scrs_tune_table_set.argtypes = [C.POINTER(_Key), C.POINTER(_Params), E]
    L.scrs_tune_table_clear.restype = None
    L.scrs_tune_table_clear.argtypes = []
    lib._tune_bound = True


def key_of(lib: Library, desc_array) -> TuneKey:
    """Key of a descriptor array (``batch.DESC_DTYPE`` numpy records)."""
    bind(lib)
    k, err = _Key(), _Error()
    lib.check(lib.lib.scrs_tune_key_of(desc_array.ctypes.data, len(desc_array), C.byref(k), C.byref(err)), err)
    return _key(k)


def entries(lib: Library) -> List[Tuple[TuneKey, TuneParams]]:
    bind(lib)
    out = []
    for i in range(int(lib.lib.scrs_tune_table_size())):
        k, p, err = _Key(), _Params(), _Error()
        lib.check(lib.lib.scrs_tune_table_entry(i, C.byref(k), C.byref(p), C.byref(err)), err)
        out.append((_key(k), _params(p)))
    return out


def set_entry(lib: Library, key: TuneKey, params: TuneParams):
    bind(lib)
    k = _Key(key.field, key.k_bucket, key.m_bucket, key.l_bucket)
    p = _Params(params.seg_rows, params.ctas_per_sm, params.drain_ms, 0)
    err = _Error()
    lib.check(lib.lib.scrs_tune_table_set(C.byref(k), C.byref(p), C.byref(err)), err)


def clear(lib: Library):
    bind(lib)
    lib.lib.scrs_tune_table_clear()


def save(lib: Library, path) -> int:
    """Write the table as JSON; returns the number of entries."""
    ents = entries(lib)
    doc = {"format": FORMAT, "entries": [{"key": asdict(k), "params": asdict(p)} for k, p in ents]}
    Path(path).write_text(json.dumps(doc, indent=1, sort_keys=True))
    return len(ents)


def load(lib: Library, path) -> int:
    """Add the entries of a JSON file written by ``save`` to the table (the
    library validates each); returns the number loaded."""
    doc = json.loads(Path(path).read_text())
    if doc.get("format") != FORMAT:
        raise ValueError(f"not a {FORMAT} file: {path}")
    n = 0
    for e in doc["entries"]:
        set_entry(lib, TuneKey(**e["key"]), TuneParams(**e["params"]))
        n += 1
    return n
