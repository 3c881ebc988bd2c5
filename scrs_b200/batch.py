"""Batched GF(256) stripes in one persistent launch (include/scrs_gpu.h
scrs_stripe_batch_*): many independent encode / decode stripes of uneven
geometry, device-resident buffers, per-stripe decode matrices built on the
device, optional CUDA-graph replay, and the one-launch-per-stripe baseline."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional, Sequence

from .api import Engine, Library, _Error, make_error, _stream_ptr

OP_ENCODE = 0
OP_DECODE = 1


class _Desc(C.Structure):
    _fields_ = [("op", C.c_int32), ("engine", C.c_int32), ("k", C.c_uint32), ("m", C.c_uint32),
                ("symbol_len", C.c_uint64), ("in_", C.c_void_p), ("out", C.c_void_p),
                ("indices", C.POINTER(C.c_uint16))]


import numpy as _np

DESC_DTYPE = _np.dtype({"names": ["op", "engine", "k", "m", "symbol_len", "in_", "out", "indices"],
                        "formats": [_np.int32, _np.int32, _np.uint32, _np.uint32, _np.uint64, _np.uint64,
                                    _np.uint64, _np.uint64],
                        "offsets": [0, 4, 8, 12, 16, 24, 32, 40], "itemsize": 48})


@dataclass
class Stripe:
    """One stripe: device pointers (ints) for ``in_ptr`` / ``out_ptr``.

    encode: in = k*L data, out = m*L repairs.
    decode: in = k received rows (row q is codeword index ``indices[q]``),
            out = k*L data.
    """

    op: int
    engine: Engine
    k: int
    m: int
    symbol_len: int
    in_ptr: int
    out_ptr: int
    indices: Optional[Sequence[int]] = None


def _bind(lib: Library):
    L = lib.lib
    if getattr(lib, "_batch_bound", False):
        return
    L.scrs_stripe_batch_create.restype = C.c_int32
    L.scrs_stripe_batch_create.argtypes = [C.c_uint64, C.c_uint64, C.POINTER(C.c_void_p), C.POINTER(_Error)]
    L.scrs_stripe_batch_destroy.restype = None
    L.scrs_stripe_batch_destroy.argtypes = [C.c_void_p]
    L.scrs_stripe_batch_set.restype = C.c_int32
    L.scrs_stripe_batch_set.argtypes = [C.c_void_p, C.POINTER(_Desc), C.c_uint64, C.POINTER(_Error)]
    L.scrs_stripe_batch_set_host.restype = C.c_int32
    L.scrs_stripe_batch_set_host.argtypes = [C.c_void_p, C.POINTER(_Desc), C.c_uint64, C.POINTER(_Error)]
    L.scrs_stripe_batch_run.restype = C.c_int32
    L.scrs_stripe_batch_run.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.POINTER(_Error)]
    L.scrs_stripe_batch_run_plain.restype = C.c_int32
    L.scrs_stripe_batch_run_plain.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(_Error)]
    L.scrs_stripe_batch_last_launches.restype = C.c_uint64
    L.scrs_stripe_batch_last_launches.argtypes = [C.c_void_p]
    L.scrs_stripe_batch_run_timed.restype = C.c_int32
    L.scrs_stripe_batch_run_timed.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_float),
                                              C.POINTER(_Error)]
    L.scrs_stripe_batch_check.restype = C.c_int32
    L.scrs_stripe_batch_check.argtypes = [C.c_void_p, C.POINTER(_Error)]
    L.scrs_stripe_batch_run_timed_drains.restype = C.c_int32
    L.scrs_stripe_batch_run_timed_drains.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(C.c_float),
                                                     C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(_Error)]
    L.scrs_stripe_batch_set_jit.restype = C.c_int32
    L.scrs_stripe_batch_set_jit.argtypes = [C.c_void_p, C.c_int32, C.POINTER(_Error)]
    L.scrs_stripe_batch_jit_stripes.restype = C.c_uint64
    L.scrs_stripe_batch_jit_stripes.argtypes = [C.c_void_p]
    L.scrs_jit_prepare.restype = C.c_int32
    L.scrs_jit_prepare.argtypes = [C.c_int32, C.c_uint32, C.c_uint32, C.c_int32, C.POINTER(C.c_uint64),
                                   C.POINTER(_Error)]
    lib._batch_bound = True


def jit_prepare(lib: Library, engine, k: int, m: int, load: bool = True) -> int:
    """Compile (and with ``load`` load) the encode kernel specialised to the
    (engine, k, m) matrix ahead of its first batch; returns its cubin size."""
    _bind(lib)
    n, err = C.c_uint64(), _Error()
    lib.check(lib.lib.scrs_jit_prepare(int(engine), k, m, 1 if load else 0, C.byref(n), C.byref(err)), err)
    return n.value


class StripeBatch:
    def __init__(self, lib: Library, max_stripes: int, max_items: int = 0):
        _bind(lib)
        self._lib = lib
        self._ptr = C.c_void_p()
        err = _Error()
        lib.check(lib.lib.scrs_stripe_batch_create(max_stripes, max_items, C.byref(self._ptr), C.byref(err)), err)
        self._keep = []

    def __del__(self):
        if getattr(self, "_ptr", None) is not None and self._ptr.value:
            self._lib.lib.scrs_stripe_batch_destroy(self._ptr)
            self._ptr = None

    def set(self, stripes: Sequence[Stripe]):
        n = len(stripes)
        arr = (_Desc * max(n, 1))()
        keep = []
        for i, s in enumerate(stripes):
            idx = None
            if s.indices is not None:
                idx = (C.c_uint16 * len(s.indices))(*[int(x) for x in s.indices])
                keep.append(idx)
            arr[i] = _Desc(int(s.op), int(s.engine), s.k, s.m, s.symbol_len, s.in_ptr, s.out_ptr,
                           C.cast(idx, C.POINTER(C.c_uint16)) if idx is not None else None)
        err = _Error()
        self._lib.check(self._lib.lib.scrs_stripe_batch_set(self._ptr, arr, n, C.byref(err)), err)
        self._keep = keep

    def run(self, stream=None, graph: bool = False):
        err = _Error()
        self._lib.check(self._lib.lib.scrs_stripe_batch_run(self._ptr, _stream_ptr(stream), 1 if graph else 0,
                                                            C.byref(err)), err)

    def set_arrays(self, op, engine, k, m, symbol_len, in_ptr, out_ptr, indices=None, host=False):
        """Bulk form of set(): numpy arrays with one entry per stripe.  For
        decode stripes, ``indices`` is a uint16 array of shape (count, k_max)
        whose row s holds that stripe's k received codeword indices."""
        import numpy as np

        n = len(op)
        desc = np.zeros(n, dtype=DESC_DTYPE)
        desc["op"], desc["engine"], desc["k"], desc["m"] = op, engine, k, m
        desc["symbol_len"], desc["in_"], desc["out"] = symbol_len, in_ptr, out_ptr
        keep = [desc]
        if indices is not None:
            idx = np.ascontiguousarray(indices, dtype=np.uint16)
            keep.append(idx)
            row_bytes = idx.shape[1] * 2
            dec = np.asarray(op) == OP_DECODE
            desc["indices"] = np.where(dec, idx.ctypes.data + np.arange(n, dtype=np.uint64) * row_bytes, 0)
        err = _Error()
        ptr = C.cast(desc.ctypes.data, C.POINTER(_Desc))
        fn = self._lib.lib.scrs_stripe_batch_set_host if host else self._lib.lib.scrs_stripe_batch_set
        self._lib.check(fn(self._ptr, ptr, n, C.byref(err)), err)
        self._keep = keep

    def run_timed(self, stream=None):
        """(plan_ms, drain_ms) of one non-graph run, bracketed by CUDA events."""
        err, a, b = _Error(), C.c_float(), C.c_float()
        self._lib.check(self._lib.lib.scrs_stripe_batch_run_timed(self._ptr, _stream_ptr(stream), C.byref(a),
                                                                  C.byref(b), C.byref(err)), err)
        return a.value, b.value

    def run_timed_drains(self, stream=None):
        """(plan_ms, specialised_drains_ms, generic_drain_ms) of one non-graph run."""
        err, a, b, c = _Error(), C.c_float(), C.c_float(), C.c_float()
        self._lib.check(self._lib.lib.scrs_stripe_batch_run_timed_drains(self._ptr, _stream_ptr(stream), C.byref(a),
                                                                         C.byref(b), C.byref(c), C.byref(err)), err)
        return a.value, b.value, c.value

    def set_jit(self, enable: bool):
        """Specialise eligible encode stripes at the next set (default on)."""
        err = _Error()
        self._lib.check(self._lib.lib.scrs_stripe_batch_set_jit(self._ptr, 1 if enable else 0, C.byref(err)), err)

    @property
    def jit_stripes(self) -> int:
        """Stripes of the current descriptors that run through specialised kernels."""
        return int(self._lib.lib.scrs_stripe_batch_jit_stripes(self._ptr))

    def run_plain(self, stream=None):
        err = _Error()
        self._lib.check(self._lib.lib.scrs_stripe_batch_run_plain(self._ptr, _stream_ptr(stream), C.byref(err)), err)

    def check(self):
        err = _Error()
        self._lib.check(self._lib.lib.scrs_stripe_batch_check(self._ptr, C.byref(err)), err)

    @property
    def last_launches(self) -> int:
        return int(self._lib.lib.scrs_stripe_batch_last_launches(self._ptr))

    def autotune(self, reps: int = 5, stream=None):
        """Time the drain's launch candidates on this batch's stripes, store the
        fastest in the library's tuning table under the batch's geometry key
        and return it (``tune.TuneParams``)."""
        from . import tune

        tune.bind(self._lib)
        p, err = tune._Params(), _Error()
        self._lib.check(self._lib.lib.scrs_stripe_batch_autotune(self._ptr, _stream_ptr(stream), reps, C.byref(p),
                                                                 C.byref(err)), err)
        return tune._params(p)

    @property
    def launch_params(self):
        """The seg_rows / ctas_per_sm a run would use now (``tune.TuneParams``)."""
        from . import tune

        tune.bind(self._lib)
        p, err = tune._Params(), _Error()
        self._lib.check(self._lib.lib.scrs_stripe_batch_launch_params(self._ptr, C.byref(p), C.byref(err)), err)
        return tune._params(p)

    @property
    def tune_key(self):
        from . import tune

        tune.bind(self._lib)
        k, err = tune._Key(), _Error()
        self._lib.check(self._lib.lib.scrs_stripe_batch_tune_key(self._ptr, C.byref(k), C.byref(err)), err)
        return tune._key(k)
