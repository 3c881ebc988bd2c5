"""Serving loop over the CUDA engines (include/scrs_gpu.h scrs_server_*):
requests of every engine with device-resident buffers, admitted as slots and
device memory free up, GF(256) requests coalesced into stripe batches, work of
different slots overlapping on the device.  ``progress()`` never blocks."""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

from .api import Library, _Error, _stream_ptr, make_error

OP_ENCODE = 0
OP_DECODE = 1


class _Request(C.Structure):
    _fields_ = [("op", C.c_int32), ("engine", C.c_int32), ("k", C.c_uint64), ("m", C.c_uint64),
                ("symbol_len", C.c_uint64), ("in_", C.c_void_p), ("out", C.c_void_p),
                ("indices", C.POINTER(C.c_uint64)), ("tag", C.c_uint64), ("stream", C.c_void_p)]


class _Completion(C.Structure):
    _fields_ = [("ticket", C.c_uint64), ("tag", C.c_uint64), ("status", C.c_int32), ("reserved", C.c_int32),
                ("submit_ns", C.c_uint64), ("done_ns", C.c_uint64)]


class _Stats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("admitted", C.c_uint64), ("completed", C.c_uint64),
                ("failed", C.c_uint64), ("batches", C.c_uint64), ("memory_in_use", C.c_uint64),
                ("resident_bytes", C.c_uint64)]


_COMPLETION_DTYPE = np.dtype([("ticket", np.uint64), ("tag", np.uint64), ("status", np.int32),
                               ("reserved", np.int32), ("submit_ns", np.uint64), ("done_ns", np.uint64)])
assert _COMPLETION_DTYPE.itemsize == C.sizeof(_Completion)


@dataclass
class Prepared:
    """A request for ``Server.submit_prepared`` (keeps its index list alive)."""
    req: _Request
    indices: Optional[np.ndarray]


@dataclass
class Completion:
    ticket: int
    tag: int
    status: int
    submit_ns: int
    done_ns: int

    @property
    def latency_ms(self) -> float:
        return (self.done_ns - self.submit_ns) / 1e6


def _bind(lib: Library):
    L = lib.lib
    if getattr(lib, "_server_bound", False):
        return
    L.scrs_server_create.restype = C.c_int32
    L.scrs_server_create.argtypes = [C.c_uint64, C.c_uint32, C.POINTER(C.c_void_p), C.POINTER(_Error)]
    L.scrs_server_destroy.restype = None
    L.scrs_server_destroy.argtypes = [C.c_void_p]
    L.scrs_server_submit.restype = C.c_int32
    L.scrs_server_submit.argtypes = [C.c_void_p, C.POINTER(_Request), C.POINTER(C.c_uint64), C.POINTER(_Error)]
    L.scrs_server_progress.restype = C.c_int32
    L.scrs_server_progress.argtypes = [C.c_void_p, C.POINTER(_Completion), C.c_uint32, C.POINTER(C.c_uint32),
                                       C.POINTER(_Error)]
    L.scrs_server_pending.restype = C.c_uint64
    L.scrs_server_pending.argtypes = [C.c_void_p]
    L.scrs_server_reserve.restype = C.c_int32
    L.scrs_server_reserve.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_uint64, C.c_uint64, C.c_uint64,
                                      C.POINTER(_Error)]
    L.scrs_server_get_stats.restype = C.c_int32
    L.scrs_server_get_stats.argtypes = [C.c_void_p, C.POINTER(_Stats)]
    lib._server_bound = True


class Server:
    """scrs_server: ``submit`` device-resident requests, call ``progress`` to
    collect completions (or ``drain`` to wait for all)."""

    def __init__(self, lib: Library, memory_budget: int, slots: int = 8):
        _bind(lib)
        self._lib = lib
        self._ptr = C.c_void_p()
        err = _Error()
        lib.check(lib.lib.scrs_server_create(memory_budget, slots, C.byref(self._ptr), C.byref(err)), err)
        self._buf = (_Completion * 256)()
        self._keep = {}

    def close(self):
        ptr = getattr(self, "_ptr", None)
        if ptr is not None and ptr.value:
            self._ptr = None  # no module global needed here (finalizers can run at interpreter exit)
            self._lib.lib.scrs_server_destroy(ptr)
            self._keep.clear()

    def __del__(self):
        self.close()

    def submit(self, op: int, engine, k: int, m: int, symbol_len: int, in_ptr: int, out_ptr: int,
               indices: Optional[Sequence[int]] = None, tag: int = 0, stream=None) -> int:
        """Queue one request.  The input is read after the work enqueued
        before this call on `stream` (default: torch's current stream)."""
        r = _Request(op, int(engine), k, m, symbol_len, in_ptr, out_ptr, None, tag, _stream_ptr(stream))
        if indices is not None:
            # one conversion for the whole list (a uint64 array passes through
            # as is); the server copies the indices before returning
            arr = np.ascontiguousarray(indices, dtype=np.uint64)
            r.indices = arr.ctypes.data_as(C.POINTER(C.c_uint64))
        t = C.c_uint64()
        err = _Error()
        self._lib.check(self._lib.lib.scrs_server_submit(self._ptr, C.byref(r), C.byref(t), C.byref(err)), err)
        return t.value

    def prepare(self, op: int, engine, k: int, m: int, symbol_len: int, in_ptr: int, out_ptr: int,
                indices: Optional[Sequence[int]] = None, tag: int = 0, stream=None) -> "Prepared":
        """A request built once and submitted any number of times with
        ``submit_prepared`` (the same buffers each time): the per-submit host
        cost is one library call."""
        arr = None if indices is None else np.ascontiguousarray(indices, dtype=np.uint64)
        r = _Request(op, int(engine), k, m, symbol_len, in_ptr, out_ptr, None, tag, _stream_ptr(stream))
        if arr is not None:
            r.indices = arr.ctypes.data_as(C.POINTER(C.c_uint64))
        return Prepared(r, arr)

    def submit_prepared(self, p: "Prepared") -> int:
        t = C.c_uint64()
        err = _Error()
        self._lib.check(self._lib.lib.scrs_server_submit(self._ptr, C.byref(p.req), C.byref(t), C.byref(err)), err)
        return t.value

    def progress_arrays(self):
        """As ``progress``, the completions as numpy arrays (tag, status,
        submit_ns, done_ns) instead of one object each."""
        chunks = []
        while True:
            n = C.c_uint32()
            err = _Error()
            self._lib.check(self._lib.lib.scrs_server_progress(self._ptr, self._buf, len(self._buf), C.byref(n),
                                                               C.byref(err)), err)
            if n.value:
                chunks.append(np.frombuffer(self._buf, dtype=_COMPLETION_DTYPE, count=n.value).copy())
            if n.value < len(self._buf):
                break
        done = np.concatenate(chunks) if chunks else np.zeros(0, _COMPLETION_DTYPE)
        return done["tag"], done["status"], done["submit_ns"], done["done_ns"]

    def progress(self) -> List[Completion]:
        out = []
        while True:
            n = C.c_uint32()
            err = _Error()
            self._lib.check(self._lib.lib.scrs_server_progress(self._ptr, self._buf, len(self._buf), C.byref(n),
                                                               C.byref(err)), err)
            for i in range(n.value):
                c = self._buf[i]
                out.append(Completion(c.ticket, c.tag, c.status, c.submit_ns, c.done_ns))
            if n.value < len(self._buf):
                return out

    def reserve(self, op: int, engine, k: int, m: int, symbol_len: int):
        """Build one tower or additive-FFT profile's engines for `op` on every
        slot (start-up; the server must be idle)."""
        err = _Error()
        self._lib.check(self._lib.lib.scrs_server_reserve(self._ptr, op, int(engine), k, m, symbol_len,
                                                          C.byref(err)), err)

    @property
    def pending(self) -> int:
        return int(self._lib.lib.scrs_server_pending(self._ptr))

    def drain(self, timeout_s: float = 120.0) -> List[Completion]:
        out = []
        t_end = time.monotonic() + timeout_s
        while self.pending:
            out += self.progress()
            if time.monotonic() > t_end:
                raise TimeoutError(f"{self.pending} requests still pending")
        return out

    def stats(self) -> dict:
        s = _Stats()
        self._lib.lib.scrs_server_get_stats(self._ptr, C.byref(s))
        return {f: getattr(s, f) for f, _ in _Stats._fields_}


def raise_for(c: Completion):
    if c.status:
        raise make_error(c.status, 0, 0)
