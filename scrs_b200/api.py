"""Python mirror of the SCRS trait surface over the C ABI in include/scrs_gpu.h.

Names, argument meaning and error behaviour follow the reference crate:

* ``Profile.resolve`` / ``Profile.recommended``  (scrs/src/selector.rs:40,67)
* ``batch_encoder`` -> ``BatchEncoder``           (selector.rs:457, codec.rs:136)
* ``batch_decoder`` -> ``BatchDecoder``           (selector.rs:270, codec.rs:157)
* ``incremental_encoder`` -> ``IncrementalEncoder`` (selector.rs:370, codec.rs:122)
* ``decoder`` -> ``Decoder`` (+ SymbolSink)       (selector.rs:117, codec.rs:180)
* ``ConfigError`` / ``EncodeError`` / ``DecodeError`` (scrs/src/error.rs)

A ``Library`` binds one shared object that exports the ABI under a symbol
prefix.  The package binds the CUDA library (prefix ``scrs_``); nothing here
falls back to another implementation when that library is missing.
"""
from __future__ import annotations

import ctypes as C
import enum
from dataclasses import dataclass
from typing import Iterable, Sequence, Tuple

import numpy as np


class Engine(enum.IntEnum):
    """scrs/src/codec.rs:30-39"""

    STANDARD_CAUCHY = 0
    GOOD_CAUCHY = 1
    TOWER = 2
    AFFT = 3


class Field(enum.IntEnum):
    """scrs/src/codec.rs:20-25"""

    GF256 = 0
    GF65536 = 1


class PushOutcomeKind(enum.IntEnum):
    """scrs/src/transport/symbol_sink.rs:11-26"""

    ADVANCED = 0
    COMPLETE = 1
    DEPENDENT = 2


@dataclass(frozen=True)
class PushOutcome:
    kind: PushOutcomeKind
    rank: int = 0
    received: int = 0

    @staticmethod
    def advanced(rank: int, received: int) -> "PushOutcome":
        return PushOutcome(PushOutcomeKind.ADVANCED, rank, received)


COMPLETE = PushOutcome(PushOutcomeKind.COMPLETE)
DEPENDENT = PushOutcome(PushOutcomeKind.DEPENDENT)

# status code -> (exception class name, variant, detail field names)
_STATUS = {
    101: ("ConfigError", "ZeroDimension", ()),
    102: ("ConfigError", "TooManySymbols", ("cap",)),
    103: ("ConfigError", "ZeroSymbolLen", ()),
    104: ("ConfigError", "OddSymbolLen", ()),
    105: ("ConfigError", "UnsupportedMode", ("engine",)),
    201: ("EncodeError", "WrongInputLen", ("expected", "got")),
    202: ("EncodeError", "IndexOutOfRange", ("index", "n")),
    203: ("EncodeError", "WrongPayloadLen", ("expected", "got")),
    204: ("EncodeError", "DuplicateData", ("index",)),
    205: ("EncodeError", "WrongOutputLen", ("expected", "got")),
    206: ("EncodeError", "ScratchMismatch", ()),
    301: ("DecodeError", "WrongCount", ("expected", "got")),
    302: ("DecodeError", "IndexOutOfRange", ("index", "n")),
    303: ("DecodeError", "DuplicateIndex", ("index",)),
    304: ("DecodeError", "WrongPayloadLen", ("expected", "got")),
    305: ("DecodeError", "TooManySymbols", ("cap", "received")),
    306: ("DecodeError", "InsufficientRank", ("rank", "k")),
    307: ("DecodeError", "WrongOutputLen", ("expected", "got")),
    308: ("DecodeError", "ScratchMismatch", ()),
    901: ("RuntimeFailure", "NullArgument", ()),
    902: ("RuntimeFailure", "Cuda", ("cuda_error", "source_line")),
    903: ("RuntimeFailure", "OutOfMemory", ("bytes",)),
    904: ("RuntimeFailure", "NoDevice", ()),
    905: ("RuntimeFailure", "Capacity", ("requested", "limit")),
    906: ("RuntimeFailure", "DeviceTimeout", ()),
    907: ("RuntimeFailure", "BadArgument", ("position",)),
    908: ("RuntimeFailure", "Jit", ("nvrtc_result",)),
}


class ScrsError(Exception):
    """Base of the three reference error enums plus runtime failures."""

    def __init__(self, code: int, variant: str, fields: dict):
        self.code = code
        self.variant = variant
        self.fields = fields
        detail = ", ".join(f"{k}: {v}" for k, v in fields.items())
        super().__init__(f"{type(self).__name__}::{variant}" + (f" {{ {detail} }}" if detail else ""))

    def __eq__(self, other):
        return (type(self) is type(other) and self.variant == other.variant
                and self.fields == other.fields)

    def __hash__(self):
        return hash((type(self).__name__, self.variant, tuple(sorted(self.fields.items()))))


class ConfigError(ScrsError):
    pass


class EncodeError(ScrsError):
    pass


class DecodeError(ScrsError):
    pass


class RuntimeFailure(ScrsError):
    pass


_CLASSES = {c.__name__: c for c in (ConfigError, EncodeError, DecodeError, RuntimeFailure)}


def make_error(code: int, a: int = 0, b: int = 0) -> ScrsError:
    cls, variant, names = _STATUS.get(code, ("RuntimeFailure", f"Status{code}", ()))
    vals = (a, b)
    fields = {n: vals[i] for i, n in enumerate(names)}
    if variant == "UnsupportedMode":
        fields["engine"] = Engine(a)
    return _CLASSES[cls](code, variant, fields)


class _Profile(C.Structure):
    _fields_ = [("engine", C.c_int32), ("reserved", C.c_int32), ("k", C.c_uint64),
                ("m", C.c_uint64), ("symbol_len", C.c_uint64)]


class _Error(C.Structure):
    _fields_ = [("code", C.c_int32), ("reserved", C.c_int32), ("a", C.c_uint64), ("b", C.c_uint64)]


class _Push(C.Structure):
    _fields_ = [("kind", C.c_int32), ("reserved", C.c_int32), ("rank", C.c_uint64),
                ("received", C.c_uint64)]


_P = C.c_void_p
_U64 = C.c_uint64
_I32 = C.c_int32
_BUF = C.c_void_p

# (name, restype, argtypes) for the host-buffer ABI shared by every binding.
_SIGNATURES = [
    ("abi_version", C.c_uint32, []),
    ("profile_resolve", _I32, [_I32, _U64, _U64, _U64, C.POINTER(_Profile), C.POINTER(_Error)]),
    ("profile_recommended", _I32, [_I32, _U64, _U64, _U64, C.POINTER(_Profile), C.POINTER(_Error)]),
    ("recommended_gf16_engine", _I32, [_U64, _U64]),
    ("batch_encoder_create", _I32, [C.POINTER(_Profile), C.POINTER(_P), C.POINTER(_Error)]),
    ("batch_encoder_destroy", None, [_P]),
    ("batch_encoder_scratch", _I32, [_P, C.POINTER(_P), C.POINTER(_Error)]),
    ("encode_scratch_destroy", None, [_P]),
    ("batch_encode_into", _I32, [_P, _BUF, _U64, _BUF, _U64, C.POINTER(_Error)]),
    ("batch_encode_into_with", _I32, [_P, _BUF, _U64, _BUF, _U64, _P, C.POINTER(_Error)]),
    ("batch_decoder_create", _I32, [C.POINTER(_Profile), C.POINTER(_P), C.POINTER(_Error)]),
    ("batch_decoder_destroy", None, [_P]),
    ("batch_decoder_scratch", _I32, [_P, C.POINTER(_P), C.POINTER(_Error)]),
    ("batch_decode_scratch_destroy", None, [_P]),
    ("batch_decode_into_with", _I32, [_P, C.POINTER(C.c_uint64), C.POINTER(C.c_void_p),
                                      C.POINTER(C.c_uint64), _U64, _BUF, _U64, _P, C.POINTER(_Error)]),
    ("batch_decode_into", _I32, [_P, C.POINTER(C.c_uint64), C.POINTER(C.c_void_p),
                                 C.POINTER(C.c_uint64), _U64, _BUF, _U64, C.POINTER(_Error)]),
    ("incremental_encoder_create", _I32, [C.POINTER(_Profile), C.POINTER(_P), C.POINTER(_Error)]),
    ("incremental_encoder_destroy", None, [_P]),
    ("inc_feed", _I32, [_P, _U64, _BUF, _U64, C.POINTER(_Error)]),
    ("inc_repair", _I32, [_P, _U64, _BUF, _U64, C.POINTER(_Error)]),
    ("inc_fed_count", _U64, [_P]),
    ("inc_reset", None, [_P]),
    ("decoder_create", _I32, [C.POINTER(_Profile), C.POINTER(_P), C.POINTER(_Error)]),
    ("decoder_destroy", None, [_P]),
    ("decoder_scratch", _I32, [_P, C.POINTER(_P), C.POINTER(_Error)]),
    ("decode_scratch_destroy", None, [_P]),
    ("dec_push", _I32, [_P, _U64, _BUF, _U64, C.POINTER(_Push), C.POINTER(_Error)]),
    ("dec_is_complete", _I32, [_P]),
    ("dec_rank", _U64, [_P]),
    ("dec_received", _U64, [_P]),
    ("dec_reset", None, [_P]),
    ("dec_finalize_into", _I32, [_P, _BUF, _U64, C.POINTER(_Error)]),
    ("dec_finalize_into_with", _I32, [_P, _BUF, _U64, _P, C.POINTER(_Error)]),
]

# Device-pointer forms exported only by the CUDA library.
_DEVICE_SIGNATURES = [
    ("batch_encode_into_with_device", _I32, [_P, _BUF, _U64, _BUF, _U64, _P, _P, C.POINTER(_Error)]),
    ("batch_decode_into_with_device", _I32, [_P, C.POINTER(C.c_uint64), _BUF, _U64, _BUF, _U64, _P, _P,
                                             C.POINTER(_Error)]),
    ("inc_feed_device", _I32, [_P, _U64, _BUF, _U64, C.POINTER(_Error)]),
    ("inc_feed_device_stream", _I32, [_P, _U64, _BUF, _U64, _P, C.POINTER(_Error)]),
    ("inc_repair_device", _I32, [_P, _U64, C.POINTER(C.c_void_p), C.POINTER(_Error)]),
    ("dec_push_device", _I32, [_P, _U64, _BUF, _U64, C.POINTER(_Push), C.POINTER(_Error)]),
    ("dec_push_device_stream", _I32, [_P, _U64, _BUF, _U64, _P, C.POINTER(_Push), C.POINTER(_Error)]),
    ("dec_finalize_into_with_device", _I32, [_P, _BUF, _U64, _P, _P, C.POINTER(_Error)]),
    ("status_name", C.c_char_p, [_I32]),
    ("alloc_count", _U64, []),
    ("batch_decode_scratch_recipe_hits", _U64, [_P]),
    ("decode_scratch_recipe_hits", _U64, [_P]),
]


class Library:
    """One loaded implementation of the ABI (CUDA library or a test checker)."""

    def __init__(self, path: str, prefix: str = "scrs_", device: bool = True):
        self.path = str(path)
        self.prefix = prefix
        self.lib = C.CDLL(self.path)
        self.device = device
        for name, res, args in _SIGNATURES + (_DEVICE_SIGNATURES if device else []):
            fn = getattr(self.lib, prefix + name)
            fn.restype = res
            fn.argtypes = args
            setattr(self, name, fn)

    def check(self, status: int, err: _Error):
        if status != 0:
            raise make_error(err.code or status, err.a, err.b)


# ---------------------------------------------------------------------------
# buffer helpers
# ---------------------------------------------------------------------------

def _is_cuda_tensor(x) -> bool:
    return getattr(x, "is_cuda", False) is True


def _host_view(x, writable=False) -> Tuple[int, int, object]:
    """(address, length, keepalive) of a host byte buffer."""
    if isinstance(x, np.ndarray):
        a = x
        if a.dtype != np.uint8:
            a = a.view(np.uint8)
        if not a.flags["C_CONTIGUOUS"]:
            if writable:
                raise ValueError("output buffer must be contiguous")
            a = np.ascontiguousarray(a)
        return a.ctypes.data, a.nbytes, a
    if isinstance(x, bytearray):
        n = len(x)
        if n == 0:
            return 0, 0, x
        buf = (C.c_char * n).from_buffer(x)
        return C.addressof(buf), n, buf
    if isinstance(x, (bytes, memoryview)):
        if writable:
            raise ValueError("output buffer must be writable")
        a = np.frombuffer(bytes(x), dtype=np.uint8)
        return (a.ctypes.data if a.size else 0), a.nbytes, a
    if hasattr(x, "data_ptr") and hasattr(x, "numel"):  # CPU torch tensor
        return x.data_ptr(), x.numel() * x.element_size(), x
    raise TypeError(f"unsupported buffer type {type(x)!r}")


def _device_view(x) -> Tuple[int, int]:
    if not x.is_contiguous():
        raise ValueError("device buffer must be contiguous")
    return x.data_ptr(), x.numel() * x.element_size()


_raw_stream = None


def _tensor_stream(t) -> int:
    """Raw handle of the current CUDA stream of tensor t's device (the stream
    torch orders t's producers on)."""
    global _raw_stream
    if _raw_stream is None:
        import torch

        get = getattr(torch._C, "_cuda_getCurrentRawStream", None)
        _raw_stream = get if get is not None else (lambda dev: torch.cuda.current_stream(dev).cuda_stream)
    return _raw_stream(t.get_device())


def _stream_ptr(stream) -> int:
    """Raw handle of `stream` (a torch stream or an int); None: torch's current
    stream of the current device (0, the legacy default stream, without torch)."""
    if stream is None:
        try:
            import torch

            get = getattr(torch._C, "_cuda_getCurrentRawStream", None)
            if get is not None:
                return get(torch.cuda.current_device())
            return torch.cuda.current_stream().cuda_stream
        except Exception:  # pragma: no cover
            return 0
    return getattr(stream, "cuda_stream", stream)


# ---------------------------------------------------------------------------
# Profile and codecs
# ---------------------------------------------------------------------------

class Profile:
    """A validated codec geometry (scrs/src/codec.rs:53-103)."""

    __slots__ = ("engine", "k", "m", "symbol_len")

    def __init__(self, engine: Engine, k: int, m: int, symbol_len: int):
        self.engine = Engine(engine)
        self.k = int(k)
        self.m = int(m)
        self.symbol_len = int(symbol_len)

    @property
    def n(self) -> int:
        return self.k + self.m

    @property
    def field(self) -> Field:
        return Field.GF256 if self.engine in (Engine.STANDARD_CAUCHY, Engine.GOOD_CAUCHY) else Field.GF65536

    def _c(self) -> _Profile:
        return _Profile(int(self.engine), 0, self.k, self.m, self.symbol_len)

    def __eq__(self, other):
        return isinstance(other, Profile) and (self.engine, self.k, self.m, self.symbol_len) == (
            other.engine, other.k, other.m, other.symbol_len)

    def __repr__(self):
        return f"Profile({self.engine.name}, k={self.k}, m={self.m}, symbol_len={self.symbol_len})"


class _Handle:
    _destroy = ""

    def __init__(self, lib: Library, ptr: C.c_void_p, profile: Profile):
        self._lib = lib
        self._ptr = ptr
        self.profile = profile

    def __del__(self):
        ptr = getattr(self, "_ptr", None)
        if ptr is not None and ptr.value:
            getattr(self._lib, self._destroy)(ptr)
            self._ptr = None

    close = __del__

    @property
    def k(self):
        return self.profile.k

    @property
    def m(self):
        return self.profile.m

    @property
    def n(self):
        return self.profile.n

    @property
    def symbol_len(self):
        return self.profile.symbol_len


class EncodeScratch(_Handle):
    _destroy = "encode_scratch_destroy"


class BatchDecodeScratch(_Handle):
    _destroy = "batch_decode_scratch_destroy"

    @property
    def recipe_hits(self) -> int:
        """Decodes whose erasure pattern was found in the device recipe cache."""
        return int(self._lib.batch_decode_scratch_recipe_hits(self._ptr))


class DecodeScratch(_Handle):
    _destroy = "decode_scratch_destroy"

    @property
    def recipe_hits(self) -> int:
        """Finalizes whose erasure pattern was found in the device recipe cache."""
        return int(self._lib.decode_scratch_recipe_hits(self._ptr))


class BatchEncoder(_Handle):
    """Block-final encoder (scrs/src/codec.rs:136-151)."""

    _destroy = "batch_encoder_destroy"

    def scratch(self) -> EncodeScratch:
        out, err = C.c_void_p(), _Error()
        self._lib.check(self._lib.batch_encoder_scratch(self._ptr, C.byref(out), C.byref(err)), err)
        return EncodeScratch(self._lib, out, self.profile)

    def encode_into(self, data, repairs):
        self._encode(data, repairs, None)

    def encode_into_with(self, data, repairs, scratch: EncodeScratch, stream=None):
        self._encode(data, repairs, scratch, stream)

    def _encode(self, data, repairs, scratch, stream=None):
        err = _Error()
        if _is_cuda_tensor(data) or _is_cuda_tensor(repairs):
            if scratch is None:
                scratch = self.scratch()
            dp, dl = _device_view(data)
            rp, rl = _device_view(repairs)
            st = self._lib.batch_encode_into_with_device(self._ptr, dp, dl, rp, rl, scratch._ptr,
                                                         _stream_ptr(stream), C.byref(err))
            self._lib.check(st, err)
            return
        dp, dl, keep1 = _host_view(data)
        rp, rl, keep2 = _host_view(repairs, writable=True)
        if scratch is None:
            st = self._lib.batch_encode_into(self._ptr, dp, dl, rp, rl, C.byref(err))
        else:
            st = self._lib.batch_encode_into_with(self._ptr, dp, dl, rp, rl, scratch._ptr, C.byref(err))
        self._lib.check(st, err)

    def encode(self, data) -> list:
        """Return the m repair symbols as bytes objects."""
        out = np.zeros(self.m * self.symbol_len, dtype=np.uint8)
        self.encode_into(data, out)
        L = self.symbol_len
        return [out[j * L:(j + 1) * L].tobytes() for j in range(self.m)]


def _symbol_arrays(symbols: Sequence[Tuple[int, object]]):
    n = len(symbols)
    idx = (C.c_uint64 * max(n, 1))()
    ptrs = (C.c_void_p * max(n, 1))()
    lens = (C.c_uint64 * max(n, 1))()
    keep = []
    for i, (index, payload) in enumerate(symbols):
        p, ln, k = _host_view(payload)
        idx[i] = int(index)
        ptrs[i] = p
        lens[i] = ln
        keep.append(k)
    return n, idx, ptrs, lens, keep


class BatchDecoder(_Handle):
    """Block-final decoder (scrs/src/codec.rs:157-175)."""

    _destroy = "batch_decoder_destroy"

    def scratch(self) -> BatchDecodeScratch:
        out, err = C.c_void_p(), _Error()
        self._lib.check(self._lib.batch_decoder_scratch(self._ptr, C.byref(out), C.byref(err)), err)
        return BatchDecodeScratch(self._lib, out, self.profile)

    def decode_into(self, symbols, out):
        self.decode_into_with(symbols, out, None)

    def decode_into_with(self, symbols, out, scratch, stream=None):
        err = _Error()
        if _is_cuda_tensor(out):
            # device form: `symbols` is (indices, payload_rows) with payload_rows a
            # CUDA tensor of count*symbol_len bytes.
            indices, rows = symbols
            if scratch is None:
                scratch = self.scratch()
            ia = np.ascontiguousarray(np.asarray(indices, dtype=np.uint64).reshape(-1))
            n = int(ia.size)
            if n == 0:
                ia = np.zeros(1, np.uint64)
            idx = ia.ctypes.data_as(C.POINTER(C.c_uint64))
            rp, _ = _device_view(rows)
            op, ol = _device_view(out)
            st = self._lib.batch_decode_into_with_device(self._ptr, idx, rp, n, op, ol, scratch._ptr,
                                                         _stream_ptr(stream), C.byref(err))
            self._lib.check(st, err)
            return
        n, idx, ptrs, lens, keep = _symbol_arrays(symbols)
        op, ol, keep_out = _host_view(out, writable=True)
        if scratch is None:
            st = self._lib.batch_decode_into(self._ptr, idx, ptrs, lens, n, op, ol, C.byref(err))
        else:
            st = self._lib.batch_decode_into_with(self._ptr, idx, ptrs, lens, n, op, ol, scratch._ptr,
                                                  C.byref(err))
        self._lib.check(st, err)

    def decode(self, symbols) -> bytes:
        out = np.zeros(self.k * self.symbol_len, dtype=np.uint8)
        self.decode_into(symbols, out)
        return out.tobytes()


class IncrementalEncoder(_Handle):
    """Streaming encoder (scrs/src/codec.rs:122-131)."""

    _destroy = "incremental_encoder_destroy"

    def feed(self, index: int, data, stream=None):
        """Feed data symbol `index`.  A CUDA tensor is copied on `stream`
        (default: the current stream of its device)."""
        if _is_cuda_tensor(data):
            # per-symbol hot path: one error struct per handle, no temporaries
            if data.is_contiguous():
                errs = self.__dict__.get("_errs")
                if errs is None:
                    e = _Error()
                    errs = self._errs = (e, C.byref(e))
                sp = _tensor_stream(data) if stream is None else _stream_ptr(stream)
                st = self._lib.inc_feed_device_stream(self._ptr, index, data.data_ptr(), data.nbytes, sp, errs[1])
                if st:
                    self._lib.check(st, errs[0])
                return
            raise ValueError("device buffer must be contiguous")
        err = _Error()
        p, ln, keep = _host_view(data)
        self._lib.check(self._lib.inc_feed(self._ptr, index, p, ln, C.byref(err)), err)

    def repair(self, index: int) -> bytes:
        err = _Error()
        out = np.zeros(self.symbol_len, dtype=np.uint8)
        self._lib.check(self._lib.inc_repair(self._ptr, index, out.ctypes.data, out.nbytes, C.byref(err)), err)
        return out.tobytes()

    def repair_device_ptr(self, index: int) -> int:
        err, ptr = _Error(), C.c_void_p()
        self._lib.check(self._lib.inc_repair_device(self._ptr, index, C.byref(ptr), C.byref(err)), err)
        return ptr.value

    def fed_count(self) -> int:
        return int(self._lib.inc_fed_count(self._ptr))

    def reset(self):
        self._lib.inc_reset(self._ptr)


class Decoder(_Handle):
    """Lazy streaming decoder (scrs/src/codec.rs:180-201 + SymbolSink)."""

    _destroy = "decoder_destroy"

    def scratch(self) -> DecodeScratch:
        out, err = C.c_void_p(), _Error()
        self._lib.check(self._lib.decoder_scratch(self._ptr, C.byref(out), C.byref(err)), err)
        return DecodeScratch(self._lib, out, self.profile)

    def push(self, index: int, payload, stream=None) -> PushOutcome:
        """Push symbol `index`.  A CUDA tensor is copied on `stream` (default:
        the current stream of its device)."""
        if _is_cuda_tensor(payload):
            # per-symbol hot path: one outcome and error struct per handle
            if not payload.is_contiguous():
                raise ValueError("device buffer must be contiguous")
            bufs = self.__dict__.get("_push_bufs")
            if bufs is None:
                o, e = _Push(), _Error()
                bufs = self._push_bufs = (o, e, C.byref(o), C.byref(e))
            o, err = bufs[0], bufs[1]
            sp = _tensor_stream(payload) if stream is None else _stream_ptr(stream)
            st = self._lib.dec_push_device_stream(self._ptr, index, payload.data_ptr(), payload.nbytes, sp, bufs[2],
                                                  bufs[3])
        else:
            err, o = _Error(), _Push()
            p, ln, keep = _host_view(payload)
            st = self._lib.dec_push(self._ptr, index, p, ln, C.byref(o), C.byref(err))
        if st:
            self._lib.check(st, err)
        kind = PushOutcomeKind(o.kind)
        if kind == PushOutcomeKind.ADVANCED:
            return PushOutcome.advanced(int(o.rank), int(o.received))
        return COMPLETE if kind == PushOutcomeKind.COMPLETE else DEPENDENT

    def is_complete(self) -> bool:
        return bool(self._lib.dec_is_complete(self._ptr))

    def rank(self) -> int:
        return int(self._lib.dec_rank(self._ptr))

    def received(self) -> int:
        return int(self._lib.dec_received(self._ptr))

    def reset(self):
        self._lib.dec_reset(self._ptr)

    def finalize_into(self, out):
        err = _Error()
        p, ln, keep = _host_view(out, writable=True)
        self._lib.check(self._lib.dec_finalize_into(self._ptr, p, ln, C.byref(err)), err)

    def finalize_into_with(self, out, scratch: DecodeScratch, stream=None):
        err = _Error()
        if _is_cuda_tensor(out):
            p, ln = _device_view(out)
            st = self._lib.dec_finalize_into_with_device(self._ptr, p, ln, scratch._ptr, _stream_ptr(stream),
                                                         C.byref(err))
        else:
            p, ln, keep = _host_view(out, writable=True)
            st = self._lib.dec_finalize_into_with(self._ptr, p, ln, scratch._ptr, C.byref(err))
        self._lib.check(st, err)

    def finalize(self) -> bytes:
        out = np.zeros(self.k * self.symbol_len, dtype=np.uint8)
        self.finalize_into(out)
        return out.tobytes()


class Api:
    """The trait-surface factories bound to one Library."""

    def __init__(self, lib: Library):
        self.lib = lib

    def resolve(self, engine, k, m, symbol_len) -> Profile:
        out, err = _Profile(), _Error()
        self.lib.check(self.lib.profile_resolve(int(engine), k, m, symbol_len, C.byref(out), C.byref(err)), err)
        return Profile(Engine(out.engine), out.k, out.m, out.symbol_len)

    def recommended(self, field, k, m, symbol_len) -> Profile:
        out, err = _Profile(), _Error()
        self.lib.check(self.lib.profile_recommended(int(field), k, m, symbol_len, C.byref(out), C.byref(err)),
                       err)
        return Profile(Engine(out.engine), out.k, out.m, out.symbol_len)

    def recommended_gf16_engine(self, k, m) -> Engine:
        return Engine(self.lib.recommended_gf16_engine(k, m))

    def _create(self, fn, cls, profile: Profile):
        out, err = C.c_void_p(), _Error()
        p = profile._c()
        self.lib.check(getattr(self.lib, fn)(C.byref(p), C.byref(out), C.byref(err)), err)
        return cls(self.lib, out, profile)

    def batch_encoder(self, profile: Profile) -> BatchEncoder:
        return self._create("batch_encoder_create", BatchEncoder, profile)

    def batch_decoder(self, profile: Profile) -> BatchDecoder:
        return self._create("batch_decoder_create", BatchDecoder, profile)

    def incremental_encoder(self, profile: Profile) -> IncrementalEncoder:
        return self._create("incremental_encoder_create", IncrementalEncoder, profile)

    def decoder(self, profile: Profile) -> Decoder:
        return self._create("decoder_create", Decoder, profile)
