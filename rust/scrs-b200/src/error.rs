//! Status codes of the C ABI (`include/scrs_gpu.h`) mapped onto the SCRS
//! error enums (`scrs/src/error.rs:12-126`).
//!
//! Every code the library returns maps to exactly one [`Failure`] variant:
//! the `1xx` codes to a [`ConfigError`] variant, `2xx` to an
//! [`EncodeError`] variant, `3xx` to a [`DecodeError`] variant, and the
//! `9xx` runtime codes (CUDA failures, device limits, timeouts: failures a
//! CPU library cannot meet) to [`RuntimeFailure`].  The detail fields come
//! from the `scrs_error` out-struct in the order the header documents.

use core::fmt;

use scrs::{ConfigError, DecodeError, EncodeError, Engine};
use scrs_b200_sys as sys;

/// A failure the GPU library reported that has no variant in the reference's
/// error enums: the raw status code and its two detail words.
#[derive(Debug, Clone, Copy, PartialEq, Eq)]
pub struct RuntimeFailure {
    /// `SCRS_ERR_*` code.
    pub code: i32,
    /// First detail word (`scrs_error::a`).
    pub a: u64,
    /// Second detail word (`scrs_error::b`).
    pub b: u64,
}

impl RuntimeFailure {
    /// The header's name of the code.
    pub fn name(&self) -> &'static str {
        match self.code {
            sys::SCRS_ERR_NULL_ARGUMENT => "NullArgument",
            sys::SCRS_ERR_CUDA => "Cuda",
            sys::SCRS_ERR_OUT_OF_MEMORY => "OutOfMemory",
            sys::SCRS_ERR_NO_DEVICE => "NoDevice",
            sys::SCRS_ERR_CAPACITY => "Capacity",
            sys::SCRS_ERR_DEVICE_TIMEOUT => "DeviceTimeout",
            sys::SCRS_ERR_BAD_ARGUMENT => "BadArgument",
            sys::SCRS_ERR_JIT => "Jit",
            _ => "Unknown",
        }
    }
}

impl fmt::Display for RuntimeFailure {
    fn fmt(&self, f: &mut fmt::Formatter<'_>) -> fmt::Result {
        write!(f, "scrs-b200 runtime failure {} ({}), details {} / {}", self.name(), self.code, self.a, self.b)
    }
}

/// Any status the library can return other than `SCRS_OK`.
#[derive(Debug, Clone, PartialEq, Eq)]
pub enum Failure {
    Config(ConfigError),
    Encode(EncodeError),
    Decode(DecodeError),
    Runtime(RuntimeFailure),
}

fn engine_of(raw: u64) -> Engine {
    match raw as i32 {
        sys::SCRS_ENGINE_STANDARD_CAUCHY => Engine::StandardCauchy,
        sys::SCRS_ENGINE_GOOD_CAUCHY => Engine::GoodCauchy,
        sys::SCRS_ENGINE_TOWER => Engine::Tower,
        _ => Engine::Afft,
    }
}

/// The engine's code on the C ABI.
pub fn engine_code(engine: Engine) -> i32 {
    match engine {
        Engine::StandardCauchy => sys::SCRS_ENGINE_STANDARD_CAUCHY,
        Engine::GoodCauchy => sys::SCRS_ENGINE_GOOD_CAUCHY,
        Engine::Tower => sys::SCRS_ENGINE_TOWER,
        Engine::Afft => sys::SCRS_ENGINE_AFFT,
    }
}

/// Map a returned status and its detail struct onto the reference's errors.
/// `rc` wins over `err.code` (the struct is only filled when it was passed).
pub fn check(rc: i32, err: &sys::scrs_error) -> Result<(), Failure> {
    let (a, b) = (err.a as usize, err.b as usize);
    let f = match rc {
        sys::SCRS_OK => return Ok(()),
        sys::SCRS_CONFIG_ZERO_DIMENSION => Failure::Config(ConfigError::ZeroDimension),
        sys::SCRS_CONFIG_TOO_MANY_SYMBOLS => Failure::Config(ConfigError::TooManySymbols { cap: a }),
        sys::SCRS_CONFIG_ZERO_SYMBOL_LEN => Failure::Config(ConfigError::ZeroSymbolLen),
        sys::SCRS_CONFIG_ODD_SYMBOL_LEN => Failure::Config(ConfigError::OddSymbolLen),
        sys::SCRS_CONFIG_UNSUPPORTED_MODE => Failure::Config(ConfigError::UnsupportedMode { engine: engine_of(err.a) }),
        sys::SCRS_ENCODE_WRONG_INPUT_LEN => Failure::Encode(EncodeError::WrongInputLen { expected: a, got: b }),
        sys::SCRS_ENCODE_INDEX_OUT_OF_RANGE => Failure::Encode(EncodeError::IndexOutOfRange { index: a, n: b }),
        sys::SCRS_ENCODE_WRONG_PAYLOAD_LEN => Failure::Encode(EncodeError::WrongPayloadLen { expected: a, got: b }),
        sys::SCRS_ENCODE_DUPLICATE_DATA => Failure::Encode(EncodeError::DuplicateData { index: a }),
        sys::SCRS_ENCODE_WRONG_OUTPUT_LEN => Failure::Encode(EncodeError::WrongOutputLen { expected: a, got: b }),
        sys::SCRS_ENCODE_SCRATCH_MISMATCH => Failure::Encode(EncodeError::ScratchMismatch),
        sys::SCRS_DECODE_WRONG_COUNT => Failure::Decode(DecodeError::WrongCount { expected: a, got: b }),
        sys::SCRS_DECODE_INDEX_OUT_OF_RANGE => Failure::Decode(DecodeError::IndexOutOfRange { index: a, n: b }),
        sys::SCRS_DECODE_DUPLICATE_INDEX => Failure::Decode(DecodeError::DuplicateIndex { index: a }),
        sys::SCRS_DECODE_WRONG_PAYLOAD_LEN => Failure::Decode(DecodeError::WrongPayloadLen { expected: a, got: b }),
        sys::SCRS_DECODE_TOO_MANY_SYMBOLS => Failure::Decode(DecodeError::TooManySymbols { cap: a, received: b }),
        sys::SCRS_DECODE_INSUFFICIENT_RANK => Failure::Decode(DecodeError::InsufficientRank { rank: a, k: b }),
        sys::SCRS_DECODE_WRONG_OUTPUT_LEN => Failure::Decode(DecodeError::WrongOutputLen { expected: a, got: b }),
        sys::SCRS_DECODE_SCRATCH_MISMATCH => Failure::Decode(DecodeError::ScratchMismatch),
        sys::SCRS_ERR_NULL_ARGUMENT
        | sys::SCRS_ERR_CUDA
        | sys::SCRS_ERR_OUT_OF_MEMORY
        | sys::SCRS_ERR_NO_DEVICE
        | sys::SCRS_ERR_CAPACITY
        | sys::SCRS_ERR_DEVICE_TIMEOUT
        | sys::SCRS_ERR_BAD_ARGUMENT
        | sys::SCRS_ERR_JIT => Failure::Runtime(RuntimeFailure { code: rc, a: err.a, b: err.b }),
        other => Failure::Runtime(RuntimeFailure { code: other, a: err.a, b: err.b }),
    };
    Err(f)
}

// The trait methods return the reference's error types, which have no room
// for a GPU runtime failure; such a failure (or a code of the wrong family,
// which would be a library bug) panics with its description, as an
// allocation failure aborts a CPU engine.

pub(crate) fn config(rc: i32, err: &sys::scrs_error) -> Result<(), ConfigError> {
    check(rc, err).map_err(|f| match f {
        Failure::Config(e) => e,
        other => panic!("scrs-b200: {other:?}"),
    })
}

pub(crate) fn encode(rc: i32, err: &sys::scrs_error) -> Result<(), EncodeError> {
    check(rc, err).map_err(|f| match f {
        Failure::Encode(e) => e,
        other => panic!("scrs-b200: {other:?}"),
    })
}

pub(crate) fn decode(rc: i32, err: &sys::scrs_error) -> Result<(), DecodeError> {
    check(rc, err).map_err(|f| match f {
        Failure::Decode(e) => e,
        other => panic!("scrs-b200: {other:?}"),
    })
}

pub(crate) fn runtime(rc: i32, err: &sys::scrs_error) {
    if let Err(f) = check(rc, err) {
        panic!("scrs-b200: {f:?}");
    }
}
