//! The B200 erasure-coding engines behind the SCRS trait family, so that a
//! Rust caller drops them in beside the CPU engines: the factories below
//! mirror `scrs::{batch_encoder, batch_decoder, incremental_encoder,
//! decoder}` (scrs/src/selector.rs:117, 270, 370, 457) and return types that
//! implement `scrs::BatchEncoder`, `scrs::BatchDecoder`,
//! `scrs::IncrementalEncoder` and `scrs::Decoder + scrs::stream::SymbolSink`
//! (scrs/src/codec.rs:106-239, scrs/src/transport/symbol_sink.rs:36-54) over
//! the C ABI of `include/scrs_gpu.h` (raw declarations: `scrs-b200-sys`).
//!
//! Buffers are host slices, as in the reference: each call copies through the
//! library's pinned staging, runs the sm_100a kernels and copies the result
//! back before it returns.  Errors come back as the reference's own enums
//! (see [`error`]); a GPU runtime failure, which those enums cannot express,
//! panics with its description.  Handles are `Send` but not `Sync`, as the
//! reference engines are `&mut`-exclusive.

pub mod error;

use core::cell::{Cell, UnsafeCell};
use core::ptr;

use scrs::stream::{PushOutcome, SymbolSink};
use scrs::{BatchDecoder, BatchEncoder, Coded, ConfigError, DecodeError, Decoder, EncodeError, Engine,
           IncrementalEncoder, Profile};
use scrs_b200_sys as sys;

pub use error::{check, engine_code, Failure, RuntimeFailure};

fn no_error() -> sys::scrs_error {
    sys::scrs_error { code: 0, reserved: 0, a: 0, b: 0 }
}

fn raw_profile(p: &Profile) -> sys::scrs_profile {
    sys::scrs_profile {
        engine: engine_code(p.engine()),
        reserved: 0,
        k: p.k() as u64,
        m: p.m() as u64,
        symbol_len: p.symbol_len() as u64,
    }
}

macro_rules! coded_from_profile {
    ($t:ty) => {
        impl Coded for $t {
            fn k(&self) -> usize {
                self.profile.k()
            }
            fn m(&self) -> usize {
                self.profile.m()
            }
            fn symbol_len(&self) -> usize {
                self.profile.symbol_len()
            }
        }
    };
}

// ---------------------------------------------------------------------------
// BatchEncoder: GF(256) Standard / Good Cauchy and the additive FFT
// ---------------------------------------------------------------------------

/// Block-final encoder on the GPU (`scrs_batch_encoder_*`).
pub struct GpuBatchEncoder {
    raw: *mut sys::scrs_batch_encoder,
    profile: Profile,
}

/// Caller-owned encode workspace (device and pinned staging of one block).
pub struct GpuEncodeScratch {
    raw: *mut sys::scrs_encode_scratch,
}

/// `batch_encoder` (selector.rs:457): `UnsupportedMode` for the tower engine.
pub fn batch_encoder(profile: &Profile) -> Result<GpuBatchEncoder, ConfigError> {
    let p = raw_profile(profile);
    let mut raw = ptr::null_mut();
    let mut err = no_error();
    let rc = unsafe { sys::scrs_batch_encoder_create(&p, &mut raw, &mut err) };
    error::config(rc, &err)?;
    Ok(GpuBatchEncoder { raw, profile: *profile })
}

impl Drop for GpuBatchEncoder {
    fn drop(&mut self) {
        unsafe { sys::scrs_batch_encoder_destroy(self.raw) }
    }
}

impl Drop for GpuEncodeScratch {
    fn drop(&mut self) {
        unsafe { sys::scrs_encode_scratch_destroy(self.raw) }
    }
}

unsafe impl Send for GpuBatchEncoder {}
unsafe impl Send for GpuEncodeScratch {}
coded_from_profile!(GpuBatchEncoder);

impl BatchEncoder for GpuBatchEncoder {
    type Scratch = GpuEncodeScratch;

    fn scratch(&self) -> GpuEncodeScratch {
        let mut raw = ptr::null_mut();
        let mut err = no_error();
        let rc = unsafe { sys::scrs_batch_encoder_scratch(self.raw, &mut raw, &mut err) };
        error::runtime(rc, &err);
        GpuEncodeScratch { raw }
    }

    fn encode_into(&self, data: &[u8], repairs: &mut [u8]) -> Result<(), EncodeError> {
        let mut err = no_error();
        let rc = unsafe {
            sys::scrs_batch_encode_into(self.raw, data.as_ptr(), data.len() as u64, repairs.as_mut_ptr(),
                                        repairs.len() as u64, &mut err)
        };
        error::encode(rc, &err)
    }

    fn encode_into_with(&self, data: &[u8], repairs: &mut [u8], scratch: &mut GpuEncodeScratch)
                        -> Result<(), EncodeError> {
        let mut err = no_error();
        let rc = unsafe {
            sys::scrs_batch_encode_into_with(self.raw, data.as_ptr(), data.len() as u64, repairs.as_mut_ptr(),
                                             repairs.len() as u64, scratch.raw, &mut err)
        };
        error::encode(rc, &err)
    }
}

// ---------------------------------------------------------------------------
// BatchDecoder: GF(256) BatchCodec, the GF(65536) engines through their lazy
// decoder (the library applies the reference's blanket impl, codec.rs:203-239)
// ---------------------------------------------------------------------------

/// Block-final decoder on the GPU (`scrs_batch_decoder_*`).
pub struct GpuBatchDecoder {
    raw: *mut sys::scrs_batch_decoder,
    profile: Profile,
    // the (index, payload) slice as the ABI's three parallel arrays; capacity
    // k reserved at creation, so decode_into_with allocates nothing
    idx: Vec<u64>,
    ptrs: Vec<*const u8>,
    lens: Vec<u64>,
}

/// Caller-owned batch-decode workspace (device recipe cache, staging).
pub struct GpuBatchDecodeScratch {
    raw: *mut sys::scrs_batch_decode_scratch,
}

/// `batch_decoder` (selector.rs:270).
pub fn batch_decoder(profile: &Profile) -> Result<GpuBatchDecoder, ConfigError> {
    let p = raw_profile(profile);
    let mut raw = ptr::null_mut();
    let mut err = no_error();
    let rc = unsafe { sys::scrs_batch_decoder_create(&p, &mut raw, &mut err) };
    error::config(rc, &err)?;
    let k = profile.k();
    Ok(GpuBatchDecoder { raw, profile: *profile, idx: Vec::with_capacity(k), ptrs: Vec::with_capacity(k),
                         lens: Vec::with_capacity(k) })
}

impl Drop for GpuBatchDecoder {
    fn drop(&mut self) {
        unsafe { sys::scrs_batch_decoder_destroy(self.raw) }
    }
}

impl Drop for GpuBatchDecodeScratch {
    fn drop(&mut self) {
        unsafe { sys::scrs_batch_decode_scratch_destroy(self.raw) }
    }
}

unsafe impl Send for GpuBatchDecoder {}
unsafe impl Send for GpuBatchDecodeScratch {}
coded_from_profile!(GpuBatchDecoder);

impl GpuBatchDecoder {
    fn stage(&mut self, symbols: &[(usize, &[u8])]) {
        self.idx.clear();
        self.ptrs.clear();
        self.lens.clear();
        for &(index, payload) in symbols {
            self.idx.push(index as u64);
            self.ptrs.push(payload.as_ptr());
            self.lens.push(payload.len() as u64);
        }
    }
}

impl BatchDecoder for GpuBatchDecoder {
    type Scratch = GpuBatchDecodeScratch;

    fn scratch(&self) -> GpuBatchDecodeScratch {
        let mut raw = ptr::null_mut();
        let mut err = no_error();
        let rc = unsafe { sys::scrs_batch_decoder_scratch(self.raw, &mut raw, &mut err) };
        error::runtime(rc, &err);
        GpuBatchDecodeScratch { raw }
    }

    fn decode_into(&mut self, symbols: &[(usize, &[u8])], out: &mut [u8]) -> Result<(), DecodeError> {
        let mut scratch = BatchDecoder::scratch(self);
        self.decode_into_with(symbols, out, &mut scratch)
    }

    fn decode_into_with(&mut self, symbols: &[(usize, &[u8])], out: &mut [u8],
                        scratch: &mut GpuBatchDecodeScratch) -> Result<(), DecodeError> {
        // the library validates in the reference's order (scratch, output
        // length, count, then each symbol); a count other than k is an error
        // there, so only an invalid call can grow the staging vectors
        self.stage(symbols);
        let mut err = no_error();
        let rc = unsafe {
            sys::scrs_batch_decode_into_with(self.raw, self.idx.as_ptr(), self.ptrs.as_ptr(), self.lens.as_ptr(),
                                             symbols.len() as u64, out.as_mut_ptr(), out.len() as u64, scratch.raw,
                                             &mut err)
        };
        error::decode(rc, &err)
    }
}

// ---------------------------------------------------------------------------
// IncrementalEncoder: GF(256) Good Cauchy and the tower engine
// ---------------------------------------------------------------------------

/// Streaming encoder on the GPU (`scrs_incremental_encoder_*`, `scrs_inc_*`).
///
/// `repair` returns a borrow, as the reference's does; the repairs live on
/// the device, so the first `repair` after a change copies all m of them into
/// a host mirror.  Only `&mut self` methods change them (and mark the mirror
/// stale), so no borrow handed out by `repair` can be outstanding when the
/// mirror is rewritten.
pub struct GpuIncrementalEncoder {
    raw: *mut sys::scrs_incremental_encoder,
    profile: Profile,
    mirror: UnsafeCell<Vec<u8>>,
    stale: Cell<bool>,
}

/// `incremental_encoder` (selector.rs:370): `UnsupportedMode` for Standard
/// Cauchy and the additive FFT.
pub fn incremental_encoder(profile: &Profile) -> Result<GpuIncrementalEncoder, ConfigError> {
    let p = raw_profile(profile);
    let mut raw = ptr::null_mut();
    let mut err = no_error();
    let rc = unsafe { sys::scrs_incremental_encoder_create(&p, &mut raw, &mut err) };
    error::config(rc, &err)?;
    Ok(GpuIncrementalEncoder { raw, profile: *profile,
                               mirror: UnsafeCell::new(vec![0u8; profile.m() * profile.symbol_len()]),
                               stale: Cell::new(true) })
}

impl Drop for GpuIncrementalEncoder {
    fn drop(&mut self) {
        unsafe { sys::scrs_incremental_encoder_destroy(self.raw) }
    }
}

unsafe impl Send for GpuIncrementalEncoder {}
coded_from_profile!(GpuIncrementalEncoder);

impl IncrementalEncoder for GpuIncrementalEncoder {
    fn feed(&mut self, index: usize, data: &[u8]) -> Result<(), EncodeError> {
        let mut err = no_error();
        let rc = unsafe { sys::scrs_inc_feed(self.raw, index as u64, data.as_ptr(), data.len() as u64, &mut err) };
        error::encode(rc, &err)?;
        self.stale.set(true);
        Ok(())
    }

    fn repair(&self, index: usize) -> Result<&[u8], EncodeError> {
        let (k, m, len) = (self.profile.k(), self.profile.m(), self.profile.symbol_len());
        if index >= m {
            return Err(EncodeError::IndexOutOfRange { index, n: k + m });
        }
        if self.stale.get() {
            // SAFETY: the mirror is stale only after a `&mut self` call, which
            // no borrow of it can outlive, so nothing reads it while it is
            // rewritten here.
            let mirror = unsafe { &mut *self.mirror.get() };
            for j in 0..m {
                let mut err = no_error();
                let rc = unsafe {
                    sys::scrs_inc_repair(self.raw, j as u64, mirror[j * len..].as_mut_ptr(), len as u64, &mut err)
                };
                error::encode(rc, &err)?;
            }
            self.stale.set(false);
        }
        // SAFETY: not stale, so no `&mut` access to the mirror happens while
        // this borrow of `self` lives.
        let mirror = unsafe { &*self.mirror.get() };
        Ok(&mirror[index * len..(index + 1) * len])
    }

    fn fed_count(&self) -> usize {
        unsafe { sys::scrs_inc_fed_count(self.raw) as usize }
    }

    fn reset(&mut self) {
        unsafe { sys::scrs_inc_reset(self.raw) }
        self.stale.set(true);
    }
}

// ---------------------------------------------------------------------------
// Decoder + SymbolSink: every engine
// ---------------------------------------------------------------------------

/// Lazy streaming decoder on the GPU (`scrs_decoder_*`, `scrs_dec_*`); it
/// also gets the reference's blanket `BatchDecoder` impl.
pub struct GpuDecoder {
    raw: *mut sys::scrs_decoder,
    profile: Profile,
}

/// Caller-owned decode workspace (device recipe cache or transform scratch).
pub struct GpuDecodeScratch {
    raw: *mut sys::scrs_decode_scratch,
}

/// `decoder` (selector.rs:117).
pub fn decoder(profile: &Profile) -> Result<GpuDecoder, ConfigError> {
    let p = raw_profile(profile);
    let mut raw = ptr::null_mut();
    let mut err = no_error();
    let rc = unsafe { sys::scrs_decoder_create(&p, &mut raw, &mut err) };
    error::config(rc, &err)?;
    Ok(GpuDecoder { raw, profile: *profile })
}

impl Drop for GpuDecoder {
    fn drop(&mut self) {
        unsafe { sys::scrs_decoder_destroy(self.raw) }
    }
}

impl Drop for GpuDecodeScratch {
    fn drop(&mut self) {
        unsafe { sys::scrs_decode_scratch_destroy(self.raw) }
    }
}

unsafe impl Send for GpuDecoder {}
unsafe impl Send for GpuDecodeScratch {}
coded_from_profile!(GpuDecoder);

impl SymbolSink for GpuDecoder {
    fn push(&mut self, idx: usize, payload: &[u8]) -> Result<PushOutcome, DecodeError> {
        let mut out = sys::scrs_push_outcome { kind: 0, reserved: 0, rank: 0, received: 0 };
        let mut err = no_error();
        let rc = unsafe {
            sys::scrs_dec_push(self.raw, idx as u64, payload.as_ptr(), payload.len() as u64, &mut out, &mut err)
        };
        error::decode(rc, &err)?;
        Ok(match out.kind {
            sys::SCRS_PUSH_COMPLETE => PushOutcome::Complete,
            sys::SCRS_PUSH_DEPENDENT => PushOutcome::Dependent,
            _ => PushOutcome::Advanced { rank: out.rank as usize, received: out.received as usize },
        })
    }

    fn is_complete(&self) -> bool {
        unsafe { sys::scrs_dec_is_complete(self.raw) != 0 }
    }

    fn finalize(mut self) -> Result<Vec<u8>, DecodeError> {
        let mut out = vec![0u8; self.profile.k() * self.profile.symbol_len()];
        self.finalize_into(&mut out)?;
        Ok(out)
    }
}

impl Decoder for GpuDecoder {
    type Scratch = GpuDecodeScratch;

    fn scratch(&self) -> GpuDecodeScratch {
        let mut raw = ptr::null_mut();
        let mut err = no_error();
        let rc = unsafe { sys::scrs_decoder_scratch(self.raw, &mut raw, &mut err) };
        error::runtime(rc, &err);
        GpuDecodeScratch { raw }
    }

    fn rank(&self) -> usize {
        unsafe { sys::scrs_dec_rank(self.raw) as usize }
    }

    fn received(&self) -> usize {
        unsafe { sys::scrs_dec_received(self.raw) as usize }
    }

    fn reset(&mut self) {
        unsafe { sys::scrs_dec_reset(self.raw) }
    }

    fn finalize_into(&mut self, out: &mut [u8]) -> Result<(), DecodeError> {
        let mut err = no_error();
        let rc = unsafe { sys::scrs_dec_finalize_into(self.raw, out.as_mut_ptr(), out.len() as u64, &mut err) };
        error::decode(rc, &err)
    }

    fn finalize_into_with(&mut self, out: &mut [u8], scratch: &mut GpuDecodeScratch) -> Result<(), DecodeError> {
        let mut err = no_error();
        let rc = unsafe {
            sys::scrs_dec_finalize_into_with(self.raw, out.as_mut_ptr(), out.len() as u64, scratch.raw, &mut err)
        };
        error::decode(rc, &err)
    }
}

/// `Engine` of a raw code, for callers that read profiles back from the ABI.
pub fn engine_of(code: i32) -> Option<Engine> {
    match code {
        sys::SCRS_ENGINE_STANDARD_CAUCHY => Some(Engine::StandardCauchy),
        sys::SCRS_ENGINE_GOOD_CAUCHY => Some(Engine::GoodCauchy),
        sys::SCRS_ENGINE_TOWER => Some(Engine::Tower),
        sys::SCRS_ENGINE_AFFT => Some(Engine::Afft),
        _ => None,
    }
}
