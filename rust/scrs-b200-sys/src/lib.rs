//! Raw declarations of `include/scrs_gpu.h` (the B200 erasure-coding engines' C ABI).
//! Generated by gen_bindings.py from the header; do not edit.
#![allow(non_camel_case_types)]

use core::ffi::{c_char, c_void};

pub const SCRS_ENGINE_STANDARD_CAUCHY: i32 = 0;
pub const SCRS_ENGINE_GOOD_CAUCHY: i32 = 1;
pub const SCRS_ENGINE_TOWER: i32 = 2;
pub const SCRS_ENGINE_AFFT: i32 = 3;
pub const SCRS_FIELD_GF256: i32 = 0;
pub const SCRS_FIELD_GF65536: i32 = 1;
pub const SCRS_OK: i32 = 0;
pub const SCRS_CONFIG_ZERO_DIMENSION: i32 = 101;
pub const SCRS_CONFIG_TOO_MANY_SYMBOLS: i32 = 102;
pub const SCRS_CONFIG_ZERO_SYMBOL_LEN: i32 = 103;
pub const SCRS_CONFIG_ODD_SYMBOL_LEN: i32 = 104;
pub const SCRS_CONFIG_UNSUPPORTED_MODE: i32 = 105;
pub const SCRS_ENCODE_WRONG_INPUT_LEN: i32 = 201;
pub const SCRS_ENCODE_INDEX_OUT_OF_RANGE: i32 = 202;
pub const SCRS_ENCODE_WRONG_PAYLOAD_LEN: i32 = 203;
pub const SCRS_ENCODE_DUPLICATE_DATA: i32 = 204;
pub const SCRS_ENCODE_WRONG_OUTPUT_LEN: i32 = 205;
pub const SCRS_ENCODE_SCRATCH_MISMATCH: i32 = 206;
pub const SCRS_DECODE_WRONG_COUNT: i32 = 301;
pub const SCRS_DECODE_INDEX_OUT_OF_RANGE: i32 = 302;
pub const SCRS_DECODE_DUPLICATE_INDEX: i32 = 303;
pub const SCRS_DECODE_WRONG_PAYLOAD_LEN: i32 = 304;
pub const SCRS_DECODE_TOO_MANY_SYMBOLS: i32 = 305;
pub const SCRS_DECODE_INSUFFICIENT_RANK: i32 = 306;
pub const SCRS_DECODE_WRONG_OUTPUT_LEN: i32 = 307;
pub const SCRS_DECODE_SCRATCH_MISMATCH: i32 = 308;
pub const SCRS_ERR_NULL_ARGUMENT: i32 = 901;
pub const SCRS_ERR_CUDA: i32 = 902;
pub const SCRS_ERR_OUT_OF_MEMORY: i32 = 903;
pub const SCRS_ERR_NO_DEVICE: i32 = 904;
pub const SCRS_ERR_CAPACITY: i32 = 905;
pub const SCRS_ERR_DEVICE_TIMEOUT: i32 = 906;
pub const SCRS_ERR_BAD_ARGUMENT: i32 = 907;
pub const SCRS_ERR_JIT: i32 = 908;
pub const SCRS_PUSH_ADVANCED: i32 = 0;
pub const SCRS_PUSH_COMPLETE: i32 = 1;
pub const SCRS_PUSH_DEPENDENT: i32 = 2;
pub const SCRS_OP_ENCODE: i32 = 0;
pub const SCRS_OP_DECODE: i32 = 1;

#[repr(C)]
pub struct scrs_batch_encoder {
    _private: [u8; 0],
}

#[repr(C)]
pub struct scrs_encode_scratch {
    _private: [u8; 0],
}

#[repr(C)]
pub struct scrs_batch_decoder {
    _private: [u8; 0],
}

#[repr(C)]
pub struct scrs_batch_decode_scratch {
    _private: [u8; 0],
}

#[repr(C)]
pub struct scrs_incremental_encoder {
    _private: [u8; 0],
}

#[repr(C)]
pub struct scrs_decoder {
    _private: [u8; 0],
}

#[repr(C)]
pub struct scrs_decode_scratch {
    _private: [u8; 0],
}

#[repr(C)]
pub struct scrs_stripe_batch {
    _private: [u8; 0],
}

#[repr(C)]
pub struct scrs_server {
    _private: [u8; 0],
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct scrs_profile {
    pub engine: i32,
    pub reserved: i32,
    pub k: u64,
    pub m: u64,
    pub symbol_len: u64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct scrs_error {
    pub code: i32,
    pub reserved: i32,
    pub a: u64,
    pub b: u64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct scrs_push_outcome {
    pub kind: i32,
    pub reserved: i32,
    pub rank: u64,
    pub received: u64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct scrs_stripe_desc {
    pub op: i32,
    pub engine: i32,
    pub k: u32,
    pub m: u32,
    pub symbol_len: u64,
    pub r#in: *const u8,
    pub out: *mut u8,
    pub indices: *const u16,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct scrs_tune_key {
    pub field: u32,
    pub k_bucket: u32,
    pub m_bucket: u32,
    pub l_bucket: u32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct scrs_tune_params {
    pub seg_rows: u32,
    pub ctas_per_sm: u32,
    pub drain_ms: f32,
    pub reserved: u32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct scrs_request {
    pub op: i32,
    pub engine: i32,
    pub k: u64,
    pub m: u64,
    pub symbol_len: u64,
    pub r#in: *const u8,
    pub out: *mut u8,
    pub indices: *const u64,
    pub tag: u64,
    pub stream: *mut c_void,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct scrs_completion {
    pub ticket: u64,
    pub tag: u64,
    pub status: i32,
    pub reserved: i32,
    pub submit_ns: u64,
    pub done_ns: u64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct scrs_server_stats {
    pub submitted: u64,
    pub admitted: u64,
    pub completed: u64,
    pub failed: u64,
    pub batches: u64,
    pub memory_in_use: u64,
    pub resident_bytes: u64,
}

extern "C" {
    pub fn scrs_abi_version() -> u32;
    pub fn scrs_status_name(code: i32) -> *const c_char;
    pub fn scrs_alloc_count() -> u64;
    pub fn scrs_profile_resolve(engine: i32, k: u64, m: u64, symbol_len: u64, out: *mut scrs_profile, err: *mut scrs_error) -> i32;
    pub fn scrs_profile_recommended(field: i32, k: u64, m: u64, symbol_len: u64, out: *mut scrs_profile, err: *mut scrs_error) -> i32;
    pub fn scrs_recommended_gf16_engine(k: u64, m: u64) -> i32;
    pub fn scrs_batch_encoder_create(profile: *const scrs_profile, out: *mut *mut scrs_batch_encoder, err: *mut scrs_error) -> i32;
    pub fn scrs_batch_encoder_destroy(enc: *mut scrs_batch_encoder);
    pub fn scrs_batch_encoder_profile(enc: *const scrs_batch_encoder, out: *mut scrs_profile) -> i32;
    pub fn scrs_batch_encoder_scratch(enc: *const scrs_batch_encoder, out: *mut *mut scrs_encode_scratch, err: *mut scrs_error) -> i32;
    pub fn scrs_encode_scratch_destroy(scratch: *mut scrs_encode_scratch);
    pub fn scrs_batch_encode_into(enc: *const scrs_batch_encoder, data: *const u8, data_len: u64, repairs: *mut u8, repairs_len: u64, err: *mut scrs_error) -> i32;
    pub fn scrs_batch_encode_into_with(enc: *const scrs_batch_encoder, data: *const u8, data_len: u64, repairs: *mut u8, repairs_len: u64, scratch: *mut scrs_encode_scratch, err: *mut scrs_error) -> i32;
    pub fn scrs_batch_encode_into_with_device(enc: *const scrs_batch_encoder, d_data: *const u8, data_len: u64, d_repairs: *mut u8, repairs_len: u64, scratch: *mut scrs_encode_scratch, stream: *mut c_void, err: *mut scrs_error) -> i32;
    pub fn scrs_batch_decoder_create(profile: *const scrs_profile, out: *mut *mut scrs_batch_decoder, err: *mut scrs_error) -> i32;
    pub fn scrs_batch_decoder_destroy(dec: *mut scrs_batch_decoder);
    pub fn scrs_batch_decoder_profile(dec: *const scrs_batch_decoder, out: *mut scrs_profile) -> i32;
    pub fn scrs_batch_decoder_scratch(dec: *const scrs_batch_decoder, out: *mut *mut scrs_batch_decode_scratch, err: *mut scrs_error) -> i32;
    pub fn scrs_batch_decode_scratch_destroy(scratch: *mut scrs_batch_decode_scratch);
    pub fn scrs_batch_decode_into_with(dec: *mut scrs_batch_decoder, indices: *const u64, payloads: *const *const u8, payload_lens: *const u64, count: u64, out: *mut u8, out_len: u64, scratch: *mut scrs_batch_decode_scratch, err: *mut scrs_error) -> i32;
    pub fn scrs_batch_decode_into(dec: *mut scrs_batch_decoder, indices: *const u64, payloads: *const *const u8, payload_lens: *const u64, count: u64, out: *mut u8, out_len: u64, err: *mut scrs_error) -> i32;
    pub fn scrs_batch_decode_into_with_device(dec: *mut scrs_batch_decoder, indices: *const u64, d_payloads: *const u8, count: u64, d_out: *mut u8, out_len: u64, scratch: *mut scrs_batch_decode_scratch, stream: *mut c_void, err: *mut scrs_error) -> i32;
    pub fn scrs_selftest_wait_timeout(limit_ns: u64, err: *mut scrs_error) -> i32;
    pub fn scrs_batch_decode_scratch_recipe_hits(scratch: *const scrs_batch_decode_scratch) -> u64;
    pub fn scrs_decode_scratch_recipe_hits(scratch: *const scrs_decode_scratch) -> u64;
    pub fn scrs_gf256_decode_static(engine: i32, k: u64, m: u64, symbol_len: u64, indices: *const u64, d_rows: *const u8, count: u64, d_out: *mut u8, out_len: u64, stream: *mut c_void, d_status: *mut i32, err: *mut scrs_error) -> i32;
    pub fn scrs_incremental_encoder_create(profile: *const scrs_profile, out: *mut *mut scrs_incremental_encoder, err: *mut scrs_error) -> i32;
    pub fn scrs_incremental_encoder_destroy(enc: *mut scrs_incremental_encoder);
    pub fn scrs_incremental_encoder_profile(enc: *const scrs_incremental_encoder, out: *mut scrs_profile) -> i32;
    pub fn scrs_inc_feed(enc: *mut scrs_incremental_encoder, index: u64, data: *const u8, data_len: u64, err: *mut scrs_error) -> i32;
    pub fn scrs_inc_feed_device_stream(enc: *mut scrs_incremental_encoder, index: u64, d_data: *const u8, data_len: u64, stream: *mut c_void, err: *mut scrs_error) -> i32;
    pub fn scrs_inc_feed_device(enc: *mut scrs_incremental_encoder, index: u64, d_data: *const u8, data_len: u64, err: *mut scrs_error) -> i32;
    pub fn scrs_inc_repair(enc: *const scrs_incremental_encoder, index: u64, dst: *mut u8, dst_len: u64, err: *mut scrs_error) -> i32;
    pub fn scrs_inc_repair_device(enc: *const scrs_incremental_encoder, index: u64, d_repair: *mut *const u8, err: *mut scrs_error) -> i32;
    pub fn scrs_inc_fed_count(enc: *const scrs_incremental_encoder) -> u64;
    pub fn scrs_inc_reset(enc: *mut scrs_incremental_encoder);
    pub fn scrs_decoder_create(profile: *const scrs_profile, out: *mut *mut scrs_decoder, err: *mut scrs_error) -> i32;
    pub fn scrs_decoder_destroy(dec: *mut scrs_decoder);
    pub fn scrs_decoder_profile(dec: *const scrs_decoder, out: *mut scrs_profile) -> i32;
    pub fn scrs_decoder_scratch(dec: *const scrs_decoder, out: *mut *mut scrs_decode_scratch, err: *mut scrs_error) -> i32;
    pub fn scrs_decode_scratch_destroy(scratch: *mut scrs_decode_scratch);
    pub fn scrs_dec_push(dec: *mut scrs_decoder, index: u64, payload: *const u8, payload_len: u64, outcome: *mut scrs_push_outcome, err: *mut scrs_error) -> i32;
    pub fn scrs_dec_push_device_stream(dec: *mut scrs_decoder, index: u64, d_payload: *const u8, payload_len: u64, stream: *mut c_void, outcome: *mut scrs_push_outcome, err: *mut scrs_error) -> i32;
    pub fn scrs_dec_push_device(dec: *mut scrs_decoder, index: u64, d_payload: *const u8, payload_len: u64, outcome: *mut scrs_push_outcome, err: *mut scrs_error) -> i32;
    pub fn scrs_dec_is_complete(dec: *const scrs_decoder) -> i32;
    pub fn scrs_dec_rank(dec: *const scrs_decoder) -> u64;
    pub fn scrs_dec_received(dec: *const scrs_decoder) -> u64;
    pub fn scrs_dec_reset(dec: *mut scrs_decoder);
    pub fn scrs_dec_finalize_into(dec: *mut scrs_decoder, out: *mut u8, out_len: u64, err: *mut scrs_error) -> i32;
    pub fn scrs_dec_finalize_into_with(dec: *mut scrs_decoder, out: *mut u8, out_len: u64, scratch: *mut scrs_decode_scratch, err: *mut scrs_error) -> i32;
    pub fn scrs_dec_finalize_into_with_device(dec: *mut scrs_decoder, d_out: *mut u8, out_len: u64, scratch: *mut scrs_decode_scratch, stream: *mut c_void, err: *mut scrs_error) -> i32;
    pub fn scrs_stripe_batch_create(max_stripes: u64, max_work_items: u64, out: *mut *mut scrs_stripe_batch, err: *mut scrs_error) -> i32;
    pub fn scrs_stripe_batch_destroy(batch: *mut scrs_stripe_batch);
    pub fn scrs_stripe_batch_set(batch: *mut scrs_stripe_batch, descs: *const scrs_stripe_desc, count: u64, err: *mut scrs_error) -> i32;
    pub fn scrs_stripe_batch_set_host(batch: *mut scrs_stripe_batch, descs: *const scrs_stripe_desc, count: u64, err: *mut scrs_error) -> i32;
    pub fn scrs_stripe_batch_run(batch: *mut scrs_stripe_batch, stream: *mut c_void, use_graph: i32, err: *mut scrs_error) -> i32;
    pub fn scrs_stripe_batch_run_plain(batch: *mut scrs_stripe_batch, stream: *mut c_void, err: *mut scrs_error) -> i32;
    pub fn scrs_stripe_batch_last_launches(batch: *const scrs_stripe_batch) -> u64;
    pub fn scrs_stripe_batch_run_timed(batch: *mut scrs_stripe_batch, stream: *mut c_void, plan_ms: *mut f32, drain_ms: *mut f32, err: *mut scrs_error) -> i32;
    pub fn scrs_stripe_batch_run_timed_drains(batch: *mut scrs_stripe_batch, stream: *mut c_void, plan_ms: *mut f32, spec_ms: *mut f32, generic_ms: *mut f32, err: *mut scrs_error) -> i32;
    pub fn scrs_stripe_batch_check(batch: *mut scrs_stripe_batch, err: *mut scrs_error) -> i32;
    pub fn scrs_tune_key_of(descs: *const scrs_stripe_desc, count: u64, key: *mut scrs_tune_key, err: *mut scrs_error) -> i32;
    pub fn scrs_stripe_batch_tune_key(batch: *const scrs_stripe_batch, key: *mut scrs_tune_key, err: *mut scrs_error) -> i32;
    pub fn scrs_stripe_batch_launch_params(batch: *const scrs_stripe_batch, params: *mut scrs_tune_params, err: *mut scrs_error) -> i32;
    pub fn scrs_stripe_batch_autotune(batch: *mut scrs_stripe_batch, stream: *mut c_void, reps: u32, chosen: *mut scrs_tune_params, err: *mut scrs_error) -> i32;
    pub fn scrs_jit_prepare(engine: i32, k: u32, m: u32, load: i32, cubin_bytes: *mut u64, err: *mut scrs_error) -> i32;
    pub fn scrs_stripe_batch_set_jit(batch: *mut scrs_stripe_batch, enable: i32, err: *mut scrs_error) -> i32;
    pub fn scrs_stripe_batch_jit_stripes(batch: *const scrs_stripe_batch) -> u64;
    pub fn scrs_tune_table_size() -> u64;
    pub fn scrs_tune_table_entry(i: u64, key: *mut scrs_tune_key, params: *mut scrs_tune_params, err: *mut scrs_error) -> i32;
    pub fn scrs_tune_table_set(key: *const scrs_tune_key, params: *const scrs_tune_params, err: *mut scrs_error) -> i32;
    pub fn scrs_tune_table_clear();
    pub fn scrs_server_create(memory_budget: u64, slots: u32, out: *mut *mut scrs_server, err: *mut scrs_error) -> i32;
    pub fn scrs_server_destroy(server: *mut scrs_server);
    pub fn scrs_server_submit(server: *mut scrs_server, req: *const scrs_request, ticket: *mut u64, err: *mut scrs_error) -> i32;
    pub fn scrs_server_progress(server: *mut scrs_server, done: *mut scrs_completion, capacity: u32, n_done: *mut u32, err: *mut scrs_error) -> i32;
    pub fn scrs_server_reserve(server: *mut scrs_server, op: i32, engine: i32, k: u64, m: u64, symbol_len: u64, err: *mut scrs_error) -> i32;
    pub fn scrs_server_pending(server: *const scrs_server) -> u64;
    pub fn scrs_server_get_stats(server: *const scrs_server, out: *mut scrs_server_stats) -> i32;
}
