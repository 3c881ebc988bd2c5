/*
 * Test infrastructure: the oracle's exported C ABI.  Same signatures as the
 * product ABI in include/scrs_gpu.h with `oracle_` in place of `scrs_`, so a
 * test can run one scenario through both libraries and compare the bytes.
 */
#ifndef SCRS_ORACLE_H
#define SCRS_ORACLE_H

#include "../include/scrs_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_batch_encoder oracle_batch_encoder;
typedef struct oracle_encode_scratch oracle_encode_scratch;
typedef struct oracle_batch_decoder oracle_batch_decoder;
typedef struct oracle_batch_decode_scratch oracle_batch_decode_scratch;
typedef struct oracle_incremental_encoder oracle_incremental_encoder;
typedef struct oracle_decoder oracle_decoder;
typedef struct oracle_decode_scratch oracle_decode_scratch;

uint32_t oracle_abi_version(void);
int32_t oracle_profile_resolve(int32_t engine, uint64_t k, uint64_t m, uint64_t L,
                               scrs_profile* out, scrs_error* err);
int32_t oracle_profile_recommended(int32_t field, uint64_t k, uint64_t m, uint64_t L,
                                   scrs_profile* out, scrs_error* err);
int32_t oracle_recommended_gf16_engine(uint64_t k, uint64_t m);

int32_t oracle_batch_encoder_create(const scrs_profile* p, oracle_batch_encoder** out,
                                    scrs_error* err);
void oracle_batch_encoder_destroy(oracle_batch_encoder* e);
int32_t oracle_batch_encoder_profile(const oracle_batch_encoder* e, scrs_profile* out);
int32_t oracle_batch_encoder_scratch(const oracle_batch_encoder* e, oracle_encode_scratch** out,
                                     scrs_error* err);
void oracle_encode_scratch_destroy(oracle_encode_scratch* s);
int32_t oracle_batch_encode_into(const oracle_batch_encoder* e, const uint8_t* data, uint64_t dl,
                                 uint8_t* rep, uint64_t rl, scrs_error* err);
int32_t oracle_batch_encode_into_with(const oracle_batch_encoder* e, const uint8_t* data,
                                      uint64_t dl, uint8_t* rep, uint64_t rl,
                                      oracle_encode_scratch* s, scrs_error* err);

int32_t oracle_batch_decoder_create(const scrs_profile* p, oracle_batch_decoder** out,
                                    scrs_error* err);
void oracle_batch_decoder_destroy(oracle_batch_decoder* b);
int32_t oracle_batch_decoder_profile(const oracle_batch_decoder* b, scrs_profile* out);
int32_t oracle_batch_decoder_scratch(const oracle_batch_decoder* b,
                                     oracle_batch_decode_scratch** out, scrs_error* err);
void oracle_batch_decode_scratch_destroy(oracle_batch_decode_scratch* s);
int32_t oracle_batch_decode_into_with(oracle_batch_decoder* b, const uint64_t* idx,
                                      const uint8_t* const* pay, const uint64_t* lens,
                                      uint64_t count, uint8_t* out, uint64_t out_len,
                                      oracle_batch_decode_scratch* s, scrs_error* err);
int32_t oracle_batch_decode_into(oracle_batch_decoder* b, const uint64_t* idx,
                                 const uint8_t* const* pay, const uint64_t* lens, uint64_t count,
                                 uint8_t* out, uint64_t out_len, scrs_error* err);

int32_t oracle_incremental_encoder_create(const scrs_profile* p,
                                          oracle_incremental_encoder** out, scrs_error* err);
void oracle_incremental_encoder_destroy(oracle_incremental_encoder* e);
int32_t oracle_incremental_encoder_profile(const oracle_incremental_encoder* e,
                                           scrs_profile* out);
int32_t oracle_inc_feed(oracle_incremental_encoder* e, uint64_t idx, const uint8_t* data,
                        uint64_t len, scrs_error* err);
int32_t oracle_inc_repair(const oracle_incremental_encoder* e, uint64_t idx, uint8_t* dst,
                          uint64_t dst_len, scrs_error* err);
uint64_t oracle_inc_fed_count(const oracle_incremental_encoder* e);
void oracle_inc_reset(oracle_incremental_encoder* e);

int32_t oracle_decoder_create(const scrs_profile* p, oracle_decoder** out, scrs_error* err);
void oracle_decoder_destroy(oracle_decoder* d);
int32_t oracle_decoder_profile(const oracle_decoder* d, scrs_profile* out);
int32_t oracle_decoder_scratch(const oracle_decoder* d, oracle_decode_scratch** out,
                               scrs_error* err);
void oracle_decode_scratch_destroy(oracle_decode_scratch* s);
int32_t oracle_dec_push(oracle_decoder* d, uint64_t idx, const uint8_t* payload, uint64_t len,
                        scrs_push_outcome* outcome, scrs_error* err);
int32_t oracle_dec_is_complete(const oracle_decoder* d);
uint64_t oracle_dec_rank(const oracle_decoder* d);
uint64_t oracle_dec_received(const oracle_decoder* d);
void oracle_dec_reset(oracle_decoder* d);
int32_t oracle_dec_finalize_into(oracle_decoder* d, uint8_t* out, uint64_t out_len,
                                 scrs_error* err);
int32_t oracle_dec_finalize_into_with(oracle_decoder* d, uint8_t* out, uint64_t out_len,
                                      oracle_decode_scratch* s, scrs_error* err);

/* ---- oracle-only entry points used by the tests ------------------------- */
uint8_t oracle_gf256_mul(uint8_t a, uint8_t b);
uint8_t oracle_gf256_mul_xtime(uint8_t a, uint8_t b);
uint8_t oracle_gf256_inv(uint8_t a);
uint8_t oracle_gf256_inv_xtime(uint8_t a);
uint8_t oracle_gf256_exp(uint32_t i);
uint16_t oracle_gf65536_mul(uint16_t a, uint16_t b);
uint16_t oracle_gf65536_square(uint16_t a);
uint16_t oracle_gf65536_inv(uint16_t a);
uint16_t oracle_gf65536_pow(uint16_t a, uint32_t e);
void oracle_gf256_coefficient_matrix(int32_t engine, uint64_t k, uint64_t m, uint8_t* out);
int32_t oracle_tower_coefficient_matrix(uint64_t k, uint64_t m, uint16_t* out);
size_t oracle_gf256_rref_decode(int32_t engine, size_t k, size_t m, size_t L,
                                const uint64_t* indices, const uint8_t* const* payloads,
                                uint8_t* out);
/* AFFT transform plan probes (transform.rs) */
int32_t oracle_afft_plan_factors(uint64_t size, uint16_t* factors, uint16_t* derivative_factors);
int32_t oracle_afft_forward(uint64_t size, uint16_t* values);
int32_t oracle_afft_inverse(uint64_t size, uint16_t* values);
int32_t oracle_afft_forward_bytes_trunc_range(uint64_t size, uint8_t* rows, uint64_t L,
                                              uint64_t active, uint64_t start, uint64_t end);
int32_t oracle_afft_inverse_truncated_bytes(uint64_t size, uint8_t* rows, uint64_t L,
                                            uint64_t active);
int32_t oracle_afft_forward_bytes(uint64_t size, uint8_t* rows, uint64_t L);
int32_t oracle_afft_encode_blocked(uint64_t k, uint64_t m, uint64_t L, const uint8_t* data,
                                   uint8_t* repairs, uint64_t width, int32_t fused);
void oracle_afft_locator(const uint8_t* known, uint64_t ts, uint16_t* values, uint16_t* derivs);
int32_t oracle_simd_active(void);
void oracle_force_scalar(int32_t on);

/* ---- CPU baseline helpers: many independent stripes over host threads --- */
/* Encodes `count` GF(256) stripes of one geometry: data[s] = in + s*k*L,
 * repairs[s] = out + s*m*L.  Returns elapsed seconds. */
double oracle_baseline_gf256_encode(int32_t engine, uint64_t k, uint64_t m, uint64_t L,
                                    const uint8_t* in, uint8_t* out, uint64_t count,
                                    int32_t threads);
/* Batch-decodes `count` stripes: received rows for stripe s at
 * in + s*k*L (indices[s*k + q] names row q), output at out + s*k*L. */
double oracle_baseline_gf256_decode(int32_t engine, uint64_t k, uint64_t m, uint64_t L,
                                    const uint8_t* in, const uint16_t* indices, uint8_t* out,
                                    uint64_t count, int32_t threads);
int32_t oracle_baseline_threads(void);
/* Runs `count` stripes of any engine and geometry (scrs_stripe_desc, every
 * pointer in HOST memory) over `threads` host threads, each taking a
 * contiguous range; *status gets the first failure (0 when all succeeded).
 * Returns elapsed seconds. */
double oracle_baseline_stripes(const scrs_stripe_desc* descs, uint64_t count, int32_t threads,
                               int32_t* status);

#ifdef __cplusplus
}
#endif
#endif
