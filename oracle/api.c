/*
 * Test infrastructure (oracle): the SCRS trait surface restated on the CPU,
 * exported with the `oracle_` prefix and the same signatures as the CUDA
 * library's `scrs_` C ABI (include/scrs_gpu.h).  Validation order follows
 * the reference so that error parity can be tested.
 */
#include <stdlib.h>

#include "oracle_afft.h"
#include "scrs_oracle.h"

/* ---- profiles: scrs/src/selector.rs:24-88, scrs/src/lib.rs:85-93 -------- */
static uint64_t engine_capacity(int32_t engine) {
    switch (engine) {
        case SCRS_ENGINE_STANDARD_CAUCHY: return 256;
        case SCRS_ENGINE_GOOD_CAUCHY: return 255;
        case SCRS_ENGINE_TOWER: return 65535;
        default: return 65536;
    }
}
static int is_gf16(int32_t engine) { return engine == SCRS_ENGINE_TOWER || engine == SCRS_ENGINE_AFFT; }

uint32_t oracle_abi_version(void) { return 0x00010000u; }

int32_t oracle_profile_resolve(int32_t engine, uint64_t k, uint64_t m, uint64_t L,
                               scrs_profile* out, scrs_error* err) {
    if (engine < 0 || engine > 3) return oerr(err, SCRS_ERR_BAD_ARGUMENT, 0, 0);
    if (k == 0 || m == 0) return oerr(err, SCRS_CONFIG_ZERO_DIMENSION, 0, 0);
    if (L == 0) return oerr(err, SCRS_CONFIG_ZERO_SYMBOL_LEN, 0, 0);
    if (is_gf16(engine) && (L % 2)) return oerr(err, SCRS_CONFIG_ODD_SYMBOL_LEN, 0, 0);
    uint64_t cap = engine_capacity(engine);
    if (k > cap || m > cap || k + m > cap) return oerr(err, SCRS_CONFIG_TOO_MANY_SYMBOLS, cap, 0);
    if (out) {
        out->engine = engine;
        out->reserved = 0;
        out->k = k, out->m = m, out->symbol_len = L;
    }
    return oerr(err, SCRS_OK, 0, 0);
}

int32_t oracle_recommended_gf16_engine(uint64_t k, uint64_t m) {
    int large = (k + m < k) || (k + m > 256);
    int high = (m > UINT64_MAX / 3) || (m * 3 >= k);
    return (large || high) ? SCRS_ENGINE_AFFT : SCRS_ENGINE_TOWER;
}

int32_t oracle_profile_recommended(int32_t field, uint64_t k, uint64_t m, uint64_t L,
                                   scrs_profile* out, scrs_error* err) {
    int32_t engine;
    if (field == SCRS_FIELD_GF256)
        engine = (k + m <= 255) ? SCRS_ENGINE_GOOD_CAUCHY : SCRS_ENGINE_STANDARD_CAUCHY;
    else if (field == SCRS_FIELD_GF65536)
        engine = oracle_recommended_gf16_engine(k, m);
    else
        return oerr(err, SCRS_ERR_BAD_ARGUMENT, 0, 0);
    return oracle_profile_resolve(engine, k, m, L, out, err);
}

static int32_t check_profile(const scrs_profile* p, scrs_error* err) {
    if (!p) return oerr(err, SCRS_ERR_NULL_ARGUMENT, 0, 0);
    return oracle_profile_resolve(p->engine, p->k, p->m, p->symbol_len, NULL, err);
}

/* ---- lazy decoder state shared by all engines ---------------------------- */
struct oracle_decoder {
    scrs_profile p;
    uint8_t* payloads; /* n * L, codeword order */
    uint8_t* have;     /* receipt bitmap (one byte per position) */
    uint64_t distinct;
    uint64_t received;
    afft_profile afft;
};

enum { SK_UNIT = 1, SK_AFFT_ENC = 2, SK_CAUCHY_BATCH = 3, SK_CAUCHY_RECIPE = 4, SK_TOWER = 5, SK_AFFT = 6 };

struct oracle_encode_scratch { int kind; scrs_profile p; };
struct oracle_batch_decode_scratch { int kind; scrs_profile p; };
struct oracle_decode_scratch { int kind; scrs_profile p; };

/* ---- BatchEncoder --------------------------------------------------------- */
struct oracle_batch_encoder {
    scrs_profile p;
    uint8_t* coeffs8;
    afft_profile afft;
};

int32_t oracle_batch_encoder_create(const scrs_profile* p, oracle_batch_encoder** out,
                                    scrs_error* err) {
    int32_t st = check_profile(p, err);
    if (st) return st;
    if (!out) return oerr(err, SCRS_ERR_NULL_ARGUMENT, 0, 0);
    if (p->engine == SCRS_ENGINE_TOWER) /* selector.rs:465 */
        return oerr(err, SCRS_CONFIG_UNSUPPORTED_MODE, (uint64_t)p->engine, 0);
    oracle_batch_encoder* e = (oracle_batch_encoder*)calloc(1, sizeof *e);
    e->p = *p;
    if (p->engine == SCRS_ENGINE_AFFT) {
        if (!afft_profile_init(&e->afft, p->k, p->m, p->symbol_len)) {
            free(e);
            return oerr(err, SCRS_CONFIG_TOO_MANY_SYMBOLS, 65536, 0);
        }
    } else {
        e->coeffs8 = (uint8_t*)malloc(p->k * p->m);
        gf8_coefficient_matrix(p->engine, p->k, p->m, e->coeffs8);
    }
    *out = e;
    return oerr(err, SCRS_OK, 0, 0);
}

void oracle_batch_encoder_destroy(oracle_batch_encoder* e) {
    if (!e) return;
    if (e->p.engine == SCRS_ENGINE_AFFT) afft_profile_free(&e->afft);
    free(e->coeffs8);
    free(e);
}

int32_t oracle_batch_encoder_profile(const oracle_batch_encoder* e, scrs_profile* out) {
    if (!e || !out) return SCRS_ERR_NULL_ARGUMENT;
    *out = e->p;
    return SCRS_OK;
}

int32_t oracle_batch_encoder_scratch(const oracle_batch_encoder* e, oracle_encode_scratch** out,
                                     scrs_error* err) {
    if (!e || !out) return oerr(err, SCRS_ERR_NULL_ARGUMENT, 0, 0);
    oracle_encode_scratch* s = (oracle_encode_scratch*)calloc(1, sizeof *s);
    s->kind = e->p.engine == SCRS_ENGINE_AFFT ? SK_AFFT_ENC : SK_UNIT;
    s->p = e->p;
    *out = s;
    return oerr(err, SCRS_OK, 0, 0);
}
void oracle_encode_scratch_destroy(oracle_encode_scratch* s) { free(s); }

/* GF(256): scrs/src/batch/codec.rs:156-192 (repairs zeroed, then every
 * (coefficient row, source) term).  AFFT: scrs/src/afft/encoder.rs:250-275. */
static int32_t encode_core(const oracle_batch_encoder* e, const uint8_t* data, uint64_t dl,
                           uint8_t* rep, uint64_t rl, scrs_error* err) {
    uint64_t k = e->p.k, m = e->p.m, L = e->p.symbol_len;
    if (dl != k * L) return oerr(err, SCRS_ENCODE_WRONG_INPUT_LEN, k * L, dl);
    if (rl != m * L) return oerr(err, SCRS_ENCODE_WRONG_OUTPUT_LEN, m * L, rl);
    if (!data || !rep) return oerr(err, SCRS_ERR_NULL_ARGUMENT, 0, 0);
    if (e->p.engine == SCRS_ENGINE_AFFT) {
        afft_encode(&e->afft, data, rep);
        return oerr(err, SCRS_OK, 0, 0);
    }
    memset(rep, 0, m * L);
    for (uint64_t i = 0; i < k; i++)
        for (uint64_t j = 0; j < m; j++) pl8_xor_scaled(rep + j * L, e->coeffs8[i * m + j], data + i * L, L);
    return oerr(err, SCRS_OK, 0, 0);
}

int32_t oracle_batch_encode_into(const oracle_batch_encoder* e, const uint8_t* data, uint64_t dl,
                                 uint8_t* rep, uint64_t rl, scrs_error* err) {
    if (!e) return oerr(err, SCRS_ERR_NULL_ARGUMENT, 0, 0);
    return encode_core(e, data, dl, rep, rl, err);
}

int32_t oracle_batch_encode_into_with(const oracle_batch_encoder* e, const uint8_t* data,
                                      uint64_t dl, uint8_t* rep, uint64_t rl,
                                      oracle_encode_scratch* s, scrs_error* err) {
    if (!e || !s) return oerr(err, SCRS_ERR_NULL_ARGUMENT, 0, 0);
    int want = e->p.engine == SCRS_ENGINE_AFFT ? SK_AFFT_ENC : SK_UNIT;
    if (s->kind != want) return oerr(err, SCRS_ENCODE_SCRATCH_MISMATCH, 0, 0); /* selector.rs:526 */
    return encode_core(e, data, dl, rep, rl, err);
}

/* ---- Decoder (lazy): decoder/streaming.rs, tower/decoder.rs, afft/decoder.rs */
int32_t oracle_decoder_create(const scrs_profile* p, oracle_decoder** out, scrs_error* err) {
    int32_t st = check_profile(p, err);
    if (st) return st;
    if (!out) return oerr(err, SCRS_ERR_NULL_ARGUMENT, 0, 0);
    oracle_decoder* d = (oracle_decoder*)calloc(1, sizeof *d);
    d->p = *p;
    uint64_t n = p->k + p->m;
    d->payloads = (uint8_t*)calloc(n * p->symbol_len, 1);
    d->have = (uint8_t*)calloc(n, 1);
    if (p->engine == SCRS_ENGINE_AFFT && !afft_profile_init(&d->afft, p->k, p->m, p->symbol_len)) {
        free(d->payloads), free(d->have), free(d);
        return oerr(err, SCRS_CONFIG_TOO_MANY_SYMBOLS, 65536, 0);
    }
    *out = d;
    return oerr(err, SCRS_OK, 0, 0);
}

void oracle_decoder_destroy(oracle_decoder* d) {
    if (!d) return;
    if (d->p.engine == SCRS_ENGINE_AFFT) afft_profile_free(&d->afft);
    free(d->payloads), free(d->have), free(d);
}

int32_t oracle_decoder_profile(const oracle_decoder* d, scrs_profile* out) {
    if (!d || !out) return SCRS_ERR_NULL_ARGUMENT;
    *out = d->p;
    return SCRS_OK;
}

static int decode_scratch_kind(int32_t engine) {
    if (engine == SCRS_ENGINE_TOWER) return SK_TOWER;
    if (engine == SCRS_ENGINE_AFFT) return SK_AFFT;
    return SK_CAUCHY_RECIPE;
}

int32_t oracle_decoder_scratch(const oracle_decoder* d, oracle_decode_scratch** out,
                               scrs_error* err) {
    if (!d || !out) return oerr(err, SCRS_ERR_NULL_ARGUMENT, 0, 0);
    oracle_decode_scratch* s = (oracle_decode_scratch*)calloc(1, sizeof *s);
    s->kind = decode_scratch_kind(d->p.engine);
    s->p = d->p;
    *out = s;
    return oerr(err, SCRS_OK, 0, 0);
}
void oracle_decode_scratch_destroy(oracle_decode_scratch* s) { free(s); }

/* SymbolSink::push, identical in all engines (decoder/streaming.rs:388-429,
 * tower/decoder.rs:372-405, afft/decoder.rs:464-500).  GF(256) reports
 * Complete at distinct >= k; the GF(65536) engines at distinct == k; both
 * coincide because distinct never exceeds k. */
int32_t oracle_dec_push(oracle_decoder* d, uint64_t idx, const uint8_t* payload, uint64_t len,
                        scrs_push_outcome* outcome, scrs_error* err) {
    if (!d) return oerr(err, SCRS_ERR_NULL_ARGUMENT, 0, 0);
    uint64_t n = d->p.k + d->p.m, L = d->p.symbol_len;
    if (idx >= n) return oerr(err, SCRS_DECODE_INDEX_OUT_OF_RANGE, idx, n);
    if (len != L) return oerr(err, SCRS_DECODE_WRONG_PAYLOAD_LEN, L, len);
    if (d->received >= n) return oerr(err, SCRS_DECODE_TOO_MANY_SYMBOLS, n, d->received);
    if (!payload) return oerr(err, SCRS_ERR_NULL_ARGUMENT, 0, 0);
    d->received++;
    scrs_push_outcome o = {0};
    if (d->distinct >= d->p.k || d->have[idx]) {
        o.kind = SCRS_PUSH_DEPENDENT;
    } else {
        memcpy(d->payloads + idx * L, payload, L);
        d->have[idx] = 1;
        d->distinct++;
        if (d->distinct >= d->p.k) {
            o.kind = SCRS_PUSH_COMPLETE;
        } else {
            o.kind = SCRS_PUSH_ADVANCED;
            o.rank = d->distinct;
            o.received = d->received;
        }
    }
    if (outcome) *outcome = o;
    return oerr(err, SCRS_OK, 0, 0);
}

int32_t oracle_dec_is_complete(const oracle_decoder* d) { return d && d->distinct >= d->p.k; }
uint64_t oracle_dec_rank(const oracle_decoder* d) { return d ? d->distinct : 0; }
uint64_t oracle_dec_received(const oracle_decoder* d) { return d ? d->received : 0; }
void oracle_dec_reset(oracle_decoder* d) {
    if (!d) return;
    memset(d->have, 0, d->p.k + d->p.m);
    d->distinct = 0;
    d->received = 0;
}

/* GF(256): build_recipe + apply_recipe_into (decoder/streaming.rs:163-352).
 * Tower: build_recipe_into + apply_recipe_into (tower/decoder.rs:218-320). */
static int32_t cauchy_finalize(const oracle_decoder* d, uint8_t* out, scrs_error* err) {
    size_t k = d->p.k, m = d->p.m, L = d->p.symbol_len;
    int gf16 = d->p.engine == SCRS_ENGINE_TOWER;
    size_t* missing = (size_t*)malloc(k * sizeof(size_t));
    size_t* present = (size_t*)malloc(k * sizeof(size_t));
    size_t* repairs = (size_t*)malloc((m + 1) * sizeof(size_t));
    size_t r = 0, pc = 0, rc = 0;
    for (size_t i = 0; i < k; i++) {
        if (d->have[i]) present[pc++] = i;
        else missing[r++] = i;
    }
    for (size_t j = 0; j < m && rc < r; j++)
        if (d->have[k + j]) repairs[rc++] = j;
    if (rc != r) {
        free(missing), free(present), free(repairs);
        return oerr(err, SCRS_DECODE_INSUFFICIENT_RANK, d->distinct, k);
    }
    for (size_t i = 0; i < r; i++) memset(out + missing[i] * L, 0, L);
    for (size_t i = 0; i < pc; i++) memcpy(out + present[i] * L, d->payloads + present[i] * L, L);
    if (r) {
        if (gf16) {
            uint16_t* rowv = (uint16_t*)malloc(r * 2), *colv = (uint16_t*)malloc(r * 2);
            uint16_t* presv = (uint16_t*)malloc((pc + 1) * 2);
            uint16_t* inv = (uint16_t*)malloc(r * r * 2), *pres = (uint16_t*)malloc((pc * r + 1) * 2);
            for (size_t t = 0; t < r; t++) rowv[t] = gf16_pow(GF16_GENERATOR, (uint32_t)(k + repairs[t]));
            for (size_t s = 0; s < r; s++) colv[s] = gf16_pow(GF16_GENERATOR, (uint32_t)missing[s]);
            for (size_t q = 0; q < pc; q++) presv[q] = gf16_pow(GF16_GENERATOR, (uint32_t)present[q]);
            gf16_rational_lagrange(rowv, colv, r, presv, pc, inv, pres);
            for (size_t s = 0; s < r; s++) {
                uint8_t* dst = out + missing[s] * L;
                for (size_t t = 0; t < r; t++)
                    pl16_xor_scaled(dst, inv[s * r + t], d->payloads + (k + repairs[t]) * L, L);
                for (size_t q = 0; q < pc; q++)
                    pl16_xor_scaled(dst, pres[q * r + s], d->payloads + present[q] * L, L);
            }
            free(rowv), free(colv), free(presv), free(inv), free(pres);
        } else {
            uint8_t* rowv = (uint8_t*)malloc(r), *colv = (uint8_t*)malloc(r), *presv = (uint8_t*)malloc(pc + 1);
            uint8_t* inv = (uint8_t*)malloc(r * r), *pres = (uint8_t*)malloc(pc * r + 1);
            for (size_t t = 0; t < r; t++) rowv[t] = gf8_y_var(d->p.engine, k, repairs[t]);
            for (size_t s = 0; s < r; s++) colv[s] = gf8_x_var(d->p.engine, k, missing[s]);
            for (size_t q = 0; q < pc; q++) presv[q] = gf8_x_var(d->p.engine, k, present[q]);
            gf8_rational_lagrange(rowv, colv, r, presv, pc, inv, pres);
            for (size_t s = 0; s < r; s++) {
                uint8_t* dst = out + missing[s] * L;
                for (size_t t = 0; t < r; t++)
                    pl8_xor_scaled(dst, inv[s * r + t], d->payloads + (k + repairs[t]) * L, L);
                for (size_t q = 0; q < pc; q++)
                    pl8_xor_scaled(dst, pres[q * r + s], d->payloads + present[q] * L, L);
            }
            free(rowv), free(colv), free(presv), free(inv), free(pres);
        }
    }
    free(missing), free(present), free(repairs);
    return oerr(err, SCRS_OK, 0, 0);
}

static int32_t finalize_core(oracle_decoder* d, uint8_t* out, uint64_t out_len,
                             oracle_decode_scratch* s, scrs_error* err) {
    uint64_t k = d->p.k, L = d->p.symbol_len;
    /* ensure_complete then output length (streaming.rs:495-502,
     * tower/decoder.rs:205-212, afft/decoder.rs:560-567) */
    if (d->distinct < k) return oerr(err, SCRS_DECODE_INSUFFICIENT_RANK, d->distinct, k);
    if (out_len != k * L) return oerr(err, SCRS_DECODE_WRONG_OUTPUT_LEN, k * L, out_len);
    if (!out) return oerr(err, SCRS_ERR_NULL_ARGUMENT, 0, 0);
    if (s) {
        int want = decode_scratch_kind(d->p.engine);
        if (s->kind != want) return oerr(err, SCRS_DECODE_SCRATCH_MISMATCH, 0, 0); /* selector.rs:239 */
        if (want != SK_CAUCHY_RECIPE &&
            (s->p.k != d->p.k || s->p.m != d->p.m || s->p.symbol_len != d->p.symbol_len))
            return oerr(err, SCRS_DECODE_SCRATCH_MISMATCH, 0, 0); /* tower/decoder.rs:219, afft/decoder.rs:244 */
    }
    if (d->p.engine == SCRS_ENGINE_AFFT) {
        afft_finalize(&d->afft, d->have, d->payloads, out);
        return oerr(err, SCRS_OK, 0, 0);
    }
    return cauchy_finalize(d, out, err);
}

int32_t oracle_dec_finalize_into(oracle_decoder* d, uint8_t* out, uint64_t out_len, scrs_error* err) {
    if (!d) return oerr(err, SCRS_ERR_NULL_ARGUMENT, 0, 0);
    return finalize_core(d, out, out_len, NULL, err);
}

int32_t oracle_dec_finalize_into_with(oracle_decoder* d, uint8_t* out, uint64_t out_len,
                                      oracle_decode_scratch* s, scrs_error* err) {
    if (!d || !s) return oerr(err, SCRS_ERR_NULL_ARGUMENT, 0, 0);
    return finalize_core(d, out, out_len, s, err);
}

/* ---- BatchDecoder --------------------------------------------------------- */
struct oracle_batch_decoder {
    scrs_profile p;
    uint8_t* coeffs8;       /* GF(256) BatchCodec */
    oracle_decoder* lazy;   /* Tower / AFFT via the blanket impl (codec.rs:203-239) */
};

int32_t oracle_batch_decoder_create(const scrs_profile* p, oracle_batch_decoder** out,
                                    scrs_error* err) {
    int32_t st = check_profile(p, err);
    if (st) return st;
    if (!out) return oerr(err, SCRS_ERR_NULL_ARGUMENT, 0, 0);
    oracle_batch_decoder* b = (oracle_batch_decoder*)calloc(1, sizeof *b);
    b->p = *p;
    if (is_gf16(p->engine)) {
        st = oracle_decoder_create(p, &b->lazy, err);
        if (st) {
            free(b);
            return st;
        }
    } else {
        b->coeffs8 = (uint8_t*)malloc(p->k * p->m);
        gf8_coefficient_matrix(p->engine, p->k, p->m, b->coeffs8);
    }
    *out = b;
    return oerr(err, SCRS_OK, 0, 0);
}

void oracle_batch_decoder_destroy(oracle_batch_decoder* b) {
    if (!b) return;
    oracle_decoder_destroy(b->lazy);
    free(b->coeffs8);
    free(b);
}

int32_t oracle_batch_decoder_profile(const oracle_batch_decoder* b, scrs_profile* out) {
    if (!b || !out) return SCRS_ERR_NULL_ARGUMENT;
    *out = b->p;
    return SCRS_OK;
}

int32_t oracle_batch_decoder_scratch(const oracle_batch_decoder* b, oracle_batch_decode_scratch** out,
                                     scrs_error* err) {
    if (!b || !out) return oerr(err, SCRS_ERR_NULL_ARGUMENT, 0, 0);
    oracle_batch_decode_scratch* s = (oracle_batch_decode_scratch*)calloc(1, sizeof *s);
    s->kind = is_gf16(b->p.engine) ? decode_scratch_kind(b->p.engine) : SK_CAUCHY_BATCH;
    s->p = b->p;
    *out = s;
    return oerr(err, SCRS_OK, 0, 0);
}
void oracle_batch_decode_scratch_destroy(oracle_batch_decode_scratch* s) { free(s); }

/* scrs/src/batch/codec.rs:278-406 */
static int32_t gf8_batch_decode(const oracle_batch_decoder* b, const uint64_t* idx,
                                const uint8_t* const* pay, const uint64_t* lens, uint64_t count,
                                uint8_t* out, uint64_t out_len, const oracle_batch_decode_scratch* s,
                                scrs_error* err) {
    uint64_t k = b->p.k, m = b->p.m, n = k + m, L = b->p.symbol_len;
    if (s->kind != SK_CAUCHY_BATCH || s->p.k != k || s->p.m != m || s->p.symbol_len != L)
        return oerr(err, SCRS_DECODE_SCRATCH_MISMATCH, 0, 0);
    if (out_len != k * L) return oerr(err, SCRS_DECODE_WRONG_OUTPUT_LEN, k * L, out_len);
    if (count != k) return oerr(err, SCRS_DECODE_WRONG_COUNT, k, count);
    if (!out || (count && (!idx || !pay || !lens))) return oerr(err, SCRS_ERR_NULL_ARGUMENT, 0, 0);
    uint8_t seen[256] = {0};
    size_t max_e = k < m ? k : m;
    uint8_t* work = (uint8_t*)malloc(max_e * L + 1);
    size_t* repair_cols = (size_t*)malloc((max_e + 1) * sizeof(size_t));
    size_t e = 0;
    int32_t st = SCRS_OK;
    for (uint64_t q = 0; q < count; q++) {
        uint64_t i = idx[q];
        if (i >= n) { st = oerr(err, SCRS_DECODE_INDEX_OUT_OF_RANGE, i, n); goto done; }
        if (seen[i]) { st = oerr(err, SCRS_DECODE_DUPLICATE_INDEX, i, 0); goto done; }
        seen[i] = 1;
        if (lens[q] != L) { st = oerr(err, SCRS_DECODE_WRONG_PAYLOAD_LEN, L, lens[q]); goto done; }
        if (i < k) {
            memcpy(out + i * L, pay[q], L);
        } else {
            repair_cols[e] = i - k;
            memcpy(work + e * L, pay[q], L);
            e++;
        }
    }
    if (e) {
        size_t* missing = (size_t*)malloc(e * sizeof(size_t));
        size_t mc = 0;
        for (size_t i = 0; i < k; i++)
            if (!seen[i]) missing[mc++] = i;
        /* subtract present data from the received repairs (codec.rs:346-380) */
        for (uint64_t q = 0; q < count; q++) {
            if (idx[q] >= k) continue;
            for (size_t t = 0; t < e; t++)
                pl8_xor_scaled(work + t * L, b->coeffs8[idx[q] * m + repair_cols[t]], pay[q], L);
        }
        uint8_t* B = (uint8_t*)malloc(e * e), *Binv = (uint8_t*)malloc(e * e);
        for (size_t t = 0; t < e; t++)
            for (size_t s2 = 0; s2 < e; s2++) B[t * e + s2] = b->coeffs8[missing[s2] * m + repair_cols[t]];
        if (!gf8_invert_square(B, e, Binv)) {
            st = oerr(err, SCRS_DECODE_INSUFFICIENT_RANK, e - 1, e);
        } else {
            for (size_t s2 = 0; s2 < e; s2++) {
                uint8_t* dst = out + missing[s2] * L;
                memset(dst, 0, L);
                for (size_t t = 0; t < e; t++) pl8_xor_scaled(dst, Binv[s2 * e + t], work + t * L, L);
            }
        }
        free(B), free(Binv), free(missing);
    }
    if (st == SCRS_OK) oerr(err, SCRS_OK, 0, 0);
done:
    free(work);
    free(repair_cols);
    return st;
}

/* Tower/AFFT: the blanket BatchDecoder impl (scrs/src/codec.rs:219-238). */
static int32_t lazy_batch_decode(oracle_batch_decoder* b, const uint64_t* idx,
                                 const uint8_t* const* pay, const uint64_t* lens, uint64_t count,
                                 uint8_t* out, uint64_t out_len, oracle_batch_decode_scratch* s,
                                 scrs_error* err) {
    if (count != b->p.k) return oerr(err, SCRS_DECODE_WRONG_COUNT, b->p.k, count);
    if (count && (!idx || !pay || !lens)) return oerr(err, SCRS_ERR_NULL_ARGUMENT, 0, 0);
    oracle_dec_reset(b->lazy);
    for (uint64_t q = 0; q < count; q++) {
        scrs_push_outcome o;
        int32_t st = oracle_dec_push(b->lazy, idx[q], pay[q], lens[q], &o, err);
        if (st) return st;
        if (o.kind == SCRS_PUSH_DEPENDENT) return oerr(err, SCRS_DECODE_DUPLICATE_INDEX, idx[q], 0);
    }
    oracle_decode_scratch ds = {s->kind, s->p};
    return finalize_core(b->lazy, out, out_len, &ds, err);
}

int32_t oracle_batch_decode_into_with(oracle_batch_decoder* b, const uint64_t* idx,
                                      const uint8_t* const* pay, const uint64_t* lens,
                                      uint64_t count, uint8_t* out, uint64_t out_len,
                                      oracle_batch_decode_scratch* s, scrs_error* err) {
    if (!b || !s) return oerr(err, SCRS_ERR_NULL_ARGUMENT, 0, 0);
    if (is_gf16(b->p.engine)) {
        if (s->kind != decode_scratch_kind(b->p.engine)) return oerr(err, SCRS_DECODE_SCRATCH_MISMATCH, 0, 0);
        return lazy_batch_decode(b, idx, pay, lens, count, out, out_len, s, err);
    }
    if (s->kind != SK_CAUCHY_BATCH) return oerr(err, SCRS_DECODE_SCRATCH_MISMATCH, 0, 0);
    return gf8_batch_decode(b, idx, pay, lens, count, out, out_len, s, err);
}

int32_t oracle_batch_decode_into(oracle_batch_decoder* b, const uint64_t* idx,
                                 const uint8_t* const* pay, const uint64_t* lens, uint64_t count,
                                 uint8_t* out, uint64_t out_len, scrs_error* err) {
    oracle_batch_decode_scratch* s = NULL;
    int32_t st = oracle_batch_decoder_scratch(b, &s, err);
    if (st) return st;
    st = oracle_batch_decode_into_with(b, idx, pay, lens, count, out, out_len, s, err);
    free(s);
    return st;
}

/* ---- IncrementalEncoder: encoder/streaming.rs:94-254, tower/encoder.rs ---- */
struct oracle_incremental_encoder {
    scrs_profile p;
    uint8_t* coeffs8;
    uint16_t* coeffs16;
    uint8_t* repairs;
    uint8_t* fed;
    uint64_t fed_count;
};

int32_t oracle_incremental_encoder_create(const scrs_profile* p, oracle_incremental_encoder** out,
                                          scrs_error* err) {
    int32_t st = check_profile(p, err);
    if (st) return st;
    if (!out) return oerr(err, SCRS_ERR_NULL_ARGUMENT, 0, 0);
    if (p->engine != SCRS_ENGINE_GOOD_CAUCHY && p->engine != SCRS_ENGINE_TOWER)
        return oerr(err, SCRS_CONFIG_UNSUPPORTED_MODE, (uint64_t)p->engine, 0); /* selector.rs:379 */
    oracle_incremental_encoder* e = (oracle_incremental_encoder*)calloc(1, sizeof *e);
    e->p = *p;
    if (p->engine == SCRS_ENGINE_TOWER) {
        e->coeffs16 = tower_coefficient_matrix(p->k, p->m);
    } else {
        e->coeffs8 = (uint8_t*)malloc(p->k * p->m);
        gf8_coefficient_matrix(p->engine, p->k, p->m, e->coeffs8);
    }
    e->repairs = (uint8_t*)calloc(p->m * p->symbol_len, 1);
    e->fed = (uint8_t*)calloc(p->k, 1);
    *out = e;
    return oerr(err, SCRS_OK, 0, 0);
}

void oracle_incremental_encoder_destroy(oracle_incremental_encoder* e) {
    if (!e) return;
    free(e->coeffs8), free(e->coeffs16), free(e->repairs), free(e->fed), free(e);
}

int32_t oracle_incremental_encoder_profile(const oracle_incremental_encoder* e, scrs_profile* out) {
    if (!e || !out) return SCRS_ERR_NULL_ARGUMENT;
    *out = e->p;
    return SCRS_OK;
}

/* encoder/streaming.rs:162-190, tower/encoder.rs:89-116 */
int32_t oracle_inc_feed(oracle_incremental_encoder* e, uint64_t idx, const uint8_t* data,
                        uint64_t len, scrs_error* err) {
    if (!e) return oerr(err, SCRS_ERR_NULL_ARGUMENT, 0, 0);
    uint64_t k = e->p.k, m = e->p.m, L = e->p.symbol_len;
    if (idx >= k) return oerr(err, SCRS_ENCODE_INDEX_OUT_OF_RANGE, idx, k + m);
    if (len != L) return oerr(err, SCRS_ENCODE_WRONG_PAYLOAD_LEN, L, len);
    if (e->fed[idx]) return oerr(err, SCRS_ENCODE_DUPLICATE_DATA, idx, 0);
    if (!data) return oerr(err, SCRS_ERR_NULL_ARGUMENT, 0, 0);
    e->fed[idx] = 1;
    e->fed_count++;
    for (uint64_t j = 0; j < m; j++) {
        if (e->coeffs16) pl16_xor_scaled(e->repairs + j * L, e->coeffs16[idx * m + j], data, L);
        else pl8_xor_scaled(e->repairs + j * L, e->coeffs8[idx * m + j], data, L);
    }
    return oerr(err, SCRS_OK, 0, 0);
}

/* encoder/streaming.rs:197-206, tower/encoder.rs:122-131 */
int32_t oracle_inc_repair(const oracle_incremental_encoder* e, uint64_t idx, uint8_t* dst,
                          uint64_t dst_len, scrs_error* err) {
    if (!e) return oerr(err, SCRS_ERR_NULL_ARGUMENT, 0, 0);
    uint64_t k = e->p.k, m = e->p.m, L = e->p.symbol_len;
    if (idx >= m) return oerr(err, SCRS_ENCODE_INDEX_OUT_OF_RANGE, idx, k + m);
    if (dst_len != L) return oerr(err, SCRS_ENCODE_WRONG_OUTPUT_LEN, L, dst_len);
    if (!dst) return oerr(err, SCRS_ERR_NULL_ARGUMENT, 0, 0);
    memcpy(dst, e->repairs + idx * L, L);
    return oerr(err, SCRS_OK, 0, 0);
}

uint64_t oracle_inc_fed_count(const oracle_incremental_encoder* e) { return e ? e->fed_count : 0; }
void oracle_inc_reset(oracle_incremental_encoder* e) {
    if (!e) return;
    memset(e->repairs, 0, e->p.m * e->p.symbol_len);
    memset(e->fed, 0, e->p.k);
    e->fed_count = 0;
}
