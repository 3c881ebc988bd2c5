/*
 * Test infrastructure (oracle): probes used by the tests to pin the
 * restatement against the reference's known answers, and the threaded CPU
 * baseline used by bench.py.
 */
#include <pthread.h>
#include <unistd.h>
#include <stdlib.h>
#include <time.h>

#include "oracle_afft.h"
#include "scrs_oracle.h"

uint8_t oracle_gf256_mul(uint8_t a, uint8_t b) { oracle_tables_init(); return gf8_mul(a, b); }
uint8_t oracle_gf256_mul_xtime(uint8_t a, uint8_t b) { return gf8_mul_xtime(a, b); }
uint8_t oracle_gf256_inv(uint8_t a) { oracle_tables_init(); return gf8_inv(a); }
uint8_t oracle_gf256_inv_xtime(uint8_t a) { return gf8_inv_xtime(a); }
uint8_t oracle_gf256_exp(uint32_t i) { oracle_tables_init(); return g_gf8_exp[i % 255]; }
uint16_t oracle_gf65536_mul(uint16_t a, uint16_t b) { oracle_tables_init(); return gf16_mul(a, b); }
uint16_t oracle_gf65536_square(uint16_t a) { oracle_tables_init(); return gf16_square(a); }
uint16_t oracle_gf65536_inv(uint16_t a) { oracle_tables_init(); return gf16_inv(a); }
uint16_t oracle_gf65536_pow(uint16_t a, uint32_t e) { oracle_tables_init(); return gf16_pow(a, e); }

void oracle_gf256_coefficient_matrix(int32_t engine, uint64_t k, uint64_t m, uint8_t* out) {
    gf8_coefficient_matrix(engine, k, m, out);
}

int32_t oracle_tower_coefficient_matrix(uint64_t k, uint64_t m, uint16_t* out) {
    uint16_t* c = tower_coefficient_matrix(k, m);
    if (!c) return SCRS_ERR_OUT_OF_MEMORY;
    memcpy(out, c, k * m * sizeof(uint16_t));
    free(c);
    return SCRS_OK;
}

int32_t oracle_afft_plan_factors(uint64_t size, uint16_t* factors, uint16_t* derivative_factors) {
    afft_plan p;
    if (!afft_plan_init(&p, size)) return SCRS_ERR_BAD_ARGUMENT;
    memcpy(factors, p.factors, size * sizeof(uint16_t));
    memcpy(derivative_factors, p.derivative_factors, p.log_size * sizeof(uint16_t));
    afft_plan_free(&p);
    return SCRS_OK;
}

int32_t oracle_afft_forward(uint64_t size, uint16_t* values) {
    afft_plan p;
    if (!afft_plan_init(&p, size)) return SCRS_ERR_BAD_ARGUMENT;
    afft_forward(&p, values);
    afft_plan_free(&p);
    return SCRS_OK;
}

int32_t oracle_afft_inverse(uint64_t size, uint16_t* values) {
    afft_plan p;
    if (!afft_plan_init(&p, size)) return SCRS_ERR_BAD_ARGUMENT;
    afft_inverse(&p, values);
    afft_plan_free(&p);
    return SCRS_OK;
}

int32_t oracle_afft_forward_bytes(uint64_t size, uint8_t* rows, uint64_t L) {
    afft_plan p;
    if (!afft_plan_init(&p, size)) return SCRS_ERR_BAD_ARGUMENT;
    afft_forward_bytes(&p, rows, L);
    afft_plan_free(&p);
    return SCRS_OK;
}

int32_t oracle_afft_forward_bytes_trunc_range(uint64_t size, uint8_t* rows, uint64_t L,
                                              uint64_t active, uint64_t start, uint64_t end) {
    afft_plan p;
    if (!afft_plan_init(&p, size)) return SCRS_ERR_BAD_ARGUMENT;
    afft_forward_bytes_trunc_range(&p, rows, L, active, start, end);
    afft_plan_free(&p);
    return SCRS_OK;
}

int32_t oracle_afft_inverse_truncated_bytes(uint64_t size, uint8_t* rows, uint64_t L,
                                            uint64_t active) {
    afft_plan p;
    if (!afft_plan_init(&p, size)) return SCRS_ERR_BAD_ARGUMENT;
    afft_inverse_truncated_bytes(&p, rows, L, active);
    afft_plan_free(&p);
    return SCRS_OK;
}

int32_t oracle_afft_encode_blocked(uint64_t k, uint64_t m, uint64_t L, const uint8_t* data,
                                   uint8_t* repairs, uint64_t width, int32_t fused) {
    afft_profile p;
    if (!afft_profile_init(&p, k, m, L)) return SCRS_ERR_BAD_ARGUMENT;
    afft_encode_blocked(&p, data, repairs, width, fused);
    afft_profile_free(&p);
    return SCRS_OK;
}

void oracle_afft_locator(const uint8_t* known, uint64_t ts, uint16_t* values, uint16_t* derivs) {
    afft_locator_evaluations(known, ts, values, derivs);
}

/* ---- CPU baseline --------------------------------------------------------- */
static double now_s(void) {
    struct timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return (double)t.tv_sec + 1e-9 * (double)t.tv_nsec;
}

int32_t oracle_baseline_threads(void) {
    long n = sysconf(_SC_NPROCESSORS_ONLN);
    return n > 0 ? (int32_t)n : 1;
}

typedef struct {
    int32_t engine, decode;
    uint64_t k, m, L, begin, end;
    const uint8_t* in;
    const uint16_t* indices;
    uint8_t* out;
} baseline_job;

/* One codec per thread; the reference is single-threaded per codec, so
 * independent stripes are spread over host threads. */
static void* baseline_worker(void* arg) {
    baseline_job* j = (baseline_job*)arg;
    scrs_profile p = {j->engine, 0, j->k, j->m, j->L};
    uint64_t k = j->k, m = j->m, L = j->L;
    if (!j->decode) {
        oracle_batch_encoder* e = NULL;
        oracle_encode_scratch* s = NULL;
        oracle_batch_encoder_create(&p, &e, NULL);
        oracle_batch_encoder_scratch(e, &s, NULL);
        for (uint64_t i = j->begin; i < j->end; i++)
            oracle_batch_encode_into_with(e, j->in + i * k * L, k * L, j->out + i * m * L, m * L, s, NULL);
        oracle_encode_scratch_destroy(s);
        oracle_batch_encoder_destroy(e);
        return NULL;
    }
    oracle_batch_decoder* d = NULL;
    oracle_batch_decode_scratch* s = NULL;
    oracle_batch_decoder_create(&p, &d, NULL);
    oracle_batch_decoder_scratch(d, &s, NULL);
    uint64_t* idx = (uint64_t*)malloc(k * sizeof(uint64_t));
    const uint8_t** pay = (const uint8_t**)malloc(k * sizeof(uint8_t*));
    uint64_t* lens = (uint64_t*)malloc(k * sizeof(uint64_t));
    for (uint64_t i = j->begin; i < j->end; i++) {
        for (uint64_t q = 0; q < k; q++) {
            idx[q] = j->indices[i * k + q];
            pay[q] = j->in + (i * k + q) * L;
            lens[q] = L;
        }
        oracle_batch_decode_into_with(d, idx, pay, lens, k, j->out + i * k * L, k * L, s, NULL);
    }
    free(idx), free(pay), free(lens);
    oracle_batch_decode_scratch_destroy(s);
    oracle_batch_decoder_destroy(d);
    return NULL;
}

static double run_baseline(baseline_job tmpl, uint64_t count, int32_t threads) {
    if (threads < 1) threads = 1;
    if ((uint64_t)threads > count) threads = count ? (int32_t)count : 1;
    pthread_t* tids = (pthread_t*)malloc((size_t)threads * sizeof(pthread_t));
    baseline_job* jobs = (baseline_job*)malloc((size_t)threads * sizeof(baseline_job));
    oracle_tables_init();
    double t0 = now_s();
    for (int32_t t = 0; t < threads; t++) {
        jobs[t] = tmpl;
        jobs[t].begin = count * (uint64_t)t / (uint64_t)threads;
        jobs[t].end = count * (uint64_t)(t + 1) / (uint64_t)threads;
        pthread_create(&tids[t], NULL, baseline_worker, &jobs[t]);
    }
    for (int32_t t = 0; t < threads; t++) pthread_join(tids[t], NULL);
    double dt = now_s() - t0;
    free(tids);
    free(jobs);
    return dt;
}

double oracle_baseline_gf256_encode(int32_t engine, uint64_t k, uint64_t m, uint64_t L,
                                    const uint8_t* in, uint8_t* out, uint64_t count,
                                    int32_t threads) {
    baseline_job j = {engine, 0, k, m, L, 0, 0, in, NULL, out};
    return run_baseline(j, count, threads);
}

double oracle_baseline_gf256_decode(int32_t engine, uint64_t k, uint64_t m, uint64_t L,
                                    const uint8_t* in, const uint16_t* indices, uint8_t* out,
                                    uint64_t count, int32_t threads) {
    baseline_job j = {engine, 1, k, m, L, 0, 0, in, indices, out};
    return run_baseline(j, count, threads);
}

/* ---- CPU baseline over stripes of any engine and geometry ----------------- */
/* Each thread takes a contiguous range of the descriptors (the caller sorts
 * them by geometry so a thread rebuilds its codecs rarely) and runs them one
 * by one through the reference's own per-engine entry points: batch encode
 * (GF(256), AFFT) or k in-order feeds and m repair reads (tower,
 * tower/encoder.rs:89-131), and batch decode (every engine; the GF(65536)
 * engines through the lazy decoder, codec.rs:203-239). */
typedef struct {
    const scrs_stripe_desc* d;
    uint64_t begin, end;
    int32_t failed;
} stripes_job;

static int same_geometry(const scrs_stripe_desc* a, const scrs_stripe_desc* b) {
    return a->op == b->op && a->engine == b->engine && a->k == b->k && a->m == b->m &&
           a->symbol_len == b->symbol_len;
}

static void* stripes_worker(void* arg) {
    stripes_job* j = (stripes_job*)arg;
    const scrs_stripe_desc* cur = NULL;
    oracle_batch_encoder* be = NULL;
    oracle_encode_scratch* bes = NULL;
    oracle_incremental_encoder* ie = NULL;
    oracle_batch_decoder* bd = NULL;
    oracle_batch_decode_scratch* bds = NULL;
    uint64_t *idx = NULL, *lens = NULL;
    const uint8_t** pay = NULL;
    uint64_t cap = 0;
    for (uint64_t i = j->begin; i < j->end && !j->failed; i++) {
        const scrs_stripe_desc* d = &j->d[i];
        const uint64_t k = d->k, m = d->m, L = d->symbol_len;
        if (!cur || !same_geometry(cur, d)) {
            oracle_encode_scratch_destroy(bes), bes = NULL;
            oracle_batch_encoder_destroy(be), be = NULL;
            oracle_incremental_encoder_destroy(ie), ie = NULL;
            oracle_batch_decode_scratch_destroy(bds), bds = NULL;
            oracle_batch_decoder_destroy(bd), bd = NULL;
            scrs_profile p = {d->engine, 0, k, m, L};
            int32_t rc;
            if (d->op == SCRS_OP_DECODE) {
                rc = oracle_batch_decoder_create(&p, &bd, NULL);
                if (!rc) rc = oracle_batch_decoder_scratch(bd, &bds, NULL);
            } else if (d->engine == SCRS_ENGINE_TOWER) {
                rc = oracle_incremental_encoder_create(&p, &ie, NULL);
            } else {
                rc = oracle_batch_encoder_create(&p, &be, NULL);
                if (!rc) rc = oracle_batch_encoder_scratch(be, &bes, NULL);
            }
            if (rc) {
                j->failed = rc;
                break;
            }
            cur = d;
        }
        int32_t rc = SCRS_OK;
        if (d->op == SCRS_OP_DECODE) {
            if (k > cap) {
                free(idx), free(lens), free((void*)pay);
                cap = k;
                idx = (uint64_t*)malloc(k * sizeof(uint64_t));
                lens = (uint64_t*)malloc(k * sizeof(uint64_t));
                pay = (const uint8_t**)malloc(k * sizeof(uint8_t*));
            }
            for (uint64_t q = 0; q < k; q++) {
                idx[q] = d->indices[q];
                pay[q] = d->in + q * L;
                lens[q] = L;
            }
            rc = oracle_batch_decode_into_with(bd, idx, pay, lens, k, d->out, k * L, bds, NULL);
        } else if (ie) {
            oracle_inc_reset(ie);
            for (uint64_t q = 0; q < k && !rc; q++) rc = oracle_inc_feed(ie, q, d->in + q * L, L, NULL);
            for (uint64_t r = 0; r < m && !rc; r++) rc = oracle_inc_repair(ie, r, d->out + r * L, L, NULL);
        } else {
            rc = oracle_batch_encode_into_with(be, d->in, k * L, d->out, m * L, bes, NULL);
        }
        if (rc) j->failed = rc;
    }
    free(idx), free(lens), free((void*)pay);
    oracle_encode_scratch_destroy(bes);
    oracle_batch_encoder_destroy(be);
    oracle_incremental_encoder_destroy(ie);
    oracle_batch_decode_scratch_destroy(bds);
    oracle_batch_decoder_destroy(bd);
    return NULL;
}

double oracle_baseline_stripes(const scrs_stripe_desc* descs, uint64_t count, int32_t threads,
                               int32_t* status) {
    if (threads < 1) threads = 1;
    if ((uint64_t)threads > count) threads = count ? (int32_t)count : 1;
    pthread_t* tids = (pthread_t*)malloc((size_t)threads * sizeof(pthread_t));
    stripes_job* jobs = (stripes_job*)calloc((size_t)threads, sizeof(stripes_job));
    oracle_tables_init();
    double t0 = now_s();
    for (int32_t t = 0; t < threads; t++) {
        jobs[t].d = descs;
        jobs[t].begin = count * (uint64_t)t / (uint64_t)threads;
        jobs[t].end = count * (uint64_t)(t + 1) / (uint64_t)threads;
        pthread_create(&tids[t], NULL, stripes_worker, &jobs[t]);
    }
    for (int32_t t = 0; t < threads; t++) pthread_join(tids[t], NULL);
    double dt = now_s() - t0;
    int32_t rc = 0;
    for (int32_t t = 0; t < threads && !rc; t++) rc = jobs[t].failed;
    if (status) *status = rc;
    free(tids);
    free(jobs);
    return dt;
}
