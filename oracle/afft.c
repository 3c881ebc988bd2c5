/*
 * Test infrastructure (oracle): the additive-FFT engine over GF(2^16),
 * restated from scrs/src/afft/{transform,encoder,decoder,profile}.rs.
 */
#include <pthread.h>
#include <stdlib.h>

#include "oracle_afft.h"

/* ---- TransformPlan: scrs/src/afft/transform.rs:30-61, :228-299 ---------- */

typedef struct {
    uint16_t coeffs[17]; /* coefficients of x^(2^j), low exponent first */
    size_t len;
    uint16_t normalizer_inverse;
} subspace_poly;

/* transform.rs:271-279 */
static uint16_t eval_linearized(const uint16_t* coeffs, size_t len, uint16_t value) {
    uint16_t power = value, result = 0;
    for (size_t i = 0; i < len; i++) {
        result ^= gf16_mul(coeffs[i], power);
        power = gf16_square(power);
    }
    return result;
}

/* transform.rs:235-243 */
static uint16_t poly_eval(const subspace_poly* p, uint16_t value) {
    return gf16_mul(eval_linearized(p->coeffs, p->len, value), p->normalizer_inverse);
}

/* transform.rs:246-269: W_0(x) = x, W_{i+1} = W_i^2 + W_i(beta_i) W_i. */
static void subspace_polynomials(size_t count, subspace_poly* out) {
    uint16_t coeffs[17] = {1};
    size_t len = 1;
    for (size_t dim = 0; dim < count; dim++) {
        uint16_t basis = (uint16_t)(1u << dim);
        uint16_t normalizer = eval_linearized(coeffs, len, basis);
        memcpy(out[dim].coeffs, coeffs, sizeof coeffs);
        out[dim].len = len;
        out[dim].normalizer_inverse = gf16_inv(normalizer);
        if (dim + 1 != count) {
            uint16_t next[17] = {0};
            for (size_t i = 0; i < len; i++) {
                next[i] ^= gf16_mul(normalizer, coeffs[i]);
                next[i + 1] ^= gf16_square(coeffs[i]);
            }
            memcpy(coeffs, next, sizeof next);
            len++;
        }
    }
}

/* transform.rs:281-299 — heap-indexed node factors, root = 1. */
static void fill_factors(uint16_t* factors, const subspace_poly* polys, size_t node,
                         size_t dim, uint16_t shift) {
    factors[node] = poly_eval(&polys[dim - 1], shift);
    if (dim > 1) {
        fill_factors(factors, polys, node * 2, dim - 1, shift);
        fill_factors(factors, polys, node * 2 + 1, dim - 1,
                     (uint16_t)(shift ^ (1u << (dim - 1))));
    }
}

/* transform.rs:41-61 */
int afft_plan_init(afft_plan* plan, size_t size) {
    memset(plan, 0, sizeof *plan);
    if (size == 0 || (size & (size - 1)) || size > AFFT_MAX_TRANSFORM_SIZE) return 0;
    oracle_tables_init();
    size_t log_size = 0;
    while (((size_t)1 << log_size) < size) log_size++;
    subspace_poly polys[16];
    subspace_polynomials(log_size, polys);
    plan->size = size;
    plan->log_size = log_size;
    plan->factors = (uint16_t*)calloc(size, sizeof(uint16_t));
    for (size_t j = 0; j < log_size; j++)
        plan->derivative_factors[j] = gf16_mul(polys[j].coeffs[0], polys[j].normalizer_inverse);
    if (log_size) fill_factors(plan->factors, polys, 1, log_size, 0);
    return 1;
}

void afft_plan_free(afft_plan* plan) {
    free(plan->factors);
    plan->factors = NULL;
}

/* ---- element-level transforms (transform.rs:75-91, :301-333) ------------ */
static void forward_node(uint16_t* v, size_t len, const uint16_t* f, size_t node, size_t dim) {
    size_t half = len / 2;
    uint16_t factor = f[node];
    for (size_t p = 0; p < half; p++) {
        uint16_t low = v[p], high = v[half + p];
        uint16_t left = low ^ gf16_mul(factor, high);
        v[p] = left;
        v[half + p] = left ^ high;
    }
    if (dim > 1) {
        forward_node(v, half, f, node * 2, dim - 1);
        forward_node(v + half, half, f, node * 2 + 1, dim - 1);
    }
}
static void inverse_node(uint16_t* v, size_t len, const uint16_t* f, size_t node, size_t dim) {
    size_t half = len / 2;
    if (dim > 1) {
        inverse_node(v, half, f, node * 2, dim - 1);
        inverse_node(v + half, half, f, node * 2 + 1, dim - 1);
    }
    uint16_t factor = f[node];
    for (size_t p = 0; p < half; p++) {
        uint16_t left = v[p], right = v[half + p];
        uint16_t high = left ^ right;
        v[p] = left ^ gf16_mul(factor, high);
        v[half + p] = high;
    }
}
void afft_forward(const afft_plan* plan, uint16_t* values) {
    if (plan->log_size) forward_node(values, plan->size, plan->factors, 1, plan->log_size);
}
void afft_inverse(const afft_plan* plan, uint16_t* values) {
    if (plan->log_size) inverse_node(values, plan->size, plan->factors, 1, plan->log_size);
}

/* ---- byte-row transforms (transform.rs:335-559) ------------------------- */
static void forward_bytes_node(uint8_t* rows, size_t nbytes, const uint16_t* f, size_t node,
                               size_t dim) {
    size_t half = nbytes / 2;
    pl16_fused_forward(rows, rows + half, f[node], half);
    if (dim > 1) {
        forward_bytes_node(rows, half, f, node * 2, dim - 1);
        forward_bytes_node(rows + half, half, f, node * 2 + 1, dim - 1);
    }
}

static void forward_bytes_range_node(uint8_t* rows, size_t nbytes, size_t L, const uint16_t* f,
                                     size_t node, size_t dim, size_t rs, size_t re) {
    size_t half = nbytes / 2, half_rows = half / L;
    pl16_fused_forward(rows, rows + half, f[node], half);
    if (dim <= 1) return;
    if (rs < half_rows)
        forward_bytes_range_node(rows, half, L, f, node * 2, dim - 1, rs, re < half_rows ? re : half_rows);
    if (re > half_rows)
        forward_bytes_range_node(rows + half, half, L, f, node * 2 + 1, dim - 1,
                                 rs > half_rows ? rs - half_rows : 0, re - half_rows);
}

/* transform.rs:387-478; rows active..end must be zero on entry. */
static void forward_bytes_trunc_range_node(uint8_t* rows, size_t nbytes, size_t L,
                                           const uint16_t* f, size_t node, size_t dim,
                                           size_t active, size_t rs, size_t re) {
    size_t half = nbytes / 2, half_rows = half / L;
    uint8_t* low = rows;
    uint8_t* high = rows + half;
    if (active <= half_rows) {
        if (dim <= 1) {
            if (re > half_rows) memcpy(high, low, active * L);
            return;
        }
        int need_low = rs < half_rows, need_high = re > half_rows;
        if (need_high) memcpy(high, low, active * L);
        if (need_low)
            forward_bytes_trunc_range_node(low, half, L, f, node * 2, dim - 1, active, rs,
                                           re < half_rows ? re : half_rows);
        if (need_high)
            forward_bytes_trunc_range_node(high, half, L, f, node * 2 + 1, dim - 1, active,
                                           rs > half_rows ? rs - half_rows : 0, re - half_rows);
        return;
    }
    pl16_fused_forward(low, high, f[node], half);
    if (dim <= 1) return;
    if (rs < half_rows)
        forward_bytes_trunc_range_node(low, half, L, f, node * 2, dim - 1, half_rows, rs,
                                       re < half_rows ? re : half_rows);
    if (re > half_rows)
        forward_bytes_trunc_range_node(high, half, L, f, node * 2 + 1, dim - 1, half_rows,
                                       rs > half_rows ? rs - half_rows : 0, re - half_rows);
}

static void inverse_bytes_node(uint8_t* rows, size_t nbytes, const uint16_t* f, size_t node,
                               size_t dim) {
    size_t half = nbytes / 2;
    if (dim > 1) {
        inverse_bytes_node(rows, half, f, node * 2, dim - 1);
        inverse_bytes_node(rows + half, half, f, node * 2 + 1, dim - 1);
    }
    pl16_fused_inverse(rows, rows + half, f[node], half);
}

/* transform.rs:480-548 */
static void inverse_truncated_bytes_node(uint8_t* rows, size_t nbytes, size_t L,
                                         const uint16_t* f, size_t node, size_t dim,
                                         size_t active) {
    size_t row_count = nbytes / L;
    if (row_count == 1) return;
    if (active == row_count) {
        inverse_bytes_node(rows, nbytes, f, node, dim);
        return;
    }
    size_t half_rows = row_count / 2, half = half_rows * L;
    uint8_t* low = rows;
    uint8_t* high = rows + half;
    if (active <= half_rows) {
        inverse_truncated_bytes_node(low, half, L, f, node * 2, dim - 1, active);
        return;
    }
    size_t right_active = active - half_rows;
    inverse_bytes_node(low, half, f, node * 2, dim - 1);
    uint8_t* known_tail = (uint8_t*)calloc(half, 1);
    size_t tail_start = right_active * L;
    memcpy(known_tail + tail_start, low + tail_start, half - tail_start);
    forward_bytes_range_node(known_tail, half, L, f, node * 2 + 1, dim - 1, 0, right_active);
    pl8_xor(high, known_tail, tail_start);
    free(known_tail);
    inverse_truncated_bytes_node(high, half, L, f, node * 2 + 1, dim - 1, right_active);
    pl16_fused_inverse(low, high, f[node], right_active * L);
}

void afft_forward_bytes(const afft_plan* p, uint8_t* rows, size_t L) {
    if (p->log_size) forward_bytes_node(rows, p->size * L, p->factors, 1, p->log_size);
}
void afft_inverse_bytes(const afft_plan* p, uint8_t* rows, size_t L) {
    if (p->log_size) inverse_bytes_node(rows, p->size * L, p->factors, 1, p->log_size);
}
/* transform.rs:109-132 */
void afft_forward_bytes_trunc_range(const afft_plan* p, uint8_t* rows, size_t L, size_t active,
                                    size_t rs, size_t re) {
    if (p->log_size && rs < re && active)
        forward_bytes_trunc_range_node(rows, p->size * L, L, p->factors, 1, p->log_size, active,
                                       rs, re);
}
/* transform.rs:142-165: subtree at node 3 over size/2 rows. */
void afft_forward_bytes_high_coset_range(const afft_plan* p, uint8_t* rows, size_t L, size_t rs,
                                         size_t re) {
    if (rs < re)
        forward_bytes_range_node(rows, (p->size / 2) * L, L, p->factors, 3, p->log_size - 1, rs,
                                 re);
}
/* transform.rs:174-186 */
void afft_inverse_truncated_bytes(const afft_plan* p, uint8_t* rows, size_t L, size_t active) {
    if (p->log_size)
        inverse_truncated_bytes_node(rows, p->size * L, L, p->factors, 1, p->log_size, active);
}
/* transform.rs:188-213: novel-basis formal derivative. */
void afft_derivative_bytes(const afft_plan* p, const uint8_t* coeffs, size_t L, uint8_t* deriv) {
    memset(deriv, 0, p->size * L);
    for (size_t index = 1; index < p->size; index++) {
        const uint8_t* src = coeffs + index * L;
        size_t remaining = index;
        while (remaining) {
            size_t bit = (size_t)__builtin_ctzll(remaining);
            size_t dst = index ^ ((size_t)1 << bit);
            pl16_xor_scaled(deriv + dst * L, p->derivative_factors[bit], src, L);
            remaining &= remaining - 1;
        }
    }
}

/* ---- Profile: scrs/src/afft/profile.rs:16-45 ---------------------------- */
static size_t next_pow2(size_t x) {
    size_t p = 1;
    while (p < x) p <<= 1;
    return p;
}
int afft_profile_init(afft_profile* pr, size_t k, size_t m, size_t L) {
    memset(pr, 0, sizeof *pr);
    if (k == 0 || m == 0 || L == 0 || (L & 1)) return 0;
    size_t n = k + m;
    if (n > AFFT_MAX_TRANSFORM_SIZE) return 0;
    pr->k = k, pr->m = m, pr->n = n, pr->L = L;
    pr->padded_k = next_pow2(k);
    pr->transform_size = next_pow2(n);
    if (!afft_plan_init(&pr->interp, pr->padded_k)) return 0;
    if (!afft_plan_init(&pr->transform, pr->transform_size)) {
        afft_plan_free(&pr->interp);
        return 0;
    }
    return 1;
}
void afft_profile_free(afft_profile* pr) {
    afft_plan_free(&pr->interp);
    afft_plan_free(&pr->transform);
}

/* ---- SystematicEncoder: scrs/src/afft/encoder.rs:25-36, :121-214 -------- */
#define STRIP_TARGET_BYTES (768u * 1024u)
static size_t strip_width(size_t rows_per_strip, size_t L) {
    size_t cap = (STRIP_TARGET_BYTES / rows_per_strip) & ~(size_t)1;
    if (cap < 2) cap = 2;
    return cap < L ? cap : L;
}

void afft_encode_blocked(const afft_profile* p, const uint8_t* data, uint8_t* repairs,
                         size_t width, int fused) {
    size_t L = p->L, k = p->k, n = p->n, m = p->m, pk = p->padded_k, ts = p->transform_size;
    size_t rows = fused ? pk : ts;
    uint8_t* strip = (uint8_t*)malloc(rows * width);
    for (size_t col = 0; col < L;) {
        size_t w = width < L - col ? width : L - col;
        for (size_t r = 0; r < k; r++) memcpy(strip + r * w, data + r * L + col, w);
        if (fused) {
            afft_inverse_truncated_bytes(&p->interp, strip, w, k);
            afft_forward_bytes_high_coset_range(&p->transform, strip, w, 0, m);
            for (size_t r = 0; r < m; r++) memcpy(repairs + r * L + col, strip + r * w, w);
        } else {
            memset(strip + k * w, 0, (ts - k) * w);
            afft_inverse_truncated_bytes(&p->interp, strip, w, k);
            afft_forward_bytes_trunc_range(&p->transform, strip, w, k, k, n);
            for (size_t r = k; r < n; r++) memcpy(repairs + (r - k) * L + col, strip + r * w, w);
        }
        col += w;
    }
    free(strip);
}

void afft_encode(const afft_profile* p, const uint8_t* data, uint8_t* repairs) {
    int fused = p->padded_k == p->k && p->transform_size == 2 * p->k && p->k >= 2;
    size_t rows = fused ? p->padded_k : p->transform_size;
    afft_encode_blocked(p, data, repairs, strip_width(rows, p->L), fused);
}

/* ---- decoder helpers: scrs/src/afft/decoder.rs:578-767 ------------------- */
#define MULT_ORDER 65535u
static uint16_t* g_log16;
static uint16_t* g_exp16;
static pthread_once_t g_log16_once = PTHREAD_ONCE_INIT;
static void build_log16(void) {
    oracle_tables_init();
    g_log16 = (uint16_t*)calloc(65536, sizeof(uint16_t));
    g_exp16 = (uint16_t*)calloc(65535, sizeof(uint16_t));
    uint16_t v = 1;
    for (uint32_t e = 0; e < MULT_ORDER; e++) {
        g_exp16[e] = v;
        g_log16[v] = (uint16_t)e;
        v = gf16_mul(v, GF16_GENERATOR);
    }
}
static void log16_init(void) { pthread_once(&g_log16_once, build_log16); }

/* decoder.rs:732-755 — Walsh-Hadamard transform with additions mod 65535. */
static void walsh_hadamard(uint32_t* v, size_t len) {
    for (size_t half = 1; half < len; half *= 2)
        for (size_t b = 0; b < len; b += 2 * half)
            for (size_t p = 0; p < half; p++) {
                uint32_t l = v[b + p], r = v[b + half + p];
                uint32_t s = l + r;
                v[b + p] = s >= MULT_ORDER ? s - MULT_ORDER : s;
                v[b + half + p] = l >= r ? l - r : l + MULT_ORDER - r;
            }
}
/* decoder.rs:757-767 */
static uint32_t mod_pow(uint32_t base, uint32_t e) {
    uint64_t r = 1, b = base;
    while (e) {
        if (e & 1) r = (r * b) % MULT_ORDER;
        b = (b * b) % MULT_ORDER;
        e >>= 1;
    }
    return (uint32_t)r;
}

/* decoder.rs:672-714 — locator L(x) = prod_{e erased}(x + e): values at known
 * points, derivatives L'(e) at erased points, via log-domain dyadic
 * convolution (log 0 is read as 0, which drops the e == x term). */
void afft_locator_evaluations(const uint8_t* known, size_t ts, uint16_t* values,
                              uint16_t* derivatives) {
    log16_init();
    uint32_t* ind = (uint32_t*)calloc(ts, sizeof(uint32_t));
    uint32_t* lg = (uint32_t*)calloc(ts, sizeof(uint32_t));
    for (size_t i = 0; i < ts; i++) {
        ind[i] = known[i] ? 0 : 1;
        lg[i] = g_log16[i];
    }
    walsh_hadamard(ind, ts);
    walsh_hadamard(lg, ts);
    for (size_t i = 0; i < ts; i++) ind[i] = (uint32_t)(((uint64_t)ind[i] * lg[i]) % MULT_ORDER);
    walsh_hadamard(ind, ts);
    size_t log_ts = (size_t)__builtin_ctzll(ts);
    uint32_t inv_size = mod_pow(32768, (uint32_t)log_ts);
    for (size_t i = 0; i < ts; i++) {
        uint32_t e = (uint32_t)(((uint64_t)ind[i] * inv_size) % MULT_ORDER);
        uint16_t prod = g_exp16[e];
        values[i] = known[i] ? prod : 0;
        derivatives[i] = known[i] ? 0 : prod;
    }
    free(ind);
    free(lg);
}

/* decoder.rs:600-617 — Lagrange generator row: coefficient of data point d
 * when evaluating at `evaluation` = L(eval) / ((eval + d) L'(d)). */
static void generator_row(size_t evaluation, const uint16_t* products, const uint16_t* derivs,
                          size_t k, uint16_t* row) {
    uint32_t num = g_log16[products[evaluation]];
    for (size_t d = 0; d < k; d++) {
        uint32_t diff = g_log16[evaluation ^ d];
        uint32_t dl = g_log16[derivs[d]];
        uint32_t e = (num + MULT_ORDER * 2 - diff - dl) % MULT_ORDER;
        row[d] = g_exp16[e];
    }
}

/* decoder.rs:619-670 — Gauss-Jordan on [A | I] over GF(65536). */
static int invert_square16(const uint16_t* a, size_t n, uint16_t* inv) {
    size_t stride = 2 * n;
    uint16_t* aug = (uint16_t*)calloc(n * stride, sizeof(uint16_t));
    for (size_t r = 0; r < n; r++) {
        memcpy(aug + r * stride, a + r * n, n * sizeof(uint16_t));
        aug[r * stride + n + r] = 1;
    }
    for (size_t c = 0; c < n; c++) {
        size_t pivot = n;
        for (size_t r = c; r < n; r++)
            if (aug[r * stride + c]) {
                pivot = r;
                break;
            }
        if (pivot == n) {
            free(aug);
            return 0;
        }
        if (pivot != c)
            for (size_t x = 0; x < stride; x++) {
                uint16_t t = aug[c * stride + x];
                aug[c * stride + x] = aug[pivot * stride + x];
                aug[pivot * stride + x] = t;
            }
        uint16_t pinv = gf16_inv(aug[c * stride + c]);
        for (size_t x = c; x < stride; x++) aug[c * stride + x] = gf16_mul(aug[c * stride + x], pinv);
        for (size_t r = 0; r < n; r++) {
            if (r == c) continue;
            uint16_t f = aug[r * stride + c];
            if (!f) continue;
            for (size_t x = c; x < stride; x++) aug[r * stride + x] ^= gf16_mul(f, aug[c * stride + x]);
        }
    }
    for (size_t r = 0; r < n; r++) memcpy(inv + r * n, aug + r * stride + n, n * sizeof(uint16_t));
    free(aug);
    return 1;
}

/* decoder.rs:256-267 — locator over the systematic set {0..k} (erased) with
 * every other transform point known; computed once per decoder. */
void afft_systematic_locator(const afft_profile* p, uint16_t* products, uint16_t* derivs) {
    uint8_t* known = (uint8_t*)malloc(p->transform_size);
    memset(known, 1, p->transform_size);
    memset(known, 0, p->k);
    afft_locator_evaluations(known, p->transform_size, products, derivs);
    free(known);
}

/* decoder.rs:269-441: reconstruct every systematic symbol from the k
 * received symbols marked in `have` (wire index order, payloads[n*L]).
 * Output must be k*L bytes. */
void afft_finalize(const afft_profile* p, const uint8_t* have, const uint8_t* payloads,
                   uint8_t* out) {
    log16_init();
    size_t L = p->L, k = p->k, n = p->n, ts = p->transform_size;
    size_t missing_count = 0;
    size_t* missing = (size_t*)malloc(k * sizeof(size_t));
    for (size_t d = 0; d < k; d++) {
        if (have[d]) {
            memcpy(out + d * L, payloads + d * L, L);
        } else {
            memset(out + d * L, 0, L);
            missing[missing_count++] = d;
        }
    }
    if (missing_count == 0) {
        free(missing);
        return;
    }
    if (missing_count <= AFFT_TARGETED_MAX_MISSING) {
        /* finalize_targeted_into, decoder.rs:360-441 */
        size_t r = missing_count;
        uint16_t* products = (uint16_t*)calloc(ts, sizeof(uint16_t));
        uint16_t* derivs = (uint16_t*)calloc(ts, sizeof(uint16_t));
        afft_systematic_locator(p, products, derivs);
        size_t repair_idx[AFFT_TARGETED_MAX_MISSING];
        size_t cnt = 0;
        for (size_t w = k; w < n && cnt < r; w++)
            if (have[w]) repair_idx[cnt++] = w;
        uint16_t* gen = (uint16_t*)malloc(r * k * sizeof(uint16_t));
        for (size_t row = 0; row < r; row++) generator_row(repair_idx[row], products, derivs, k, gen + row * k);
        uint16_t sys[AFFT_TARGETED_MAX_MISSING * AFFT_TARGETED_MAX_MISSING];
        uint16_t inv[AFFT_TARGETED_MAX_MISSING * AFFT_TARGETED_MAX_MISSING];
        for (size_t row = 0; row < r; row++)
            for (size_t c = 0; c < r; c++) sys[row * r + c] = gen[row * k + missing[c]];
        invert_square16(sys, r, inv);
        uint8_t* resid = (uint8_t*)malloc(r * L);
        uint8_t* rec = (uint8_t*)calloc(r * L, 1);
        for (size_t row = 0; row < r; row++) memcpy(resid + row * L, payloads + repair_idx[row] * L, L);
        for (size_t d = 0; d < k; d++) {
            if (!have[d]) continue;
            for (size_t row = 0; row < r; row++)
                pl16_xor_scaled(resid + row * L, gen[row * k + d], payloads + d * L, L);
        }
        for (size_t rr = 0; rr < r; rr++)
            for (size_t orow = 0; orow < r; orow++)
                pl16_xor_scaled(rec + orow * L, inv[orow * r + rr], resid + rr * L, L);
        for (size_t row = 0; row < r; row++) memcpy(out + missing[row] * L, rec + row * L, L);
        free(products), free(derivs), free(gen), free(resid), free(rec), free(missing);
        return;
    }
    /* complete path, decoder.rs:294-357 */
    uint8_t* known = (uint8_t*)calloc(ts, 1);
    for (size_t w = 0; w < n; w++)
        if (have[w]) known[w] = 1;
    uint16_t* values = (uint16_t*)calloc(ts, sizeof(uint16_t));
    uint16_t* derivs = (uint16_t*)calloc(ts, sizeof(uint16_t));
    afft_locator_evaluations(known, ts, values, derivs);
    uint8_t* work0 = (uint8_t*)calloc(ts * L, 1);
    uint8_t* work1 = (uint8_t*)calloc(ts * L, 1);
    for (size_t w = 0; w < n; w++)
        if (have[w]) pl16_xor_scaled(work0 + w * L, values[w], payloads + w * L, L);
    afft_inverse_bytes(&p->transform, work0, L);
    afft_derivative_bytes(&p->transform, work0, L, work1);
    afft_forward_bytes(&p->transform, work1, L);
    for (size_t i = 0; i < missing_count; i++) {
        size_t d = missing[i];
        pl16_xor_scaled(out + d * L, gf16_inv(derivs[d]), work1 + d * L, L);
    }
    free(known), free(values), free(derivs), free(work0), free(work1), free(missing);
}
