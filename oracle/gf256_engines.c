/*
 * Test infrastructure (oracle): GF(256) coefficient sets, the reduced
 * closed-form Cauchy solve and the Gauss-Jordan helpers, restated from the
 * SCRS reference.
 */
#include <stdlib.h>

#include "oracle_internal.h"

/* Standard Cauchy X = {0..k}, Y = {k..k+m} (scrs/src/matrices/cauchy.rs:87-95,
 * :151-157); Good Cauchy X = g^i, Y = g^(k+j) with g = 3 and exponents mod 255
 * (scrs/src/matrices/good_cauchy.rs:76-88, :195-201, :211-215). */
uint8_t gf8_x_var(int32_t engine, size_t k, size_t i) {
    (void)k;
    if (engine == SCRS_ENGINE_STANDARD_CAUCHY) return (uint8_t)i;
    return g_gf8_exp[i % 255];
}
uint8_t gf8_y_var(int32_t engine, size_t k, size_t j) {
    if (engine == SCRS_ENGINE_STANDARD_CAUCHY) return (uint8_t)(k + j);
    return g_gf8_exp[(k + j) % 255];
}

/* Coefficients in source-major order (coding_matrix.rs:40-49).
 * Standard: C[i][j] = inv(x_i + y_j)   (cauchy.rs:38-47, :98-101).
 * Good: diagonal factorization C[i][j] = g^-i * 1/(1 + g^(k+j-i))
 *       (good_cauchy.rs:125-144). */
void gf8_coefficient_matrix(int32_t engine, size_t k, size_t m, uint8_t* coeffs) {
    oracle_tables_init();
    if (engine == SCRS_ENGINE_STANDARD_CAUCHY) {
        for (size_t i = 0; i < k; i++)
            for (size_t j = 0; j < m; j++) {
                uint8_t denom = (uint8_t)i ^ (uint8_t)(k + j);
                coeffs[i * m + j] = denom ? gf8_inv(denom) : 0;
            }
        return;
    }
    size_t max_d = k + m - 1;
    uint8_t* base = (uint8_t*)calloc(max_d + 1, 1);
    for (size_t d = 1; d <= max_d; d++) base[d] = gf8_inv((uint8_t)(1 ^ g_gf8_exp[d % 255]));
    for (size_t i = 0; i < k; i++) {
        uint8_t scale = i == 0 ? 1 : gf8_inv(g_gf8_exp[i % 255]);
        for (size_t j = 0; j < m; j++) coeffs[i * m + j] = gf8_mul(scale, base[k + j - i]);
    }
    free(base);
}

/* scrs/src/decoder/cauchy_inverse.rs:50-212.  A[i][j] = 1/(row_i + col_j);
 * R_i = prod_h(row_i+col_h)/prod_{l!=i}(row_i+row_l);
 * C_j = prod_l(col_j+row_l)/prod_{h!=j}(col_j+col_h);
 * inverse[j][i] = R_i C_j / (col_j + row_i);
 * present[z][j] = C_j prod_{h!=j}(z+col_h) / prod_l(z+row_l).
 * The r <= 2 closed forms (:170-212) compute the same values. */
void gf8_rational_lagrange(const uint8_t* row, const uint8_t* col, size_t r,
                           const uint8_t* pres, size_t p, uint8_t* inverse,
                           uint8_t* present) {
    if (r == 0) return;
    uint8_t* rf = (uint8_t*)malloc(r);
    uint8_t* cf = (uint8_t*)malloc(r);
    for (size_t i = 0; i < r; i++) {
        uint8_t cross = 1, within = 1;
        for (size_t h = 0; h < r; h++) cross = gf8_mul(cross, row[i] ^ col[h]);
        for (size_t l = 0; l < r; l++)
            if (l != i) within = gf8_mul(within, row[i] ^ row[l]);
        rf[i] = gf8_mul(cross, gf8_inv(within));
    }
    for (size_t j = 0; j < r; j++) {
        uint8_t cross = 1, within = 1;
        for (size_t l = 0; l < r; l++) cross = gf8_mul(cross, col[j] ^ row[l]);
        for (size_t h = 0; h < r; h++)
            if (h != j) within = gf8_mul(within, col[j] ^ col[h]);
        cf[j] = gf8_mul(cross, gf8_inv(within));
    }
    for (size_t j = 0; j < r; j++)
        for (size_t i = 0; i < r; i++)
            inverse[j * r + i] = gf8_mul(gf8_mul(rf[i], cf[j]), gf8_inv(col[j] ^ row[i]));
    for (size_t z = 0; z < p; z++) {
        uint8_t rowprod = 1;
        for (size_t l = 0; l < r; l++) rowprod = gf8_mul(rowprod, pres[z] ^ row[l]);
        uint8_t rinv = gf8_inv(rowprod);
        for (size_t j = 0; j < r; j++) {
            uint8_t allbut = 1;
            for (size_t h = 0; h < r; h++)
                if (h != j) allbut = gf8_mul(allbut, pres[z] ^ col[h]);
            present[z * r + j] = gf8_mul(gf8_mul(cf[j], allbut), rinv);
        }
    }
    free(rf);
    free(cf);
}

/* scrs/src/batch/codec.rs:525-562 — Gauss-Jordan with partial pivoting on a
 * row-major e x e matrix (destroyed); returns 0 when singular. */
int gf8_invert_square(uint8_t* a, size_t e, uint8_t* inv) {
    memset(inv, 0, e * e);
    for (size_t i = 0; i < e; i++) inv[i * e + i] = 1;
    for (size_t col = 0; col < e; col++) {
        size_t pivot = e;
        for (size_t r = col; r < e; r++)
            if (a[r * e + col]) {
                pivot = r;
                break;
            }
        if (pivot == e) return 0;
        if (pivot != col)
            for (size_t c = 0; c < e; c++) {
                uint8_t t = a[col * e + c];
                a[col * e + c] = a[pivot * e + c];
                a[pivot * e + c] = t;
                t = inv[col * e + c];
                inv[col * e + c] = inv[pivot * e + c];
                inv[pivot * e + c] = t;
            }
        uint8_t scale = gf8_inv(a[col * e + col]);
        for (size_t c = 0; c < e; c++) {
            a[col * e + c] = gf8_mul(a[col * e + c], scale);
            inv[col * e + c] = gf8_mul(inv[col * e + c], scale);
        }
        for (size_t r = 0; r < e; r++) {
            if (r == col) continue;
            uint8_t f = a[r * e + col];
            if (!f) continue;
            for (size_t c = 0; c < e; c++) {
                a[r * e + c] ^= gf8_mul(f, a[col * e + c]);
                inv[r * e + c] ^= gf8_mul(f, inv[col * e + c]);
            }
        }
    }
    return 1;
}

/* Naive full-RREF decode used by the reference as the correctness oracle of
 * its fast decoder (scrs/src/batch/codec.rs:412-459 with
 * scrs/src/matrices/elimination.rs:39-63).  Returns the rank. */
size_t oracle_gf256_rref_decode(int32_t engine, size_t k, size_t m, size_t L,
                                const uint64_t* indices,
                                const uint8_t* const* payloads, uint8_t* out) {
    oracle_tables_init();
    size_t stride = k + L;
    uint8_t* coeffs = (uint8_t*)malloc(k * m);
    uint8_t* buf = (uint8_t*)calloc(k * stride, 1);
    gf8_coefficient_matrix(engine, k, m, coeffs);
    for (size_t row = 0; row < k; row++) {
        size_t idx = (size_t)indices[row];
        if (idx < k) {
            buf[row * stride + idx] = 1;
        } else {
            for (size_t col = 0; col < k; col++) buf[row * stride + col] = coeffs[col * m + (idx - k)];
        }
        memcpy(buf + row * stride + k, payloads[row], L);
    }
    size_t rank = 0;
    for (size_t c = 0; c < stride && rank < k; c++) {
        size_t pivot = k;
        for (size_t r = rank; r < k; r++)
            if (buf[r * stride + c]) {
                pivot = r;
                break;
            }
        if (pivot == k) continue;
        if (pivot != rank)
            for (size_t x = 0; x < stride; x++) {
                uint8_t t = buf[rank * stride + x];
                buf[rank * stride + x] = buf[pivot * stride + x];
                buf[pivot * stride + x] = t;
            }
        uint8_t pv = buf[rank * stride + c];
        if (pv != 1) {
            uint8_t iv = gf8_inv(pv);
            for (size_t x = 0; x < stride; x++) buf[rank * stride + x] = gf8_mul(buf[rank * stride + x], iv);
        }
        for (size_t r = 0; r < k; r++) {
            if (r == rank) continue;
            uint8_t f = buf[r * stride + c];
            if (!f) continue;
            for (size_t x = 0; x < stride; x++) buf[r * stride + x] ^= gf8_mul(f, buf[rank * stride + x]);
        }
        rank++;
    }
    if (rank == k)
        for (size_t r = 0; r < k; r++) memcpy(out + r * L, buf + r * stride + k, L);
    free(buf);
    free(coeffs);
    return rank;
}
