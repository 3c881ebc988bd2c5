/*
 * Test infrastructure (oracle): Tower Cauchy coefficients over GF((2^8)^2)
 * and the reduced closed-form solve, restated from the SCRS reference.
 */
#include <stdlib.h>

#include "oracle_internal.h"

/* scrs/src/tower/cauchy.rs:69-106: powers g^0..g^(n-1);
 * base[d] = 1/(1+g^d) (batch inversion, cauchy.rs:111-128, gives the same
 * reciprocals as one inversion each); row scale g^-i;
 * C[i][j] = g^-i * base[k+j-i].  Returns NULL on allocation failure. */
uint16_t* tower_coefficient_matrix(size_t k, size_t m) {
    oracle_tables_init();
    size_t n = k + m;
    uint16_t* coeffs = (uint16_t*)malloc(k * m * sizeof(uint16_t));
    uint16_t* base = (uint16_t*)calloc(n, sizeof(uint16_t));
    if (!coeffs || !base) {
        free(coeffs);
        free(base);
        return NULL;
    }
    uint16_t power = 1;
    for (size_t d = 0; d < n; d++) {
        if (d) base[d] = gf16_inv((uint16_t)(1 ^ power));
        power = gf16_mul(power, GF16_GENERATOR);
    }
    uint16_t ginv = gf16_inv(GF16_GENERATOR);
    uint16_t scale = 1;
    for (size_t i = 0; i < k; i++) {
        for (size_t j = 0; j < m; j++) coeffs[i * m + j] = gf16_mul(scale, base[k + j - i]);
        scale = gf16_mul(scale, ginv);
    }
    free(base);
    return coeffs;
}

/* scrs/src/tower/decoder.rs:433-546, the GF(65536) form of the rational
 * Lagrange factors (same formulas as decoder/cauchy_inverse.rs:29-49). */
void gf16_rational_lagrange(const uint16_t* row, const uint16_t* col, size_t r,
                            const uint16_t* pres, size_t p, uint16_t* inverse,
                            uint16_t* present) {
    if (r == 0) return;
    uint16_t* rf = (uint16_t*)malloc(r * sizeof(uint16_t));
    uint16_t* cf = (uint16_t*)malloc(r * sizeof(uint16_t));
    uint16_t* prefix = (uint16_t*)malloc((r + 1) * sizeof(uint16_t));
    uint16_t* suffix = (uint16_t*)malloc((r + 1) * sizeof(uint16_t));
    for (size_t i = 0; i < r; i++) {
        uint16_t cross = 1, within = 1;
        for (size_t h = 0; h < r; h++) cross = gf16_mul(cross, row[i] ^ col[h]);
        for (size_t l = 0; l < r; l++)
            if (l != i) within = gf16_mul(within, row[i] ^ row[l]);
        rf[i] = gf16_mul(cross, gf16_inv(within));
    }
    for (size_t j = 0; j < r; j++) {
        uint16_t cross = 1, within = 1;
        for (size_t l = 0; l < r; l++) cross = gf16_mul(cross, col[j] ^ row[l]);
        for (size_t h = 0; h < r; h++)
            if (h != j) within = gf16_mul(within, col[j] ^ col[h]);
        cf[j] = gf16_mul(cross, gf16_inv(within));
    }
    for (size_t j = 0; j < r; j++)
        for (size_t i = 0; i < r; i++)
            inverse[j * r + i] = gf16_mul(gf16_mul(rf[i], cf[j]), gf16_inv(col[j] ^ row[i]));
    for (size_t z = 0; z < p; z++) {
        uint16_t rowprod = 1;
        for (size_t l = 0; l < r; l++) rowprod = gf16_mul(rowprod, pres[z] ^ row[l]);
        uint16_t rinv = gf16_inv(rowprod);
        prefix[0] = 1;
        for (size_t j = 0; j < r; j++) prefix[j + 1] = gf16_mul(prefix[j], pres[z] ^ col[j]);
        suffix[r] = 1;
        for (size_t j = r; j-- > 0;) suffix[j] = gf16_mul(suffix[j + 1], pres[z] ^ col[j]);
        for (size_t j = 0; j < r; j++)
            present[z * r + j] = gf16_mul(gf16_mul(cf[j], gf16_mul(prefix[j], suffix[j + 1])), rinv);
    }
    free(rf);
    free(cf);
    free(prefix);
    free(suffix);
}
