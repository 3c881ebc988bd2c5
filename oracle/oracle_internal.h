/*
 * Test infrastructure, not product code.
 *
 * The oracle is a CPU restatement of the SCRS reference algorithms (Rust crate
 * scrs, files cited per function as scrs/src/<path>:<line>).  It is used only
 * as the checker in tests/, by __graft_entry__.smoke(), and as the timed CPU
 * baseline in bench.py.  It exports the same C ABI as the CUDA library with
 * the prefix `oracle_` in place of `scrs_` (declared in oracle/scrs_oracle.h),
 * so a test harness can run one scenario on both and compare bytes.
 *
 * Parity pinning: the reference crate cannot be compiled in this image (no
 * Rust toolchain), so the restatement is pinned by the reference's own
 * known-answer tests (tests/golden/reference_kats.json, extracted from the
 * reference test sources by tests/golden/make_kats.py) and by its
 * definitional oracles (byte-wise Cauchy sums, Lagrange interpolation at the
 * AFFT evaluation points, RREF decode, direct locator products).
 */
#ifndef SCRS_ORACLE_INTERNAL_H
#define SCRS_ORACLE_INTERNAL_H

#include <stddef.h>
#include <stdint.h>
#include <string.h>

#include "../include/scrs_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- GF(256): scrs/src/algebra/gf256.rs ---------------------------------- */
#define GF8_POLY_LOW 0x1Bu /* gf256.rs:32, polynomial 0x11B (gf256.rs:29) */
#define GF8_GENERATOR 0x03u /* gf256.rs:39 */

extern uint8_t g_gf8_exp[255]; /* gf256.rs:261 */
extern uint8_t g_gf8_log[256]; /* gf256.rs:265 */

void oracle_tables_init(void);
uint8_t gf8_mul_xtime(uint8_t a, uint8_t b); /* gf256.rs:79 */
uint8_t gf8_inv_xtime(uint8_t a);            /* gf256.rs:105 */
uint8_t gf8_mul(uint8_t a, uint8_t b);       /* gf256.rs:135 */
uint8_t gf8_inv(uint8_t a);                  /* gf256.rs:150 */
uint8_t gf8_div(uint8_t a, uint8_t b);       /* gf256.rs:167 */

/* ---- GF((2^8)^2): scrs/src/algebra/gf65536.rs ----------------------------- */
#define GF16_DELTA 0x20u       /* gf65536.rs:20 */
#define GF16_GENERATOR 0x0108u /* gf65536.rs:26 */
uint16_t gf16_mul(uint16_t x, uint16_t y); /* gf65536.rs:79 */
uint16_t gf16_square(uint16_t x);          /* gf65536.rs:93 */
uint16_t gf16_inv(uint16_t x);             /* gf65536.rs:104 */
uint16_t gf16_div(uint16_t x, uint16_t y); /* gf65536.rs:119 */
uint16_t gf16_pow(uint16_t x, uint32_t e); /* gf65536.rs:132 */

/* ---- payload kernels ------------------------------------------------------ */
/* dst ^= c * src over GF(256) bytes (scrs/src/payload.rs:6). */
void pl8_xor_scaled(uint8_t* dst, uint8_t c, const uint8_t* src, size_t len);
void pl8_xor(uint8_t* dst, const uint8_t* src, size_t len);
/* dst ^= c * src over interleaved GF(65536) elements (tower/payload.rs:7). */
void pl16_xor_scaled(uint8_t* dst, uint16_t c, const uint8_t* src, size_t len);
/* low ^= c*high; high ^= low (tower/payload.rs:58). */
void pl16_fused_forward(uint8_t* low, uint8_t* high, uint16_t c, size_t len);
/* high ^= low; low ^= c*high (tower/payload.rs:103). */
void pl16_fused_inverse(uint8_t* low, uint8_t* high, uint16_t c, size_t len);
/* 1 when the GFNI+AVX2 payload path is active (scrs/src/simd/dispatch.rs:32). */
int oracle_simd_active(void);
void oracle_force_scalar(int on);

/* ---- error helpers -------------------------------------------------------- */
static inline int32_t oerr(scrs_error* err, int32_t code, uint64_t a, uint64_t b) {
    if (err) {
        err->code = code;
        err->reserved = 0;
        err->a = a;
        err->b = b;
    }
    return code;
}

/* ---- GF(256) coefficient sets (matrices/cauchy.rs, good_cauchy.rs) ------- */
uint8_t gf8_x_var(int32_t engine, size_t k, size_t i);
uint8_t gf8_y_var(int32_t engine, size_t k, size_t j);
/* Source-major k x m coefficients, coeffs[i*m + j] (coding_matrix.rs:40). */
void gf8_coefficient_matrix(int32_t engine, size_t k, size_t m, uint8_t* coeffs);
/* Closed-form reduced Cauchy solve (decoder/cauchy_inverse.rs:50-212):
 * inverse[s*r + t] (missing s, repair row t), present[p*r + s]. */
void gf8_rational_lagrange(const uint8_t* row_vars, const uint8_t* col_vars,
                           size_t r, const uint8_t* present_vars, size_t p,
                           uint8_t* inverse, uint8_t* present);
int gf8_invert_square(uint8_t* matrix, size_t e, uint8_t* inv);

/* ---- tower (tower/cauchy.rs) ---------------------------------------------- */
uint16_t* tower_coefficient_matrix(size_t k, size_t m); /* malloc'd k*m */
void gf16_rational_lagrange(const uint16_t* row_vars, const uint16_t* col_vars,
                            size_t r, const uint16_t* present_vars, size_t p,
                            uint16_t* inverse, uint16_t* present);

#ifdef __cplusplus
}
#endif
#endif
