/*
 * Test infrastructure (oracle): GF(256) / GF((2^8)^2) arithmetic and the
 * payload multiply-XOR kernels, restated from the SCRS reference.
 */
#include <immintrin.h>
#include <pthread.h>
#include <stdlib.h>

#include "oracle_internal.h"

uint8_t g_gf8_exp[255];
uint8_t g_gf8_log[256];
/* Full product table, derived from EXP/LOG; a lookup form of gf256.rs:135. */
static uint8_t g_gf8_mul[256][256];
static int g_simd = 0;
static int g_force_scalar = 0;
static pthread_once_t g_once = PTHREAD_ONCE_INIT;

/* scrs/src/algebra/gf256.rs:79-98 — shift-and-XOR reference multiply. */
uint8_t gf8_mul_xtime(uint8_t a, uint8_t b) {
    uint8_t acc = 0;
    for (int i = 0; i < 8; i++) {
        if ((b >> i) & 1) acc ^= a;
        uint8_t hi = a & 0x80;
        a = (uint8_t)(a << 1);
        if (hi) a ^= GF8_POLY_LOW;
    }
    return acc;
}

/* scrs/src/algebra/gf256.rs:105-123 — Fermat inverse a^254. */
uint8_t gf8_inv_xtime(uint8_t a) {
    if (a == 0) return 0;
    uint8_t result = 1;
    for (int i = 0; i < 8; i++) {
        result = gf8_mul_xtime(result, result);
        if ((254u >> (7 - i)) & 1) result = gf8_mul_xtime(result, a);
    }
    return result;
}

static void init_tables(void) {
    /* gf256.rs:268-290: EXP[i] = 3^i, LOG inverts EXP, LOG[0] left 0. */
    uint8_t v = 1;
    for (int i = 0; i < 255; i++) {
        g_gf8_exp[i] = v;
        v = gf8_mul_xtime(v, GF8_GENERATOR);
    }
    memset(g_gf8_log, 0, sizeof g_gf8_log);
    for (int i = 0; i < 255; i++) g_gf8_log[g_gf8_exp[i]] = (uint8_t)i;
    for (int a = 0; a < 256; a++)
        for (int b = 0; b < 256; b++) {
            uint8_t p = 0;
            if (a && b) p = g_gf8_exp[(g_gf8_log[a] + g_gf8_log[b]) % 255];
            g_gf8_mul[a][b] = p;
        }
#if defined(__x86_64__)
    __builtin_cpu_init();
    g_simd = __builtin_cpu_supports("avx2") && __builtin_cpu_supports("gfni");
#endif
    const char* force = getenv("SCRS_ORACLE_SCALAR");
    if (force && force[0] == '1') g_force_scalar = 1;
}

void oracle_tables_init(void) { pthread_once(&g_once, init_tables); }
int oracle_simd_active(void) {
    oracle_tables_init();
    return g_simd && !g_force_scalar;
}
void oracle_force_scalar(int on) {
    oracle_tables_init();
    g_force_scalar = on ? 1 : 0;
}

/* scrs/src/algebra/gf256.rs:135-146 */
uint8_t gf8_mul(uint8_t a, uint8_t b) {
    if (a == 0 || b == 0) return 0;
    return g_gf8_exp[(g_gf8_log[a] + g_gf8_log[b]) % 255];
}
/* scrs/src/algebra/gf256.rs:150-162 */
uint8_t gf8_inv(uint8_t a) {
    if (a == 0) return 0;
    return g_gf8_exp[(255 - g_gf8_log[a]) % 255];
}
/* scrs/src/algebra/gf256.rs:167-176 */
uint8_t gf8_div(uint8_t a, uint8_t b) {
    if (a == 0 || b == 0) return 0;
    return gf8_mul(a, gf8_inv(b));
}

/* scrs/src/algebra/gf65536.rs:79-89 — Karatsuba, u^2 = u + DELTA. */
uint16_t gf16_mul(uint16_t x, uint16_t y) {
    uint8_t a = (uint8_t)x, b = (uint8_t)(x >> 8);
    uint8_t c = (uint8_t)y, d = (uint8_t)(y >> 8);
    uint8_t ac = gf8_mul(a, c);
    uint8_t bd = gf8_mul(b, d);
    uint8_t constant = ac ^ gf8_mul(GF16_DELTA, bd);
    uint8_t extension = gf8_mul(a ^ b, c ^ d) ^ ac;
    return (uint16_t)(constant | ((uint16_t)extension << 8));
}
/* scrs/src/algebra/gf65536.rs:93-98 */
uint16_t gf16_square(uint16_t x) {
    uint8_t a = (uint8_t)x, b = (uint8_t)(x >> 8);
    uint8_t a2 = gf8_mul(a, a), b2 = gf8_mul(b, b);
    return (uint16_t)((a2 ^ gf8_mul(GF16_DELTA, b2)) | ((uint16_t)b2 << 8));
}
/* scrs/src/algebra/gf65536.rs:104-114 — conjugate over norm. */
uint16_t gf16_inv(uint16_t x) {
    uint8_t a = (uint8_t)x, b = (uint8_t)(x >> 8);
    if (a == 0 && b == 0) return 0;
    uint8_t norm = gf8_mul(a, a) ^ gf8_mul(a, b) ^ gf8_mul(GF16_DELTA, gf8_mul(b, b));
    uint8_t ni = gf8_inv(norm);
    return (uint16_t)(gf8_mul(a ^ b, ni) | ((uint16_t)gf8_mul(b, ni) << 8));
}
/* scrs/src/algebra/gf65536.rs:119-128 */
uint16_t gf16_div(uint16_t x, uint16_t y) {
    if (x == 0 || y == 0) return 0;
    return gf16_mul(x, gf16_inv(y));
}
/* scrs/src/algebra/gf65536.rs:132-143 */
uint16_t gf16_pow(uint16_t x, uint32_t e) {
    uint16_t base = x, result = 1;
    while (e) {
        if (e & 1) result = gf16_mul(result, base);
        base = gf16_square(base);
        e >>= 1;
    }
    return result;
}

/* ---- payload kernels ------------------------------------------------------ */

void pl8_xor(uint8_t* dst, const uint8_t* src, size_t len) {
    size_t i = 0;
    for (; i + 8 <= len; i += 8) {
        uint64_t a, b;
        memcpy(&a, dst + i, 8);
        memcpy(&b, src + i, 8);
        a ^= b;
        memcpy(dst + i, &a, 8);
    }
    for (; i < len; i++) dst[i] ^= src[i];
}

#if defined(__x86_64__)
/* GFNI path: gf2p8mulb multiplies bytes modulo 0x11B, the reference field
 * (scrs/src/simd/x86.rs:63-140 uses the same instruction). */
__attribute__((target("avx2,gfni"))) static void pl8_xor_scaled_gfni(
    uint8_t* dst, uint8_t c, const uint8_t* src, size_t len) {
    const __m256i cv = _mm256_set1_epi8((char)c);
    size_t i = 0;
    for (; i + 32 <= len; i += 32) {
        __m256i s = _mm256_loadu_si256((const __m256i*)(src + i));
        __m256i d = _mm256_loadu_si256((const __m256i*)(dst + i));
        d = _mm256_xor_si256(d, _mm256_gf2p8mul_epi8(s, cv));
        _mm256_storeu_si256((__m256i*)(dst + i), d);
    }
    const uint8_t* row = g_gf8_mul[c];
    for (; i < len; i++) dst[i] ^= row[src[i]];
}

/* Tower AXPY with two gf2p8mulb per vector: for interleaved [a,b] pairs,
 * lo' = c0*a + DELTA*c1*b and hi' = c1*a + (c0+c1)*b (gf65536.rs:79-89),
 * the same same/cross factor split as tower/payload.rs:257 factor_words. */
__attribute__((target("avx2,gfni"))) static void pl16_xor_scaled_gfni(
    uint8_t* dst, uint16_t c, const uint8_t* src, size_t len) {
    uint8_t c0 = (uint8_t)c, c1 = (uint8_t)(c >> 8);
    uint8_t same_lo = c0, same_hi = c0 ^ c1;
    uint8_t cross_lo = gf8_mul(GF16_DELTA, c1), cross_hi = c1;
    const __m256i same = _mm256_set1_epi16((short)(same_lo | (same_hi << 8)));
    const __m256i cross = _mm256_set1_epi16((short)(cross_lo | (cross_hi << 8)));
    const __m256i swap = _mm256_setr_epi8(1, 0, 3, 2, 5, 4, 7, 6, 9, 8, 11, 10, 13, 12, 15, 14,
                                          1, 0, 3, 2, 5, 4, 7, 6, 9, 8, 11, 10, 13, 12, 15, 14);
    size_t i = 0;
    for (; i + 32 <= len; i += 32) {
        __m256i s = _mm256_loadu_si256((const __m256i*)(src + i));
        __m256i d = _mm256_loadu_si256((const __m256i*)(dst + i));
        __m256i sw = _mm256_shuffle_epi8(s, swap);
        __m256i p = _mm256_xor_si256(_mm256_gf2p8mul_epi8(s, same), _mm256_gf2p8mul_epi8(sw, cross));
        _mm256_storeu_si256((__m256i*)(dst + i), _mm256_xor_si256(d, p));
    }
    for (; i + 2 <= len; i += 2) {
        uint16_t x = (uint16_t)(src[i] | (src[i + 1] << 8));
        uint16_t p = gf16_mul(x, c);
        dst[i] ^= (uint8_t)p;
        dst[i + 1] ^= (uint8_t)(p >> 8);
    }
}

__attribute__((target("avx2,gfni"))) static void pl16_fused_forward_gfni(
    uint8_t* low, uint8_t* high, uint16_t c, size_t len) {
    uint8_t c0 = (uint8_t)c, c1 = (uint8_t)(c >> 8);
    const __m256i same = _mm256_set1_epi16((short)(c0 | ((c0 ^ c1) << 8)));
    const __m256i cross = _mm256_set1_epi16((short)(gf8_mul(GF16_DELTA, c1) | (c1 << 8)));
    const __m256i swap = _mm256_setr_epi8(1, 0, 3, 2, 5, 4, 7, 6, 9, 8, 11, 10, 13, 12, 15, 14,
                                          1, 0, 3, 2, 5, 4, 7, 6, 9, 8, 11, 10, 13, 12, 15, 14);
    size_t i = 0;
    for (; i + 32 <= len; i += 32) {
        __m256i h = _mm256_loadu_si256((const __m256i*)(high + i));
        __m256i l = _mm256_loadu_si256((const __m256i*)(low + i));
        __m256i p = _mm256_xor_si256(_mm256_gf2p8mul_epi8(h, same),
                                     _mm256_gf2p8mul_epi8(_mm256_shuffle_epi8(h, swap), cross));
        l = _mm256_xor_si256(l, p);
        h = _mm256_xor_si256(h, l);
        _mm256_storeu_si256((__m256i*)(low + i), l);
        _mm256_storeu_si256((__m256i*)(high + i), h);
    }
    for (; i + 2 <= len; i += 2) {
        uint16_t lo = (uint16_t)(low[i] | (low[i + 1] << 8));
        uint16_t hi = (uint16_t)(high[i] | (high[i + 1] << 8));
        uint16_t nl = lo ^ gf16_mul(c, hi);
        uint16_t nh = hi ^ nl;
        low[i] = (uint8_t)nl, low[i + 1] = (uint8_t)(nl >> 8);
        high[i] = (uint8_t)nh, high[i + 1] = (uint8_t)(nh >> 8);
    }
}

__attribute__((target("avx2,gfni"))) static void pl16_fused_inverse_gfni(
    uint8_t* low, uint8_t* high, uint16_t c, size_t len) {
    uint8_t c0 = (uint8_t)c, c1 = (uint8_t)(c >> 8);
    const __m256i same = _mm256_set1_epi16((short)(c0 | ((c0 ^ c1) << 8)));
    const __m256i cross = _mm256_set1_epi16((short)(gf8_mul(GF16_DELTA, c1) | (c1 << 8)));
    const __m256i swap = _mm256_setr_epi8(1, 0, 3, 2, 5, 4, 7, 6, 9, 8, 11, 10, 13, 12, 15, 14,
                                          1, 0, 3, 2, 5, 4, 7, 6, 9, 8, 11, 10, 13, 12, 15, 14);
    size_t i = 0;
    for (; i + 32 <= len; i += 32) {
        __m256i h = _mm256_loadu_si256((const __m256i*)(high + i));
        __m256i l = _mm256_loadu_si256((const __m256i*)(low + i));
        h = _mm256_xor_si256(h, l);
        __m256i p = _mm256_xor_si256(_mm256_gf2p8mul_epi8(h, same),
                                     _mm256_gf2p8mul_epi8(_mm256_shuffle_epi8(h, swap), cross));
        l = _mm256_xor_si256(l, p);
        _mm256_storeu_si256((__m256i*)(low + i), l);
        _mm256_storeu_si256((__m256i*)(high + i), h);
    }
    for (; i + 2 <= len; i += 2) {
        uint16_t lo = (uint16_t)(low[i] | (low[i + 1] << 8));
        uint16_t hi = (uint16_t)(high[i] | (high[i + 1] << 8));
        uint16_t nh = hi ^ lo;
        uint16_t nl = lo ^ gf16_mul(c, nh);
        low[i] = (uint8_t)nl, low[i + 1] = (uint8_t)(nl >> 8);
        high[i] = (uint8_t)nh, high[i + 1] = (uint8_t)(nh >> 8);
    }
}
#endif

/* scrs/src/payload.rs:6-29 (scalar form): zero and one short-circuit. */
void pl8_xor_scaled(uint8_t* dst, uint8_t c, const uint8_t* src, size_t len) {
    if (c == 0 || len == 0) return;
    if (c == 1) {
        pl8_xor(dst, src, len);
        return;
    }
#if defined(__x86_64__)
    if (g_simd && !g_force_scalar) {
        pl8_xor_scaled_gfni(dst, c, src, len);
        return;
    }
#endif
    const uint8_t* row = g_gf8_mul[c];
    for (size_t i = 0; i < len; i++) dst[i] ^= row[src[i]];
}

/* scrs/src/tower/payload.rs:7-51 and the scalar form :187-205. */
void pl16_xor_scaled(uint8_t* dst, uint16_t c, const uint8_t* src, size_t len) {
    if (c == 0 || len == 0) return;
    if (c == 1) {
        pl8_xor(dst, src, len);
        return;
    }
#if defined(__x86_64__)
    if (g_simd && !g_force_scalar) {
        pl16_xor_scaled_gfni(dst, c, src, len);
        return;
    }
#endif
    for (size_t i = 0; i + 2 <= len; i += 2) {
        uint16_t x = (uint16_t)(src[i] | (src[i + 1] << 8));
        uint16_t p = gf16_mul(x, c);
        dst[i] ^= (uint8_t)p;
        dst[i + 1] ^= (uint8_t)(p >> 8);
    }
}

/* scrs/src/tower/payload.rs:58-98 and scalar :207-222. */
void pl16_fused_forward(uint8_t* low, uint8_t* high, uint16_t c, size_t len) {
    if (c == 0) { /* payload.rs:62-66: high ^= low only */
        pl8_xor(high, low, len);
        return;
    }
#if defined(__x86_64__)
    if (g_simd && !g_force_scalar) {
        pl16_fused_forward_gfni(low, high, c, len);
        return;
    }
#endif
    for (size_t i = 0; i + 2 <= len; i += 2) {
        uint16_t lo = (uint16_t)(low[i] | (low[i + 1] << 8));
        uint16_t hi = (uint16_t)(high[i] | (high[i + 1] << 8));
        uint16_t nl = lo ^ gf16_mul(c, hi);
        uint16_t nh = hi ^ nl;
        low[i] = (uint8_t)nl, low[i + 1] = (uint8_t)(nl >> 8);
        high[i] = (uint8_t)nh, high[i + 1] = (uint8_t)(nh >> 8);
    }
}

/* scrs/src/tower/payload.rs:103-143 and scalar :224-239. */
void pl16_fused_inverse(uint8_t* low, uint8_t* high, uint16_t c, size_t len) {
    if (c == 0) {
        pl8_xor(high, low, len);
        return;
    }
#if defined(__x86_64__)
    if (g_simd && !g_force_scalar) {
        pl16_fused_inverse_gfni(low, high, c, len);
        return;
    }
#endif
    for (size_t i = 0; i + 2 <= len; i += 2) {
        uint16_t lo = (uint16_t)(low[i] | (low[i + 1] << 8));
        uint16_t hi = (uint16_t)(high[i] | (high[i + 1] << 8));
        uint16_t nh = hi ^ lo;
        uint16_t nl = lo ^ gf16_mul(c, nh);
        low[i] = (uint8_t)nl, low[i + 1] = (uint8_t)(nl >> 8);
        high[i] = (uint8_t)nh, high[i + 1] = (uint8_t)(nh >> 8);
    }
}
