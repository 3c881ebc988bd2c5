// Bit-sliced constant multiplication over GF(256) and GF((2^8)^2).
//
// Multiplying a byte by a constant c is GF(2)-linear: an 8x8 bit matrix M_c
// with M_c[r][s] = bit r of c*x^s (the XOR form of the Cauchy code, Bloemer
// et al. 1995).  With 32 bytes bit-sliced into 8 planes, acc ^= c*x becomes
// acc[r] ^= XOR_{s: M_c[r][s]} plane[s].  Coefficients are warp-uniform at
// run time, so a jump table selects one of the compile-time XOR networks
// below; no table lookups touch the payload.
#pragma once

#include "common.cuh"
#if defined(__CUDA_ARCH__)
#include "brx_dispatch.cuh"
#endif

namespace scrs {

template <int C>
SCRS_HD void mulacc8(uint32_t (&acc)[8], const uint32_t (&p)[8]) {
#pragma unroll
    for (int r = 0; r < 8; r++) {
        uint32_t t = 0;
#pragma unroll
        for (int s = 0; s < 8; s++)
            if (gf8_matrix_bit(C, r, s)) t ^= p[s];
        acc[r] ^= t;
    }
}

// Same map applied to both components of 16-plane GF((2^8)^2) data: a GF(256)
// scalar c multiplies a + b*u componentwise.
template <int C>
SCRS_HD void mulacc8x2(uint32_t (&acc)[16], const uint32_t (&p)[16]) {
#pragma unroll
    for (int h = 0; h < 16; h += 8)
#pragma unroll
        for (int r = 0; r < 8; r++) {
            uint32_t t = 0;
#pragma unroll
            for (int s = 0; s < 8; s++)
                if (gf8_matrix_bit(C, r, s)) t ^= p[h + s];
            acc[h + r] ^= t;
        }
}

#define SCRS_R16(M, B) \
    M(B + 0) M(B + 1) M(B + 2) M(B + 3) M(B + 4) M(B + 5) M(B + 6) M(B + 7) M(B + 8) M(B + 9) M(B + 10) \
        M(B + 11) M(B + 12) M(B + 13) M(B + 14) M(B + 15)
#define SCRS_R256(M)                                                                                    \
    SCRS_R16(M, 0) SCRS_R16(M, 16) SCRS_R16(M, 32) SCRS_R16(M, 48) SCRS_R16(M, 64) SCRS_R16(M, 80)      \
        SCRS_R16(M, 96) SCRS_R16(M, 112) SCRS_R16(M, 128) SCRS_R16(M, 144) SCRS_R16(M, 160)             \
            SCRS_R16(M, 176) SCRS_R16(M, 192) SCRS_R16(M, 208) SCRS_R16(M, 224) SCRS_R16(M, 240)

// Host reference forms of the multiply (the device code dispatches through
// the generated jump tables in brx_dispatch.cuh instead).
// One 256-way switch per coefficient.
SCRS_HD void mul8_byte(uint32_t c, uint32_t (&acc)[8], const uint32_t (&p)[8]) {
#define SCRS_CASE8(N) \
    case (N): mulacc8<(N)>(acc, p); break;
    switch (c & 255u) { SCRS_R256(SCRS_CASE8) }
#undef SCRS_CASE8
}

// c = lo + 16*hi: two 16-way switches.
SCRS_HD void mul8_nibble(uint32_t c, uint32_t (&acc)[8], const uint32_t (&p)[8]) {
#define SCRS_CASE8L(N) \
    case (N): mulacc8<(N)>(acc, p); break;
#define SCRS_CASE8H(N) \
    case (N): mulacc8<((N) << 4)>(acc, p); break;
    switch (c & 15u) { SCRS_R16(SCRS_CASE8L, 0) }
    switch ((c >> 4) & 15u) { SCRS_R16(SCRS_CASE8H, 0) }
#undef SCRS_CASE8L
#undef SCRS_CASE8H
}

// acc ^= v * x for a GF(256) scalar v applied to both tower components.
SCRS_HD void mul8x2_nibble(uint32_t v, uint32_t (&acc)[16], const uint32_t (&p)[16]) {
#define SCRS_CASE16L(N) \
    case (N): mulacc8x2<(N)>(acc, p); break;
#define SCRS_CASE16H(N) \
    case (N): mulacc8x2<((N) << 4)>(acc, p); break;
    switch (v & 15u) { SCRS_R16(SCRS_CASE16L, 0) }
    switch ((v >> 4) & 15u) { SCRS_R16(SCRS_CASE16H, 0) }
#undef SCRS_CASE16L
#undef SCRS_CASE16H
}

// x <- u * x in the tower basis: (a + b u) u = DELTA*b + (a + b) u
// (u^2 = u + DELTA, scrs/src/algebra/gf65536.rs:7).
SCRS_HD void mul_by_u(uint32_t (&x)[16]) {
    uint32_t lo[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    uint32_t b[8];
#pragma unroll
    for (int s = 0; s < 8; s++) b[s] = x[8 + s];
    mulacc8<kGf16Delta>(lo, b);
#pragma unroll
    for (int s = 0; s < 8; s++) {
        x[8 + s] ^= x[s];  // hi = a + b
        x[s] = lo[s];      // lo = DELTA * b
    }
}

template <bool kUniform>
SCRS_HD void mul8x2_dispatch(uint32_t v, uint32_t (&acc)[16], const uint32_t (&p)[16]) {
#if defined(__CUDA_ARCH__)
    if (kUniform)
        brx_mul8x2_nib(v & 15u, (v >> 4) & 15u, acc, p);
    else
        brx_mul8x2_nib_div(v & 15u, (v >> 4) & 15u, acc, p);
#else
    mul8x2_nibble(v, acc, p);
#endif
}

// acc ^= c * x over GF((2^8)^2), c = c0 + c1*u:  c*x = c0*x + c1*(u*x).
// The loop runs the same two jump tables twice (x, then u*x) so the code
// holds one copy of each.  kUniform: c is the same in every lane of the warp.
template <bool kUniform = true>
SCRS_HD void mul16(uint32_t c, uint32_t (&acc)[16], const uint32_t (&p)[16]) {
    uint32_t x[16];
#pragma unroll
    for (int i = 0; i < 16; i++) x[i] = p[i];
    uint32_t c0 = c & 0xFFu, c1 = (c >> 8) & 0xFFu;
#pragma unroll 1
    for (int t = 0; t < 2; t++) {
        uint32_t v = t ? c1 : c0;
        if (v) mul8x2_dispatch<kUniform>(v, acc, x);
        if (t == 0) {
            if (c1 == 0) break;
            mul_by_u(x);
        }
    }
}

// acc ^= c * x over GF((2^8)^2) without branches, for a constant that may
// differ in every lane (shift-and-add over the coefficient's bits, on the
// planes).  c = c0 + c1*u: c*x = c0*x + c1*(u*x), and a GF(256) scalar v
// times both tower components is XOR_{i: bit i of v} 2^i * x, each 2^i * x
// one xtime step (multiply by 2 modulo 0x11B: shift the planes up, fold
// plane 7 into planes 0, 1, 3, 4) from the last.  About 2.5x the work of one
// jump-table product, the same for every lane whatever its constant, so it
// serves a warp whose lanes hold many different constants.
SCRS_HD void mul8x2_masked(uint32_t v, uint32_t (&acc)[16], uint32_t (&y)[16]) {
#pragma unroll
    for (int i = 0; i < 8; i++) {
        const uint32_t m = 0u - ((v >> i) & 1u);
#pragma unroll
        for (int q = 0; q < 16; q++) acc[q] ^= y[q] & m;
        if (i == 7) break;
#pragma unroll
        for (int h = 0; h < 16; h += 8) {
            const uint32_t top = y[h + 7];
#pragma unroll
            for (int r = 7; r > 0; r--) y[h + r] = y[h + r - 1];
            y[h] = top;
            y[h + 1] ^= top;
            y[h + 3] ^= top;
            y[h + 4] ^= top;
        }
    }
}

SCRS_HD void mul16_masked(uint32_t c, uint32_t (&acc)[16], const uint32_t (&p)[16]) {
    uint32_t y[16];
#pragma unroll
    for (int i = 0; i < 16; i++) y[i] = p[i];
    mul8x2_masked(c & 0xFFu, acc, y);
#pragma unroll
    for (int i = 0; i < 16; i++) y[i] = p[i];
    mul_by_u(y);
    mul8x2_masked((c >> 8) & 0xFFu, acc, y);
}

}  // namespace scrs
