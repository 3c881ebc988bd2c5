// Host-side field arithmetic for coefficient setup (the layer above the
// payload kernels).  Coefficient tables are built once per codec on the host,
// as the reference builds them at construction.
#pragma once

#include <stdint.h>

#include <vector>

#include "../../include/scrs_gpu.h"

namespace scrs {
namespace hf {

struct Tables {
    uint8_t exp[510];
    uint8_t log[256];
    Tables() {
        // EXP[i] = 3^i mod 0x11B, LOG inverts it (scrs/src/algebra/gf256.rs:252-311).
        uint32_t v = 1;
        for (int i = 0; i < 255; i++) {
            exp[i] = exp[i + 255] = (uint8_t)v;
            log[v] = (uint8_t)i;
            uint32_t x2 = v << 1;
            if (x2 & 0x100) x2 ^= 0x11B;
            v = x2 ^ v;  // v * 3 = v*2 + v
        }
        log[0] = 0;
    }
};

inline const Tables& tables() {
    static const Tables t;
    return t;
}

inline uint8_t mul8(uint8_t a, uint8_t b) {
    if (!a || !b) return 0;
    const Tables& t = tables();
    return t.exp[t.log[a] + t.log[b]];
}
inline uint8_t inv8(uint8_t a) { return a ? tables().exp[255 - tables().log[a]] : 0; }

constexpr uint8_t kDelta = 0x20;
constexpr uint16_t kGen16 = 0x0108;

// (a + b u)(c + d u) with u^2 = u + DELTA (scrs/src/algebra/gf65536.rs:79).
inline uint16_t mul16(uint16_t x, uint16_t y) {
    uint8_t a = (uint8_t)x, b = (uint8_t)(x >> 8), c = (uint8_t)y, d = (uint8_t)(y >> 8);
    uint8_t ac = mul8(a, c), bd = mul8(b, d);
    return (uint16_t)((ac ^ mul8(kDelta, bd)) | ((uint16_t)(mul8(a ^ b, c ^ d) ^ ac) << 8));
}
inline uint16_t inv16(uint16_t x) {  // gf65536.rs:104
    uint8_t a = (uint8_t)x, b = (uint8_t)(x >> 8);
    if (!x) return 0;
    uint8_t norm = mul8(a, a) ^ mul8(a, b) ^ mul8(kDelta, mul8(b, b));
    uint8_t ni = inv8(norm);
    return (uint16_t)(mul8(a ^ b, ni) | ((uint16_t)mul8(b, ni) << 8));
}

// GF(256) Cauchy coefficients, source-major [k][m].
// Standard: 1/(i + (k+j)) (cauchy.rs:38, :98); Good: g^-i / (1 + g^(k+j-i))
// (good_cauchy.rs:125-144).
inline void gf8_coefficients(int32_t engine, uint32_t k, uint32_t m, uint8_t* out) {
    const Tables& t = tables();
    if (engine == SCRS_ENGINE_STANDARD_CAUCHY) {
        for (uint32_t i = 0; i < k; i++)
            for (uint32_t j = 0; j < m; j++) {
                uint8_t d = (uint8_t)i ^ (uint8_t)(k + j);
                out[i * m + j] = inv8(d);
            }
        return;
    }
    std::vector<uint8_t> base(k + m, 0);
    for (uint32_t d = 1; d < k + m; d++) base[d] = inv8((uint8_t)(1 ^ t.exp[d % 255]));
    for (uint32_t i = 0; i < k; i++) {
        uint8_t scale = i == 0 ? 1 : inv8(t.exp[i % 255]);
        for (uint32_t j = 0; j < m; j++) out[i * m + j] = mul8(scale, base[k + j - i]);
    }
}

// g^0 .. g^(n-1) for the tower generator (tower/cauchy.rs:74-80).
inline void tower_powers(uint32_t n, uint16_t* out) {
    uint16_t v = 1;
    for (uint32_t i = 0; i < n; i++) {
        out[i] = v;
        v = mul16(v, kGen16);
    }
}

// Tower coefficients [k][m]: g^-i / (1 + g^(k+j-i)) (tower/cauchy.rs:69-106).
inline void tower_coefficients(uint32_t k, uint32_t m, const uint16_t* powers, uint16_t* out) {
    std::vector<uint16_t> base(k + m, 0);
    for (uint32_t d = 1; d < k + m; d++) base[d] = inv16((uint16_t)(1 ^ powers[d]));
    uint16_t ginv = inv16(kGen16), scale = 1;
    for (uint32_t i = 0; i < k; i++) {
        for (uint32_t j = 0; j < m; j++) out[(size_t)i * m + j] = mul16(scale, base[k + j - i]);
        scale = mul16(scale, ginv);
    }
}

}  // namespace hf
}  // namespace scrs
