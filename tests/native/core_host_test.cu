// Host-side check of the bit-sliced GF(256)/GF((2^8)^2) core used by the
// kernels (scrs_b200/csrc/gf_mul_core.cuh), against scalar field arithmetic
// written from scrs/src/algebra/gf256.rs and gf65536.rs.  Built and run by
// tests/test_native_core.py; needs nvcc but no GPU.
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "../../scrs_b200/csrc/gf_mul_core.cuh"

using namespace scrs;

static uint8_t mul8s(uint8_t a, uint8_t b) { return gf8_mul_ce(a, b); }
static uint16_t mul16s(uint16_t x, uint16_t y) {
    uint8_t a = x, b = x >> 8, c = y, d = y >> 8;
    uint8_t ac = mul8s(a, c), bd = mul8s(b, d);
    return (uint16_t)((ac ^ mul8s(0x20, bd)) | ((mul8s(a ^ b, c ^ d) ^ ac) << 8));
}

static uint64_t rng = 0x9E3779B97F4A7C15ull;
static uint32_t next32() {
    rng ^= rng << 13;
    rng ^= rng >> 7;
    rng ^= rng << 17;
    return (uint32_t)rng;
}

int main() {
    int failures = 0;
    // bitslice8: planes hold bit s of every byte; involution.
    for (int trial = 0; trial < 200; trial++) {
        uint32_t w[8], orig[8];
        for (int i = 0; i < 8; i++) orig[i] = w[i] = next32();
        bitslice8(w);
        int ones_in = 0, ones_out = 0;
        for (int i = 0; i < 8; i++) ones_in += __builtin_popcount(orig[i]), ones_out += __builtin_popcount(w[i]);
        for (int s = 0; s < 8; s++) {
            int cnt = 0;
            for (int byte = 0; byte < 32; byte++) cnt += (((const uint8_t*)orig)[byte] >> s) & 1;
            if (cnt != __builtin_popcount(w[s])) failures++;
        }
        if (ones_in != ones_out) failures++;
        bitslice8(w);
        if (memcmp(w, orig, sizeof w)) failures++;
    }
    // mul8 (both strategies): acc ^= c * x bytewise.
    for (int c = 0; c < 256; c++) {
        uint32_t x[8], acc0[8], acc1[8], p[8];
        for (int i = 0; i < 8; i++) x[i] = next32(), acc0[i] = acc1[i] = next32();
        uint8_t expect[32];
        for (int b = 0; b < 32; b++) expect[b] = ((uint8_t*)acc0)[b] ^ mul8s((uint8_t)c, ((uint8_t*)x)[b]);
        memcpy(p, x, sizeof p);
        bitslice8(p);
        bitslice8(acc0);
        bitslice8(acc1);
        mul8_byte((uint32_t)c, acc0, p);
        mul8_nibble((uint32_t)c, acc1, p);
        bitslice8(acc0);
        bitslice8(acc1);
        if (memcmp(acc0, expect, 32) || memcmp(acc1, expect, 32)) {
            if (failures < 10) printf("mul8 mismatch c=%d\n", c);
            failures++;
        }
    }
    // bitslice16 + mul16: acc ^= c * x over interleaved [a,b] elements.
    for (int trial = 0; trial < 3000; trial++) {
        uint16_t c = trial < 4 ? (uint16_t)(trial == 0 ? 0 : trial == 1 ? 1 : trial == 2 ? 0x100 : 0xFFFF) : (uint16_t)next32();
        uint32_t x[16], acc[16], p[16];
        for (int i = 0; i < 16; i++) x[i] = next32(), acc[i] = next32();
        uint16_t expect[32];
        for (int e = 0; e < 32; e++) expect[e] = ((uint16_t*)acc)[e] ^ mul16s(c, ((uint16_t*)x)[e]);
        memcpy(p, x, sizeof p);
        bitslice16(p);
        bitslice16(acc);
        uint32_t acc2[16];
        memcpy(acc2, acc, sizeof acc2);
        mul16(c, acc, p);
        bitslice16(acc);
        if (memcmp(acc, expect, 64)) {
            if (failures < 10) printf("mul16 mismatch c=%04x\n", c);
            failures++;
        }
        mul16_masked(c, acc2, p);  // the branch-free form
        bitslice16(acc2);
        if (memcmp(acc2, expect, 64)) {
            if (failures < 10) printf("mul16_masked mismatch c=%04x\n", c);
            failures++;
        }
        // plane layout: w[s] = bit s of component a, w[8+s] = bit s of b.
        uint32_t q[16];
        memcpy(q, x, sizeof q);
        bitslice16(q);
        for (int s = 0; s < 8; s++) {
            int ca = 0, cb = 0;
            for (int e = 0; e < 32; e++) {
                ca += (((uint8_t*)x)[2 * e] >> s) & 1;
                cb += (((uint8_t*)x)[2 * e + 1] >> s) & 1;
            }
            if (ca != __builtin_popcount(q[s]) || cb != __builtin_popcount(q[8 + s])) failures++;
        }
    }
    printf("%s (%d failures)\n", failures ? "FAIL" : "PASS", failures);
    return failures ? 1 : 0;
}
