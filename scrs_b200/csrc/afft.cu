// Additive FFT over GF(2^16) on sm_100a: transform passes, formal
// derivative, erasure locator (Walsh-Hadamard in the log domain) and the
// encode/decode pipelines built from them.
//
// Rows between stages are kept bit-sliced in HBM: a row of L bytes is stored
// as G = ceil(L/64) groups of 64 bytes, each group the 16 bit planes of 32
// field elements (scrs_b200/csrc/common.cuh bitslice16).  Bytes are sliced
// once on the way in (the first transform pass) and unsliced once on the way
// out (the last).
#include <algorithm>
#include <map>
#include <mutex>
#include <new>
#include <type_traits>

#include "afft_engine.h"
#include "gf_mul_core.cuh"
#include "host_field.h"

namespace scrs {

namespace {

constexpr uint32_t kMult = 65535u;  // multiplicative group order (afft/decoder.rs:580)
constexpr uint32_t kTargetedMax = 5;  // TARGETED_MAX_MISSING (afft/decoder.rs:578)

// ---- GF(2^16) log/exp tables in device memory (afft/decoder.rs:587-598) --------
struct Log16Tables {
    DevBuf log;  // uint16[65536]
    DevBuf exp;  // uint16[65535]
};

std::mutex g_log_mu;
std::map<int, Log16Tables*> g_log_tables;

cudaError_t log16_tables(const uint16_t** d_log, const uint16_t** d_exp) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(g_log_mu);
    auto it = g_log_tables.find(dev);
    if (it == g_log_tables.end()) {
        std::vector<uint16_t> lg(65536, 0), ex(65535);
        uint16_t v = 1;
        for (uint32_t i = 0; i < kMult; i++) {
            ex[i] = v;
            lg[v] = (uint16_t)i;
            v = hf::mul16(v, hf::kGen16);
        }
        Log16Tables* t = new (std::nothrow) Log16Tables();
        if (!t) return cudaErrorMemoryAllocation;
        if ((e = t->log.ensure(65536 * 2)) != cudaSuccess || (e = t->exp.ensure(65535 * 2)) != cudaSuccess ||
            (e = upload_now(t->log.p, lg.data(), 65536 * 2)) != cudaSuccess ||
            (e = upload_now(t->exp.p, ex.data(), 65535 * 2)) != cudaSuccess) {
            delete t;
            return e;
        }
        it = g_log_tables.emplace(dev, t).first;
    }
    *d_log = it->second->log.as<uint16_t>();
    *d_exp = it->second->exp.as<uint16_t>();
    return cudaSuccess;
}

// ---- transform plan on the host (scrs/src/afft/transform.rs:228-299) -------------
struct SubspacePoly {
    uint16_t coeffs[17];
    int len;
    uint16_t norm_inv;
};

uint16_t sq16(uint16_t x) { return hf::mul16(x, x); }

uint16_t eval_linearized(const uint16_t* c, int len, uint16_t v) {
    uint16_t power = v, r = 0;
    for (int i = 0; i < len; i++) {
        r ^= hf::mul16(c[i], power);
        power = sq16(power);
    }
    return r;
}

void subspace_polynomials(int count, SubspacePoly* out) {
    uint16_t c[17] = {1};
    int len = 1;
    for (int dim = 0; dim < count; dim++) {
        uint16_t norm = eval_linearized(c, len, (uint16_t)(1u << dim));
        std::copy(c, c + 17, out[dim].coeffs);
        out[dim].len = len;
        out[dim].norm_inv = hf::inv16(norm);
        if (dim + 1 != count) {
            uint16_t nx[17] = {0};
            for (int i = 0; i < len; i++) {
                nx[i] ^= hf::mul16(norm, c[i]);
                nx[i + 1] ^= sq16(c[i]);
            }
            std::copy(nx, nx + 17, c);
            len++;
        }
    }
}

void fill_factors(std::vector<uint16_t>& f, const SubspacePoly* polys, size_t node, int dim, uint16_t shift) {
    const SubspacePoly& p = polys[dim - 1];
    f[node] = hf::mul16(eval_linearized(p.coeffs, p.len, shift), p.norm_inv);
    if (dim > 1) {
        fill_factors(f, polys, node * 2, dim - 1, shift);
        fill_factors(f, polys, node * 2 + 1, dim - 1, (uint16_t)(shift ^ (1u << (dim - 1))));
    }
}

// ---- device helpers --------------------------------------------------------------
__device__ __forceinline__ uint32_t add_mod(uint32_t a, uint32_t b) {
    uint32_t s = a + b;
    return s >= kMult ? s - kMult : s;
}
__device__ __forceinline__ uint32_t sub_mod(uint32_t a, uint32_t b) { return a >= b ? a - b : a + kMult - b; }


// ---- erasure locator (decoder.rs:672-755) ----------------------------------------
// log L(x) for every point x is a Walsh-Hadamard transform (mod 65535) of the
// product of two transforms: one of the erasure indicator, one of the
// logarithm table's first ts entries.  The second depends on ts alone, so the
// codec computes it once (log_walsh_host), with the final transform's 1/ts
// folded in; a decode runs two transforms.  Every level of a Walsh-Hadamard
// transform is exact arithmetic mod 65535 and the levels commute, so any
// grouping of levels into rounds gives the reference's residues.
//
// In one CTA (ts <= kLocatorOneCtaTs): round A takes index bits [0, 5 + R2)
// per warp, bits 0-4 across the lanes (shuffles) and bits 5.. through
// registers; round B takes the remaining RB <= 5 bits through registers,
// consecutive threads on consecutive entries (no bank conflicts).  The
// indicator is read straight from the known-point mask, the product with the
// log transform happens on the first transform's last store, and the
// second's last store writes values and derivatives.
constexpr uint32_t kLocatorOneCtaTs = 16384;
// Round A of a 2^14 transform has 32 blocks of 512 entries, round B 512
// groups: 16 warps serve both without idle threads.
constexpr int kLocatorThreads = 512;

template <int R2, class Load, class Store>
__device__ __forceinline__ void wht_round_lanes(int D, Load load, Store store) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const uint32_t ts = 1u << D;
    const int lane_bits = D < 5 ? D : 5;
    const uint32_t span = 32u << R2;
    const uint32_t nblk = ts > span ? ts / span : 1u;
    for (uint32_t b = warp; b < nblk; b += nwarps) {
        uint32_t x[1 << R2];
#pragma unroll
        for (int j = 0; j < (1 << R2); j++) {
            const uint32_t idx = b * span + 32u * j + lane;
            x[j] = idx < ts ? load(idx) : 0u;
        }
#pragma unroll
        for (int s = 0; s < R2; s++)
#pragma unroll
            for (int j = 0; j < (1 << R2); j++)
                if (!(j & (1 << s))) {
                    const uint32_t a = x[j], c = x[j | (1 << s)];
                    x[j] = add_mod(a, c);
                    x[j | (1 << s)] = sub_mod(a, c);
                }
        for (int s = 0; s < lane_bits; s++) {
            const bool upper = (lane >> s) & 1u;
#pragma unroll
            for (int j = 0; j < (1 << R2); j++) {
                const uint32_t y = __shfl_xor_sync(0xFFFFFFFFu, x[j], 1u << s);
                x[j] = upper ? sub_mod(y, x[j]) : add_mod(x[j], y);
            }
        }
#pragma unroll
        for (int j = 0; j < (1 << R2); j++) {
            const uint32_t idx = b * span + 32u * j + lane;
            if (idx < ts) store(idx, x[j]);
        }
    }
}

template <int RB, class Load, class Store>
__device__ __forceinline__ void wht_round_regs(int D, int lo, Load load, Store store) {
    const uint32_t groups = 1u << (D - RB);
    for (uint32_t g = threadIdx.x; g < groups; g += blockDim.x) {
        const uint32_t base = ((g >> lo) << (lo + RB)) | (g & ((1u << lo) - 1u));
        uint32_t x[1 << RB];
#pragma unroll
        for (int j = 0; j < (1 << RB); j++) x[j] = load(base + ((uint32_t)j << lo));
#pragma unroll
        for (int s = 0; s < RB; s++)
#pragma unroll
            for (int j = 0; j < (1 << RB); j++)
                if (!(j & (1 << s))) {
                    const uint32_t a = x[j], c = x[j | (1 << s)];
                    x[j] = add_mod(a, c);
                    x[j | (1 << s)] = sub_mod(a, c);
                }
#pragma unroll
        for (int j = 0; j < (1 << RB); j++) store(base + ((uint32_t)j << lo), x[j]);
    }
}

template <int R2, int RB>
__device__ void locator_cta(const uint8_t* known, int D, const uint32_t* lw, const uint16_t* exp16,
                            uint16_t* values, uint16_t* derivs, uint32_t* v) {
    auto indicator = [&](uint32_t i) -> uint32_t { return known[i] ? 0u : 1u; };
    auto ld = [&](uint32_t i) -> uint32_t { return v[i]; };
    auto st = [&](uint32_t i, uint32_t x) { v[i] = x; };
    auto st_mul = [&](uint32_t i, uint32_t x) { v[i] = (uint32_t)(((uint64_t)x * lw[i]) % kMult); };
    auto st_out = [&](uint32_t i, uint32_t x) {
        const uint16_t prod = exp16[x];
        const bool have = known[i] != 0;
        values[i] = have ? prod : 0;
        derivs[i] = have ? 0 : prod;
    };
    if constexpr (RB == 0) {
        wht_round_lanes<R2>(D, indicator, st_mul);
        __syncthreads();
        wht_round_lanes<R2>(D, ld, st_out);
    } else {
        wht_round_lanes<R2>(D, indicator, st);
        __syncthreads();
        wht_round_regs<RB>(D, 5 + R2, ld, st_mul);
        __syncthreads();
        wht_round_lanes<R2>(D, ld, st);
        __syncthreads();
        wht_round_regs<RB>(D, 5 + R2, ld, st_out);
    }
}

__global__ void __launch_bounds__(kLocatorThreads) locator_one_cta_kernel(const uint8_t* known, int D, const uint32_t* lw,
                                                               const uint16_t* exp16, uint16_t* values,
                                                               uint16_t* derivs) {
    extern __shared__ uint32_t sm_loc[];
    pdl_trigger();  // the first transform pass may start slicing its rows
    const int r2 = D <= 5 ? 0 : min(4, D - 5);
    const int rb = D <= 9 ? 0 : D - 9;
    switch (r2 * 8 + rb) {
        case 0: locator_cta<0, 0>(known, D, lw, exp16, values, derivs, sm_loc); break;
        case 8: locator_cta<1, 0>(known, D, lw, exp16, values, derivs, sm_loc); break;
        case 16: locator_cta<2, 0>(known, D, lw, exp16, values, derivs, sm_loc); break;
        case 24: locator_cta<3, 0>(known, D, lw, exp16, values, derivs, sm_loc); break;
        case 32: locator_cta<4, 0>(known, D, lw, exp16, values, derivs, sm_loc); break;
        case 33: locator_cta<4, 1>(known, D, lw, exp16, values, derivs, sm_loc); break;
        case 34: locator_cta<4, 2>(known, D, lw, exp16, values, derivs, sm_loc); break;
        case 35: locator_cta<4, 3>(known, D, lw, exp16, values, derivs, sm_loc); break;
        case 36: locator_cta<4, 4>(known, D, lw, exp16, values, derivs, sm_loc); break;
        case 37: locator_cta<4, 5>(known, D, lw, exp16, values, derivs, sm_loc); break;
        default: break;  // D > 14 takes the multi-CTA path
    }
}

// Larger transforms: passes over index bits [lo, lo + nb), one CTA per group
// of 2^nb entries that differ only in those bits.  The first pass of the
// first transform reads the indicator from the known-point mask (in_mode 1);
// the last pass of the first transform multiplies by the log transform
// (out_mode 1); the last pass of the second writes values and derivatives
// (out_mode 2).
__global__ void __launch_bounds__(1024) wht_pass_kernel(uint32_t* v, int lo, int nb, int in_mode, int out_mode,
                                                        const uint8_t* known, const uint32_t* lw,
                                                        const uint16_t* exp16, uint16_t* values, uint16_t* derivs) {
    extern __shared__ uint32_t sv[];
    pdl_trigger();  // the next pass (or, after the last, the first transform pass) may start its set-up
    const uint32_t gsize = 1u << nb;
    const uint32_t gidx = blockIdx.x;
    const uint32_t base = ((gidx >> lo) << (lo + nb)) | (gidx & ((1u << lo) - 1u));
    pdl_wait();  // v is the previous pass's output
    for (uint32_t t = threadIdx.x; t < gsize; t += blockDim.x) {
        const uint32_t i = base + (t << lo);
        sv[t] = in_mode ? (known[i] ? 0u : 1u) : v[i];
    }
    __syncthreads();
    for (int s = 0; s < nb; s++) {
        for (uint32_t p = threadIdx.x; p < gsize / 2; p += blockDim.x) {
            const uint32_t i = ((p >> s) << (s + 1)) | (p & ((1u << s) - 1u));
            const uint32_t a = sv[i], c = sv[i + (1u << s)];
            sv[i] = add_mod(a, c);
            sv[i + (1u << s)] = sub_mod(a, c);
        }
        __syncthreads();
    }
    for (uint32_t t = threadIdx.x; t < gsize; t += blockDim.x) {
        const uint32_t i = base + (t << lo), x = sv[t];
        if (out_mode == 0) {
            v[i] = x;
        } else if (out_mode == 1) {
            v[i] = (uint32_t)(((uint64_t)x * lw[i]) % kMult);
        } else {
            const uint16_t prod = exp16[x];
            const bool have = known[i] != 0;
            values[i] = have ? prod : 0;
            derivs[i] = have ? 0 : prod;
        }
    }
}

__device__ __forceinline__ void load_group_bytes(const uint8_t* row, uint32_t g, uint64_t L, uint32_t (&w)[16]) {
    const uint64_t pos = (uint64_t)g * 64;
    if (pos + 64 <= L && (reinterpret_cast<uintptr_t>(row + pos) & 15) == 0) {
#pragma unroll
        for (int q = 0; q < 4; q++) {
            uint4 v = __ldg(reinterpret_cast<const uint4*>(row + pos) + q);
            w[4 * q] = v.x, w[4 * q + 1] = v.y, w[4 * q + 2] = v.z, w[4 * q + 3] = v.w;
        }
        return;
    }
#pragma unroll
    for (int t = 0; t < 16; t++) {
        uint32_t x = 0;
        for (int b = 0; b < 4; b++) {
            uint64_t p = pos + 4 * t + b;
            if (p < L) x |= (uint32_t)row[p] << (8 * b);
        }
        w[t] = x;
    }
}

__device__ __forceinline__ void store_group_bytes(uint8_t* row, uint32_t g, uint64_t L, const uint32_t (&w)[16]) {
    const uint64_t pos = (uint64_t)g * 64;
    if (pos + 64 <= L && (reinterpret_cast<uintptr_t>(row + pos) & 15) == 0) {
#pragma unroll
        for (int q = 0; q < 4; q++)
            reinterpret_cast<uint4*>(row + pos)[q] = make_uint4(w[4 * q], w[4 * q + 1], w[4 * q + 2], w[4 * q + 3]);
        return;
    }
    for (int t = 0; t < 16; t++)
        for (int b = 0; b < 4; b++) {
            uint64_t p = pos + 4 * t + b;
            if (p < L) row[p] = (uint8_t)(w[t] >> (8 * b));
        }
}

__device__ __forceinline__ void load_planes(const uint8_t* p, uint32_t (&w)[16]) {
#pragma unroll
    for (int q = 0; q < 4; q++) {
        uint4 v = reinterpret_cast<const uint4*>(p)[q];
        w[4 * q] = v.x, w[4 * q + 1] = v.y, w[4 * q + 2] = v.z, w[4 * q + 3] = v.w;
    }
}
__device__ __forceinline__ void store_planes(uint8_t* p, const uint32_t (&w)[16]) {
#pragma unroll
    for (int q = 0; q < 4; q++)
        reinterpret_cast<uint4*>(p)[q] = make_uint4(w[4 * q], w[4 * q + 1], w[4 * q + 2], w[4 * q + 3]);
}

// Novel-basis formal derivative in gather form (transform.rs:188-213):
// out[j] = sum over bits b with j_b = 0 of df[b] * in[j | 2^b].
struct DerivFactors {
    uint16_t f[16];
};

__global__ void __launch_bounds__(128) derivative_kernel(const uint8_t* in, uint8_t* out, uint32_t ts, uint32_t G,
                                                         int D, DerivFactors df) {
    pdl_trigger();
    pdl_wait();  // `in` is the transform pass's output
    const uint64_t total = (uint64_t)ts * G;
    for (uint64_t x = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; x < total;
         x += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t j = (uint32_t)(x / G), g = (uint32_t)(x % G);
        uint32_t acc[16], cur[16], nxt[16];
#pragma unroll
        for (int t = 0; t < 16; t++) acc[t] = 0, cur[t] = 0, nxt[t] = 0;
        // the partner row of bit b + 1 is loaded while bit b's product runs;
        // b stays the same across the warp (the factor table jump is uniform)
        auto fetch = [&](int b, uint32_t (&w)[16]) {
            if (b < D && !((j >> b) & 1u)) load_planes(in + ((uint64_t)(j | (1u << b)) * G + g) * 64, w);
        };
        fetch(0, cur);
#pragma unroll 1
        for (int b = 0; b < D; b++) {
            fetch(b + 1, nxt);
            if (!((j >> b) & 1u)) mul16<true>(df.f[b], acc, cur);
#pragma unroll
            for (int t = 0; t < 16; t++) cur[t] = nxt[t];
        }
        store_planes(out + ((uint64_t)j * G + g) * 64, acc);
    }
}

// dst row rows[t] = src row (row_map ? row_map[rows[t]] : rows[t]), L bytes
// each, in units of `unit` bytes (16 when both bases are 16-byte aligned and
// L is a multiple of 16, else 1).
// With `chain` (launched with programmatic dependent launch right after the
// decode's locator, whose output it does not read) the copy runs beside the
// locator and waits for it only before exiting, so the next kernel's wait on
// this one also covers the locator.
template <int kUnit>
__global__ void copy_rows_kernel(const uint8_t* src, uint8_t* dst, uint64_t L, const uint16_t* rows,
                                 uint32_t count, const uint16_t* row_map, int chain) {
    using U = typename std::conditional<kUnit == 16, uint4, uint8_t>::type;
    if (chain) pdl_trigger();
    const uint64_t per = L / kUnit;
    const uint64_t total = (uint64_t)count * per;
    for (uint64_t x = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; x < total;
         x += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t t = x / per, q = x - t * per;
        const uint64_t r = rows[t];
        const uint64_t s = row_map ? row_map[r] : r;
        reinterpret_cast<U*>(dst + r * L)[q] = reinterpret_cast<const U*>(src + s * L)[q];
    }
    if (chain) pdl_wait();
}

// ---- transform passes ---------------------------------------------------------
// Several butterfly levels of a transform of 2^D rows on a shared-memory tile
// (transform.rs:301-333 forward_node / inverse_node, flattened by level).
// Rows p and p + 2^(D-1-l) pair at level l with node factor
// factors[root*2^l + (p >> (D-l))]: rows that agree in their top l bits share
// it.  A tile holds the rows that differ only in the c "level bits"
// [D-l0-c, D-l0) of the pass's levels [l0, l0+c) and in the e lowest row
// bits, for gn <= gt column groups.  The low bits lie below every level bit,
// so rows that differ only in them share every factor of the pass: lanes run
// over (group, low bits) first, and a level whose factor blocks of
// gn * 2^(e + b) butterflies (b: the level's pair bit among the level bits)
// are whole warps sends each warp through one factor.  Elsewhere (the
// deepest levels of a transform, which have no lower bits) the lanes of a
// warp are served factor by factor, each group with the uniform jump table,
// so the kernel holds a single copy of the multiply code.
//
// A pass runs one or two phases on the same tile (root, direction): the
// encode of a power-of-two k runs its inverse left half-transform's top
// levels and its forward right half-transform's top levels in one launch.
// With `slice` (the first pass of a transform) the tile is loaded from byte
// rows, bit-sliced and scaled on the way in; with `unslice` (the last pass)
// the output rows are scaled, converted back to bytes and stored to the
// caller's output instead of the work array (see PassIo).
constexpr int kTileThreads = 256;
constexpr uint32_t kTileElems = 1024;  // (row, group) elements of 64 bytes: 64 KiB
constexpr uint32_t kTileNominal = 512; // elements the deepest pass's tile aims at (32 KiB)

struct PassPhases {
    uint32_t root[2];
    int32_t forward[2];
    int32_t n;
};

struct PassIo {
    // slice (first pass): tile row r <- the bit-sliced bytes of payload row
    // (row_map ? row_map[r] : r) of src, times in_scale[r] when given, for
    // r < n_src that are known (known == nullptr: all); zero otherwise
    const uint8_t* src;
    const uint8_t* known;
    const uint16_t* row_map;
    const uint16_t* in_scale;
    uint32_t n_src;
    // unslice (last pass): rows r in [out_lo, out_hi) that are not known,
    // divided by out_derivs[r] when given, as bytes to dst row r - out_lo
    uint32_t out_lo, out_hi;
    uint8_t* dst;
    const uint16_t* out_derivs;
    const uint16_t* log16;
    const uint16_t* exp16;
    uint64_t L;
    // the slice's byte rows, row map and known mask were complete before the
    // decode's locator started (it is launched without programmatic
    // serialisation, after their upload): the first pass reads them before
    // waiting on the kernel before it (the locator, or the present-row copy
    // chained after it), and waits only for in_scale
    int32_t early_read;
};

// acc ^= f * x for every lane of the calling warp (all 32 lanes call it
// together; a lane with nothing to multiply passes f = 0), each lane with its
// own factor.  A warp whose lanes hold one or two distinct factors serves
// them one at a time, every group through the uniform jump table (brx.idx.uni
// is valid there: all active lanes share the index); with more, every lane
// runs the branch-free product (mul16_masked), whose cost does not grow with
// the number of factors.
// `uniform`: the caller knows every lane holds the same f (block-uniform
// flag), so the warp skips the match and ballots on its critical path.
__device__ __forceinline__ void mul16_lanes(uint32_t f, uint32_t (&acc)[16], const uint32_t (&x)[16],
                                            bool uniform = false) {
    const int lane = threadIdx.x & 31;
    if (!uniform) {
        const unsigned same = __match_any_sync(0xFFFFFFFFu, f);
        const unsigned leaders = __ballot_sync(0xFFFFFFFFu, (unsigned)(__ffs(same) - 1) == (unsigned)lane);
        if (__popc(leaders) > 2) {
            if (f) mul16_masked(f, acc, x);
            return;
        }
    }
    unsigned left = 0xFFFFFFFFu;
    while (left) {
        const uint32_t fl = uniform ? f : __shfl_sync(0xFFFFFFFFu, f, __ffs(left) - 1);
        const bool mine = uniform || (((left >> lane) & 1u) && f == fl);
        const unsigned grp = uniform ? 0xFFFFFFFFu : __ballot_sync(0xFFFFFFFFu, mine);
        if (mine && fl) mul16<true>(fl, acc, x);
        left &= ~grp;
    }
}

__global__ void __launch_bounds__(kTileThreads) afft_tile_kernel(uint8_t* work, uint32_t G, int D, int l0, int c,
                                                                int e, uint32_t gt, PassPhases ph,
                                                                const uint16_t* factors, PassIo io, int slice,
                                                                int unslice) {
    extern __shared__ __align__(16) uint8_t tile[];
    const uint32_t col_tiles = (G + gt - 1) / gt;
    const int low_bits = D - l0 - c;   // row bits below the level bits
    const int mid_bits = low_bits - e; // of which the tile fixes these
    const uint32_t tid = threadIdx.x;
    uint32_t t = blockIdx.x;
    const uint32_t ct = t % col_tiles;
    t /= col_tiles;
    const uint32_t mid = t & ((1u << mid_bits) - 1u);
    const uint32_t hi = t >> mid_bits;
    const uint32_t g0 = ct * gt;
    const uint32_t gn = min(gt, G - g0);
    const uint32_t rows = 1u << (c + e);
    const uint32_t low_mask = (1u << e) - 1u;
    // tile row i = (level bits << e) | low bits
    auto row_of = [&](uint32_t i) {
        return (hi << (D - l0)) | ((i >> e) << low_bits) | (mid << e) | (i & low_mask);
    };
    auto piece = [&](uint32_t i, uint32_t q, uint32_t g) { return tile + ((size_t)(i * 4 + q) * gt + g) * 16; };
    // Loops that multiply run whole warps: every lane of a warp takes the same
    // iterations (x0 is the warp's first element), lanes past the end with
    // nothing to do, so that mul16_lanes always has all 32 lanes.
    const uint32_t lane = tid & 31u;
    // The node factors of the pass, after the tile: at tile level lam the rows
    // whose level bits above the pair bit read u share factor
    // factors[(root << l) + (hi << lam) + u]; entry (1 << lam) - 1 + u of the
    // phase's table, 2^c - 1 entries per phase.
    uint16_t* fac = reinterpret_cast<uint16_t*>(tile + (size_t)rows * gt * 64);
    const uint32_t per_phase = (1u << c) - 1u;
    for (uint32_t x = tid; x < (uint32_t)ph.n * per_phase; x += blockDim.x) {
        const uint32_t p = x / per_phase, at = x - p * per_phase;
        const int lam = 31 - __clz(at + 1);
        const uint32_t u = at + 1 - (1u << lam);
        fac[x] = factors[((uint64_t)ph.root[p] << (l0 + lam)) + ((uint64_t)hi << lam) + u];
    }
    // the node factors are fixed per transform; the rows are the previous
    // kernel's output, or (io.early_read) were complete before it started
    pdl_trigger();
    if (slice) {
        if (!io.early_read) pdl_wait();
        // bytes in, bit-sliced, unscaled
        for (uint32_t x = tid; x < rows * gn; x += blockDim.x) {
            const uint32_t g = x % gn, i = x / gn;
            const uint32_t r = row_of(i);
            uint32_t w[16];
#pragma unroll
            for (int q = 0; q < 16; q++) w[q] = 0;
            if (r < io.n_src && (!io.known || io.known[r])) {
                load_group_bytes(io.src + (uint64_t)(io.row_map ? io.row_map[r] : r) * io.L, g0 + g, io.L, w);
                bitslice16(w);
            }
#pragma unroll
            for (int q = 0; q < 4; q++)
                *reinterpret_cast<uint4*>(piece(i, q, g)) = make_uint4(w[4 * q], w[4 * q + 1], w[4 * q + 2], w[4 * q + 3]);
        }
        if (io.early_read) pdl_wait();
        // times the locator value of each row (the previous kernel's output);
        // every thread rescales the elements it stored
        if (io.in_scale) {
            for (uint32_t x0 = tid - lane; x0 < rows * gn; x0 += blockDim.x) {
                const uint32_t x = x0 + lane;
                const bool valid = x < rows * gn;
                const uint32_t g = valid ? x % gn : 0u, i = valid ? x / gn : 0u;
                const uint32_t r = row_of(i);
                const bool have = valid && r < io.n_src && (!io.known || io.known[r]);
                uint32_t w[16], acc[16];
#pragma unroll
                for (int q = 0; q < 16; q++) acc[q] = 0, w[q] = 0;
                if (valid) {
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        const uint4 v = *reinterpret_cast<const uint4*>(piece(i, q, g));
                        w[4 * q] = v.x, w[4 * q + 1] = v.y, w[4 * q + 2] = v.z, w[4 * q + 3] = v.w;
                    }
                }
                mul16_lanes(have ? io.in_scale[r] : 0u, acc, w);
                if (!valid) continue;
#pragma unroll
                for (int q = 0; q < 4; q++)
                    *reinterpret_cast<uint4*>(piece(i, q, g)) =
                        make_uint4(acc[4 * q], acc[4 * q + 1], acc[4 * q + 2], acc[4 * q + 3]);
            }
        }
    } else {
        pdl_wait();
        // the copies are asynchronous, so every thread has all of its loads in flight
        for (uint32_t x = tid; x < rows * gn * 4; x += blockDim.x) {
            const uint32_t q = x & 3, g = (x >> 2) % gn, i = (x >> 2) / gn;
            cp_async_16(piece(i, q, g), work + ((uint64_t)row_of(i) * G + g0 + g) * 64 + 16 * q);
        }
    }
    if (!slice) cp_async_wait_all();
    __syncthreads();
    const uint32_t items = (rows / 2) * gn;
    const bool gpow = (gn & (gn - 1u)) == 0;  // the column split by shift and mask
    const int gsh = __ffs(gn) - 1;
    for (int p = 0; p < ph.n; p++) {
        const bool fwd = ph.forward[p] != 0;
        for (int s = 0; s < c; s++) {
            const int lam = fwd ? s : c - 1 - s;  // tile-local level
            const int b = c - 1 - lam;            // pair bit among the level bits
            const uint16_t* lf = fac + p * per_phase + (1u << lam) - 1u;
            // every warp holds one factor when its 32 items agree in all bits
            // from the pair bit up: items (low bits, group) of 2^(e+b) * gn
            // share the factor index r >> b
            const bool uni = gpow && (items & 31u) == 0 && ((gn << e) << b) >= 32u;
            for (uint32_t x0 = tid - lane; x0 < items; x0 += blockDim.x) {
                const uint32_t x = x0 + lane;
                const bool valid = x < items;
                const uint32_t g = !valid ? 0u : gpow ? (x & (gn - 1u)) : x % gn;
                uint32_t r = !valid ? 0u : gpow ? (x >> gsh) : x / gn;
                const uint32_t low = r & low_mask;
                r >>= e;
                const uint32_t lev_lo = ((r >> b) << (b + 1)) | (r & ((1u << b) - 1u));
                const uint32_t ilo = (lev_lo << e) | low, ihi = ilo | (1u << (b + e));
                const uint32_t f = valid ? lf[r >> b] : 0u;
                uint32_t wl[16], wh[16];
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    const uint4 a = *reinterpret_cast<const uint4*>(piece(ilo, q, g));
                    const uint4 h = *reinterpret_cast<const uint4*>(piece(ihi, q, g));
                    wl[4 * q] = a.x, wl[4 * q + 1] = a.y, wl[4 * q + 2] = a.z, wl[4 * q + 3] = a.w;
                    wh[4 * q] = h.x, wh[4 * q + 1] = h.y, wh[4 * q + 2] = h.z, wh[4 * q + 3] = h.w;
                }
                // forward: low ^= f*high, high ^= low;  inverse: high ^= low, low ^= f*high
                if (!fwd) {
#pragma unroll
                    for (int q = 0; q < 16; q++) wh[q] ^= wl[q];
                }
                mul16_lanes(f, wl, wh, uni);
                if (fwd) {
#pragma unroll
                    for (int q = 0; q < 16; q++) wh[q] ^= wl[q];
                }
                if (!valid) continue;
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    *reinterpret_cast<uint4*>(piece(ilo, q, g)) =
                        make_uint4(wl[4 * q], wl[4 * q + 1], wl[4 * q + 2], wl[4 * q + 3]);
                    *reinterpret_cast<uint4*>(piece(ihi, q, g)) =
                        make_uint4(wh[4 * q], wh[4 * q + 1], wh[4 * q + 2], wh[4 * q + 3]);
                }
            }
            __syncthreads();
        }
    }
    if (unslice) {
        for (uint32_t x0 = tid - lane; x0 < rows * gn; x0 += blockDim.x) {
            const uint32_t x = x0 + lane;
            const bool valid = x < rows * gn;
            const uint32_t g = valid ? x % gn : 0u, i = valid ? x / gn : 0u;
            const uint32_t r = row_of(i);
            const bool out = valid && r >= io.out_lo && r < io.out_hi && !(io.known && io.known[r]);
            uint32_t w[16], acc[16];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const uint4 v = *reinterpret_cast<const uint4*>(piece(i, q, g));
                w[4 * q] = v.x, w[4 * q + 1] = v.y, w[4 * q + 2] = v.z, w[4 * q + 3] = v.w;
            }
            if (io.out_derivs) {
                // 1 / L'(r) through the log tables (decoder.rs:348-356)
                const uint32_t d = out ? io.out_derivs[r] : 0u;
                const uint32_t f = d ? io.exp16[(kMult - io.log16[d]) % kMult] : 0u;
#pragma unroll
                for (int q = 0; q < 16; q++) acc[q] = 0;
                mul16_lanes(f, acc, w);
            } else {
#pragma unroll
                for (int q = 0; q < 16; q++) acc[q] = w[q];
            }
            if (!out) continue;
            bitslice16(acc);
            store_group_bytes(io.dst + (uint64_t)(r - io.out_lo) * io.L, g0 + g, io.L, acc);
        }
        return;
    }
    for (uint32_t x = tid; x < rows * gn * 4; x += blockDim.x) {
        const uint32_t q = x & 3, g = (x >> 2) % gn, i = (x >> 2) / gn;
        *reinterpret_cast<uint4*>(work + ((uint64_t)row_of(i) * G + g0 + g) * 64 + 16 * q) =
            *reinterpret_cast<const uint4*>(piece(i, q, g));
    }
}

int grid_for(uint64_t items, int threads) {
    uint64_t g = (items + threads - 1) / threads;
    return (int)std::max<uint64_t>(1, std::min<uint64_t>(g, 148ull * 32));
}

cudaError_t launch_derivative(const uint8_t* in, uint8_t* out, uint32_t ts, uint32_t G, int D,
                              const uint16_t* deriv_factors, cudaStream_t st) {
    DerivFactors df{};
    std::copy(deriv_factors, deriv_factors + 16, df.f);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid_for((uint64_t)ts * G, 128));
    cfg.blockDim = dim3(128);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, derivative_kernel, in, out, ts, G, D, df);
}

int log2_floor(uint32_t v) {
    int r = 0;
    while (v >>= 1) r++;
    return r;
}

// Column groups per tile: a power of two, at most 16 (whole rows up to L = 1 KiB).
uint32_t tile_groups(uint32_t G) {
    uint32_t gt = 1;
    while (gt * 2 <= std::min<uint32_t>(G, 16)) gt *= 2;
    return gt;
}

struct PassPlan {
    int l0, c, e;
};

// Passes of a transform of 2^D rows, top-down: the deepest pass has no row
// bits below its levels (e = 0) and takes log2(kTileNominal / gt) levels;
// the passes above it take the low bits a uniform factor per warp needs
// (gt * 2^e >= 32) and at most log2(kTileElems / gt) - e levels each, as
// few passes as that allows with the levels spread evenly.
std::vector<PassPlan> plan_passes(int D, uint32_t gt) {
    std::vector<PassPlan> out;
    if (D <= 0) return out;
    const int c_last = std::min(D, log2_floor(kTileNominal / gt));
    const int rest = D - c_last;
    if (rest > 0) {
        const int e = std::max(0, 5 - log2_floor(gt));
        const int c_max = std::max(1, log2_floor(kTileElems / gt) - e);
        const int n = (rest + c_max - 1) / c_max;
        for (int q = 0, l0 = 0; q < n; q++) {
            const int c = rest / n + (q < rest % n ? 1 : 0);
            out.push_back({l0, c, std::min(e, D - l0 - c)});
            l0 += c;
        }
    }
    out.push_back({rest, c_last, 0});
    return out;
}

// Shared memory after the tile: the node factors of up to two phases of a
// pass of at most 10 levels (2 * (2^10 - 1) uint16).
constexpr size_t kFactorSmem = 2 * 1024 * 2;

cudaError_t set_tile_attr() {
    static std::atomic<uint64_t> attr{0};
    return once_per_device(attr, [] {
        return cudaFuncSetAttribute(afft_tile_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)(kTileElems * 64 + kFactorSmem));
    });
}

cudaError_t launch_pass(uint8_t* work, uint32_t G, int D, const PassPlan& P, uint32_t gt, const PassPhases& ph,
                        const uint16_t* factors, const PassIo& io, int slice, int unslice, cudaStream_t st) {
    const uint32_t col_tiles = (G + gt - 1) / gt;
    const uint32_t tiles = (1u << (D - P.c - P.e)) * col_tiles;
    const size_t rows = (size_t)1 << (P.c + P.e);
    const size_t smem = rows * gt * 64 + (size_t)std::max(ph.n, 1) * (((size_t)1 << P.c) - 1) * 2;
    // one butterfly per thread and level: a multiple of 32 threads, at most kTileThreads
    const uint32_t bfly = (uint32_t)(rows / 2) * gt;
    const int threads = (int)std::min<uint32_t>(kTileThreads, std::max<uint32_t>(32, (bfly + 31) / 32 * 32));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(tiles);
    cfg.blockDim = dim3(threads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, afft_tile_kernel, work, G, D, P.l0, P.c, P.e, gt, ph, factors, io, slice, unslice);
}

// Full transform of 2^D bit-sliced rows (heap root `root`: 1 for the whole
// transform; 2 and 3 for the halves below it, each of 2^D rows, D one less),
// forward (top-down) or inverse (bottom-up).  With io.src the first pass
// slices the rows in from bytes (see PassIo); with io.dst the last pass
// writes its output rows as bytes instead of back to the work array.
cudaError_t run_transform(uint8_t* work, uint32_t G, int D, const uint16_t* factors, bool forward,
                          cudaStream_t st, uint32_t root = 1, const PassIo& io = PassIo{}) {
    cudaError_t e = set_tile_attr();
    if (e != cudaSuccess) return e;
    const uint32_t gt = tile_groups(G);
    std::vector<PassPlan> plan = plan_passes(D, gt);
    if (!forward) std::reverse(plan.begin(), plan.end());
    const PassPhases ph{{root, 0}, {forward ? 1 : 0, 0}, 1};
    for (size_t q = 0; q < plan.size(); q++) {
        e = launch_pass(work, G, D, plan[q], gt, ph, factors, io, q == 0 && io.src, q + 1 == plan.size() && io.dst,
                        st);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// Encode of a power-of-two k (ts = 2k, m <= k): the k data rows bit-sliced
// into the work array, the inverse transform over them as the left half
// (heap root 2), the forward transform of the result as the right half
// (root 3), its first m rows unsliced into the repairs.  The inverse's top
// pass and the forward's top pass share one launch; the first pass slices
// the data on the way in, the last one unslices the repairs on the way out.
cudaError_t run_encode_halves(uint8_t* work, uint32_t G, int D, const uint16_t* factors, const uint8_t* data,
                              uint32_t k, uint32_t m, uint64_t L, uint8_t* repairs, cudaStream_t st) {
    cudaError_t e = set_tile_attr();
    if (e != cudaSuccess) return e;
    const uint32_t gt = tile_groups(G);
    const std::vector<PassPlan> plan = plan_passes(D, gt);  // top-down
    const size_t np = plan.size();
    PassIo io{};
    io.src = data;
    io.n_src = k;
    io.dst = repairs;
    io.out_lo = 0;
    io.out_hi = m;
    io.L = L;
    if (np == 0) {  // k = 1: no levels; the one data row is the repair
        const PassPhases none{{0, 0}, {0, 0}, 0};
        return launch_pass(work, G, 0, PassPlan{0, 0, 0}, gt, none, factors, io, 1, 1, st);
    }
    // inverse, bottom-up: plan[np-1] .. plan[1]; then plan[0] inverse + forward;
    // then forward top-down: plan[1] .. plan[np-1]
    for (size_t q = np; q-- > 1;) {
        const PassPhases inv{{2, 0}, {0, 0}, 1};
        e = launch_pass(work, G, D, plan[q], gt, inv, factors, io, q == np - 1, 0, st);
        if (e != cudaSuccess) return e;
    }
    const PassPhases both{{2, 3}, {0, 1}, 2};
    e = launch_pass(work, G, D, plan[0], gt, both, factors, io, np == 1, np == 1, st);
    if (e != cudaSuccess) return e;
    for (size_t q = 1; q < np; q++) {
        const PassPhases fw{{3, 0}, {1, 0}, 1};
        e = launch_pass(work, G, D, plan[q], gt, fw, factors, io, 0, q == np - 1, st);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

uint32_t mod_pow(uint32_t base, uint32_t e) {
    uint64_t r = 1, b = base;
    while (e) {
        if (e & 1) r = r * b % kMult;
        b = b * b % kMult;
        e >>= 1;
    }
    return (uint32_t)r;
}

// One Walsh-Hadamard transform of v (2^D entries) as passes of at most 8
// index bits, enough groups per pass to spread over the SMs; in_mode and
// out_mode as wht_pass_kernel, applied on the first and last pass.
cudaError_t run_wht(uint32_t* v, uint32_t ts, int D, int in_mode, int out_mode, const uint8_t* known,
                    const uint32_t* lw, const uint16_t* exp16, uint16_t* values, uint16_t* derivs,
                    cudaStream_t st) {
    static std::atomic<uint64_t> attr{0};
    cudaError_t ea = once_per_device(attr, [] {
        return cudaFuncSetAttribute(wht_pass_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 8192 * 4);
    });
    if (ea != cudaSuccess) return ea;
    const int n_pass = (D + 7) / 8;
    for (int q = 0, lo = 0; q < n_pass; q++) {
        const int nb = (D - lo + (n_pass - q) - 1) / (n_pass - q);
        const uint32_t groups = ts >> nb, gsize = 1u << nb;
        // chained after the pass before it (programmatic dependent launch);
        // the locator's first pass follows the upload, a copy, and is plain
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(groups);
        cfg.blockDim = dim3(std::min<uint32_t>(1024, std::max<uint32_t>(32, gsize / 2)));
        cfg.dynamicSmemBytes = gsize * 4;
        cfg.stream = st;
        cfg.attrs = attr;
        cfg.numAttrs = (q == 0 && in_mode) ? 0 : 1;
        cudaError_t e = cudaLaunchKernelEx(&cfg, wht_pass_kernel, v, lo, nb, q == 0 ? in_mode : 0,
                                           q + 1 == n_pass ? out_mode : 0, known, lw, exp16, values, derivs);
        if (e != cudaSuccess) return e;
        lo += nb;
    }
    return cudaSuccess;
}

// The logarithm table's first ts entries (log 0 = 0, as the device table),
// Walsh-Hadamard transformed mod 65535 (decoder.rs:691-694), times the final
// transform's 1/ts (decoder.rs:700-703).
std::vector<uint32_t> log_walsh_host(uint32_t ts, int D) {
    static const std::vector<uint32_t> lg = [] {
        std::vector<uint32_t> t(65536, 0);
        uint16_t v = 1;
        for (uint32_t i = 0; i < kMult; i++) {
            t[v] = i;
            v = hf::mul16(v, hf::kGen16);
        }
        return t;
    }();
    std::vector<uint32_t> w(lg.begin(), lg.begin() + ts);
    for (uint32_t h = 1; h < ts; h <<= 1)
        for (uint32_t b = 0; b < ts; b += 2 * h)
            for (uint32_t p = b; p < b + h; p++) {
                const uint32_t a = w[p], c = w[p + h];
                w[p] = a + c >= kMult ? a + c - kMult : a + c;
                w[p + h] = a >= c ? a - c : a + kMult - c;
            }
    const uint64_t inv = mod_pow(32768, (uint32_t)D);
    for (auto& e : w) e = (uint32_t)(e * inv % kMult);
    return w;
}

}  // namespace

int32_t afft_locator_device(const uint8_t* d_known, uint32_t ts, const uint32_t* log_walsh, uint32_t* wa,
                            uint16_t* values, uint16_t* derivs, cudaStream_t st, scrs_error* err) {
    const uint16_t *lg, *ex;
    SCRS_CUDA(log16_tables(&lg, &ex));
    int D = 0;
    while ((1u << D) < ts) D++;
    if (ts <= kLocatorOneCtaTs) {
        static std::atomic<uint64_t> attr{0};
        SCRS_CUDA(once_per_device(attr, [] {
            return cudaFuncSetAttribute(locator_one_cta_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)(kLocatorOneCtaTs * sizeof(uint32_t)));
        }));
        locator_one_cta_kernel<<<1, kLocatorThreads, ts * sizeof(uint32_t), st>>>(d_known, D, log_walsh, ex, values,
                                                                                   derivs);
        SCRS_CUDA(cudaGetLastError());
        return SCRS_OK;
    }
    SCRS_CUDA(run_wht(wa, ts, D, 1, 1, d_known, log_walsh, ex, values, derivs, st));
    SCRS_CUDA(run_wht(wa, ts, D, 0, 2, d_known, log_walsh, ex, values, derivs, st));
    return SCRS_OK;
}

// ---- targeted decode (afft/decoder.rs:360-441) --------------------------------
// With r <= 5 missing data symbols and exactly r received repairs, the repairs
// are linear in the data through the systematic generator rows
// G[t][i] = L_S(e_t) / ((e_t + i) L_S'(i)) (generator_row, decoder.rs:600-619),
// so the missing symbols are A^-1 (repairs + G_P d_P) with A = G restricted
// to the missing columns: one k x r coefficient table and one multiply-XOR
// pass instead of two transforms.
__device__ __forceinline__ uint32_t lmul(const uint16_t* lg, const uint16_t* ex, uint32_t a, uint32_t b) {
    if (!a || !b) return 0;
    uint32_t e = (uint32_t)lg[a] + lg[b];
    return ex[e >= kMult ? e - kMult : e];
}

// gen[t*k + i] = G[t][i] for the r received repairs at evaluation points rep[t].
// Launched chained after the present-row copy, whose output it does not read:
// it runs beside it and waits for it only before exiting.
__global__ void targeted_gen_kernel(const uint16_t* sys_values, const uint16_t* sys_derivs, const uint16_t* lg,
                                    const uint16_t* ex, const uint16_t* rep, uint32_t r, uint32_t k, uint16_t* gen) {
    pdl_trigger();
    for (uint64_t x = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; x < (uint64_t)r * k;
         x += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t t = (uint32_t)(x / k), i = (uint32_t)(x - (uint64_t)t * k);
        const uint32_t e = rep[t];
        uint32_t lv = (uint32_t)lg[sys_values[e]] + 2 * kMult - lg[e ^ i] - lg[sys_derivs[i]];
        gen[x] = ex[lv % kMult];
    }
    pdl_wait();
}

// Fused coefficients, rows 0..r-1 the received repairs (A^-1 columns), rows
// r.. the present data rows: row z, output s = sum_t (A^-1)[s][t] G[t][present[z]].
__global__ void targeted_fuse_kernel(const uint16_t* gen, const uint16_t* inv_g, const uint16_t* present, uint32_t r,
                                     uint32_t k, const uint16_t* lg, const uint16_t* ex, uint16_t* coef) {
    __shared__ uint32_t inv[kTargetedMax * kTargetedMax];
    pdl_trigger();
    for (uint32_t x = threadIdx.x; x < r * r; x += blockDim.x) inv[x] = inv_g[x];  // uploaded, not computed
    pdl_wait();  // gen is the previous kernel's output
    __syncthreads();
    for (uint64_t x = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; x < (uint64_t)k * r;
         x += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t row = (uint32_t)(x / r), s = (uint32_t)(x - (uint64_t)row * r);
        uint32_t v;
        if (row < r) {
            v = inv[s * r + row];
        } else {
            const uint32_t p = present[row - r];
            v = 0;
            for (uint32_t t = 0; t < r; t++) v ^= lmul(lg, ex, inv[s * r + t], gen[(size_t)t * k + p]);
        }
        coef[x] = (uint16_t)v;
    }
}

// ---- AfftCodec -------------------------------------------------------------------
int32_t AfftCodec::init(uint64_t k_, uint64_t m_, uint64_t L_, scrs_error* err) {
    k = k_, m = m_, L = L_, n = k + m;
    // profile.rs:16-38 (the caller already validated dimensions and parity)
    if (n > 65536) return set_err(err, SCRS_CONFIG_TOO_MANY_SYMBOLS, 65536);
    padded_k = 1;
    while (padded_k < k) padded_k <<= 1;
    ts = 1;
    log_ts = 0;
    while (ts < n) ts <<= 1, log_ts++;
    SubspacePoly polys[16];
    subspace_polynomials((int)log_ts, polys);
    std::vector<uint16_t> f(ts, 0);
    for (uint32_t j = 0; j < log_ts; j++) deriv_factors[j] = hf::mul16(polys[j].coeffs[0], polys[j].norm_inv);
    if (log_ts) fill_factors(f, polys, 1, (int)log_ts, 0);
    SCRS_CUDA(factors.ensure(ts * 2));
    SCRS_CUDA(cudaMemcpy(factors.p, f.data(), ts * 2, cudaMemcpyHostToDevice));
    const std::vector<uint32_t> lw = log_walsh_host((uint32_t)ts, (int)log_ts);
    SCRS_CUDA(log_walsh.ensure(ts * 4));
    SCRS_CUDA(cudaMemcpy(log_walsh.p, lw.data(), ts * 4, cudaMemcpyHostToDevice));
    // Encode locator: known = [0, k), erased = [k, ts), fixed per geometry.
    SCRS_CUDA(enc_values.ensure(ts * 2));
    SCRS_CUDA(enc_derivs.ensure(ts * 2));
    DevBuf known, wa;
    std::vector<uint8_t> hk(ts, 0);
    std::fill(hk.begin(), hk.begin() + k, 1);
    SCRS_CUDA(known.ensure(ts));
    SCRS_CUDA(wa.ensure(ts * 4));
    SCRS_CUDA(cudaMemcpy(known.p, hk.data(), ts, cudaMemcpyHostToDevice));
    int32_t r = afft_locator_device(known.as<uint8_t>(), (uint32_t)ts, log_walsh.as<uint32_t>(), wa.as<uint32_t>(),
                                    enc_values.as<uint16_t>(), enc_derivs.as<uint16_t>(), 0, err);
    if (r) return r;
    // Systematic locator for the targeted decode: known = [k, ts), erased = [0, k).
    SCRS_CUDA(sys_values.ensure(ts * 2));
    SCRS_CUDA(sys_derivs.ensure(ts * 2));
    SCRS_CUDA(cudaStreamSynchronize(0));  // `known` is rewritten below
    for (uint64_t i = 0; i < ts; i++) hk[i] = i >= k ? 1 : 0;
    SCRS_CUDA(cudaMemcpy(known.p, hk.data(), ts, cudaMemcpyHostToDevice));
    r = afft_locator_device(known.as<uint8_t>(), (uint32_t)ts, log_walsh.as<uint32_t>(), wa.as<uint32_t>(),
                            sys_values.as<uint16_t>(), sys_derivs.as<uint16_t>(), 0, err);
    if (r) return r;
    SCRS_CUDA(cudaStreamSynchronize(0));  // the locators ran on the legacy stream
    // host copies for the targeted decode's r x r solve
    h_sys_values.resize(ts);
    h_sys_derivs.resize(ts);
    SCRS_CUDA(cudaMemcpy(h_sys_values.data(), sys_values.p, ts * 2, cudaMemcpyDeviceToHost));
    SCRS_CUDA(cudaMemcpy(h_sys_derivs.data(), sys_derivs.p, ts * 2, cudaMemcpyDeviceToHost));
    return SCRS_OK;
}

int32_t AfftWorkspace::init_encode(const AfftCodec& c, scrs_error* err) {
    k = c.k, m = c.m, L = c.L;
    const uint64_t G = (c.L + 63) / 64;
    SCRS_CUDA(work0.ensure(c.ts * G * 64));
    SCRS_CUDA(work1.ensure(c.ts * G * 64));
    SCRS_CUDA(known.ensure(c.ts));
    std::vector<uint8_t> hk(c.ts, 0);
    std::fill(hk.begin(), hk.begin() + c.k, 1);
    SCRS_CUDA(upload_now(known.p, hk.data(), c.ts));
    return SCRS_OK;
}

AfftWorkspace::~AfftWorkspace() {
    for (int i = 0; i < 2; i++) {
        if (!staged[i]) continue;
        if (stage_pending[i]) cudaEventSynchronize(staged[i]);  // copies still reading the area
        cudaEventDestroy(staged[i]);
    }
}

int32_t AfftWorkspace::stage_acquire(scrs_error* err) {
    cur ^= 1;
    if (stage_pending[cur]) SCRS_CUDA(cudaEventSynchronize(staged[cur]));
    stage_pending[cur] = false;
    return SCRS_OK;
}

int32_t AfftWorkspace::stage_release(cudaStream_t st, scrs_error* err) {
    SCRS_CUDA(cudaEventRecord(staged[cur], st));
    stage_pending[cur] = true;
    return SCRS_OK;
}

int32_t AfftWorkspace::init_decode(const AfftCodec& c, scrs_error* err) {
    k = c.k, m = c.m, L = c.L;
    const uint64_t G = (c.L + 63) / 64;
    SCRS_CUDA(work0.ensure(c.ts * G * 64));
    SCRS_CUDA(work1.ensure(c.ts * G * 64));
    SCRS_CUDA(wht_a.ensure(c.ts * 4));
    SCRS_CUDA(values.ensure(c.ts * 2));
    SCRS_CUDA(derivs.ensure(c.ts * 2));
    const size_t rows_bytes = (2 * c.k + 8) * 2;
    const size_t lists_elems = c.targeted_list_elems();
    off_map = (rows_bytes + 15) & ~(size_t)15;
    off_known = (off_map + c.n * 2 + 15) & ~(size_t)15;
    off_lists = (off_known + c.ts + 15) & ~(size_t)15;
    for (int i = 0; i < 2; i++) {
        SCRS_CUDA(stage[i].ensure(off_lists + lists_elems * 2));
        memset(stage[i].p, 0, stage[i].bytes);
        if (!staged[i]) SCRS_CUDA(cudaEventCreateWithFlags(&staged[i], cudaEventDisableTiming));
    }
    SCRS_CUDA(up.ensure(off_lists + lists_elems * 2));
    SCRS_CUDA(tgen.ensure(kTargetedMax * c.k * 2));
    SCRS_CUDA(tcoef.ensure(kTargetedMax * c.k * 2));
    return SCRS_OK;
}

int32_t AfftCodec::encode(const uint8_t* d_data, uint8_t* d_repairs, AfftWorkspace& ws, int32_t* status,
                          cudaStream_t st, scrs_error* err) const {
    (void)status;
    const uint32_t G = (uint32_t)((L + 63) / 64);
    if (2 * k == ts) {
        // k a power of two (and m <= k): the data points are the left half of
        // the transform's points and the repair points the first m of the right
        // half.  The top butterfly level of a forward transform whose upper
        // coefficients are zero copies the lower half into the upper, so the
        // repairs are the right half-transform of the left half-transform's
        // inverse of the data: two transforms of k points, no locator, no
        // derivative (the reference encoder is this IFFT-then-forward form,
        // afft/encoder.rs:150-250).
        SCRS_CUDA(run_encode_halves(ws.work0.as<uint8_t>(), G, (int)log_ts - 1, factors.as<uint16_t>(), d_data,
                                    (uint32_t)k, (uint32_t)m, L, d_repairs, st));
        return SCRS_OK;
    }
    // general k: the erasure-decode form with E = [k, ts) (see afft_engine.h)
    const uint16_t *lg, *ex;
    SCRS_CUDA(log16_tables(&lg, &ex));
    PassIo in{};
    in.src = d_data;
    in.known = ws.known.as<uint8_t>();
    in.in_scale = enc_values.as<uint16_t>();
    in.n_src = (uint32_t)k;
    in.L = L;
    SCRS_CUDA(run_transform(ws.work0.as<uint8_t>(), G, (int)log_ts, factors.as<uint16_t>(), false, st, 1, in));
    SCRS_CUDA(launch_derivative(ws.work0.as<uint8_t>(), ws.work1.as<uint8_t>(), (uint32_t)ts, G, (int)log_ts,
                                deriv_factors, st));
    PassIo out{};
    out.known = ws.known.as<uint8_t>();
    out.out_lo = (uint32_t)k;
    out.out_hi = (uint32_t)(k + m);
    out.dst = d_repairs;
    out.out_derivs = enc_derivs.as<uint16_t>();
    out.log16 = lg;
    out.exp16 = ex;
    out.L = L;
    SCRS_CUDA(run_transform(ws.work1.as<uint8_t>(), G, (int)log_ts, factors.as<uint16_t>(), true, st, 1, out));
    return SCRS_OK;
}

int32_t AfftCodec::decode(const uint8_t* d_payloads, const uint8_t* have, uint8_t* d_out, AfftWorkspace& ws,
                          int32_t* status, cudaStream_t st, scrs_error* err, const uint16_t* row_map) const {
    (void)status;
    const uint32_t G = (uint32_t)((L + 63) / 64);
    const uint16_t *lg, *ex;
    SCRS_CUDA(log16_tables(&lg, &ex));
    // missing data rows (afft/decoder.rs:276-286) and present data rows
    int32_t rc = ws.stage_acquire(err);
    if (rc) return rc;
    uint8_t* stage = ws.stage_ptr();
    uint16_t* miss = reinterpret_cast<uint16_t*>(stage);
    uint16_t* pres = miss + k;
    uint32_t nm = 0, np = 0;
    for (uint64_t d = 0; d < k; d++) {
        if (have[d])
            pres[np++] = (uint16_t)d;
        else
            miss[nm++] = (uint16_t)d;
    }
    // Everything the decode uploads sits in one stage area laid out as its
    // device mirror (rows | codeword -> payload map | known mask | targeted
    // lists), so it goes up in one copy.
    size_t upload = (2 * k + 8) * 2;
    if (row_map) {
        memcpy(stage + ws.off_map, row_map, n * 2);
        upload = ws.off_map + n * 2;
    }
    const bool targeted = nm > 0 && nm <= kTargetedMax;
    if (targeted) {
        rc = targeted_lists(have, ws, err, row_map, miss, nm, pres, np);
        if (rc) {
            const int32_t rr = ws.stage_release(st, err);
            return rc ? rc : rr;
        }
        upload = ws.off_lists + targeted_list_elems() * 2;
    } else if (nm > 0) {
        uint8_t* known = stage + ws.off_known;
        memcpy(known, have, n);  // receipt flags are 0 / 1
        memset(known + n, 0, ts - n);
        upload = ws.off_known + ts;
    }
    SCRS_CUDA(cudaMemcpyAsync(ws.up.p, stage, upload, cudaMemcpyHostToDevice, st));
    rc = ws.stage_release(st, err);
    if (rc) return rc;
    const uint8_t* dev = ws.up.as<uint8_t>();
    const uint16_t* d_pres = reinterpret_cast<const uint16_t*>(dev) + k;
    const uint16_t* d_map = row_map ? reinterpret_cast<const uint16_t*>(dev + ws.off_map) : nullptr;
    const uint8_t* d_known = dev + ws.off_known;
    // the present data rows, straight from the payloads into the output
    // chain: trigger the next kernel at once and wait for the previous one
    // before exiting; attr: launched with programmatic dependent launch
    auto copy_present = [&](int chain, bool attr_on) -> cudaError_t {
        if (!np) return cudaSuccess;
        const bool vec = L % 16 == 0 && (reinterpret_cast<uintptr_t>(d_payloads) & 15) == 0 &&
                         (reinterpret_cast<uintptr_t>(d_out) & 15) == 0;
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(vec ? grid_for((uint64_t)np * (L / 16), 256) : grid_for((uint64_t)np * L, 256));
        cfg.blockDim = dim3(256);
        cfg.stream = st;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = attr;
        cfg.numAttrs = attr_on ? 1 : 0;
        return vec ? cudaLaunchKernelEx(&cfg, copy_rows_kernel<16>, d_payloads, d_out, L, d_pres, np, d_map, chain)
                   : cudaLaunchKernelEx(&cfg, copy_rows_kernel<1>, d_payloads, d_out, L, d_pres, np, d_map, chain);
    };
    if (nm == 0) {
        SCRS_CUDA(copy_present(0, false));
        return SCRS_OK;
    }
    if (targeted) {
        // after the upload (a copy, not a kernel): launched plainly, it lets
        // the targeted kernels chained after it start beside it
        SCRS_CUDA(copy_present(np ? 1 : 0, false));
        return decode_targeted(d_payloads, d_out, ws, status, st, err, nm, np > 0);
    }
    int32_t r = afft_locator_device(d_known, (uint32_t)ts, log_walsh.as<uint32_t>(), ws.wht_a.as<uint32_t>(),
                                    ws.values.as<uint16_t>(), ws.derivs.as<uint16_t>(), st, err);
    if (r) return r;
    // the copy runs beside the locator (it reads none of its output) and
    // exits after it, so the first pass's wait covers both
    SCRS_CUDA(copy_present(1, true));
    PassIo in{};
    in.src = d_payloads;
    in.known = d_known;
    in.row_map = d_map;
    in.in_scale = ws.values.as<uint16_t>();
    in.n_src = (uint32_t)ts;
    in.L = L;
    in.early_read = 1;  // the previous kernels are the locator and the chained copy
    SCRS_CUDA(run_transform(ws.work0.as<uint8_t>(), G, (int)log_ts, factors.as<uint16_t>(), false, st, 1, in));
    SCRS_CUDA(launch_derivative(ws.work0.as<uint8_t>(), ws.work1.as<uint8_t>(), (uint32_t)ts, G, (int)log_ts,
                                deriv_factors, st));
    // the missing data rows: rows of [0, k) not known
    PassIo out{};
    out.known = d_known;
    out.out_lo = 0;
    out.out_hi = (uint32_t)k;
    out.dst = d_out;
    out.out_derivs = ws.derivs.as<uint16_t>();
    out.log16 = lg;
    out.exp16 = ex;
    out.L = L;
    SCRS_CUDA(run_transform(ws.work1.as<uint8_t>(), G, (int)log_ts, factors.as<uint16_t>(), true, st, 1, out));
    return SCRS_OK;
}

// Targeted lists in the stage area (at off_lists): in_rows[k] (the received
// repairs' payload rows, then the present data rows'), out_rows[5],
// rep[5] (the repairs' evaluation points), missing[5], present[k], then room
// for the r x r inverse the device writes.
size_t AfftCodec::targeted_list_elems() const { return 3 * k + 4 * kTargetedMax + kTargetedMax * kTargetedMax + 8; }

int32_t AfftCodec::targeted_lists(const uint8_t* have, AfftWorkspace& ws, scrs_error* err, const uint16_t* row_map,
                                  const uint16_t* miss, uint32_t nm, const uint16_t* pres, uint32_t np) const {
    uint16_t* h = reinterpret_cast<uint16_t*>(ws.stage_ptr() + ws.off_lists);  // acquired by decode()
    uint16_t* in_rows = h;
    uint16_t* out_rows = in_rows + k;
    uint16_t* rep = out_rows + kTargetedMax;
    uint16_t* mis = rep + kTargetedMax;
    uint16_t* prs = mis + kTargetedMax;
    uint32_t nr = 0;
    for (uint64_t w = k; w < n && nr < nm; w++)
        if (have[w]) rep[nr++] = (uint16_t)w;
    if (nr != nm) return set_err(err, SCRS_DECODE_INSUFFICIENT_RANK, k, k - nm + nr);
    auto payload_row = [&](uint32_t w) { return row_map ? row_map[w] : (uint16_t)w; };
    for (uint32_t t = 0; t < nm; t++) in_rows[t] = payload_row(rep[t]), out_rows[t] = miss[t], mis[t] = miss[t];
    for (uint32_t z = 0; z < np; z++) in_rows[nm + z] = payload_row(pres[z]), prs[z] = pres[z];
    // A[t][s] = G[t][missing s], G[t][i] = L_S(e_t) / ((e_t + i) L_S'(i))
    // (generator_row, decoder.rs:600-619), inverted by Gauss-Jordan over
    // GF(2^16) (invert_square_into, decoder.rs:619-670): r <= 5, so on the
    // host, into the list area after the present rows (uploaded with it).
    uint16_t a[kTargetedMax][2 * kTargetedMax];
    for (uint32_t t = 0; t < nm; t++)
        for (uint32_t s = 0; s < nm; s++) {
            const uint16_t d = hf::mul16((uint16_t)(rep[t] ^ miss[s]), h_sys_derivs[miss[s]]);
            a[t][s] = hf::mul16(h_sys_values[rep[t]], hf::inv16(d));
            a[t][nm + s] = t == s;
        }
    for (uint32_t col = 0; col < nm; col++) {
        uint32_t piv = col;
        while (piv < nm && !a[piv][col]) piv++;
        if (piv == nm) return set_err(err, SCRS_DECODE_INSUFFICIENT_RANK, k, k - 1);
        if (piv != col)
            for (uint32_t q = 0; q < 2 * nm; q++) std::swap(a[col][q], a[piv][q]);
        const uint16_t pinv = hf::inv16(a[col][col]);
        for (uint32_t q = 0; q < 2 * nm; q++) a[col][q] = hf::mul16(a[col][q], pinv);
        for (uint32_t t = 0; t < nm; t++) {
            if (t == col || !a[t][col]) continue;
            const uint16_t f = a[t][col];
            for (uint32_t q = 0; q < 2 * nm; q++) a[t][q] ^= hf::mul16(f, a[col][q]);
        }
    }
    uint16_t* inv = prs + k;
    for (uint32_t s = 0; s < nm; s++)
        for (uint32_t t = 0; t < nm; t++) inv[s * nm + t] = a[s][nm + t];
    return SCRS_OK;
}

// The launches are chained (programmatic dependent launch): each kernel may
// start while the one before it runs, reads that kernel's output only after
// waiting for it, and has waited for it by the time it exits, so the last
// one's completion covers them all.
int32_t AfftCodec::decode_targeted(const uint8_t* d_payloads, uint8_t* d_out, AfftWorkspace& ws, int32_t* status,
                                   cudaStream_t st, scrs_error* err, uint32_t nm, bool after_copy) const {
    const uint16_t *lg, *ex;
    SCRS_CUDA(log16_tables(&lg, &ex));
    const uint16_t* d_in_rows = reinterpret_cast<const uint16_t*>(ws.up.as<uint8_t>() + ws.off_lists);
    const uint16_t* d_out_rows = d_in_rows + k;
    const uint16_t* d_rep = d_out_rows + kTargetedMax;
    const uint16_t* d_mis = d_rep + kTargetedMax;
    const uint16_t* d_prs = d_mis + kTargetedMax;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.blockDim = dim3(256);
    cfg.stream = st;
    cfg.attrs = attr;
    // after the upload alone (a copy, not a kernel) the first launch is plain
    cfg.numAttrs = after_copy ? 1 : 0;
    cfg.gridDim = dim3(grid_for((uint64_t)nm * k, 256));
    SCRS_CUDA(cudaLaunchKernelEx(&cfg, targeted_gen_kernel, sys_values.as<uint16_t>(), sys_derivs.as<uint16_t>(), lg,
                                 ex, d_rep, nm, (uint32_t)k, ws.tgen.as<uint16_t>()));
    const uint16_t* d_inv = d_prs + k;  // r*r entries of A^-1 after the present list
    cfg.numAttrs = 1;
    cfg.gridDim = dim3(grid_for((uint64_t)k * nm, 256));
    SCRS_CUDA(cudaLaunchKernelEx(&cfg, targeted_fuse_kernel, (const uint16_t*)ws.tgen.as<uint16_t>(), d_inv, d_prs,
                                 nm, (uint32_t)k, lg, ex, ws.tcoef.as<uint16_t>()));
    MxkTask T{};
    T.in = d_payloads;
    T.out = d_out;
    T.coef = ws.tcoef.p;
    T.in_rows = d_in_rows;
    T.out_rows = d_out_rows;
    T.L = L;
    T.in_stride = L;
    T.out_stride = L;
    T.n_in = (uint32_t)k;
    T.n_out = nm;
    T.ld = nm;
    T.n_items = n_chunks(L, true);
    T.aligned = (L % 16 == 0 && aligned16(d_payloads) && aligned16(d_out)) ? 1u : 0u;
    // k inputs: the launch splits them over CTAs (input-split form) when the
    // output rows allow 4-byte atomics, else walks them per chunk
    SCRS_CUDA(launch_mxk_single(T, 1, status, 0, st, /*chain=*/true));
    return SCRS_OK;
}

}  // namespace scrs
