// Additive FFT over GF(2^16) on sm_100a: transform passes, formal
// derivative, erasure locator (Walsh-Hadamard in the log domain) and the
// encode/decode pipelines built from them.
//
// Rows between stages are kept bit-sliced in HBM: a row of L bytes is stored
// as G = ceil(L/64) groups of 64 bytes, each group the 16 bit planes of 32
// field elements (scrs_b200/csrc/common.cuh bitslice16).  Bytes are sliced
// once on the way in (scale_in) and unsliced once on the way out (scale_out).
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
constexpr int kPassThreads = 256;
constexpr int kTileBytes = 64 * 1024;
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

// Walsh-Hadamard butterflies over index bits [lo, lo + nb) (decoder.rs:732-755);
// one CTA per group of 2^nb elements that differ only in those bits.
__global__ void __launch_bounds__(1024) wht_pass_kernel(uint32_t* v, uint32_t ts, int lo, int nb) {
    extern __shared__ uint32_t sv[];
    const uint32_t gsize = 1u << nb;
    const uint32_t gidx = blockIdx.x;
    const uint32_t base = ((gidx >> lo) << (lo + nb)) | (gidx & ((1u << lo) - 1u));
    for (uint32_t t = threadIdx.x; t < gsize; t += blockDim.x) sv[t] = v[base + ((size_t)t << lo)];
    __syncthreads();
    for (uint32_t half = 1; half < gsize; half <<= 1) {
        for (uint32_t p = threadIdx.x; p < gsize / 2; p += blockDim.x) {
            uint32_t i = ((p / half) * 2 * half) + (p % half);
            uint32_t a = sv[i], b = sv[i + half];
            sv[i] = add_mod(a, b);
            sv[i + half] = sub_mod(a, b);
        }
        __syncthreads();
    }
    for (uint32_t t = threadIdx.x; t < gsize; t += blockDim.x) v[base + ((size_t)t << lo)] = sv[t];
}

__global__ void locator_init_kernel(const uint8_t* known, uint32_t ts, const uint16_t* log16, uint32_t* a,
                                    uint32_t* b) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < ts; i += gridDim.x * blockDim.x) {
        a[i] = known[i] ? 0u : 1u;
        b[i] = log16[i];
    }
}

__global__ void locator_mul_kernel(uint32_t* a, const uint32_t* b, uint32_t ts) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < ts; i += gridDim.x * blockDim.x)
        a[i] = (uint32_t)(((uint64_t)a[i] * b[i]) % kMult);
}

// The whole locator in one CTA for transforms of at most kLocatorOneCtaTs
// points: the same steps as locator_init -> 2 WHTs -> locator_mul -> WHT ->
// locator_finish, on shared-memory copies of both arrays (one launch instead
// of nine; at these sizes launch gaps, not arithmetic, set the time).
constexpr uint32_t kLocatorOneCtaTs = 16384;

__device__ __forceinline__ void wht_block(uint32_t* v, uint32_t ts) {
    for (uint32_t half = 1; half < ts; half <<= 1) {
        for (uint32_t p = threadIdx.x; p < ts / 2; p += blockDim.x) {
            const uint32_t i = ((p / half) * 2 * half) + (p % half);
            const uint32_t a = v[i], b = v[i + half];
            v[i] = add_mod(a, b);
            v[i + half] = sub_mod(a, b);
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(1024) locator_one_cta_kernel(const uint8_t* known, uint32_t ts, uint32_t inv_size,
                                                               const uint16_t* log16, const uint16_t* exp16,
                                                               uint16_t* values, uint16_t* derivs) {
    extern __shared__ uint32_t sm_loc[];
    uint32_t* a = sm_loc;
    uint32_t* b = sm_loc + ts;
    for (uint32_t i = threadIdx.x; i < ts; i += blockDim.x) {
        a[i] = known[i] ? 0u : 1u;
        b[i] = log16[i];
    }
    __syncthreads();
    wht_block(a, ts);
    wht_block(b, ts);
    for (uint32_t i = threadIdx.x; i < ts; i += blockDim.x) a[i] = (uint32_t)(((uint64_t)a[i] * b[i]) % kMult);
    __syncthreads();
    wht_block(a, ts);
    for (uint32_t i = threadIdx.x; i < ts; i += blockDim.x) {
        const uint32_t e = (uint32_t)(((uint64_t)a[i] * inv_size) % kMult);
        const uint16_t prod = exp16[e];
        values[i] = known[i] ? prod : 0;
        derivs[i] = known[i] ? 0 : prod;
    }
}

__global__ void locator_finish_kernel(const uint32_t* a, const uint8_t* known, uint32_t ts, uint32_t inv_size,
                                      const uint16_t* exp16, uint16_t* values, uint16_t* derivs) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < ts; i += gridDim.x * blockDim.x) {
        uint32_t e = (uint32_t)(((uint64_t)a[i] * inv_size) % kMult);
        uint16_t prod = exp16[e];
        values[i] = known[i] ? prod : 0;
        derivs[i] = known[i] ? 0 : prod;
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

// work[i] = planes(values[i] * payload_i) for known i < n_rows_src, else 0
// (the product evaluations of F*L, decoder.rs:320-333).  known == nullptr:
// every row is known; values == nullptr: the rows are sliced unscaled.
__global__ void __launch_bounds__(128) scale_in_kernel(const uint8_t* payloads, uint64_t L, uint32_t G,
                                                       const uint8_t* known, const uint16_t* values,
                                                       uint32_t ts, uint8_t* work, const uint16_t* row_map) {
    const uint64_t total = (uint64_t)ts * G;
    for (uint64_t x = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; x < total;
         x += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t row = (uint32_t)(x / G), g = (uint32_t)(x % G);
        uint32_t acc[16];
#pragma unroll
        for (int t = 0; t < 16; t++) acc[t] = 0;
        if (!known || known[row]) {
            uint32_t w[16];
            const uint64_t src = row_map ? row_map[row] : row;
            load_group_bytes(payloads + src * L, g, L, w);
            bitslice16(w);
            if (values) {
                mul16<false>(values[row], acc, w);
            } else {
#pragma unroll
                for (int t = 0; t < 16; t++) acc[t] = w[t];
            }
        }
        store_planes(work + ((uint64_t)row * G + g) * 64, acc);
    }
}

// Novel-basis formal derivative in gather form (transform.rs:188-213):
// out[j] = sum over bits b with j_b = 0 of df[b] * in[j | 2^b].
struct DerivFactors {
    uint16_t f[16];
};

__global__ void __launch_bounds__(128) derivative_kernel(const uint8_t* in, uint8_t* out, uint32_t ts, uint32_t G,
                                                         int D, DerivFactors df) {
    const uint64_t total = (uint64_t)ts * G;
    for (uint64_t x = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; x < total;
         x += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t j = (uint32_t)(x / G), g = (uint32_t)(x % G);
        uint32_t acc[16];
#pragma unroll
        for (int t = 0; t < 16; t++) acc[t] = 0;
        for (int b = 0; b < D; b++) {
            if ((j >> b) & 1u) continue;
            uint32_t w[16];
            load_planes(in + ((uint64_t)(j | (1u << b)) * G + g) * 64, w);
            mul16<true>(df.f[b], acc, w);
        }
        store_planes(out + ((uint64_t)j * G + g) * 64, acc);
    }
}

// out row dst[t] = bytes(inv(derivs[src[t]]) * work[src[t]]) (decoder.rs:348-356);
// derivs == nullptr: the rows are unsliced unscaled.
__global__ void __launch_bounds__(128) scale_out_kernel(const uint8_t* work, uint32_t G, uint64_t L,
                                                        const uint16_t* rows_src, const uint16_t* rows_dst,
                                                        uint32_t count, const uint16_t* derivs,
                                                        const uint16_t* log16, const uint16_t* exp16,
                                                        uint8_t* out) {
    const uint64_t total = (uint64_t)count * G;
    for (uint64_t x = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; x < total;
         x += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t t = (uint32_t)(x / G), g = (uint32_t)(x % G);
        const uint32_t src = rows_src[t];
        uint32_t w[16], acc[16];
        load_planes(work + ((uint64_t)src * G + g) * 64, w);
        if (derivs) {
            const uint16_t d = derivs[src];
            const uint16_t f = d ? exp16[(kMult - log16[d]) % kMult] : 0;
#pragma unroll
            for (int q = 0; q < 16; q++) acc[q] = 0;
            mul16<false>(f, acc, w);
        } else {
#pragma unroll
            for (int q = 0; q < 16; q++) acc[q] = w[q];
        }
        bitslice16(acc);
        store_group_bytes(out + (uint64_t)rows_dst[t] * L, g, L, acc);
    }
}

// dst row rows[t] = src row (row_map ? row_map[rows[t]] : rows[t]), L bytes
// each, in units of `unit` bytes (16 when both bases are 16-byte aligned and
// L is a multiple of 16, else 1).
template <int kUnit>
__global__ void copy_rows_kernel(const uint8_t* src, uint8_t* dst, uint64_t L, const uint16_t* rows,
                                 uint32_t count, const uint16_t* row_map) {
    using U = typename std::conditional<kUnit == 16, uint4, uint8_t>::type;
    const uint64_t per = L / kUnit;
    const uint64_t total = (uint64_t)count * per;
    for (uint64_t x = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; x < total;
         x += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t t = x / per, q = x - t * per;
        const uint64_t r = rows[t];
        const uint64_t s = row_map ? row_map[r] : r;
        reinterpret_cast<U*>(dst + r * L)[q] = reinterpret_cast<const U*>(src + s * L)[q];
    }
}

// Several butterfly levels of one transform on a shared-memory tile
// (transform.rs:301-333 forward_node / inverse_node, flattened by level).
// Rows p and p + 2^(D-1-l) pair at level l; the node factor is
// factors[root*2^l + (p >> (D-l))].  A tile holds the 2^c rows that differ
// only in the c index bits of levels [l0, l0+c), for gt groups of columns.
__global__ void __launch_bounds__(kPassThreads) afft_pass_kernel(uint8_t* work, uint32_t G, int D, uint32_t root,
                                                                 int l0, int c, int forward,
                                                                 const uint16_t* factors, uint32_t gt) {
    extern __shared__ __align__(16) uint8_t tile[];
    const uint32_t col_tiles = (G + gt - 1) / gt;
    const uint32_t low_bits = (uint32_t)(D - l0 - c);
    const uint32_t tid = threadIdx.x;
    const uint32_t rows_in_tile = 1u << c;
    // tile id -> (high index, low index, column tile)
    uint32_t tidx = blockIdx.x;
    const uint32_t ct = tidx % col_tiles;
    tidx /= col_tiles;
    const uint32_t lo = tidx & ((1u << low_bits) - 1u);
    const uint32_t hi = tidx >> low_bits;
    const uint32_t g0 = ct * gt;
    const uint32_t gn = min(gt, G - g0);
    auto row_of = [&](uint32_t i) { return (hi << (D - l0)) | (i << low_bits) | lo; };
    // load: element (i, g, q) = 16 bytes, smem at ((i*4 + q)*gt + g)*16; the
    // copies are asynchronous, so every thread has all of its loads in flight
    const uint32_t pieces = rows_in_tile * gn * 4;
    for (uint32_t x = tid; x < pieces; x += blockDim.x) {
        const uint32_t q = x & 3, g = (x >> 2) % gn, i = (x >> 2) / gn;
        cp_async_16(tile + ((size_t)(i * 4 + q) * gt + g) * 16,
                    work + ((uint64_t)row_of(i) * G + g0 + g) * 64 + 16 * q);
    }
    cp_async_wait_all();
    __syncthreads();
    const uint32_t pairs = rows_in_tile / 2;
    for (int s = 0; s < c; s++) {
        const int lam = forward ? s : c - 1 - s;  // tile-local level
        const int l = l0 + lam;
        const uint32_t b = (uint32_t)(c - 1 - lam);  // tile index bit of this level
        for (uint32_t x = tid; x < pairs * gn; x += blockDim.x) {
            const uint32_t g = x % gn, pi = x / gn;
            const uint32_t ilo = ((pi >> b) << (b + 1)) | (pi & ((1u << b) - 1u));
            const uint32_t ihi = ilo | (1u << b);
            const uint32_t node = (root << l) + (row_of(ilo) >> (D - l));
            const uint32_t f = factors[node];
            uint32_t wl[16], wh[16];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                uint4 a = *reinterpret_cast<const uint4*>(tile + ((size_t)(ilo * 4 + q) * gt + g) * 16);
                uint4 h = *reinterpret_cast<const uint4*>(tile + ((size_t)(ihi * 4 + q) * gt + g) * 16);
                wl[4 * q] = a.x, wl[4 * q + 1] = a.y, wl[4 * q + 2] = a.z, wl[4 * q + 3] = a.w;
                wh[4 * q] = h.x, wh[4 * q + 1] = h.y, wh[4 * q + 2] = h.z, wh[4 * q + 3] = h.w;
            }
            if (forward) {  // low ^= f*high; high ^= low
                if (f) mul16<false>(f, wl, wh);
#pragma unroll
                for (int q = 0; q < 16; q++) wh[q] ^= wl[q];
            } else {  // high ^= low; low ^= f*high
#pragma unroll
                for (int q = 0; q < 16; q++) wh[q] ^= wl[q];
                if (f) mul16<false>(f, wl, wh);
            }
#pragma unroll
            for (int q = 0; q < 4; q++) {
                *reinterpret_cast<uint4*>(tile + ((size_t)(ilo * 4 + q) * gt + g) * 16) =
                    make_uint4(wl[4 * q], wl[4 * q + 1], wl[4 * q + 2], wl[4 * q + 3]);
                *reinterpret_cast<uint4*>(tile + ((size_t)(ihi * 4 + q) * gt + g) * 16) =
                    make_uint4(wh[4 * q], wh[4 * q + 1], wh[4 * q + 2], wh[4 * q + 3]);
            }
        }
        __syncthreads();
    }
    for (uint32_t x = tid; x < pieces; x += blockDim.x) {
        const uint32_t q = x & 3, g = (x >> 2) % gn, i = (x >> 2) / gn;
        *reinterpret_cast<uint4*>(work + ((uint64_t)row_of(i) * G + g0 + g) * 64 + 16 * q) =
            *reinterpret_cast<const uint4*>(tile + ((size_t)(i * 4 + q) * gt + g) * 16);
    }
}

int grid_for(uint64_t items, int threads) {
    uint64_t g = (items + threads - 1) / threads;
    return (int)std::max<uint64_t>(1, std::min<uint64_t>(g, 148ull * 32));
}

// Full transform of 2^D bit-sliced rows (heap root 1), forward or inverse.
// root: heap index of the transform's root node (1: the whole transform of
// 2^D rows; 2 and 3: the halves below it, each of 2^D rows, D one less).
cudaError_t run_transform(uint8_t* work, uint32_t G, int D, const uint16_t* factors, bool forward,
                          cudaStream_t st, uint32_t root = 1) {
    static std::atomic<uint64_t> attr{0};
    cudaError_t ea = once_per_device(attr, [] {
        return cudaFuncSetAttribute(afft_pass_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kTileBytes);
    });
    if (ea != cudaSuccess) return ea;
    // Column groups per tile: up to 8 of one row pair, so that the lanes of a
    // warp (consecutive groups of a few pairs) mostly share the butterfly
    // factor, and tiles stay small enough for two-level-count passes
    // (k = m = 4096, L = 1024: 8 groups give 2 passes of 6-7 levels, 16 gave 3).
    const uint32_t gt = std::min<uint32_t>(G, 8);
    int cmax = 1;
    while (cmax < D && ((size_t)2 << cmax) * gt * 64 <= (size_t)kTileBytes) cmax++;
    const uint32_t col_tiles = (G + gt - 1) / gt;
    // The fewest passes the tile size allows (a pass more costs more than the
    // parallelism it adds), levels spread evenly over them.
    const int n_pass = (D + cmax - 1) / cmax;
    std::vector<std::pair<int, int>> passes;  // (l0, c) top-down
    for (int q = 0, l0 = 0; q < n_pass; q++) {
        const int c = D / n_pass + (q < D % n_pass ? 1 : 0);
        passes.push_back({l0, c});
        l0 += c;
    }
    if (!forward) std::reverse(passes.begin(), passes.end());
    for (auto& pc : passes) {
        const int l0 = pc.first, c = pc.second;
        const uint32_t tiles = (1u << (D - c)) * col_tiles;
        const size_t smem = ((size_t)1 << c) * gt * 64;
        // one butterfly per thread and level (a multiple of 32, at most kPassThreads)
        const uint32_t bfly = (1u << (c - 1)) * gt;
        const int threads = (int)std::min<uint32_t>(kPassThreads, std::max<uint32_t>(32, (bfly + 31) / 32 * 32));
        afft_pass_kernel<<<tiles, threads, smem, st>>>(work, G, D, root, l0, c, forward ? 1 : 0, factors, gt);
        cudaError_t e = cudaGetLastError();
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

cudaError_t run_wht(uint32_t* v, uint32_t ts, int D, cudaStream_t st) {
    static std::atomic<uint64_t> attr{0};
    cudaError_t ea = once_per_device(attr, [] {
        return cudaFuncSetAttribute(wht_pass_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 8192 * 4);
    });
    if (ea != cudaSuccess) return ea;
    // passes of at most 8 index bits: enough groups per pass to spread over
    // the SMs (one CTA per group of 2^nb elements)
    std::vector<std::pair<int, int>> passes;
    const int n_pass = (D + 7) / 8;
    for (int q = 0, lo = 0; q < n_pass; q++) {
        const int nb = (D - lo + (n_pass - q) - 1) / (n_pass - q);
        passes.push_back({lo, nb});
        lo += nb;
    }
    for (auto& p : passes) {
        uint32_t groups = ts >> p.second;
        uint32_t gsize = 1u << p.second;
        wht_pass_kernel<<<groups, std::min<uint32_t>(1024, std::max<uint32_t>(32, gsize / 2)), gsize * 4, st>>>(
            v, ts, p.first, p.second);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace

int32_t afft_locator_device(const uint8_t* d_known, uint32_t ts, uint32_t* wa, uint32_t* wb, uint16_t* values,
                            uint16_t* derivs, cudaStream_t st, scrs_error* err) {
    const uint16_t *lg, *ex;
    SCRS_CUDA(log16_tables(&lg, &ex));
    int D = 0;
    while ((1u << D) < ts) D++;
    if (ts <= kLocatorOneCtaTs) {
        static std::atomic<uint64_t> attr{0};
        SCRS_CUDA(once_per_device(attr, [] {
            return cudaFuncSetAttribute(locator_one_cta_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)(2 * kLocatorOneCtaTs * sizeof(uint32_t)));
        }));
        locator_one_cta_kernel<<<1, 1024, 2 * ts * sizeof(uint32_t), st>>>(d_known, ts, mod_pow(32768, (uint32_t)D),
                                                                           lg, ex, values, derivs);
        SCRS_CUDA(cudaGetLastError());
        return SCRS_OK;
    }
    const int g = grid_for(ts, 256);
    locator_init_kernel<<<g, 256, 0, st>>>(d_known, ts, lg, wa, wb);
    SCRS_CUDA(cudaGetLastError());
    SCRS_CUDA(run_wht(wa, ts, D, st));
    SCRS_CUDA(run_wht(wb, ts, D, st));
    locator_mul_kernel<<<g, 256, 0, st>>>(wa, wb, ts);
    SCRS_CUDA(cudaGetLastError());
    SCRS_CUDA(run_wht(wa, ts, D, st));
    locator_finish_kernel<<<g, 256, 0, st>>>(wa, d_known, ts, mod_pow(32768, (uint32_t)D), ex, values, derivs);
    SCRS_CUDA(cudaGetLastError());
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
__device__ __forceinline__ uint32_t linv(const uint16_t* lg, const uint16_t* ex, uint32_t a) {
    return ex[(kMult - lg[a]) % kMult];
}

// gen[t*k + i] = G[t][i] for the r received repairs at evaluation points rep[t].
__global__ void targeted_gen_kernel(const uint16_t* sys_values, const uint16_t* sys_derivs, const uint16_t* lg,
                                    const uint16_t* ex, const uint16_t* rep, uint32_t r, uint32_t k, uint16_t* gen) {
    for (uint64_t x = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; x < (uint64_t)r * k;
         x += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t t = (uint32_t)(x / k), i = (uint32_t)(x - (uint64_t)t * k);
        const uint32_t e = rep[t];
        uint32_t lv = (uint32_t)lg[sys_values[e]] + 2 * kMult - lg[e ^ i] - lg[sys_derivs[i]];
        gen[x] = ex[lv % kMult];
    }
}

// One thread: invert A (r x r, GF(2^16) Gauss-Jordan; invertible for every
// supported pattern) into inv[s*r + t] = (A^-1)[s][t].
__global__ void targeted_invert_kernel(const uint16_t* gen, const uint16_t* missing, uint32_t r, uint32_t k,
                                       const uint16_t* lg, const uint16_t* ex, uint16_t* inv, int32_t* status) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    uint32_t a[kTargetedMax][2 * kTargetedMax];
    for (uint32_t t = 0; t < r; t++)
        for (uint32_t s = 0; s < r; s++) {
            a[t][s] = gen[(size_t)t * k + missing[s]];
            a[t][r + s] = t == s;
        }
    bool ok = true;
    for (uint32_t col = 0; col < r && ok; col++) {
        uint32_t piv = col;
        while (piv < r && !a[piv][col]) piv++;
        if (piv == r) {
            ok = false;
            break;
        }
        if (piv != col)
            for (uint32_t q = 0; q < 2 * r; q++) {
                const uint32_t tmp = a[col][q];
                a[col][q] = a[piv][q];
                a[piv][q] = tmp;
            }
        const uint32_t pinv = linv(lg, ex, a[col][col]);
        for (uint32_t q = 0; q < 2 * r; q++) a[col][q] = lmul(lg, ex, a[col][q], pinv);
        for (uint32_t t = 0; t < r; t++) {
            if (t == col || !a[t][col]) continue;
            const uint32_t f = a[t][col];
            for (uint32_t q = 0; q < 2 * r; q++) a[t][q] ^= lmul(lg, ex, f, a[col][q]);
        }
    }
    if (!ok && status) atomicCAS(status, 0, SCRS_DECODE_INSUFFICIENT_RANK);
    for (uint32_t s = 0; s < r; s++)
        for (uint32_t t = 0; t < r; t++) inv[s * r + t] = ok ? (uint16_t)a[s][r + t] : 0;
}

// Fused coefficients, rows 0..r-1 the received repairs (A^-1 columns), rows
// r.. the present data rows: row z, output s = sum_t (A^-1)[s][t] G[t][present[z]].
__global__ void targeted_fuse_kernel(const uint16_t* gen, const uint16_t* inv_g, const uint16_t* present, uint32_t r,
                                     uint32_t k, const uint16_t* lg, const uint16_t* ex, uint16_t* coef) {
    __shared__ uint32_t inv[kTargetedMax * kTargetedMax];
    for (uint32_t x = threadIdx.x; x < r * r; x += blockDim.x) inv[x] = inv_g[x];
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
    // Encode locator: known = [0, k), erased = [k, ts), fixed per geometry.
    SCRS_CUDA(enc_values.ensure(ts * 2));
    SCRS_CUDA(enc_derivs.ensure(ts * 2));
    DevBuf known, wa, wb;
    std::vector<uint8_t> hk(ts, 0);
    std::fill(hk.begin(), hk.begin() + k, 1);
    SCRS_CUDA(known.ensure(ts));
    SCRS_CUDA(wa.ensure(ts * 4));
    SCRS_CUDA(wb.ensure(ts * 4));
    SCRS_CUDA(cudaMemcpy(known.p, hk.data(), ts, cudaMemcpyHostToDevice));
    int32_t r = afft_locator_device(known.as<uint8_t>(), (uint32_t)ts, wa.as<uint32_t>(), wb.as<uint32_t>(),
                                    enc_values.as<uint16_t>(), enc_derivs.as<uint16_t>(), 0, err);
    if (r) return r;
    // Systematic locator for the targeted decode: known = [k, ts), erased = [0, k).
    SCRS_CUDA(sys_values.ensure(ts * 2));
    SCRS_CUDA(sys_derivs.ensure(ts * 2));
    SCRS_CUDA(cudaStreamSynchronize(0));  // `known` is rewritten below
    for (uint64_t i = 0; i < ts; i++) hk[i] = i >= k ? 1 : 0;
    SCRS_CUDA(cudaMemcpy(known.p, hk.data(), ts, cudaMemcpyHostToDevice));
    r = afft_locator_device(known.as<uint8_t>(), (uint32_t)ts, wa.as<uint32_t>(), wb.as<uint32_t>(),
                            sys_values.as<uint16_t>(), sys_derivs.as<uint16_t>(), 0, err);
    if (r) return r;
    SCRS_CUDA(cudaStreamSynchronize(0));  // the locators ran on the legacy stream
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
    std::vector<uint16_t> host_rows(2 * c.m);
    for (uint64_t t = 0; t < c.m; t++) host_rows[t] = (uint16_t)(c.k + t), host_rows[c.m + t] = (uint16_t)t;
    SCRS_CUDA(rows.ensure(host_rows.size() * 2));
    SCRS_CUDA(upload_now(rows.p, host_rows.data(), host_rows.size() * 2));
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
    SCRS_CUDA(known.ensure(c.ts));
    SCRS_CUDA(wht_a.ensure(c.ts * 4));
    SCRS_CUDA(wht_b.ensure(c.ts * 4));
    SCRS_CUDA(values.ensure(c.ts * 2));
    SCRS_CUDA(derivs.ensure(c.ts * 2));
    SCRS_CUDA(row_map.ensure(c.n * 2));
    const size_t rows_bytes = (2 * c.k + 8) * 2;
    const size_t lists_elems = 3 * c.k + 4 * kTargetedMax + kTargetedMax * kTargetedMax + 8;
    off_map = (rows_bytes + 15) & ~(size_t)15;
    off_known = (off_map + c.n * 2 + 15) & ~(size_t)15;
    off_lists = (off_known + c.ts + 15) & ~(size_t)15;
    for (int i = 0; i < 2; i++) {
        SCRS_CUDA(stage[i].ensure(off_lists + lists_elems * 2));
        memset(stage[i].p, 0, stage[i].bytes);
        if (!staged[i]) SCRS_CUDA(cudaEventCreateWithFlags(&staged[i], cudaEventDisableTiming));
    }
    SCRS_CUDA(rows.ensure(rows_bytes));
    SCRS_CUDA(tgen.ensure(kTargetedMax * c.k * 2));
    SCRS_CUDA(tcoef.ensure(kTargetedMax * c.k * 2));
    SCRS_CUDA(tlists.ensure((3 * c.k + 4 * kTargetedMax + kTargetedMax * kTargetedMax + 8) * 2));
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
        scale_in_kernel<<<grid_for(k * G, 128), 128, 0, st>>>(d_data, L, G, nullptr, nullptr, (uint32_t)k,
                                                              ws.work0.as<uint8_t>(), nullptr);
        SCRS_CUDA(cudaGetLastError());
        SCRS_CUDA(run_transform(ws.work0.as<uint8_t>(), G, (int)log_ts - 1, factors.as<uint16_t>(), false, st, 2));
        SCRS_CUDA(run_transform(ws.work0.as<uint8_t>(), G, (int)log_ts - 1, factors.as<uint16_t>(), true, st, 3));
        scale_out_kernel<<<grid_for(m * G, 128), 128, 0, st>>>(ws.work0.as<uint8_t>(), G, L,
                                                               ws.rows.as<uint16_t>() + m, ws.rows.as<uint16_t>() + m,
                                                               (uint32_t)m, nullptr, nullptr, nullptr, d_repairs);
        SCRS_CUDA(cudaGetLastError());
        return SCRS_OK;
    }
    const uint16_t *lg, *ex;
    SCRS_CUDA(log16_tables(&lg, &ex));
    scale_in_kernel<<<grid_for(ts * G, 128), 128, 0, st>>>(d_data, L, G, ws.known.as<uint8_t>(),
                                                           enc_values.as<uint16_t>(), (uint32_t)ts,
                                                           ws.work0.as<uint8_t>(), nullptr);
    SCRS_CUDA(cudaGetLastError());
    SCRS_CUDA(run_transform(ws.work0.as<uint8_t>(), G, (int)log_ts, factors.as<uint16_t>(), false, st));
    DerivFactors df{};
    std::copy(deriv_factors, deriv_factors + 16, df.f);
    derivative_kernel<<<grid_for(ts * G, 128), 128, 0, st>>>(ws.work0.as<uint8_t>(), ws.work1.as<uint8_t>(),
                                                             (uint32_t)ts, G, (int)log_ts, df);
    SCRS_CUDA(cudaGetLastError());
    SCRS_CUDA(run_transform(ws.work1.as<uint8_t>(), G, (int)log_ts, factors.as<uint16_t>(), true, st));
    scale_out_kernel<<<grid_for(m * G, 128), 128, 0, st>>>(ws.work1.as<uint8_t>(), G, L, ws.rows.as<uint16_t>(),
                                                           ws.rows.as<uint16_t>() + m, (uint32_t)m,
                                                           enc_derivs.as<uint16_t>(), lg, ex, d_repairs);
    SCRS_CUDA(cudaGetLastError());
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
    SCRS_CUDA(cudaMemcpyAsync(ws.rows.p, miss, (2 * k + 8) * 2, cudaMemcpyHostToDevice, st));
    const uint16_t* d_miss = ws.rows.as<uint16_t>();
    const uint16_t* d_pres = ws.rows.as<uint16_t>() + k;
    const uint16_t* d_map = nullptr;
    if (row_map) {
        memcpy(stage + ws.off_map, row_map, n * 2);
        SCRS_CUDA(cudaMemcpyAsync(ws.row_map.p, stage + ws.off_map, n * 2, cudaMemcpyHostToDevice, st));
        d_map = ws.row_map.as<uint16_t>();
    }
    if (np) {
        const bool vec = L % 16 == 0 && (reinterpret_cast<uintptr_t>(d_payloads) & 15) == 0 &&
                         (reinterpret_cast<uintptr_t>(d_out) & 15) == 0;
        if (vec)
            copy_rows_kernel<16><<<grid_for((uint64_t)np * (L / 16), 256), 256, 0, st>>>(d_payloads, d_out, L,
                                                                                            d_pres, np, d_map);
        else
            copy_rows_kernel<1><<<grid_for((uint64_t)np * L, 256), 256, 0, st>>>(d_payloads, d_out, L, d_pres, np,
                                                                                   d_map);
        SCRS_CUDA(cudaGetLastError());
    }
    if (nm == 0) return ws.stage_release(st, err);
    if (nm <= kTargetedMax) {
        rc = decode_targeted(d_payloads, have, d_out, ws, status, st, err, row_map, miss, nm, pres, np);
        const int32_t rr = ws.stage_release(st, err);  // after its list upload, on every path
        return rc ? rc : rr;
    }
    uint8_t* known = stage + ws.off_known;
    memcpy(known, have, n);  // receipt flags are 0 / 1
    memset(known + n, 0, ts - n);
    SCRS_CUDA(cudaMemcpyAsync(ws.known.p, known, ts, cudaMemcpyHostToDevice, st));
    rc = ws.stage_release(st, err);
    if (rc) return rc;
    int32_t r = afft_locator_device(ws.known.as<uint8_t>(), (uint32_t)ts, ws.wht_a.as<uint32_t>(),
                                    ws.wht_b.as<uint32_t>(), ws.values.as<uint16_t>(), ws.derivs.as<uint16_t>(), st,
                                    err);
    if (r) return r;
    scale_in_kernel<<<grid_for(ts * G, 128), 128, 0, st>>>(d_payloads, L, G, ws.known.as<uint8_t>(),
                                                           ws.values.as<uint16_t>(), (uint32_t)ts,
                                                           ws.work0.as<uint8_t>(), d_map);
    SCRS_CUDA(cudaGetLastError());
    SCRS_CUDA(run_transform(ws.work0.as<uint8_t>(), G, (int)log_ts, factors.as<uint16_t>(), false, st));
    DerivFactors df{};
    std::copy(deriv_factors, deriv_factors + 16, df.f);
    derivative_kernel<<<grid_for(ts * G, 128), 128, 0, st>>>(ws.work0.as<uint8_t>(), ws.work1.as<uint8_t>(),
                                                             (uint32_t)ts, G, (int)log_ts, df);
    SCRS_CUDA(cudaGetLastError());
    SCRS_CUDA(run_transform(ws.work1.as<uint8_t>(), G, (int)log_ts, factors.as<uint16_t>(), true, st));
    scale_out_kernel<<<grid_for((uint64_t)nm * G, 128), 128, 0, st>>>(ws.work1.as<uint8_t>(), G, L, d_miss, d_miss,
                                                                      nm, ws.derivs.as<uint16_t>(), lg, ex, d_out);
    SCRS_CUDA(cudaGetLastError());
    return SCRS_OK;
}

int32_t AfftCodec::decode_targeted(const uint8_t* d_payloads, const uint8_t* have, uint8_t* d_out,
                                   AfftWorkspace& ws, int32_t* status, cudaStream_t st, scrs_error* err,
                                   const uint16_t* row_map, const uint16_t* miss, uint32_t nm, const uint16_t* pres,
                                   uint32_t np) const {
    const uint16_t *lg, *ex;
    SCRS_CUDA(log16_tables(&lg, &ex));
    // lists: in_rows[k] (repairs then present), out_rows[nm], rep[nm] (evaluation points),
    // missing[nm], present[np]
    const size_t n_lists = 3 * k + 4 * kTargetedMax + kTargetedMax * kTargetedMax + 8;
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
    SCRS_CUDA(cudaMemcpyAsync(ws.tlists.p, h, n_lists * 2, cudaMemcpyHostToDevice, st));
    const uint16_t* d_in_rows = ws.tlists.as<uint16_t>();
    const uint16_t* d_out_rows = d_in_rows + k;
    const uint16_t* d_rep = d_out_rows + kTargetedMax;
    const uint16_t* d_mis = d_rep + kTargetedMax;
    const uint16_t* d_prs = d_mis + kTargetedMax;
    targeted_gen_kernel<<<grid_for((uint64_t)nm * k, 256), 256, 0, st>>>(
        sys_values.as<uint16_t>(), sys_derivs.as<uint16_t>(), lg, ex, d_rep, nm, (uint32_t)k, ws.tgen.as<uint16_t>());
    SCRS_CUDA(cudaGetLastError());
    uint16_t* d_inv = const_cast<uint16_t*>(d_prs) + k;  // r*r entries after the present list
    targeted_invert_kernel<<<1, 32, 0, st>>>(ws.tgen.as<uint16_t>(), d_mis, nm, (uint32_t)k, lg, ex, d_inv, status);
    SCRS_CUDA(cudaGetLastError());
    targeted_fuse_kernel<<<grid_for((uint64_t)k * nm, 256), 256, 0, st>>>(ws.tgen.as<uint16_t>(), d_inv, d_prs, nm,
                                                                         (uint32_t)k, lg, ex, ws.tcoef.as<uint16_t>());
    SCRS_CUDA(cudaGetLastError());
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
    SCRS_CUDA(launch_mxk_single(T, 1, status, 0, st));
    return SCRS_OK;
}

}  // namespace scrs
