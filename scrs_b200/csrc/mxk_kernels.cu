// Multiply-XOR stripe kernels for sm_100a.
//
// One CTA (4 warps) owns one column chunk of one stripe: 1 KiB of every row
// for GF(256), 2 KiB for GF((2^8)^2).  Per segment of input rows:
//   1. one thread issues a TMA bulk copy (cp.async.bulk, no multicast) per
//      input row into shared memory; all threads wait on one mbarrier;
//   2. each warp bit-slices its share of the staged rows in place (and writes
//      decode's present rows straight through to the output);
//   3. each warp produces whole output rows: for every input row it reads the
//      row's planes and applies the warp-uniform coefficient through the
//      jump-tabled XOR networks, then converts back to bytes and stores.
// Inputs are read from HBM once and outputs written once, which is the
// algorithmic traffic (k+m)*L for encode and 2*k*L for decode.  A persistent
// grid drains a device work queue of (stripe, chunk) items, so thousands of
// uneven stripes run in one launch.
#include <algorithm>

#include "gf_mul_core.cuh"
#include "kernels.cuh"

namespace scrs {

namespace {

constexpr int kSmemHeader = 128;

__device__ __forceinline__ uint64_t umin64(uint64_t a, uint64_t b) { return a < b ? a : b; }
__device__ __forceinline__ uint32_t umin32(uint32_t a, uint32_t b) { return a < b ? a : b; }

__device__ __forceinline__ uint4 load_piece(const uint8_t* row, uint64_t pos, uint64_t L, bool aligned) {
    uint4 v = make_uint4(0, 0, 0, 0);
    if (pos >= L) return v;
    if (aligned && pos + 16 <= L) return __ldg(reinterpret_cast<const uint4*>(row + pos));
    uint8_t b[16];
#pragma unroll
    for (int t = 0; t < 16; t++) b[t] = (pos + t < L) ? row[pos + t] : 0;
    v.x = b[0] | (b[1] << 8) | (b[2] << 16) | ((uint32_t)b[3] << 24);
    v.y = b[4] | (b[5] << 8) | (b[6] << 16) | ((uint32_t)b[7] << 24);
    v.z = b[8] | (b[9] << 8) | (b[10] << 16) | ((uint32_t)b[11] << 24);
    v.w = b[12] | (b[13] << 8) | (b[14] << 16) | ((uint32_t)b[15] << 24);
    return v;
}

__device__ __forceinline__ void store_piece(uint8_t* row, uint64_t pos, uint64_t L, bool aligned, uint4 v) {
    if (pos >= L) return;
    if (aligned && pos + 16 <= L) {
        *reinterpret_cast<uint4*>(row + pos) = v;
        return;
    }
    uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int t = 0; t < 16; t++)
        if (pos + t < L) row[pos + t] = (uint8_t)(w[t >> 2] >> (8 * (t & 3)));
}

__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

template <int kGf16>
__device__ __forceinline__ uint32_t piece_pos(int pc, int lane) {
    return (uint32_t)pc * 512u + 16u * (uint32_t)lane;
}

template <int kGf16, int kStrategy>
__device__ __forceinline__ void mul_planes(uint32_t c, uint32_t (&acc)[FieldGeom<kGf16>::kLaneBytes / 4],
                                           const uint32_t (&p)[FieldGeom<kGf16>::kLaneBytes / 4]) {
    if constexpr (kGf16)
        mul16(c, acc, p);
    else
        mul8<kStrategy>(c, acc, p);
}

template <int kGf16>
__device__ __forceinline__ void bitslice_lane(uint32_t (&w)[FieldGeom<kGf16>::kLaneBytes / 4]) {
    if constexpr (kGf16)
        bitslice16(w);
    else
        bitslice8(w);
}

// Process one (task, chunk) item; returns false on a device wait timeout.
template <int kGf16, int kStrategy>
__device__ bool process_item(const MxkTask& T, uint32_t chunk, uint8_t* planes, uint8_t* coef_s, uint64_t* bar,
                             uint32_t& phase, int seg_cap, int32_t* status) {
    using G = FieldGeom<kGf16>;
    constexpr int W = G::kLaneBytes / 4;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint64_t L = T.L;
    const uint64_t off = (uint64_t)chunk * G::kChunk;
    const uint32_t bytes_here = (uint32_t)umin64(G::kChunk, L - off);
    const uint32_t n_in = T.n_in, n_out = T.n_out, ld = T.ld;
    const bool aligned = T.aligned != 0;

    for (uint32_t og = 0; og == 0 || og < n_out; og += kMaxOutGroup) {
        const uint32_t og_n = n_out > og ? umin32(kMaxOutGroup, n_out - og) : 0;
        const bool need_pass = og == 0 && T.pass_rows != nullptr;
        if (og_n == 0 && !need_pass) break;
        for (uint32_t seg = 0; seg < n_in; seg += seg_cap) {
            const uint32_t seg_n = umin32((uint32_t)seg_cap, n_in - seg);
            // ---- stage the segment's rows in shared memory
            if (aligned) {
                if (tid == 0) {
                    fence_proxy_async_smem();
                    mbar_arrive_expect_tx(bar, seg_n * bytes_here);
                    for (uint32_t i = 0; i < seg_n; i++) {
                        uint32_t r = T.in_rows ? T.in_rows[seg + i] : seg + i;
                        tma_load_1d(planes + (size_t)i * G::kChunk, T.in + (uint64_t)r * T.in_stride + off,
                                    bytes_here, bar);
                    }
                }
                bool ok = mbar_wait_bounded(bar, phase, status);
                phase ^= 1u;
                if (!__syncthreads_and(ok)) return false;
            } else {
                for (uint32_t i = warp; i < seg_n; i += 4) {
                    uint32_t r = T.in_rows ? T.in_rows[seg + i] : seg + i;
                    const uint8_t* row = T.in + (uint64_t)r * T.in_stride;
#pragma unroll
                    for (int pc = 0; pc < G::kPieces; pc++) {
                        uint32_t pp = piece_pos<kGf16>(pc, lane);
                        *reinterpret_cast<uint4*>(planes + (size_t)i * G::kChunk + pp) =
                            load_piece(row, off + pp, L, false);
                    }
                }
                __syncthreads();
            }
            // ---- pass-through copies and in-place bit-slicing
            for (uint32_t i = warp; i < seg_n; i += 4) {
                uint8_t* base = planes + (size_t)i * G::kChunk;
                uint32_t w[W];
#pragma unroll
                for (int pc = 0; pc < G::kPieces; pc++) {
                    uint4 v = *reinterpret_cast<const uint4*>(base + piece_pos<kGf16>(pc, lane));
                    w[4 * pc] = v.x, w[4 * pc + 1] = v.y, w[4 * pc + 2] = v.z, w[4 * pc + 3] = v.w;
                }
                if (need_pass) {
                    uint16_t pr = T.pass_rows[seg + i];
                    if (pr != kNoRow) {
                        uint8_t* orow = T.out + (uint64_t)pr * T.out_stride;
#pragma unroll
                        for (int pc = 0; pc < G::kPieces; pc++)
                            store_piece(orow, off + piece_pos<kGf16>(pc, lane), L, aligned,
                                        make_uint4(w[4 * pc], w[4 * pc + 1], w[4 * pc + 2], w[4 * pc + 3]));
                    }
                }
                if (og_n) {
                    bitslice_lane<kGf16>(w);
#pragma unroll
                    for (int pc = 0; pc < G::kPieces; pc++)
                        *reinterpret_cast<uint4*>(base + piece_pos<kGf16>(pc, lane)) =
                            make_uint4(w[4 * pc], w[4 * pc + 1], w[4 * pc + 2], w[4 * pc + 3]);
                }
            }
            // ---- coefficients of this (output group, segment)
            for (uint32_t x = tid; x < seg_n * og_n; x += kThreads) {
                uint32_t i = x / og_n, j = x - i * og_n;
                size_t crow = T.coef_rows ? T.coef_rows[seg + i] : seg + i;
                size_t src = crow * ld + og + j;
                if constexpr (kGf16)
                    reinterpret_cast<uint16_t*>(coef_s)[x] = reinterpret_cast<const uint16_t*>(T.coef)[src];
                else
                    coef_s[x] = reinterpret_cast<const uint8_t*>(T.coef)[src];
            }
            __syncthreads();
            // ---- output rows, one per warp at a time
            for (uint32_t j = warp; j < og_n; j += 4) {
                uint32_t acc[W];
                uint32_t orow_idx = T.out_rows ? T.out_rows[og + j] : og + j;
                uint8_t* orow = T.out + (uint64_t)orow_idx * T.out_stride;
                if (seg == 0 && !T.accumulate) {
#pragma unroll
                    for (int t = 0; t < W; t++) acc[t] = 0;
                } else {  // existing output (accumulate) or partial sums of earlier segments
#pragma unroll
                    for (int pc = 0; pc < G::kPieces; pc++) {
                        uint4 v = load_piece(orow, off + piece_pos<kGf16>(pc, lane), L, aligned);
                        acc[4 * pc] = v.x, acc[4 * pc + 1] = v.y, acc[4 * pc + 2] = v.z, acc[4 * pc + 3] = v.w;
                    }
                    bitslice_lane<kGf16>(acc);
                }
                for (uint32_t i = 0; i < seg_n; i++) {
                    uint32_t c;
                    if constexpr (kGf16)
                        c = reinterpret_cast<const uint16_t*>(coef_s)[i * og_n + j];
                    else
                        c = coef_s[i * og_n + j];
                    if (c == 0) continue;
                    const uint8_t* base = planes + (size_t)i * G::kChunk;
                    uint32_t p[W];
#pragma unroll
                    for (int pc = 0; pc < G::kPieces; pc++) {
                        uint4 v = *reinterpret_cast<const uint4*>(base + piece_pos<kGf16>(pc, lane));
                        p[4 * pc] = v.x, p[4 * pc + 1] = v.y, p[4 * pc + 2] = v.z, p[4 * pc + 3] = v.w;
                    }
                    mul_planes<kGf16, kStrategy>(c, acc, p);
                }
                bitslice_lane<kGf16>(acc);
#pragma unroll
                for (int pc = 0; pc < G::kPieces; pc++)
                    store_piece(orow, off + piece_pos<kGf16>(pc, lane), L, aligned,
                                make_uint4(acc[4 * pc], acc[4 * pc + 1], acc[4 * pc + 2], acc[4 * pc + 3]));
            }
            __syncthreads();
        }
    }
    return true;
}

template <int kGf16, int kStrategy>
__device__ __forceinline__ void mxk_smem_setup(uint8_t* smem, int seg_cap, uint64_t*& bar, uint8_t*& planes,
                                               uint8_t*& coef_s) {
    using G = FieldGeom<kGf16>;
    bar = reinterpret_cast<uint64_t*>(smem);
    planes = smem + kSmemHeader;
    coef_s = planes + (size_t)seg_cap * G::kChunk;
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        fence_mbar_init();
    }
    __syncthreads();
}

template <int kGf16, int kStrategy>
__global__ void __launch_bounds__(kThreads) mxk_kernel(const MxkTask* __restrict__ tasks, uint32_t n_tasks,
                                                       uint32_t total_items, uint32_t* work_counter,
                                                       int32_t* status, int seg_cap) {
    extern __shared__ __align__(128) uint8_t smem[];
    volatile uint32_t* item_sh = reinterpret_cast<volatile uint32_t*>(smem + 16);
    uint64_t* bar;
    uint8_t *planes, *coef_s;
    mxk_smem_setup<kGf16, kStrategy>(smem, seg_cap, bar, planes, coef_s);
    uint32_t phase = 0;
    for (uint32_t iter = 0;; iter++) {
        uint32_t item;
        if (work_counter) {
            if (threadIdx.x == 0) *item_sh = atomicAdd(work_counter, 1u);
            __syncthreads();
            item = *item_sh;
        } else {
            item = blockIdx.x + iter * gridDim.x;
        }
        if (item >= total_items) break;
        uint32_t lo = 0, hi = n_tasks - 1;
        while (lo < hi) {
            uint32_t mid = (lo + hi + 1) >> 1;
            if (tasks[mid].item_begin <= item)
                lo = mid;
            else
                hi = mid - 1;
        }
        const MxkTask T = tasks[lo];
        if (!process_item<kGf16, kStrategy>(T, item - T.item_begin, planes, coef_s, bar, phase, seg_cap, status))
            break;
        __syncthreads();
    }
}

// One task passed by value (kernel parameter space), CTAs striding over its
// row chunks: the single-stripe launch used by the per-codec entry points and
// by the one-launch-per-stripe baseline.
template <int kGf16, int kStrategy>
__global__ void __launch_bounds__(kThreads) mxk_single_kernel(const MxkTask T, int32_t* status, int seg_cap) {
    extern __shared__ __align__(128) uint8_t smem[];
    uint64_t* bar;
    uint8_t *planes, *coef_s;
    mxk_smem_setup<kGf16, kStrategy>(smem, seg_cap, bar, planes, coef_s);
    uint32_t phase = 0;
    for (uint32_t item = blockIdx.x; item < T.n_items; item += gridDim.x) {
        if (!process_item<kGf16, kStrategy>(T, item, planes, coef_s, bar, phase, seg_cap, status)) break;
        __syncthreads();
    }
}

// ---- closed-form Cauchy solve on the device --------------------------------
struct Gf8Tables {
    uint8_t log[256];
    uint8_t exp[512];
};

__device__ __forceinline__ uint32_t m8(const Gf8Tables& t, uint32_t a, uint32_t b) {
    return (a && b) ? t.exp[t.log[a] + t.log[b]] : 0u;
}
__device__ __forceinline__ uint32_t i8(const Gf8Tables& t, uint32_t a) { return a ? t.exp[255 - t.log[a]] : 0u; }

// GF((2^8)^2) product and inverse (scrs/src/algebra/gf65536.rs:79-114).
__device__ __forceinline__ uint32_t m16(const Gf8Tables& t, uint32_t x, uint32_t y) {
    uint32_t a = x & 0xFF, b = x >> 8, c = y & 0xFF, d = y >> 8;
    uint32_t ac = m8(t, a, c), bd = m8(t, b, d);
    return (ac ^ m8(t, kGf16Delta, bd)) | ((m8(t, a ^ b, c ^ d) ^ ac) << 8);
}
__device__ __forceinline__ uint32_t i16(const Gf8Tables& t, uint32_t x) {
    uint32_t a = x & 0xFF, b = x >> 8;
    if (x == 0) return 0;
    uint32_t norm = m8(t, a, a) ^ m8(t, a, b) ^ m8(t, kGf16Delta, m8(t, b, b));
    uint32_t ni = i8(t, norm);
    return m8(t, a ^ b, ni) | (m8(t, b, ni) << 8);
}

template <int kGf16>
struct FieldOps {
    const Gf8Tables& t;
    __device__ uint32_t mul(uint32_t a, uint32_t b) const { return kGf16 ? m16(t, a, b) : m8(t, a, b); }
    __device__ uint32_t inv(uint32_t a) const { return kGf16 ? i16(t, a) : i8(t, a); }
};

template <int kGf16>
__device__ __forceinline__ uint32_t x_var(const CauchyPlanTask& P, const Gf8Tables& t, uint32_t i) {
    if (kGf16) return P.powers[i];  // g^i (tower/cauchy.rs:44-49)
    if (P.engine == SCRS_ENGINE_STANDARD_CAUCHY) return i & 0xFF;  // cauchy.rs:88
    return t.exp[i % 255];                                          // good_cauchy.rs:78
}
template <int kGf16>
__device__ __forceinline__ uint32_t y_var(const CauchyPlanTask& P, const Gf8Tables& t, uint32_t j) {
    if (kGf16) return P.powers[P.k + j];
    if (P.engine == SCRS_ENGINE_STANDARD_CAUCHY) return (P.k + j) & 0xFF;
    return t.exp[(P.k + j) % 255];
}

__constant__ uint8_t c_gf8_exp[255];
__constant__ uint8_t c_gf8_log[256];

// One CTA per decode.  rf/cf are the rational-Lagrange row/column factors
// R_i = prod_h(row_i+col_h)/prod_{l!=i}(row_i+row_l) and
// C_j = prod_l(col_j+row_l)/prod_{h!=j}(col_j+col_h)
// (decoder/cauchy_inverse.rs:29-49); the inverse is R_i C_j / (col_j+row_i)
// and a present column z gets C_j * prod_h(z+col_h) / ((z+col_j) prod_l(z+row_l)).
template <int kGf16>
__device__ void cauchy_plan_body(const CauchyPlanTask& P) {
    __shared__ Gf8Tables tb;
    for (int i = threadIdx.x; i < 512; i += blockDim.x) {
        if (i < 256) tb.log[i] = c_gf8_log[i];
        tb.exp[i] = c_gf8_exp[i % 255];
    }
    __syncthreads();
    FieldOps<kGf16> F{tb};
    const uint32_t r = P.r;
    if (r == 0) return;
    // row vars, col vars, rf, cf: 4*r words in shared memory, or in the
    // task's global scratch when r is too large for shared memory.
    extern __shared__ uint32_t dyn[];
    uint32_t* rv = P.work ? P.work : dyn;
    uint32_t* cv = rv + r;
    uint32_t* rf = rv + 2 * r;
    uint32_t* cf = rv + 3 * r;
    for (uint32_t t = threadIdx.x; t < r; t += blockDim.x) {
        rv[t] = y_var<kGf16>(P, tb, P.repairs[t]);
        cv[t] = x_var<kGf16>(P, tb, P.missing[t]);
    }
    __syncthreads();
    for (uint32_t t = threadIdx.x; t < 2 * r; t += blockDim.x) {
        const bool is_row = t < r;
        const uint32_t u = is_row ? t : t - r;
        const uint32_t v = is_row ? rv[u] : cv[u];
        const uint32_t* other = is_row ? cv : rv;
        const uint32_t* same = is_row ? rv : cv;
        uint32_t cross = 1, within = 1;
        for (uint32_t h = 0; h < r; h++) {
            cross = F.mul(cross, v ^ other[h]);
            if (h != u) within = F.mul(within, v ^ same[h]);
        }
        (is_row ? rf : cf)[u] = F.mul(cross, F.inv(within));
    }
    __syncthreads();
    const uint32_t ld = P.ld;
    for (uint32_t x = threadIdx.x; x < r * r; x += blockDim.x) {
        uint32_t t = x / r, s = x - t * r;  // input row t (repair), output s (missing)
        uint32_t val = F.mul(F.mul(rf[t], cf[s]), F.inv(cv[s] ^ rv[t]));
        if (kGf16)
            reinterpret_cast<uint16_t*>(P.coef)[(size_t)t * ld + s] = (uint16_t)val;
        else
            reinterpret_cast<uint8_t*>(P.coef)[(size_t)t * ld + s] = (uint8_t)val;
    }
    for (uint32_t z = threadIdx.x; z < P.p; z += blockDim.x) {
        uint32_t zv = x_var<kGf16>(P, tb, P.present[z]);
        uint32_t rp = 1, cp = 1;
        for (uint32_t h = 0; h < r; h++) {
            rp = F.mul(rp, zv ^ rv[h]);
            cp = F.mul(cp, zv ^ cv[h]);
        }
        uint32_t f = F.mul(cp, F.inv(rp));
        size_t row = (size_t)(r + z) * ld;
        for (uint32_t s = 0; s < r; s++) {
            uint32_t val = F.mul(F.mul(cf[s], f), F.inv(zv ^ cv[s]));
            if (kGf16)
                reinterpret_cast<uint16_t*>(P.coef)[row + s] = (uint16_t)val;
            else
                reinterpret_cast<uint8_t*>(P.coef)[row + s] = (uint8_t)val;
        }
    }
}

template <int kGf16>
__global__ void __launch_bounds__(256) cauchy_plan_kernel(const CauchyPlanTask* __restrict__ tasks) {
    const CauchyPlanTask P = tasks[blockIdx.x];
    cauchy_plan_body<kGf16>(P);
}

template <int kGf16>
__global__ void __launch_bounds__(256) cauchy_plan_single(const CauchyPlanTask P) {
    cauchy_plan_body<kGf16>(P);
}

bool g_tables_uploaded = false;

cudaError_t ensure_tables() {
    if (g_tables_uploaded) return cudaSuccess;
    uint8_t ex[255], lg[256] = {0};
    uint8_t v = 1;
    for (int i = 0; i < 255; i++) {
        ex[i] = v;
        lg[v] = (uint8_t)i;
        v = gf8_mul_ce(v, 3);
    }
    cudaError_t e = cudaMemcpyToSymbol(c_gf8_exp, ex, sizeof ex);
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_gf8_log, lg, sizeof lg);
    if (e == cudaSuccess) g_tables_uploaded = true;
    return e;
}

template <int kGf16, int kStrategy>
cudaError_t set_mxk_attrs() {
    using G = FieldGeom<kGf16>;
    static bool done = false;
    if (done) return cudaSuccess;
    int bytes = (int)mxk_smem_bytes(kGf16, G::kSeg);
    cudaError_t e = cudaFuncSetAttribute(mxk_kernel<kGf16, kStrategy>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(mxk_single_kernel<kGf16, kStrategy>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) done = true;
    return e;
}

template <int kGf16, int kStrategy>
cudaError_t launch_single_impl(const MxkTask& T, int32_t* status, int grid, cudaStream_t stream) {
    using G = FieldGeom<kGf16>;
    if (T.n_items == 0 || (T.n_out == 0 && T.pass_rows == nullptr)) return cudaSuccess;
    cudaError_t e = set_mxk_attrs<kGf16, kStrategy>();
    if (e != cudaSuccess) return e;
    int seg_cap = std::max(1, std::min((int)T.n_in, G::kSeg));
    if (grid <= 0 || grid > (int)T.n_items) grid = (int)T.n_items;
    mxk_single_kernel<kGf16, kStrategy><<<grid, kThreads, mxk_smem_bytes(kGf16, T.n_in), stream>>>(T, status,
                                                                                                 seg_cap);
    return cudaGetLastError();
}

template <int kGf16, int kStrategy>
cudaError_t launch_mxk_impl(const MxkTask* tasks, uint32_t n_tasks, uint32_t total_items, uint32_t* counter,
                            int32_t* status, int max_in, int grid, cudaStream_t stream) {
    using G = FieldGeom<kGf16>;
    if (total_items == 0 || n_tasks == 0) return cudaSuccess;
    int seg_cap = std::max(1, std::min(max_in, G::kSeg));
    size_t smem = mxk_smem_bytes(kGf16, max_in);
    cudaError_t e = set_mxk_attrs<kGf16, kStrategy>();
    if (e != cudaSuccess) return e;
    if (grid <= 0) grid = (int)total_items;
    mxk_kernel<kGf16, kStrategy><<<grid, kThreads, smem, stream>>>(tasks, n_tasks, total_items, counter, status,
                                                                     seg_cap);
    return cudaGetLastError();
}

}  // namespace

size_t mxk_smem_bytes(int gf16, int max_in) {
    int chunk = gf16 ? FieldGeom<1>::kChunk : FieldGeom<0>::kChunk;
    int segmax = gf16 ? FieldGeom<1>::kSeg : FieldGeom<0>::kSeg;
    int elem = gf16 ? 2 : 1;
    int seg = std::max(1, std::min(max_in, segmax));
    return (size_t)kSmemHeader + (size_t)seg * chunk + (size_t)seg * kMaxOutGroup * elem;
}

int mxk_ctas_per_sm(int gf16, int max_in) {
    int n = 0;
    size_t smem = mxk_smem_bytes(gf16, max_in);
    cudaError_t e = gf16 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, mxk_kernel<1, 1>, kThreads, smem)
                         : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, mxk_kernel<0, 0>, kThreads, smem);
    if (e != cudaSuccess || n < 1) n = 1;
    return n;
}

cudaError_t launch_gf256_mxk(const MxkTask* tasks, uint32_t n_tasks, uint32_t total_items, uint32_t* counter,
                             int32_t* status, int max_in, int strategy, int grid, cudaStream_t stream) {
    if (strategy == 0)
        return launch_mxk_impl<0, 0>(tasks, n_tasks, total_items, counter, status, max_in, grid, stream);
    return launch_mxk_impl<0, 1>(tasks, n_tasks, total_items, counter, status, max_in, grid, stream);
}

cudaError_t launch_gf16_mxk(const MxkTask* tasks, uint32_t n_tasks, uint32_t total_items, uint32_t* counter,
                            int32_t* status, int max_in, int grid, cudaStream_t stream) {
    return launch_mxk_impl<1, 1>(tasks, n_tasks, total_items, counter, status, max_in, grid, stream);
}

cudaError_t launch_mxk_single(const MxkTask& task, int gf16, int strategy, int32_t* status, int grid,
                              cudaStream_t stream) {
    if (gf16) return launch_single_impl<1, 1>(task, status, grid, stream);
    if (strategy == 0) return launch_single_impl<0, 0>(task, status, grid, stream);
    return launch_single_impl<0, 1>(task, status, grid, stream);
}

cudaError_t launch_cauchy_plan_single(const CauchyPlanTask& task, int gf16, cudaStream_t stream) {
    if (task.r == 0) return cudaSuccess;
    cudaError_t e = ensure_tables();
    if (e != cudaSuccess) return e;
    size_t smem = task.work ? 0 : (size_t)4 * task.r * sizeof(uint32_t);
    if (smem > 48 * 1024) {
        auto fn = gf16 ? cauchy_plan_single<1> : cauchy_plan_single<0>;
        e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    if (gf16)
        cauchy_plan_single<1><<<1, 256, smem, stream>>>(task);
    else
        cauchy_plan_single<0><<<1, 256, smem, stream>>>(task);
    return cudaGetLastError();
}

cudaError_t launch_cauchy_plan(const CauchyPlanTask* tasks, uint32_t n_tasks, int gf16, uint32_t max_smem_r,
                               cudaStream_t stream) {
    if (n_tasks == 0) return cudaSuccess;
    cudaError_t e = ensure_tables();
    if (e != cudaSuccess) return e;
    size_t smem = (size_t)4 * max_smem_r * sizeof(uint32_t);
    if (smem > 48 * 1024) {
        auto fn = gf16 ? cauchy_plan_kernel<1> : cauchy_plan_kernel<0>;
        e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    if (gf16)
        cauchy_plan_kernel<1><<<n_tasks, 256, smem, stream>>>(tasks);
    else
        cauchy_plan_kernel<0><<<n_tasks, 256, smem, stream>>>(tasks);
    return cudaGetLastError();
}

}  // namespace scrs
