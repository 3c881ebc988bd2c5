// Multiply-XOR stripe kernels for sm_100a.
//
// One CTA (4 warps) owns one 2 KiB column chunk of one stripe; every lane
// owns 64 bytes of each row (two sets of 8 GF(256) bit planes, or one set of
// 16 GF(2^16) planes).
// For each segment of up to 16 input rows:
//   1. one thread issues a TMA bulk copy (cp.async.bulk, into this CTA only) per
//      input row into shared memory; all threads wait on the stage's mbarrier;
//   2. each warp bit-slices its share of the staged rows in place (and writes
//      decode's present rows straight through to the output);
//   3. each warp produces whole output rows: for every input row it reads the
//      row's planes and applies the warp-uniform coefficient through the
//      generated jump tables (brx_dispatch.cuh), then converts back to bytes.
// A jump whose target changes from one use to the next is the expensive part
// of a multiply, so nothing else (no memory access) sits on the path from one
// jump to the next: each warp holds its output's coefficients in registers.
// Inputs are read from HBM once and outputs written once: the algorithmic
// traffic is (k+m)*L for encode and 2*k*L for decode.  The persistent form
// drains a device work queue of (stripe, chunk) items.
#include <algorithm>

#include "gf_mul_core.cuh"
#include "kernels.cuh"
#include "mxk_device.cuh"

namespace scrs {

namespace {

// Coefficient of input row seg + lane for output og + j, or 0 past the segment.
template <int kGf16>
__device__ __forceinline__ uint32_t lane_coef(const MxkTask& T, uint32_t seg, uint32_t seg_n, uint32_t og, uint32_t j,
                                              int lane) {
    if ((uint32_t)lane >= seg_n) return 0;
    const size_t crow = T.coef_rows ? T.coef_rows[seg + lane] : seg + lane;
    const size_t src = crow * T.ld + og + j;
    if constexpr (kGf16)
        return __ldg(reinterpret_cast<const uint16_t*>(T.coef) + src);
    else
        return __ldg(reinterpret_cast<const uint8_t*>(T.coef) + src);
}

template <int kGf16>
__device__ __forceinline__ void load_out_planes(const uint8_t* orow, uint64_t off, int lane, uint64_t L,
                                                bool aligned, typename Lane<kGf16>::Words& w) {
#pragma unroll
    for (int pc = 0; pc < Lane<kGf16>::kPieces; pc++) {
        const uint4 v = load_piece(orow, off + piece_pos(pc, lane), L, aligned);
        w[4 * pc] = v.x, w[4 * pc + 1] = v.y, w[4 * pc + 2] = v.z, w[4 * pc + 3] = v.w;
    }
    bitslice_lane<kGf16>(w);
}

// One output row of one chunk: out = XOR_i c_i * x_i over the staged (bit-sliced)
// rows x_i, plus the row's existing content when `existing` (accumulate mode or
// the partial sum of earlier segments).  `c` is lane i's coefficient c_i.
//
// Horner on nibbles.  GF(256): c*x = 16*(hi*x) + lo*x, so the whole sum is
// 16 * (XOR_i hi_i x_i) + XOR_i lo_i x_i.  GF((2^8)^2), c = c0 + c1*u with
// GF(256) components: c*x = c0*x + c1*(u*x), so the sum is
// 16 * XOR_i (hi(c0_i) x_i + hi(c1_i) u x_i) + XOR_i (lo(c0_i) x_i + lo(c1_i) u x_i)
// (a GF(256) scalar multiplies both tower components alike, and u*x is a
// fixed XOR network computed on the fly).  Either way one 16-way table
// (v*x for v < 16, the cheapest half of the multiplication table) serves every
// step from a single jump site, so it stays in the SM's instruction cache; a
// 256-way or two 16-way tables do not, and their misses cost more than the
// second pass over the staged rows.  The warp runs a step list of
// (i * chunk bytes) | (u-flag << 4) | nibble entries: the high-nibble pass,
// the x16 fold, then the low-nibble pass.
//
// Between the segments of a stripe whose chunk is a whole aligned span of the
// row (`sliced_in` / `sliced_out`), the partial sum stays in the output row
// in bit-sliced form: each lane stores its plane words where its bytes go and
// reads them back for the next segment, so only the last segment converts
// back to bytes.
template <int kGf16>
__device__ __forceinline__ void output_row(const uint8_t* buf, uint32_t c, uint16_t* steps, uint32_t seg_n, int lane,
                                           bool existing, uint8_t* orow, uint64_t off, uint64_t L, bool aligned,
                                           bool full, bool atomic_out, bool sliced_in = false,
                                           bool sliced_out = false) {
    using G = FieldGeom<kGf16>;
    using Words = typename Lane<kGf16>::Words;
    constexpr int kWords = Lane<kGf16>::kWords;
    static_assert(kWords == 16, "one 16-plane set per lane");
    Words acc;
    // nibbles of the x-term (c0, or the GF(256) coefficient) and the u-term (c1)
    const uint32_t cx = c & 0xFFu, cu = kGf16 ? (c >> 8) & 0xFFu : 0u;
    const uint32_t below = (1u << lane) - 1u;
    // step entries: (i * chunk bytes) | (u-flag << 4) | nibble; pass 0 (high
    // nibbles) is entries [0, n0), pass 1 (low nibbles) [n0, n_steps)
    static_assert((G::kSegMax - 1) * G::kChunk + 31 < 65536, "step entries hold i * chunk | 31 in 16 bits");
    uint32_t n0 = 0, n_steps = 0;
#pragma unroll
    for (int pass = 0; pass < 2; pass++) {
        const uint32_t vx = pass ? cx & 15u : cx >> 4, vu = pass ? cu & 15u : cu >> 4;
        const uint32_t mx = __ballot_sync(0xFFFFFFFFu, vx != 0), mu = __ballot_sync(0xFFFFFFFFu, vu != 0);
        const uint32_t at = n_steps + __popc(mx & below) + __popc(mu & below);
        const uint32_t row = (uint32_t)lane * G::kChunk;
        if (vx) steps[at] = (uint16_t)(row | vx);
        if (vu) steps[at + (vx != 0)] = (uint16_t)(row | 16u | vu);
        n_steps += __popc(mx) + __popc(mu);
        if (pass == 0) n0 = n_steps;
    }
    __syncwarp();
#pragma unroll
    for (int t = 0; t < kWords; t++) acc[t] = 0;
    const uint8_t* lane_buf = buf + 16 * lane;
    uint32_t s = 0;
    uint32_t d = steps[0];
#pragma unroll 1
    for (int pass = 0; pass < 2; pass++) {  // one loop body, so one jump site
        const uint32_t end = pass ? n_steps : n0;
        for (; s < end; s++) {
            const uint32_t dn = steps[s + 1];
            Words p;
            const uint8_t* src = lane_buf + (d & ~31u);
#pragma unroll
            for (int pc = 0; pc < 4; pc++) {
                const uint4 v = *reinterpret_cast<const uint4*>(src + pc * 512);
                p[4 * pc] = v.x, p[4 * pc + 1] = v.y, p[4 * pc + 2] = v.z, p[4 * pc + 3] = v.w;
            }
            if (kGf16 && (d & 16u)) mul_by_u(p);
#if defined(__CUDA_ARCH__)
            brx_mul8x2_lo(d & 15u, acc, p);
#endif
            d = dn;
        }
        if (pass == 0) {  // high nibbles done: acc = 16 * acc, plus the existing content
#pragma unroll
            for (int h = 0; h < kWords; h += 8) {
                uint32_t t16[8] = {0, 0, 0, 0, 0, 0, 0, 0};
                mulacc8<16>(t16, *reinterpret_cast<const uint32_t(*)[8]>(&acc[h]));
#pragma unroll
                for (int r = 0; r < 8; r++) acc[h + r] = t16[r];
            }
            if (existing) {
                Words e;
                if (sliced_in) {
#pragma unroll
                    for (int pc = 0; pc < Lane<kGf16>::kPieces; pc++) {
                        const uint4 v = *reinterpret_cast<const uint4*>(orow + off + piece_pos(pc, lane));
                        e[4 * pc] = v.x, e[4 * pc + 1] = v.y, e[4 * pc + 2] = v.z, e[4 * pc + 3] = v.w;
                    }
                } else {
                    load_out_planes<kGf16>(orow, off, lane, L, aligned, e);
                }
#pragma unroll
                for (int t = 0; t < kWords; t++) acc[t] ^= e[t];
            }
        }
    }
    __syncwarp();  // the list is rebuilt for the warp's next output row
    if (sliced_out) {
        store_pieces<Lane<kGf16>::kPieces>(orow, off, 0, lane, L, true, true, acc);
        return;
    }
    bitslice_lane<kGf16>(acc);
    if (atomic_out) {  // partial sum of an input range: XOR into the (zeroed) output
#pragma unroll
        for (int pc = 0; pc < Lane<kGf16>::kPieces; pc++) {
            const uint64_t pos = off + piece_pos(pc, lane);
#pragma unroll
            for (int w = 0; w < 4; w++)
                if (pos + 4 * w + 4 <= L) atomicXor(reinterpret_cast<unsigned int*>(orow + pos + 4 * w), acc[4 * pc + w]);
        }
        return;
    }
    store_pieces<Lane<kGf16>::kPieces>(orow, off, 0, lane, L, aligned, full, acc);
}

// Process one item: outputs [out_lo, out_hi) of chunk `chunk` of task T.
// When `first_issued`, the TMA copies of the first stage (segment 0) were
// already issued into `buf` on `bar`.  kShape (see launch_gf256_mxk): what T
// is known to satisfy; the paths it rules out are compiled out.  Returns
// false on a wait timeout.
template <int kGf16, int kShape = kShapeAny>
__device__ bool process_item(const MxkTask& T, uint32_t chunk, uint8_t* buf, uint8_t* steps_base, uint64_t* bar,
                             uint32_t& phase, int seg_cap, int32_t* status, uint32_t out_lo, uint32_t out_hi,
                             bool first_issued, uint32_t in_lo = 0, uint32_t in_hi = 0xFFFFFFFFu,
                             bool atomic_out = false) {
    using G = FieldGeom<kGf16>;
    constexpr int kPieces = Lane<kGf16>::kPieces;
    // GF(256) rows are bit-sliced in two independent 32-byte halves per lane,
    // which balances the work over the 4 warps for any row count.
    constexpr int kUnitPieces = kGf16 ? kPieces : kPieces / 2;
    constexpr int kUnitsPerRow = kPieces / kUnitPieces;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint64_t L = T.L;
    const uint64_t off = (uint64_t)chunk * G::kChunk;
    const uint32_t n_in = umin32(T.n_in, in_hi);
    const bool aligned = (kShape & kShapeAligned) || T.aligned != 0;
    const bool full = (kShape & kShapeWhole) || (aligned && off + G::kChunk <= L);
    uint16_t* steps = reinterpret_cast<uint16_t*>(steps_base + warp * kStepBytes);

    for (uint32_t og = out_lo; og == out_lo || og < out_hi; og += kMaxOutGroup) {
        const uint32_t og_n = out_hi > og ? umin32(kMaxOutGroup, out_hi - og) : 0;
        const bool need_pass = og == 0 && T.pass_rows != nullptr;
        if (og_n == 0 && !need_pass) break;
        for (uint32_t seg = in_lo; seg < n_in; seg += seg_cap) {
            const uint32_t seg_n = umin32((uint32_t)seg_cap, n_in - seg);
            const bool prefetched = first_issued && og == out_lo && seg == in_lo;
            // this warp's first output's coefficients, loaded while the rows arrive
            uint32_t c = (uint32_t)warp < og_n ? lane_coef<kGf16>(T, seg, seg_n, og, warp, lane) : 0u;
            // ---- stage the segment's rows in shared memory
            if (aligned) {
                if (warp == 0 && !prefetched) issue_stage<kGf16>(T, chunk, seg, seg_n, buf, bar, lane);
                bool ok = mbar_wait_bounded(bar, phase, status);
                phase ^= 1u;
                if (!__syncthreads_and(ok)) return false;
            } else {
                for (uint32_t i = warp; i < seg_n; i += 4) {
                    const uint32_t r = T.in_rows ? T.in_rows[seg + i] : seg + i;
                    const uint8_t* row = T.in + (uint64_t)r * T.in_stride;
#pragma unroll
                    for (int pc = 0; pc < kPieces; pc++) {
                        const uint32_t pp = piece_pos(pc, lane);
                        *reinterpret_cast<uint4*>(buf + (size_t)i * G::kChunk + pp) = load_piece(row, off + pp, L, false);
                    }
                }
                __syncthreads();
            }
            // ---- pass-through copies and in-place bit-slicing, per (row, half)
            for (uint32_t u = warp; u < seg_n * kUnitsPerRow; u += 4) {
                const uint32_t i = u / kUnitsPerRow;
                const int pc0 = (int)(u - i * kUnitsPerRow) * kUnitPieces;
                uint8_t* base = buf + (size_t)i * G::kChunk;
                uint32_t w[4 * kUnitPieces];
#pragma unroll
                for (int q = 0; q < kUnitPieces; q++) {
                    const uint4 v = *reinterpret_cast<const uint4*>(base + piece_pos(pc0 + q, lane));
                    w[4 * q] = v.x, w[4 * q + 1] = v.y, w[4 * q + 2] = v.z, w[4 * q + 3] = v.w;
                }
                if (need_pass) {
                    const uint16_t pr = T.pass_rows[seg + i];
                    if (pr != kNoRow)
                        store_pieces<kUnitPieces>(T.out + (uint64_t)pr * T.out_stride, off, pc0, lane, L, aligned, full,
                                                  w);
                }
                if (og_n) {
                    if constexpr (kGf16)
                        bitslice16(*reinterpret_cast<uint32_t(*)[16]>(w));
                    else
                        bitslice8(*reinterpret_cast<uint32_t(*)[8]>(w));
#pragma unroll
                    for (int q = 0; q < kUnitPieces; q++)
                        *reinterpret_cast<uint4*>(base + piece_pos(pc0 + q, lane)) =
                            make_uint4(w[4 * q], w[4 * q + 1], w[4 * q + 2], w[4 * q + 3]);
                }
            }
            __syncthreads();
            // ---- output rows, one per warp at a time
            // partial sums between segments stay bit-sliced when the chunk is
            // a whole aligned span of the row
            const bool sliced = !(kShape & kShapeOneSeg) && !atomic_out && full;
            const bool sliced_in = sliced && seg != in_lo;
            const bool sliced_out = sliced && seg + (uint32_t)seg_cap < n_in;
            for (uint32_t j = warp; j < og_n; j += 4) {
                if (j != (uint32_t)warp) c = lane_coef<kGf16>(T, seg, seg_n, og, j, lane);
                const uint32_t orow_idx = T.out_rows ? T.out_rows[og + j] : og + j;
                output_row<kGf16>(buf, c, steps, seg_n, lane,
                                  !(kShape & kShapeOneSeg) && !atomic_out && (seg != in_lo || T.accumulate),
                                  T.out + (uint64_t)orow_idx * T.out_stride, off, L, aligned, full, atomic_out,
                                  sliced_in, sliced_out);
            }
            __syncthreads();
        }
    }
    return true;
}

// Persistent drain: items are claimed from work_counter (or strided by grid
// when it is nullptr) one ahead of use, so the claim's latency is hidden.
// Warp 0 loads the current item's descriptor and issues its first stage's
// copies before the CTA meets at the barrier.
// Aligned shapes fit 9 CTAs per SM without spilling (2 % faster on cfg1
// decodes than 8); the unaligned ones keep the registers of 8.
template <int kGf16, int kShape>
__global__ void __launch_bounds__(kThreads, (kShape & kShapeAligned) ? 9 : 8) mxk_kernel(const MxkTask* __restrict__ tasks,
                                                          const uint32_t* __restrict__ item_task,
                                                          uint32_t item_lo, uint32_t total_items,
                                                          uint32_t* work_counter, int32_t* status, int seg_cap) {
    extern __shared__ __align__(128) uint8_t smem[];
    const SmemLayout S = layout<kGf16>(smem, seg_cap);
    const int tid = threadIdx.x;
    uint32_t claims = 0;
    auto claim = [&]() -> uint32_t {
        const uint32_t v = item_lo + (work_counter ? atomicAdd(work_counter, 1u) : blockIdx.x + claims * gridDim.x);
        claims++;
        return v;
    };
    if (tid == 0) {
        mbar_init(S.bar, 1);
        fence_mbar_init();
        S.item[1] = claim();
    }
    uint32_t phase = 0;
    for (;;) {
        if (tid == 0) {
            const uint32_t cur = S.item[1];
            S.item[0] = cur;
            S.item[1] = cur < total_items ? claim() : total_items;
        }
        __syncthreads();
        const uint32_t item = S.item[0];
        if (item >= total_items) return;
        if (tid < 32) {
            if (tid < (int)kTaskWords)
                S.task[tid] = __ldg(reinterpret_cast<const uint32_t*>(tasks + __ldg(item_task + item)) + tid);
            __syncwarp();
            const MxkTask& T = *reinterpret_cast<const MxkTask*>(S.task);
            if (((kShape & kShapeAligned) || T.aligned) && item_loads(T, 0, T.n_out))
                issue_stage<kGf16>(T, item - T.item_begin, 0, umin32((uint32_t)seg_cap, T.n_in), S.buf, S.bar, tid);
        }
        __syncthreads();
        const MxkTask& T = *reinterpret_cast<const MxkTask*>(S.task);
        const bool issued = ((kShape & kShapeAligned) || T.aligned) && item_loads(T, 0, T.n_out);
        if (!process_item<kGf16, kShape>(T, item - T.item_begin, S.buf, S.steps, S.bar, phase, seg_cap, status, 0, T.n_out,
                                 issued))
            return;
        __syncthreads();
    }
}

// One task passed by value (kernel parameter space).  Items are (row chunk,
// output range) with `per` outputs each, so a stripe with few row chunks
// still spreads over the SMs (the chunk's rows are then staged once per
// output range, mostly from L2).
template <int kGf16>
__global__ void __launch_bounds__(kThreads, 8) mxk_single_kernel(const MxkTask T, int32_t* status,
                                                                            int seg_cap, uint32_t per) {
    extern __shared__ __align__(128) uint8_t smem[];
    const SmemLayout S = layout<kGf16>(smem, seg_cap);
    if (threadIdx.x == 0) {
        mbar_init(S.bar, 1);
        fence_mbar_init();
    }
    __syncthreads();
    uint32_t phase = 0;
    const uint32_t splits = T.n_out ? (T.n_out + per - 1) / per : 1;
    const uint32_t items = T.n_items * splits;
    for (uint32_t item = blockIdx.x; item < items; item += gridDim.x) {
        const uint32_t chunk = item % T.n_items, sp = item / T.n_items;
        const uint32_t lo = sp * per, hi = min(T.n_out, lo + per);
        if (!process_item<kGf16>(T, chunk, S.buf, S.steps, S.bar, phase, seg_cap, status, lo, hi, false)) break;
        __syncthreads();
    }
}

// Many inputs: items are (row chunk, output range of `per` outputs, block of
// seg_cap inputs); each CTA XORs its block's partial sums into the outputs
// with atomicXor (outputs zeroed beforehand unless accumulating), so all
// input blocks run in parallel instead of one CTA walking every segment and
// re-reading its partial sums.
// With `chain` (programmatic dependent launch) the set-up overlaps the kernel
// before, and the items start once it has completed (its coefficients and
// zeroed outputs visible).
template <int kGf16>
__global__ void __launch_bounds__(kThreads, 8) mxk_ksplit_kernel(const MxkTask T, int32_t* status, int seg_cap,
                                                                 uint32_t per, int chain) {
    extern __shared__ __align__(128) uint8_t smem[];
    const SmemLayout S = layout<kGf16>(smem, seg_cap);
    if (threadIdx.x == 0) {
        mbar_init(S.bar, 1);
        fence_mbar_init();
    }
    if (chain) {
        pdl_trigger();
        pdl_wait();
    }
    __syncthreads();
    uint32_t phase = 0;
    const uint32_t blocks = (T.n_in + seg_cap - 1) / seg_cap;
    const uint32_t splits = T.n_out ? (T.n_out + per - 1) / per : 1;
    const uint32_t items = T.n_items * splits * blocks;
    for (uint32_t item = blockIdx.x; item < items; item += gridDim.x) {
        const uint32_t chunk = item % T.n_items, rest = item / T.n_items;
        const uint32_t sp = rest % splits, blk = rest / splits;
        const uint32_t lo = blk * (uint32_t)seg_cap;
        const uint32_t olo = sp * per, ohi = min(T.n_out, olo + per);
        if (!process_item<kGf16>(T, chunk, S.buf, S.steps, S.bar, phase, seg_cap, status, olo, ohi, false, lo,
                                 lo + (uint32_t)seg_cap, true))
            break;
        __syncthreads();
    }
}

// Zero the output rows of T (4-byte words; L % 4 == 0).
// With `chain` (programmatic dependent launch after the kernel that builds the
// task's coefficients) the zeroing runs beside that kernel and waits for it
// only before exiting.
__global__ void zero_out_rows_kernel(const MxkTask T, int chain) {
    if (chain) pdl_trigger();
    const uint64_t words = T.L / 4;
    for (uint64_t x = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; x < (uint64_t)T.n_out * words;
         x += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t j = (uint32_t)(x / words);
        const uint32_t r = T.out_rows ? T.out_rows[j] : j;
        reinterpret_cast<uint32_t*>(T.out + (uint64_t)r * T.out_stride)[x - (uint64_t)j * words] = 0;
    }
    if (chain) pdl_wait();
}

// ---- bounded-wait self-test -------------------------------------------------
// Waits on an mbarrier that nothing arrives on: the bounded wait must give up
// after limit_ns and report SCRS_ERR_DEVICE_TIMEOUT through the status word,
// leaving the context usable.  No copy is in flight, so nothing is left to
// drain before returning.
__global__ void wait_selftest_kernel(int32_t* status, uint64_t limit_ns) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x != 0) return;
    mbar_init(&bar, 1);
    fence_mbar_init();
    mbar_wait_bounded(&bar, 0, status, limit_ns);
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(&bar)) : "memory");
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

// Batched plans with r <= kWarpPlanMaxR: one warp per decode (a whole CTA per
// decode leaves most of its threads idle when r is a handful).  The same
// closed form as cauchy_plan_body; rv/cv/rf/cf live in per-warp shared
// scratch.
constexpr uint32_t kWarpPlanMaxR = 64;
constexpr int kPlanWarps = 8;

template <int kGf16>
__global__ void __launch_bounds__(32 * kPlanWarps) cauchy_plan_warp_kernel(const CauchyPlanTask* __restrict__ tasks,
                                                                          uint32_t n_tasks) {
    __shared__ Gf8Tables tb;
    __shared__ uint32_t scratch[kPlanWarps][4 * kWarpPlanMaxR];
    for (int i = threadIdx.x; i < 512; i += blockDim.x) {
        if (i < 256) tb.log[i] = c_gf8_log[i];
        tb.exp[i] = c_gf8_exp[i % 255];
    }
    __syncthreads();
    FieldOps<kGf16> F{tb};
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    uint32_t* rv = scratch[wib];
    uint32_t* cv = rv + kWarpPlanMaxR;
    uint32_t* rf = rv + 2 * kWarpPlanMaxR;
    uint32_t* cf = rv + 3 * kWarpPlanMaxR;
    for (uint32_t t = blockIdx.x * kPlanWarps + wib; t < n_tasks; t += gridDim.x * kPlanWarps) {
        const CauchyPlanTask P = tasks[t];
        const uint32_t r = P.r;
        for (uint32_t u = lane; u < r; u += 32) {
            rv[u] = y_var<kGf16>(P, tb, P.repairs[u]);
            cv[u] = x_var<kGf16>(P, tb, P.missing[u]);
        }
        __syncwarp();
        for (uint32_t u = lane; u < 2 * r; u += 32) {
            const bool is_row = u < r;
            const uint32_t q = is_row ? u : u - r;
            const uint32_t v = is_row ? rv[q] : cv[q];
            const uint32_t* other = is_row ? cv : rv;
            const uint32_t* same = is_row ? rv : cv;
            uint32_t cross = 1, within = 1;
            for (uint32_t h = 0; h < r; h++) {
                cross = F.mul(cross, v ^ other[h]);
                if (h != q) within = F.mul(within, v ^ same[h]);
            }
            (is_row ? rf : cf)[q] = F.mul(cross, F.inv(within));
        }
        __syncwarp();
        const uint32_t ld = P.ld;
        for (uint32_t x = lane; x < r * r; x += 32) {
            const uint32_t a = x / r, b = x - a * r;  // input row a (repair), output b (missing)
            const uint32_t val = F.mul(F.mul(rf[a], cf[b]), F.inv(cv[b] ^ rv[a]));
            if (kGf16)
                reinterpret_cast<uint16_t*>(P.coef)[(size_t)a * ld + b] = (uint16_t)val;
            else
                reinterpret_cast<uint8_t*>(P.coef)[(size_t)a * ld + b] = (uint8_t)val;
        }
        for (uint32_t x = lane; x < P.p * r; x += 32) {
            const uint32_t z = x / r, b = x - z * r;  // present row z, output b
            const uint32_t zv = x_var<kGf16>(P, tb, P.present[z]);
            uint32_t rp = 1, cp = 1;
            for (uint32_t h = 0; h < r; h++) {
                rp = F.mul(rp, zv ^ rv[h]);
                cp = F.mul(cp, zv ^ cv[h]);
            }
            const uint32_t val = F.mul(F.mul(F.mul(cp, F.inv(rp)), cf[b]), F.inv(zv ^ cv[b]));
            const size_t at = (size_t)(r + z) * ld + b;
            if (kGf16)
                reinterpret_cast<uint16_t*>(P.coef)[at] = (uint16_t)val;
            else
                reinterpret_cast<uint8_t*>(P.coef)[at] = (uint8_t)val;
        }
        __syncwarp();  // scratch is reused by the warp's next decode
    }
}

// Constant tables are per device: upload once on each device used.

cudaError_t ensure_tables() {
    static std::atomic<uint64_t> done{0};
    return once_per_device(done, [] {
        uint8_t ex[255], lg[256] = {0};
        uint8_t v = 1;
        for (int i = 0; i < 255; i++) {
            ex[i] = v;
            lg[v] = (uint8_t)i;
            v = gf8_mul_ce(v, 3);
        }
        // complete on the device before any plan kernel (on a non-blocking stream) reads it
        cudaError_t e = cudaMemcpyToSymbolAsync(c_gf8_exp, ex, sizeof ex, 0, cudaMemcpyHostToDevice,
                                                cudaStreamPerThread);
        if (e == cudaSuccess)
            e = cudaMemcpyToSymbolAsync(c_gf8_log, lg, sizeof lg, 0, cudaMemcpyHostToDevice, cudaStreamPerThread);
        if (e == cudaSuccess) e = cudaStreamSynchronize(cudaStreamPerThread);
        return e;
    });
}

// Shared memory of a launch staging seg_rows input rows per segment.
size_t smem_bytes(int gf16, int seg_rows) {
    const int chunk = gf16 ? FieldGeom<1>::kChunk : FieldGeom<0>::kChunk;
    const int segmax = gf16 ? FieldGeom<1>::kSegMax : FieldGeom<0>::kSegMax;
    const int seg = std::max(1, std::min(seg_rows, segmax));
    return (size_t)kSmemHeader + (size_t)seg * chunk;
}

// The persistent drain's instantiations, indexed by [field][drain_index(shape)]
// (GF(256) stripes, tower stripes).
using DrainFn = void (*)(const MxkTask*, const uint32_t*, uint32_t, uint32_t, uint32_t*, int32_t*, int);
constexpr DrainFn kDrains[2][6] = {{mxk_kernel<0, kShapeAny>,
                                    mxk_kernel<0, kShapeAligned>,
                                    mxk_kernel<0, kShapeAligned | kShapeWhole>,
                                    mxk_kernel<0, kShapeOneSeg>,
                                    mxk_kernel<0, kShapeOneSeg | kShapeAligned>,
                                    mxk_kernel<0, kShapeOneSeg | kShapeAligned | kShapeWhole>},
                                   {mxk_kernel<1, kShapeAny>,
                                    mxk_kernel<1, kShapeAligned>,
                                    mxk_kernel<1, kShapeAligned | kShapeWhole>,
                                    mxk_kernel<1, kShapeOneSeg>,
                                    mxk_kernel<1, kShapeOneSeg | kShapeAligned>,
                                    mxk_kernel<1, kShapeOneSeg | kShapeAligned | kShapeWhole>}};

int drain_index(int shape) {
    const bool aligned = shape & kShapeAligned, whole = aligned && (shape & kShapeWhole);
    return (shape & kShapeOneSeg ? 3 : 0) + (whole ? 2 : aligned ? 1 : 0);
}

template <int kGf16>
cudaError_t set_mxk_attrs() {
    using G = FieldGeom<kGf16>;
    static std::atomic<uint64_t> done{0};
    return once_per_device(done, [] {
        const int smem = (int)smem_bytes(kGf16, G::kSegMax);
        cudaError_t e =
            cudaFuncSetAttribute(mxk_single_kernel<kGf16>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(mxk_ksplit_kernel<kGf16>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        for (auto fn : kDrains[kGf16])  // the persistent drains of stripe batches
            if (e == cudaSuccess) e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        return e;
    });
}

// Input-split launch (see mxk_ksplit_kernel): outputs are zeroed first unless
// the task accumulates; about four outputs per item.
template <int kGf16>
cudaError_t launch_ksplit_impl(const MxkTask& T, int32_t* status, cudaStream_t stream, bool chain = false) {
    using G = FieldGeom<kGf16>;
    cudaError_t ea = set_mxk_attrs<kGf16>();
    if (ea != cudaSuccess) return ea;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.blockDim = dim3(kThreads);
    cfg.stream = stream;
    cfg.attrs = attr;
    cfg.numAttrs = chain ? 1 : 0;
    if (!T.accumulate && T.n_out) {
        const uint64_t words = (uint64_t)T.n_out * (T.L / 4);
        cudaLaunchConfig_t zc = cfg;
        zc.gridDim = dim3((unsigned)std::min<uint64_t>((words + 255) / 256, 148 * 16));
        zc.blockDim = dim3(256);
        cudaError_t e = cudaLaunchKernelEx(&zc, zero_out_rows_kernel, T, (int)chain);
        if (e != cudaSuccess) return e;
    }
    const int seg_cap = std::max(1, std::min((int)T.n_in, G::kSeg));
    const uint32_t per = std::max<uint32_t>(1, std::min<uint32_t>(T.n_out, 4));
    const uint32_t splits = T.n_out ? (T.n_out + per - 1) / per : 1;
    const uint64_t items = (uint64_t)T.n_items * splits * ((T.n_in + seg_cap - 1) / seg_cap);
    const int grid = (int)std::min<uint64_t>(items, 148u * 8u);
    cfg.gridDim = dim3(grid);
    cfg.dynamicSmemBytes = smem_bytes(kGf16, seg_cap);
    return cudaLaunchKernelEx(&cfg, mxk_ksplit_kernel<kGf16>, T, status, seg_cap, per, (int)chain);
}

// Whether partial sums of T's outputs can be combined with 4-byte atomicXor.
bool ksplit_ok(const MxkTask& T) {
    return T.L % 4 == 0 && T.out_stride % 4 == 0 && (reinterpret_cast<uintptr_t>(T.out) & 3u) == 0 && T.n_out > 0;
}

template <int kGf16>
cudaError_t launch_single_impl(const MxkTask& T, int32_t* status, int grid, cudaStream_t stream, bool chain) {
    using G = FieldGeom<kGf16>;
    if (T.n_items == 0 || (T.n_out == 0 && T.pass_rows == nullptr)) return cudaSuccess;
    cudaError_t e = set_mxk_attrs<kGf16>();
    if (e != cudaSuccess) return e;
    int seg_cap = std::max(1, std::min((int)T.n_in, G::kSeg));
    // More than one segment of inputs: split the inputs over CTAs instead.
    if ((int)T.n_in > seg_cap && ksplit_ok(T)) return launch_ksplit_impl<kGf16>(T, status, stream, chain);
    // Split the outputs when the row chunks alone cannot fill the GPU, keeping
    // at least one output per warp in each split (every split re-stages and
    // re-slices the chunk's input rows).
    constexpr uint32_t kTargetItems = 2 * 148;
    uint32_t per = std::max<uint32_t>(T.n_out, 1);
    if (T.n_items < kTargetItems && T.n_out > 4) {
        const uint32_t splits = std::min<uint32_t>((T.n_out + 3) / 4, (kTargetItems + T.n_items - 1) / T.n_items);
        per = (T.n_out + splits - 1) / splits;
    }
    const uint32_t items = T.n_items * (T.n_out ? (T.n_out + per - 1) / per : 1);
    if (grid <= 0 || grid > (int)items) grid = (int)items;
    mxk_single_kernel<kGf16><<<grid, kThreads, smem_bytes(kGf16, seg_cap), stream>>>(T, status, seg_cap, per);
    return cudaGetLastError();
}

}  // namespace

int mxk_default_seg(int max_in) { return std::max(1, std::min(max_in, FieldGeom<0>::kSeg)); }

cudaError_t prepare_batch_kernels() {
    cudaError_t e = ensure_tables();
    if (e == cudaSuccess) e = set_mxk_attrs<0>();
    if (e == cudaSuccess) e = set_mxk_attrs<1>();
    return e;
}

int mxk_ctas_per_sm(int seg_rows, int shape, int gf16) {
    int n = 0;
    if ((gf16 ? set_mxk_attrs<1>() : set_mxk_attrs<0>()) != cudaSuccess) return 1;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kDrains[gf16 ? 1 : 0][drain_index(shape)],
                                                                  kThreads, smem_bytes(gf16, seg_rows));
    if (e != cudaSuccess || n < 1) n = 1;
    return n;
}

cudaError_t launch_gf256_mxk(const MxkTask* tasks, const uint32_t* item_task, uint32_t item_lo, uint32_t item_end,
                             uint32_t* counter, int32_t* status, int seg_rows, int grid, cudaStream_t stream,
                             int shape, int gf16) {
    if (item_end <= item_lo) return cudaSuccess;
    if (seg_rows < 1 || seg_rows > (gf16 ? FieldGeom<1>::kSegMax : FieldGeom<0>::kSegMax)) return cudaErrorInvalidValue;
    cudaError_t e = gf16 ? set_mxk_attrs<1>() : set_mxk_attrs<0>();
    if (e != cudaSuccess) return e;
    if (grid <= 0 || grid > (int)(item_end - item_lo)) grid = (int)(item_end - item_lo);
    const auto fn = kDrains[gf16 ? 1 : 0][drain_index(shape)];
    fn<<<grid, kThreads, smem_bytes(gf16, seg_rows), stream>>>(tasks, item_task, item_lo, item_end, counter, status,
                                                                 seg_rows);
    return cudaGetLastError();
}

cudaError_t launch_mxk_single(const MxkTask& task, int gf16, int32_t* status, int grid, cudaStream_t stream,
                              bool chain) {
    if (gf16) return launch_single_impl<1>(task, status, grid, stream, chain);
    return launch_single_impl<0>(task, status, grid, stream, chain);
}

cudaError_t launch_mxk_ksplit(const MxkTask& T, int gf16, int32_t* status, cudaStream_t stream) {
    if (T.n_items == 0 || T.n_in == 0) return cudaSuccess;
    if (gf16) return launch_ksplit_impl<1>(T, status, stream);
    return launch_ksplit_impl<0>(T, status, stream);
}

cudaError_t launch_wait_selftest(int32_t* status, uint64_t limit_ns, cudaStream_t stream) {
    wait_selftest_kernel<<<1, 32, 0, stream>>>(status, limit_ns);
    return cudaGetLastError();
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

cudaError_t launch_cauchy_plan(const CauchyPlanTask* tasks, uint32_t n_tasks, int gf16, uint32_t max_r,
                               cudaStream_t stream) {
    if (n_tasks == 0) return cudaSuccess;
    cudaError_t e = ensure_tables();
    if (e != cudaSuccess) return e;
    if (max_r <= kWarpPlanMaxR) {
        const uint32_t grid = std::min<uint32_t>((n_tasks + kPlanWarps - 1) / kPlanWarps, 148u * 8u);
        if (gf16)
            cauchy_plan_warp_kernel<1><<<grid, 32 * kPlanWarps, 0, stream>>>(tasks, n_tasks);
        else
            cauchy_plan_warp_kernel<0><<<grid, 32 * kPlanWarps, 0, stream>>>(tasks, n_tasks);
        return cudaGetLastError();
    }
    size_t smem = (size_t)4 * std::min(max_r, kPlanSmemMaxR) * sizeof(uint32_t);
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
