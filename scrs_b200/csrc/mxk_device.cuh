// Device pieces of the multiply-XOR kernels shared by the precompiled kernels
// (mxk_kernels.cu) and the kernels specialised to one coefficient matrix at
// run time (mxk_spec.cuh, compiled by jit.cu): the shared-memory header,
// row-chunk loads and stores, and the TMA staging of input rows.
#pragma once

#include "common.cuh"
#include "kernels.cuh"

namespace scrs {
namespace {

// Shared-memory header: mbarrier (0), item words (8, 12), task descriptor
// (16), one step list per warp (kStepOffset).
constexpr int kStepOffset = 128;
constexpr int kStepBytes = 144;  // u16 steps, 2 per GF(256) or 4 per GF(2^16) input, + 1 read-ahead
constexpr int kSmemHeader = kStepOffset + 4 * kStepBytes;
// step entries: 2 per GF(256) input, 4 per GF(2^16) input, plus the read-ahead
static_assert(2 * (4 * FieldGeom<1>::kSegMax + 1) <= kStepBytes, "step list too short");
static_assert(2 * (2 * FieldGeom<0>::kSegMax + 1) <= kStepBytes, "step list too short");
static_assert(FieldGeom<0>::kSegMax <= 32 && FieldGeom<1>::kSegMax <= 32, "one lane per staged row");
constexpr uint32_t kTaskWords = (sizeof(MxkTask) + 3) / 4;
static_assert(kTaskWords <= 32, "task descriptor must fit one warp's loads");
static_assert(16 + kTaskWords * 4 <= kStepOffset, "header too small");

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

// Byte offset of a lane's piece pc (16 bytes) within a chunk row: piece pc
// of all 32 lanes is one contiguous, coalesced 512-byte span.
__device__ __forceinline__ uint32_t piece_pos(int pc, int lane) { return (uint32_t)pc * 512u + 16u * (uint32_t)lane; }

template <int kGf16>
struct Lane {
    static constexpr int kPieces = FieldGeom<kGf16>::kPieces;
    static constexpr int kWords = 4 * kPieces;
    using Words = uint32_t[kWords];
};

template <int kGf16>
__device__ __forceinline__ void bitslice_lane(typename Lane<kGf16>::Words& w) {
    if constexpr (kGf16) {
        bitslice16(w);
    } else {
#pragma unroll
        for (int h = 0; h < Lane<0>::kWords; h += 8) bitslice8(*reinterpret_cast<uint32_t(*)[8]>(&w[h]));
    }
}

// Issue the TMA copies of input rows [seg, seg + seg_n) of one chunk.  Called
// by all 32 lanes of one warp: lane i < seg_n resolves and copies row seg + i,
// so the row-number loads overlap instead of following one another.
template <int kGf16>
__device__ __forceinline__ void issue_stage(const MxkTask& T, uint32_t chunk, uint32_t seg, uint32_t seg_n,
                                            uint8_t* buf, uint64_t* bar, int lane) {
    using G = FieldGeom<kGf16>;
    const uint64_t off = (uint64_t)chunk * G::kChunk;
    const uint32_t bytes = (uint32_t)umin64(G::kChunk, T.L - off);
    const uint8_t* src = nullptr;
    if ((uint32_t)lane < seg_n) {
        const uint32_t r = T.in_rows ? T.in_rows[seg + lane] : seg + lane;
        src = T.in + (uint64_t)r * T.in_stride + off;
    }
    if (lane == 0) mbar_arrive_expect_tx(bar, seg_n * bytes);
    __syncwarp();
    if ((uint32_t)lane < seg_n) {
        fence_proxy_async_smem();
        tma_load_1d(buf + (size_t)lane * G::kChunk, src, bytes, bar);
    }
}

// Whether an item reads any input rows at all.
__device__ __forceinline__ bool item_loads(const MxkTask& T, uint32_t out_lo, uint32_t out_hi) {
    return T.n_in && (out_hi > out_lo || (out_lo == 0 && T.pass_rows != nullptr));
}

// Store `n` 16-byte pieces starting at piece pc0 of this lane.  `full`: the
// whole chunk lies inside an aligned row, so no bounds checks are needed.
template <int kN>
__device__ __forceinline__ void store_pieces(uint8_t* row, uint64_t off, int pc0, int lane, uint64_t L, bool aligned,
                                             bool full, const uint32_t* w) {
    if (full) {
#pragma unroll
        for (int q = 0; q < kN; q++)
            *reinterpret_cast<uint4*>(row + off + piece_pos(pc0 + q, lane)) =
                make_uint4(w[4 * q], w[4 * q + 1], w[4 * q + 2], w[4 * q + 3]);
    } else {
#pragma unroll
        for (int q = 0; q < kN; q++)
            store_piece(row, off + piece_pos(pc0 + q, lane), L, aligned,
                        make_uint4(w[4 * q], w[4 * q + 1], w[4 * q + 2], w[4 * q + 3]));
    }
}

// Shared memory: [header: mbarrier | item words | task descriptor | step
// lists] [staged rows: seg_cap * chunk bytes].
struct SmemLayout {
    uint64_t* bar;
    volatile uint32_t* item;  // [0] the item being processed, [1] the next one
    uint32_t* task;
    uint8_t* steps;
    uint8_t* buf;
};

template <int kGf16>
__device__ __forceinline__ SmemLayout layout(uint8_t* smem, int seg_cap) {
    uint8_t* buf = smem + kSmemHeader;
    (void)seg_cap;
    return SmemLayout{reinterpret_cast<uint64_t*>(smem), reinterpret_cast<volatile uint32_t*>(smem + 8),
                      reinterpret_cast<uint32_t*>(smem + 16), smem + kStepOffset, buf};
}

}  // namespace
}  // namespace scrs
