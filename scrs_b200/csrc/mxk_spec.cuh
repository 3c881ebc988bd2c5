// Persistent drain of GF(256) encode stripes that share one coefficient
// matrix, compiled at run time (jit.cu) with that matrix's XOR networks
// inlined.  jit.cu places before this file, in namespace scrs::spec:
//   constexpr uint32_t kK, kM, kGroups;   // inputs, outputs, ceil(kM / 2)
//   void group(uint32_t g, const uint8_t* half, uint32_t (&a0)[8], uint32_t (&a1)[8]);
// group(g, ...) XORs C[i][2g] * x_i into a0 and C[i][2g+1] * x_i into a1 for
// every input i, reading the 8 planes of x_i's half-lane at half + i * chunk
// (and + 512).  Each product is the whole-byte network of its constant with
// shared XOR pairs, so there is no coefficient load, no jump table and no
// nibble fold: about a third fewer XORs per product than the generic kernel's
// nibble steps, and no per-step dispatch.
//
// Work items are (stripe, chunk) as in mxk_kernel: the rows are staged by TMA
// and bit-sliced in place per (row, half); then warp w takes half w & 1 of
// every lane's 64 bytes and the output pairs w >> 1, w >> 1 + 2, ..., so two
// warps run each generated code path (the instruction footprint is
// ceil(m/2) paths, not m).
#pragma once

namespace scrs {

extern "C" __global__ void __launch_bounds__(kThreads, 10)
    scrs_spec_drain(const MxkTask* __restrict__ tasks, const uint32_t* __restrict__ item_task, uint32_t item_lo,
                    uint32_t total_items, uint32_t* work_counter, int32_t* status) {
    using G = FieldGeom<0>;
    extern __shared__ __align__(128) uint8_t smem[];
    const SmemLayout S = layout<0>(smem, (int)spec::kK);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) {
        mbar_init(S.bar, 1);
        fence_mbar_init();
        S.item[1] = item_lo + atomicAdd(work_counter, 1u);
    }
    uint32_t phase = 0;
    for (;;) {
        if (tid == 0) {  // claim the next item one ahead of use
            const uint32_t cur = S.item[1];
            S.item[0] = cur;
            S.item[1] = cur < total_items ? item_lo + atomicAdd(work_counter, 1u) : total_items;
        }
        __syncthreads();
        const uint32_t item = S.item[0];
        if (item >= total_items) return;
        if (tid < 32) {
            if (tid < (int)kTaskWords)
                S.task[tid] = __ldg(reinterpret_cast<const uint32_t*>(tasks + __ldg(item_task + item)) + tid);
            __syncwarp();
            const MxkTask& T = *reinterpret_cast<const MxkTask*>(S.task);
            if (T.aligned) issue_stage<0>(T, item - T.item_begin, 0, spec::kK, S.buf, S.bar, tid);
        }
        __syncthreads();
        const MxkTask& T = *reinterpret_cast<const MxkTask*>(S.task);
        const uint64_t L = T.L;
        const uint64_t off = (uint64_t)(item - T.item_begin) * G::kChunk;
        const bool aligned = T.aligned != 0;
        const bool full = aligned && off + G::kChunk <= L;
        if (aligned) {
            const bool ok = mbar_wait_bounded(S.bar, phase, status);
            phase ^= 1u;
            if (!__syncthreads_and(ok)) return;
        } else {
            for (uint32_t i = warp; i < spec::kK; i += 4) {
                const uint8_t* row = T.in + (uint64_t)i * T.in_stride;
#pragma unroll
                for (int pc = 0; pc < G::kPieces; pc++) {
                    const uint32_t pp = piece_pos(pc, lane);
                    *reinterpret_cast<uint4*>(S.buf + (size_t)i * G::kChunk + pp) = load_piece(row, off + pp, L, false);
                }
            }
            __syncthreads();
        }
        // bit-slice the staged rows in place, one (row, half) per warp at a time
        for (uint32_t u = warp; u < 2 * spec::kK; u += 4) {
            uint8_t* base = S.buf + (size_t)(u >> 1) * G::kChunk;
            const int pc0 = (int)(u & 1) * 2;
            uint32_t w[8];
#pragma unroll
            for (int q = 0; q < 2; q++) {
                const uint4 v = *reinterpret_cast<const uint4*>(base + piece_pos(pc0 + q, lane));
                w[4 * q] = v.x, w[4 * q + 1] = v.y, w[4 * q + 2] = v.z, w[4 * q + 3] = v.w;
            }
            bitslice8(w);
#pragma unroll
            for (int q = 0; q < 2; q++)
                *reinterpret_cast<uint4*>(base + piece_pos(pc0 + q, lane)) =
                    make_uint4(w[4 * q], w[4 * q + 1], w[4 * q + 2], w[4 * q + 3]);
        }
        __syncthreads();
        const int h = warp & 1;
        const uint8_t* half = S.buf + 16 * lane + h * 1024;
        for (uint32_t g = (uint32_t)warp >> 1; g < spec::kGroups; g += 2) {
            uint32_t a0[8], a1[8];
#pragma unroll
            for (int t = 0; t < 8; t++) a0[t] = 0, a1[t] = 0;
            spec::group(g, half, a0, a1);
            bitslice8(a0);
            store_pieces<2>(T.out + (uint64_t)(2 * g) * T.out_stride, off, 2 * h, lane, L, aligned, full, a0);
            if (2 * g + 1 < spec::kM) {
                bitslice8(a1);
                store_pieces<2>(T.out + (uint64_t)(2 * g + 1) * T.out_stride, off, 2 * h, lane, L, aligned, full, a1);
            }
        }
        __syncthreads();
    }
}

}  // namespace scrs
