// Device work descriptors and launch entry points shared by the kernels and
// the host engine code.
#pragma once

#ifndef __CUDACC_RTC__  // the run-time compiler (jit.cu) sees only the device parts
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <mutex>
#endif

namespace scrs {

#ifndef __CUDACC_RTC__
// Per-device one-time set-up (function attributes such as the dynamic
// shared-memory limit are set per device): runs `set` for the current device
// until it succeeds once.  The device's bit in `done_mask` is published only
// after `set` succeeded, and set-up runs under a lock, so no thread launches
// on a half-set-up device.
template <class F>
cudaError_t once_per_device(std::atomic<uint64_t>& done_mask, F&& set) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return set();
    const uint64_t bit = 1ull << dev;
    if (done_mask.load(std::memory_order_acquire) & bit) return cudaSuccess;
    static std::mutex mu;
    std::lock_guard<std::mutex> lock(mu);
    if (done_mask.load(std::memory_order_relaxed) & bit) return cudaSuccess;
    e = set();
    if (e == cudaSuccess) done_mask.fetch_or(bit, std::memory_order_release);
    return e;
}
#endif

constexpr uint16_t kNoRow = 0xFFFFu;
constexpr int kThreads = 128;   // 4 warps per CTA
constexpr int kMaxOutGroup = 64; // outputs computed per pass over the inputs

// Field-dependent geometry: bytes a lane owns and the CTA's column chunk.
// A GF(256) lane holds two 32-byte plane sets, a GF(2^16) lane one 64-byte set.
template <int kGf16>
struct FieldGeom {
    static constexpr int kLaneBytes = 64;
    static constexpr int kChunk = 32 * kLaneBytes;     // bytes per row per CTA
    static constexpr int kPieces = kLaneBytes / 16;    // 16-byte pieces per lane
    static constexpr int kSeg = 16;                    // input rows staged per segment (default)
    static constexpr int kSegMax = kGf16 ? 16 : 32;    // most rows a segment may stage
    static constexpr int kElem = kGf16 ? 2 : 1;        // coefficient bytes
};

// One stripe's multiply-XOR job: out_rows[j] = XOR_i coef[i][j] * in_rows[i]
// for j < n_out, plus verbatim copies in -> pass_rows (decode's present data).
struct MxkTask {
    const uint8_t* in;        // row r of the input is in + r * in_stride
    uint8_t* out;             // row r of the output is out + r * out_stride
    const void* coef;         // [n_in][ld] elements (uint8 or uint16)
    const uint16_t* in_rows;  // n_in input row numbers (nullptr: 0..n_in-1)
    const uint16_t* out_rows; // n_out output row numbers (nullptr: 0..n_out-1)
    const uint16_t* pass_rows;// n_in output rows for verbatim copies (kNoRow: none)
    const uint16_t* coef_rows;// n_in coefficient rows (nullptr: input position)
    uint64_t L;               // bytes per row
    uint64_t in_stride;
    uint64_t out_stride;
    uint32_t n_in;
    uint32_t n_out;
    uint32_t ld;
    uint32_t item_begin;      // first work item (row chunk) of this task
    uint32_t n_items;         // ceil(L / chunk)
    uint32_t aligned;         // all rows 16-byte aligned and L % 16 == 0
    uint32_t accumulate;      // 1: out ^= sum (incremental feed); 0: out = sum
    uint32_t pad;
};

// Closed-form reduced Cauchy solve for one decode (decoder/cauchy_inverse.rs:50-167,
// tower/decoder.rs:433-546).  Rows of `coef`: first the r received repairs
// (coefficients of the inverse A^-1), then the p present data symbols (the
// fused coefficients), each row holding r output coefficients.
struct CauchyPlanTask {
    uint32_t r;
    uint32_t p;
    uint32_t ld;              // row stride of coef, in elements
    uint32_t engine;          // SCRS_ENGINE_*
    uint32_t k;
    uint32_t pad;
    const uint16_t* missing;  // r data indices
    const uint16_t* repairs;  // r repair columns j (codeword index k + j)
    const uint16_t* present;  // p data indices
    const uint16_t* powers;   // GF(65536): g^i for i < k + m
    void* coef;
    uint32_t* work;           // 4*r words of global scratch, or nullptr (shared memory)
};

#ifndef __CUDACC_RTC__
// Launchers (return cudaError_t of the launch).
// Persistent drain of the work items [item_lo, item_end): item i belongs to
// tasks[item_task[i]] (row chunk i - item_begin of that task).  work_counter
// (zeroed before the launch) hands items out dynamically; nullptr strides
// items by grid instead.
// seg_rows: input rows staged per segment, 1..FieldGeom<0>::kSegMax.
// shape: flags of what every task of the range is known to satisfy, so that
// a kernel without the other paths runs (less code for the instruction
// cache): kShapeAligned (aligned != 0), kShapeWhole (only with kShapeAligned:
// L a multiple of the row chunk, so every chunk is full), kShapeOneSeg
// (n_in <= seg_rows and accumulate == 0: no partial sums carried from one
// segment to the next).
constexpr int kShapeAny = 0, kShapeAligned = 1, kShapeWhole = 2, kShapeOneSeg = 4;
// gf16 != 0: tower stripes (GF((2^8)^2), seg_rows at most FieldGeom<1>::kSegMax).
cudaError_t launch_gf256_mxk(const MxkTask* tasks, const uint32_t* item_task, uint32_t item_lo, uint32_t item_end,
                             uint32_t* work_counter, int32_t* status, int seg_rows, int grid, cudaStream_t stream,
                             int shape = kShapeAny, int gf16 = 0);
// One task by value; grid <= 0 means one CTA per row chunk (or the
// input-split form for more than one segment of inputs, see below).  `chain`:
// the input-split form's launches use programmatic dependent launch, so they
// may start while the kernel before them on the stream runs (they wait for it
// before reading the coefficients); the single-kernel form ignores it.
cudaError_t launch_mxk_single(const MxkTask& task, int gf16, int32_t* status, int grid, cudaStream_t stream,
                              bool chain = false);
cudaError_t launch_cauchy_plan_single(const CauchyPlanTask& task, int gf16, cudaStream_t stream);
// Input-split form: inputs split into blocks over CTAs, partial sums XORed
// (atomicXor) into the outputs, which the launch zeroes first unless the task
// accumulates; needs L and the output rows 4-byte aligned.  launch_mxk_single
// takes this form by itself when a task has more than one segment of inputs.
cudaError_t launch_mxk_ksplit(const MxkTask& task, int gf16, int32_t* status, cudaStream_t stream);
// One bounded wait that nothing completes (limit_ns of global time).
cudaError_t launch_wait_selftest(int32_t* status, uint64_t limit_ns, cudaStream_t stream);
// max_r: the largest r among the tasks (all of them, with or without `work`).
cudaError_t launch_cauchy_plan(const CauchyPlanTask* tasks, uint32_t n_tasks, int gf16, uint32_t max_r,
                               cudaStream_t stream);
// Largest r the plan kernel keeps in shared memory.
constexpr uint32_t kPlanSmemMaxR = 12288;
// Input rows per segment when nothing else is chosen: all of them up to kSeg.
int mxk_default_seg(int max_in);
// Most CTAs of the persistent drain (GF(256), or tower with gf16) one SM
// holds with seg_rows rows staged per segment (shared memory and registers
// permitting).
int mxk_ctas_per_sm(int seg_rows, int shape = kShapeAny, int gf16 = 0);
// The one-time per-device set-up of the batch kernels (decode-plan tables,
// shared-memory limits).  Must precede a stream capture of them: the set-up
// synchronises, which a capturing thread may not do.
cudaError_t prepare_batch_kernels();
#endif  // __CUDACC_RTC__

}  // namespace scrs
