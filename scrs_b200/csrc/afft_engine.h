// Additive-FFT engine over GF(2^16) on the device (scrs/src/afft/*.rs).
//
// Every systematic encode and erasure decode is the same computation: given
// the code polynomial F (degree < k, novel basis) at a known point set, with
// erased set E and locator L(x) = prod_{e in E}(x + e),
//   F(e) = (F L)'(e) / L'(e)  for e in E
// (scrs/src/afft/decoder.rs:294-357).  Encode takes E = [k, ts) and reads the
// repairs at points k..n-1; decode takes E = the untransmitted and lost points
// and reads the missing data points.  F is unique, so the repairs equal the
// reference's truncated-transform encode (afft/encoder.rs:150-214) byte for
// byte.
#pragma once

#include <stdint.h>

#include <vector>

#include "runtime.h"

namespace scrs {

class AfftWorkspace;

class AfftCodec {
   public:
    int32_t init(uint64_t k, uint64_t m, uint64_t L, scrs_error* err);
    // d_data: k rows; d_repairs: m rows.
    int32_t encode(const uint8_t* d_data, uint8_t* d_repairs, AfftWorkspace& ws, int32_t* status,
                   cudaStream_t st, scrs_error* err) const;
    // d_payloads: rows of received symbols; row of codeword index i is
    // row_map[i] (host array of n entries) or i when row_map is nullptr.  Only
    // rows with have[i] != 0 are read.  d_out: k rows of data.
    int32_t decode(const uint8_t* d_payloads, const uint8_t* have, uint8_t* d_out, AfftWorkspace& ws,
                   int32_t* status, cudaStream_t st, scrs_error* err, const uint16_t* row_map = nullptr) const;

    // r <= 5 missing data symbols: one coefficient table + multiply-XOR pass.
    // targeted_lists fills the lists in the workspace's stage area (host);
    // decode_targeted runs the device part once they are uploaded.
    size_t targeted_list_elems() const;
    int32_t targeted_lists(const uint8_t* have, AfftWorkspace& ws, scrs_error* err, const uint16_t* row_map,
                           const uint16_t* miss, uint32_t nm, const uint16_t* pres, uint32_t np) const;
    // after_copy: the kernel before it on the stream is the present-row copy
    // (its launches are chained after it, see afft.cu)
    int32_t decode_targeted(const uint8_t* d_payloads, uint8_t* d_out, AfftWorkspace& ws, int32_t* status,
                            cudaStream_t st, scrs_error* err, uint32_t nm, bool after_copy = false) const;

    uint64_t k = 0, m = 0, n = 0, L = 0, padded_k = 0, ts = 0;
    uint32_t log_ts = 0;
    DevBuf factors;                 // uint16[ts], heap layout (transform.rs:30-61)
    DevBuf log_walsh;               // uint32[ts]: transformed log table, times 1/ts (decoder.rs:691-703)
    uint16_t deriv_factors[16] = {};
    DevBuf enc_values, enc_derivs;  // encode locator for E = [k, ts): uint16[ts]
    // Systematic locator L_S(x) = prod_{i<k}(x + i) (decoder.rs:256-266):
    // sys_values[e] = L_S(e) for e >= k, sys_derivs[i] = L_S'(i) for i < k.
    DevBuf sys_values, sys_derivs;
    std::vector<uint16_t> h_sys_values, h_sys_derivs;  // host copies (targeted r x r solve)
};

class AfftWorkspace {
   public:
    AfftWorkspace() = default;
    AfftWorkspace(const AfftWorkspace&) = delete;
    AfftWorkspace& operator=(const AfftWorkspace&) = delete;
    ~AfftWorkspace();
    int32_t init_encode(const AfftCodec& c, scrs_error* err);
    int32_t init_decode(const AfftCodec& c, scrs_error* err);
    // Host side of a decode's uploads (row lists, codeword -> payload row map,
    // known-point mask, targeted lists) in pinned memory, so the copies are
    // asynchronous.  Two areas used in turn: a decode waits only for the
    // copies of the decode before the previous one before it rewrites an area.
    int32_t stage_acquire(scrs_error* err);
    int32_t stage_release(cudaStream_t st, scrs_error* err);
    uint8_t* stage_ptr() const { return stage[cur].as<uint8_t>(); }
    PinnedBuf stage[2];
    cudaEvent_t staged[2] = {nullptr, nullptr};
    bool stage_pending[2] = {false, false};
    int cur = 0;
    size_t off_map = 0, off_known = 0, off_lists = 0;  // byte offsets in an area (rows at 0)
    DevBuf work0, work1;            // ts * L bytes, bit-sliced rows
    DevBuf known;                   // uint8[ts]: the encode's known-point mask
    DevBuf wht_a;                   // uint32[ts]: locator transform (ts > 16384)
    DevBuf values, derivs;          // uint16[ts]
    DevBuf up;                      // device mirror of a decode's stage area, uploaded in one copy
    DevBuf tgen, tcoef;             // targeted decode: generator rows, fused coefficients
    uint64_t k = 0, m = 0, L = 0;
};

// Locator evaluations for a known-point mask (decoder.rs:672-714), on the
// device: values[x] = L(x) for known x, derivs[x] = L'(x) for erased x.
// log_walsh: the codec's transformed log table; wa: uint32[ts] of work space
// (used when ts > 16384).
int32_t afft_locator_device(const uint8_t* d_known, uint32_t ts, const uint32_t* log_walsh, uint32_t* wa,
                            uint16_t* values, uint16_t* derivs, cudaStream_t st, scrs_error* err);

}  // namespace scrs
