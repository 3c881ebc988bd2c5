// Shared device/host helpers for the sm_100a erasure-coding kernels.
#pragma once

#ifndef __CUDACC_RTC__  // the run-time compiler (jit.cu) supplies stdint.h and the status codes
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/scrs_gpu.h"
#endif

#define SCRS_HD __host__ __device__ __forceinline__

namespace scrs {

// ---- GF(256): polynomial 0x11B, generator 3 (scrs/src/algebra/gf256.rs) ----
// Compile-time product used to build the per-coefficient XOR networks.
__host__ __device__ constexpr uint8_t gf8_mul_ce(uint8_t a, uint8_t b) {
    uint8_t acc = 0;
    for (int i = 0; i < 8; i++) {
        if ((b >> i) & 1) acc ^= a;
        uint8_t hi = a & 0x80;
        a = (uint8_t)(a << 1);
        if (hi) a ^= 0x1B;
    }
    return acc;
}

// Bit r of (c * x^s): entry (r, s) of the 8x8 GF(2) matrix of "multiply by c".
__host__ __device__ constexpr bool gf8_matrix_bit(int c, int r, int s) {
    return (gf8_mul_ce((uint8_t)c, (uint8_t)(1u << s)) >> r) & 1;
}

constexpr uint8_t kGf16Delta = 0x20;    // u^2 + u + 0x20 (gf65536.rs:20)
constexpr uint16_t kGf16Gen = 0x0108;   // gf65536.rs:26

// ---- bit-slicing ------------------------------------------------------------
// 8 words (32 bytes) <-> 8 bit planes.  Three delta swaps exchange the word
// index bits (q2 q1 q0) with the in-byte bit index (s2 s1 s0); the map is an
// involution, so the same call converts planes back to bytes.  After the call
// w[s] holds bit s of the 32 bytes.
// Exchange the bits of b selected by M with the bits of a selected by M << D.
template <int D, uint32_t M>
SCRS_HD void delta_swap(uint32_t& a, uint32_t& b) {
    const uint32_t t = ((a >> D) ^ b) & M;
    b ^= t;
    a ^= t << D;
}

SCRS_HD void bitslice8(uint32_t (&w)[8]) {
    delta_swap<4, 0x0F0F0F0Fu>(w[0], w[4]);
    delta_swap<4, 0x0F0F0F0Fu>(w[1], w[5]);
    delta_swap<4, 0x0F0F0F0Fu>(w[2], w[6]);
    delta_swap<4, 0x0F0F0F0Fu>(w[3], w[7]);
    delta_swap<2, 0x33333333u>(w[0], w[2]);
    delta_swap<2, 0x33333333u>(w[1], w[3]);
    delta_swap<2, 0x33333333u>(w[4], w[6]);
    delta_swap<2, 0x33333333u>(w[5], w[7]);
    delta_swap<1, 0x55555555u>(w[0], w[1]);
    delta_swap<1, 0x55555555u>(w[2], w[3]);
    delta_swap<1, 0x55555555u>(w[4], w[5]);
    delta_swap<1, 0x55555555u>(w[6], w[7]);
}

// 16 words (64 bytes of interleaved [a, b] GF(2^16) elements) <-> 16 planes.
// Word index bits (q3..q0) swap with (byte-in-word bit 0, s2, s1, s0); after
// the call w[s] = bit s of the `a` components and w[8 + s] = bit s of the
// `b` components of the 32 elements.  Involution.
SCRS_HD void bitslice16(uint32_t (&w)[16]) {
#pragma unroll
    for (int q = 0; q < 8; q++) delta_swap<8, 0x00FF00FFu>(w[q], w[q + 8]);
#pragma unroll
    for (int h = 0; h < 16; h += 8) {
#pragma unroll
        for (int q = 0; q < 4; q++) delta_swap<4, 0x0F0F0F0Fu>(w[h + q], w[h + q + 4]);
#pragma unroll
        for (int q = 0; q < 2; q++) {
            delta_swap<2, 0x33333333u>(w[h + q], w[h + q + 2]);
            delta_swap<2, 0x33333333u>(w[h + q + 4], w[h + q + 6]);
        }
#pragma unroll
        for (int q = 0; q < 8; q += 2) delta_swap<1, 0x55555555u>(w[h + q], w[h + q + 1]);
    }
}

// ---- bounded waits -------------------------------------------------------------
// Every device-side wait gives up after kWaitLimitNs of global time (checked
// every 64 polls) and reports SCRS_ERR_DEVICE_TIMEOUT through the launch's
// status word.
constexpr uint64_t kWaitLimitNs = 2000000000ull;

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Programmatic dependent launch: a kernel launched with the programmatic
// stream serialization attribute may start while the kernel before it on the
// stream is still running.  It reads nothing that kernel writes before
// pdl_wait(), which returns once that kernel has completed and its writes are
// visible (at once for a kernel launched without the attribute);
// pdl_trigger() lets the next such kernel start its own prologue.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

__device__ __forceinline__ void report_status(int32_t* status, int32_t code) {
    if (status) atomicCAS(status, 0, code);
}

// ---- mbarrier + TMA bulk copy (PTX) -----------------------------------------
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count));
}

__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

// Returns true when the phase with the given parity has completed.  A
// thread whose phase is still open is suspended by the hardware until the
// phase completes or about kWaitSuspendNs pass, so waiting costs few issue
// slots.
constexpr uint32_t kWaitSuspendNs = 20000;
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity), "n"(kWaitSuspendNs)
        : "memory");
    return done != 0;
}

// Bounded wait: false (and a status report) when the time limit runs out.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, int32_t* status,
                                                  uint64_t limit_ns = kWaitLimitNs) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    for (;;) {
        for (int i = 0; i < 64; i++)
            if (mbar_try_wait(bar, parity)) return true;
        if (global_ns() - t0 > limit_ns) break;
    }
    report_status(status, SCRS_ERR_DEVICE_TIMEOUT);
    return false;
}

// 1-D bulk copy global -> shared, completing on `bar` (both addresses 16-byte
// aligned, bytes a multiple of 16), into this CTA's shared memory only.
__device__ __forceinline__ void tma_load_1d(void* smem_dst, const void* gmem_src, uint32_t bytes,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(smem_dst)),
        "l"(gmem_src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

// 16-byte asynchronous global -> shared copy (no register staging), so a
// thread keeps many tile loads in flight; cp_async_wait_all() waits for this
// thread's copies.
__device__ __forceinline__ void cp_async_16(void* smem_dst, const void* gmem_src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(smem_dst)), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

}  // namespace scrs
