// Host runtime helpers shared by the engine implementations: status
// reporting, device/pinned buffers, per-handle streams.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <atomic>
#include <vector>

#include "../../include/scrs_gpu.h"
#include "kernels.cuh"

namespace scrs {

inline int32_t set_err(scrs_error* err, int32_t code, uint64_t a = 0, uint64_t b = 0) {
    if (err) {
        err->code = code;
        err->reserved = 0;
        err->a = a;
        err->b = b;
    }
    return code;
}

#define SCRS_CUDA(expr)                                                   \
    do {                                                                  \
        cudaError_t _e = (expr);                                          \
        if (_e != cudaSuccess) {                                          \
            if (_e == cudaErrorMemoryAllocation) cudaGetLastError();      \
            return set_err(err, SCRS_ERR_CUDA, (uint64_t)_e, __LINE__);   \
        }                                                                 \
    } while (0)

// Device and pinned-host allocations the library has made (cudaMalloc,
// cudaHostAlloc), for scrs_alloc_count: every allocation goes through the
// three helpers below.
inline std::atomic<uint64_t> g_alloc_calls{0};

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    cudaError_t ensure(size_t n) {
        if (n <= bytes && p) return cudaSuccess;
        release();
        if (n == 0) n = 16;
        g_alloc_calls.fetch_add(1, std::memory_order_relaxed);
        cudaError_t e = cudaMalloc(&p, n);
        if (e == cudaSuccess) bytes = n;
        else p = nullptr;
        return e;
    }
    // As ensure(), but a reallocation takes twice the current size when that
    // is larger, so a buffer that grows in small steps reallocates (and
    // synchronises the device in cudaFree) only a logarithmic number of times.
    cudaError_t ensure_grow(size_t n) {
        if (n <= bytes && p) return cudaSuccess;
        return ensure(n > 2 * bytes ? n : 2 * bytes);
    }
    template <class T>
    T* as() const { return reinterpret_cast<T*>(p); }
};

struct PinnedBuf {
    void* p = nullptr;
    size_t bytes = 0;
    PinnedBuf() = default;
    PinnedBuf(const PinnedBuf&) = delete;
    PinnedBuf& operator=(const PinnedBuf&) = delete;
    ~PinnedBuf() { release(); }
    void release() {
        if (p) cudaFreeHost(p);
        p = nullptr;
        bytes = 0;
    }
    cudaError_t ensure(size_t n) {
        if (n <= bytes && p) return cudaSuccess;
        release();
        if (n == 0) n = 16;
        g_alloc_calls.fetch_add(1, std::memory_order_relaxed);
        cudaError_t e = cudaHostAlloc(&p, n, cudaHostAllocDefault);
        if (e == cudaSuccess) bytes = n;
        else p = nullptr;
        return e;
    }
    template <class T>
    T* as() const { return reinterpret_cast<T*>(p); }
};

// Mapped host status word written by kernels on a device-side failure
// (for example a bounded wait that ran out).  Read after the stream syncs.
struct StatusWord {
    int32_t* host = nullptr;
    int32_t* dev = nullptr;
    cudaError_t init() {
        g_alloc_calls.fetch_add(1, std::memory_order_relaxed);
        cudaError_t e = cudaHostAlloc(reinterpret_cast<void**>(&host), 64, cudaHostAllocMapped);
        if (e != cudaSuccess) return e;
        *host = 0;
        return cudaHostGetDevicePointer(reinterpret_cast<void**>(&dev), host, 0);
    }
    ~StatusWord() {
        if (host) cudaFreeHost(host);
    }
};

// A stream owned by a handle, plus the device it was created on.
struct OwnedStream {
    cudaStream_t s = nullptr;
    int device = 0;
    int sm_count = 0;
    cudaError_t init() {
        cudaError_t e = cudaGetDevice(&device);
        if (e != cudaSuccess) return e;
        e = cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, device);
        if (e != cudaSuccess) return e;
        return cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    }
    ~OwnedStream() {
        if (s) cudaStreamDestroy(s);
    }
};

inline bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// Upload of set-up data from pageable host memory, complete on the device
// when this returns.  A plain cudaMemcpy from pageable memory may return once
// the bytes are staged, before the DMA has landed, and the kernels that read
// these buffers run on non-blocking streams that are not ordered after it.
inline cudaError_t upload_now(void* dst, const void* src, size_t bytes, cudaStream_t st = cudaStreamPerThread) {
    if (bytes == 0) return cudaSuccess;
    cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    return e;
}

inline uint32_t chunk_bytes(bool gf16) { return gf16 ? (uint32_t)FieldGeom<1>::kChunk : (uint32_t)FieldGeom<0>::kChunk; }

inline uint32_t n_chunks(uint64_t L, bool gf16) {
    uint64_t c = chunk_bytes(gf16);
    return (uint32_t)((L + c - 1) / c);
}

// Check the status word after a synchronised run.
inline int32_t take_status(StatusWord& st, scrs_error* err) {
    int32_t code = *st.host;
    if (code) {
        *st.host = 0;
        return set_err(err, code, 0, 0);
    }
    return SCRS_OK;
}

}  // namespace scrs
