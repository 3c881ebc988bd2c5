// Run-time specialised GF(256) encode drain (jit.cu, mxk_spec.cuh).
#pragma once

#include <stdint.h>

#include <string>

#include "../../include/scrs_gpu.h"
#include "kernels.cuh"

namespace scrs {

// Largest k * m specialised: the generated code grows with the number of
// products, and past this size its instruction footprint costs more than the
// jump-table kernel.
constexpr uint32_t kJitMaxProducts = 64;

struct JitKernel {
    const void* kernel = nullptr;  // cudaKernel_t, launchable with cudaLaunchKernel
    int smem = 0;
    int ctas_per_sm = 0;
    uint64_t cubin_bytes = 0;
};

// Whether an encode of k inputs and m outputs is specialised.
bool jit_eligible(uint32_t k, uint32_t m);
// The generated CUDA source for one matrix (for tests and inspection).
std::string jit_source(int32_t engine, uint32_t k, uint32_t m);
// Compile (once per process) and, with load_it, load the kernel for the
// current device.  SCRS_ERR_JIT (a = nvrtcResult) when NVRTC fails.
int32_t jit_kernel(int32_t engine, uint32_t k, uint32_t m, bool load_it, JitKernel* out, scrs_error* err);
// Persistent launch over items [item_lo, item_end) (counter zeroed before).
cudaError_t launch_jit(const JitKernel& jk, const MxkTask* tasks, const uint32_t* item_task, uint32_t item_lo,
                       uint32_t item_end, uint32_t* counter, int32_t* status, int grid, cudaStream_t stream);

}  // namespace scrs
