// Run-time specialisation of the GF(256) encode drain to one coefficient
// matrix (mxk_spec.cuh): the XOR network of every coefficient is generated
// as straight-line CUDA, compiled for sm_100a by NVRTC and loaded as a
// library kernel.  Encode matrices are fixed per (engine, k, m), so a batch
// of such stripes reuses one compiled kernel; compiled kernels are cached
// for the life of the process.
#include "jit.h"

#include <dlfcn.h>
#include <nvrtc.h>

#include <algorithm>
#include <map>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>
#include <tuple>
#include <vector>

#include "host_field.h"
#include "jit_sources.inc"  // kJitHeaderNames / kJitHeaderTexts / kJitHeaderCount (build.py)
#include "mxk_device.cuh"
#include "runtime.h"

namespace scrs {
namespace {

// ---- the XOR network of one constant (same construction as gen_brx.py) -------
// rows[r] = the planes s with bit r of (c * x^s) set: acc[r] ^= XOR of them.
std::vector<std::vector<int>> rows_of(uint8_t c) {
    std::vector<std::vector<int>> rows(8);
    for (int s = 0; s < 8; s++) {
        const uint8_t col = hf::mul8(c, (uint8_t)(1u << s));
        for (int r = 0; r < 8; r++)
            if ((col >> r) & 1) rows[r].push_back(s);
    }
    return rows;
}

int xor_cost(const std::vector<std::vector<int>>& rows) {
    int n = 0;
    for (auto& r : rows) n += ((int)r.size() + 1) / 2;  // 3-input XORs into the accumulator
    return n;
}

// Greedy sharing: while some pair of operands occurs in two or more rows and
// XORing it once into a temporary lowers the count, take the pair with the
// largest gain (the first in (a, b) order among equals).  Temporaries are
// operands 8, 9, ...
std::vector<std::pair<int, int>> share_pairs(std::vector<std::vector<int>>& rows) {
    std::vector<std::pair<int, int>> pairs;
    for (;;) {
        std::map<std::pair<int, int>, int> count;
        for (auto& r : rows) {
            std::vector<int> s = r;
            std::sort(s.begin(), s.end());
            for (size_t i = 0; i < s.size(); i++)
                for (size_t j = i + 1; j < s.size(); j++) count[{s[i], s[j]}]++;
        }
        int best_gain = 0;
        std::pair<int, int> best{-1, -1};
        std::vector<std::vector<int>> best_rows;
        const int t = 8 + (int)pairs.size();
        for (auto& kv : count) {
            if (kv.second < 2) continue;
            const int a = kv.first.first, b = kv.first.second;
            std::vector<std::vector<int>> nr = rows;
            for (auto& r : nr) {
                const bool ha = std::find(r.begin(), r.end(), a) != r.end();
                const bool hb = std::find(r.begin(), r.end(), b) != r.end();
                if (ha && hb) {
                    r.erase(std::remove_if(r.begin(), r.end(), [&](int x) { return x == a || x == b; }), r.end());
                    r.push_back(t);
                }
            }
            const int gain = xor_cost(rows) - xor_cost(nr) - 1;
            if (gain > best_gain) {
                best_gain = gain;
                best = kv.first;
                best_rows = std::move(nr);
            }
        }
        if (best_gain <= 0) return pairs;
        pairs.push_back(best);
        rows = std::move(best_rows);
    }
}

// The products of one input's planes p with the constants of one output
// group: a0 ^= c0 * p and, when `two`, a1 ^= c1 * p.  The 16 rows of both
// networks share their common plane pairs: 7 % fewer XORs than sharing within
// each constant alone on the k = 10, m = 4 Cauchy matrices (the compiled
// kernel runs 0.6 % faster, the compiler already finding part of it).
void emit_networks(std::ostringstream& o, uint8_t c0, uint8_t c1, bool two, int& tmp) {
    auto rows = rows_of(c0);
    if (two) {
        const auto r1 = rows_of(c1);
        rows.insert(rows.end(), r1.begin(), r1.end());
    }
    const auto pairs = share_pairs(rows);
    std::vector<std::string> name(8 + pairs.size());
    for (int s = 0; s < 8; s++) name[s] = "p[" + std::to_string(s) + "]";
    for (size_t q = 0; q < pairs.size(); q++) {
        name[8 + q] = "t" + std::to_string(tmp++);
        o << "        const uint32_t " << name[8 + q] << " = " << name[pairs[q].first] << " ^ "
          << name[pairs[q].second] << ";\n";
    }
    for (size_t r = 0; r < rows.size(); r++) {
        if (rows[r].empty()) continue;
        o << "        " << (r < 8 ? "a0" : "a1") << "[" << (r % 8) << "] ^=";
        for (size_t i = 0; i < rows[r].size(); i++) o << (i ? " ^ " : " ") << name[rows[r][i]];
        o << ";\n";
    }
}

// ---- NVRTC, loaded on first use ----------------------------------------------------
// The library does not link NVRTC: without it, nothing is specialised and
// every stripe runs on the precompiled kernels.
struct Nvrtc {
    bool ok = false;
    nvrtcResult (*create)(nvrtcProgram*, const char*, const char*, int, const char* const*, const char* const*);
    nvrtcResult (*compile)(nvrtcProgram, int, const char* const*);
    nvrtcResult (*cubin_size)(nvrtcProgram, size_t*);
    nvrtcResult (*cubin)(nvrtcProgram, char*);
    nvrtcResult (*destroy)(nvrtcProgram*);
};

const Nvrtc& nvrtc() {
    static Nvrtc n = [] {
        Nvrtc r{};
        void* h = nullptr;
        for (const char* name : {"libnvrtc.so.12", "libnvrtc.so", "/usr/local/cuda/lib64/libnvrtc.so.12"})
            if ((h = dlopen(name, RTLD_NOW | RTLD_LOCAL))) break;
        if (!h) return r;
        r.create = reinterpret_cast<decltype(r.create)>(dlsym(h, "nvrtcCreateProgram"));
        r.compile = reinterpret_cast<decltype(r.compile)>(dlsym(h, "nvrtcCompileProgram"));
        r.cubin_size = reinterpret_cast<decltype(r.cubin_size)>(dlsym(h, "nvrtcGetCUBINSize"));
        r.cubin = reinterpret_cast<decltype(r.cubin)>(dlsym(h, "nvrtcGetCUBIN"));
        r.destroy = reinterpret_cast<decltype(r.destroy)>(dlsym(h, "nvrtcDestroyProgram"));
        r.ok = r.create && r.compile && r.cubin_size && r.cubin && r.destroy;
        return r;
    }();
    return n;
}

// ---- compiled kernels ------------------------------------------------------------
struct Compiled {
    int32_t status = SCRS_OK;  // SCRS_ERR_JIT when the compile failed (detail = nvrtcResult)
    uint64_t detail = 0;
    std::vector<char> cubin;
    cudaLibrary_t lib = nullptr;
    cudaKernel_t kernel = nullptr;
    std::atomic<uint64_t> attr_done{0};  // devices whose shared-memory limit is set
    int ctas_per_sm = 0;
};

using Key = std::tuple<int32_t, uint32_t, uint32_t>;
std::mutex g_mu;
std::map<Key, std::unique_ptr<Compiled>>& cache() {
    static std::map<Key, std::unique_ptr<Compiled>> c;
    return c;
}

void compile(Compiled& c, int32_t engine, uint32_t k, uint32_t m) {
    const Nvrtc& nv = nvrtc();
    if (!nv.ok) {  // no NVRTC in this process
        c.status = SCRS_ERR_JIT;
        c.detail = (uint64_t)NVRTC_ERROR_INTERNAL_ERROR;
        return;
    }
    const std::string src = jit_source(engine, k, m);
    nvrtcProgram prog = nullptr;
    nvrtcResult r = nv.create(&prog, src.c_str(), "scrs_spec.cu", kJitHeaderCount, kJitHeaderTexts, kJitHeaderNames);
    if (r == NVRTC_SUCCESS) {
        const char* opts[] = {"--gpu-architecture=sm_100a", "-std=c++17"};
        r = nv.compile(prog, 2, opts);
        size_t n = 0;
        if (r == NVRTC_SUCCESS) r = nv.cubin_size(prog, &n);
        if (r == NVRTC_SUCCESS) {
            c.cubin.resize(n);
            r = nv.cubin(prog, c.cubin.data());
        }
    }
    if (prog) nv.destroy(&prog);
    if (r != NVRTC_SUCCESS) {
        c.status = SCRS_ERR_JIT;
        c.detail = (uint64_t)r;
        c.cubin.clear();
    }
}

int32_t load(Compiled& c, scrs_error* err) {
    if (!c.lib) {
        SCRS_CUDA(cudaLibraryLoadData(&c.lib, c.cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0));
        SCRS_CUDA(cudaLibraryGetKernel(&c.kernel, c.lib, "scrs_spec_drain"));
    }
    return SCRS_OK;
}

}  // namespace

bool jit_eligible(uint32_t k, uint32_t m) {
    return k >= 1 && m >= 1 && k <= (uint32_t)FieldGeom<0>::kSegMax && k * m <= kJitMaxProducts;
}

std::string jit_source(int32_t engine, uint32_t k, uint32_t m) {
    std::vector<uint8_t> C((size_t)k * m);
    hf::gf8_coefficients(engine, k, m, C.data());
    const uint32_t groups = (m + 1) / 2;
    std::ostringstream o;
    o << "// generated: GF(256) engine " << engine << ", k = " << k << ", m = " << m << "\n";
    o << "#include <stdint.h>\nenum { SCRS_ERR_DEVICE_TIMEOUT = " << (int)SCRS_ERR_DEVICE_TIMEOUT << " };\n";
    o << "#include \"mxk_device.cuh\"\nnamespace scrs {\nnamespace spec {\n";
    o << "constexpr uint32_t kK = " << k << ", kM = " << m << ", kGroups = " << groups << ";\n";
    o << "__device__ __forceinline__ void group(uint32_t g, const uint8_t* half, uint32_t (&a0)[8], "
         "uint32_t (&a1)[8]) {\n    switch (g) {\n";
    for (uint32_t g = 0; g < groups; g++) {
        o << "    case " << g << ":\n";
        for (uint32_t i = 0; i < k; i++) {
            o << "    {\n        uint32_t p[8];\n";
            o << "        const uint8_t* src = half + " << i * (uint32_t)FieldGeom<0>::kChunk << ";\n";
            o << "        { const uint4 v = *reinterpret_cast<const uint4*>(src); "
                 "p[0] = v.x; p[1] = v.y; p[2] = v.z; p[3] = v.w; }\n";
            o << "        { const uint4 v = *reinterpret_cast<const uint4*>(src + 512); "
                 "p[4] = v.x; p[5] = v.y; p[6] = v.z; p[7] = v.w; }\n";
            int tmp = 0;
            const bool two = 2 * g + 1 < m;
            emit_networks(o, C[(size_t)i * m + 2 * g], two ? C[(size_t)i * m + 2 * g + 1] : 0, two, tmp);
            o << "    }\n";
        }
        o << "        break;\n";
    }
    o << "    }\n}\n}  // namespace spec\n}  // namespace scrs\n#include \"mxk_spec.cuh\"\n";
    return o.str();
}

int32_t jit_kernel(int32_t engine, uint32_t k, uint32_t m, bool load_it, JitKernel* out, scrs_error* err) {
    if (engine != SCRS_ENGINE_STANDARD_CAUCHY && engine != SCRS_ENGINE_GOOD_CAUCHY)
        return set_err(err, SCRS_ERR_BAD_ARGUMENT, 1, (uint64_t)engine);
    if (!jit_eligible(k, m)) return set_err(err, SCRS_ERR_BAD_ARGUMENT, 2, (uint64_t)k * m);
    std::lock_guard<std::mutex> lock(g_mu);
    auto& slot = cache()[Key(engine, k, m)];
    if (!slot) {
        slot.reset(new (std::nothrow) Compiled());
        if (!slot) return set_err(err, SCRS_ERR_OUT_OF_MEMORY, sizeof(Compiled));
        compile(*slot, engine, k, m);
    }
    Compiled& c = *slot;
    if (c.status) return set_err(err, c.status, c.detail);
    if (out) out->cubin_bytes = c.cubin.size();
    if (!load_it) return set_err(err, SCRS_OK);
    int32_t rc = load(c, err);
    if (rc) return rc;
    const int smem = (int)(kSmemHeader + (size_t)k * FieldGeom<0>::kChunk);
    const cudaError_t e = once_per_device(c.attr_done, [&] {
        cudaError_t r = cudaFuncSetAttribute((const void*)c.kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (r == cudaSuccess)
            r = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c.ctas_per_sm, (const void*)c.kernel, kThreads, smem);
        if (c.ctas_per_sm < 1) c.ctas_per_sm = 1;
        return r;
    });
    if (e != cudaSuccess) return set_err(err, SCRS_ERR_CUDA, (uint64_t)e, __LINE__);
    if (out) {
        out->kernel = (const void*)c.kernel;
        out->smem = smem;
        out->ctas_per_sm = c.ctas_per_sm;
    }
    return set_err(err, SCRS_OK);
}

cudaError_t launch_jit(const JitKernel& jk, const MxkTask* tasks, const uint32_t* item_task, uint32_t item_lo,
                       uint32_t item_end, uint32_t* counter, int32_t* status, int grid, cudaStream_t stream) {
    if (item_end <= item_lo) return cudaSuccess;
    if (grid <= 0 || grid > (int)(item_end - item_lo)) grid = (int)(item_end - item_lo);
    void* args[] = {(void*)&tasks, (void*)&item_task, (void*)&item_lo, (void*)&item_end, (void*)&counter,
                    (void*)&status};
    return cudaLaunchKernel(jk.kernel, dim3(grid), dim3(kThreads), args, (size_t)jk.smem, stream);
}

}  // namespace scrs

using namespace scrs;

extern "C" int32_t scrs_jit_prepare(int32_t engine, uint32_t k, uint32_t m, int32_t load, uint64_t* cubin_bytes,
                                    scrs_error* err) {
    JitKernel jk{};
    int32_t rc = jit_kernel(engine, k, m, load != 0, &jk, err);
    if (!rc && cubin_bytes) *cubin_bytes = jk.cubin_bytes;
    return rc;
}
