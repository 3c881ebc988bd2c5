// GF(256) batch decode that allocates nothing.
//
// The regular decode entry points keep their reconstruction recipe (row
// lists and the closed-form coefficient matrix the device planner writes) in
// memory allocated when the codec or its scratch is created.  Some callers
// cannot make that allocation at all: cudaMalloc may synchronise the whole
// device, which a packet-receive loop reconstructing stripes under a latency
// budget cannot afford, and a serving process that reserved its device
// memory pool at start-up has no headroom left for per-codec buffers.  This
// entry point serves them: the recipe lives in one file-scope device array
// of fixed size, so a call needs no cudaMalloc, cudaFree or other allocating
// routine; the caller supplies the received rows and the output.
//
// Limits and sharing:
//  - the array holds kStaticRecipeBytes; a decode whose recipe needs more
//    (2*(3k + 3r) bytes of row lists, rounded up to 16, plus k*r coefficient
//    bytes, r = erased data symbols) is rejected with SCRS_ERR_CAPACITY
//    (a = bytes needed, b = kStaticRecipeBytes) before any device work is
//    queued;
//  - every call, on every stream, writes the same array, and the array keeps
//    the last call's recipe: two calls whose device work overlaps (different
//    streams, no ordering between them) race on it and can return wrong data,
//    so order such calls on one stream or synchronise between them;
//  - no part of the array needs to start at zero: each call writes every row
//    list entry and coefficient its kernels read before they read it;
//  - the row lists travel to the device as a kernel argument (at most 768
//    uint16), so the call never waits on the host for a copy;
//  - the first call on each device does the one-time set-up there, with that
//    device current: it looks up the array's device address
//    (cudaGetSymbolAddress) and uploads the field tables and kernel limits the
//    decode kernels use, whatever the erasure count; make that first call
//    before any stream capture on that device;
//  - a bounded device wait that runs out (the kernels never hang) is reported
//    through the caller's optional device status word, not the return code,
//    since the call returns before the device work runs.
#include <mutex>

#include "runtime.h"

using namespace scrs;

namespace {

constexpr size_t kStaticRecipeBytes = 16 * 1024;
constexpr int kMaxDevices = 64;
// in_rows[k] pass_rows[k] out_rows[r] missing[r] repairs[r] present[k-r]
// with r <= m and k + m <= 256
constexpr uint32_t kMaxListWords = 3 * 256;

// The recipe scratch: row lists (uint16) followed by the coefficient matrix.
static __device__ __align__(256) uint8_t g_static_recipe[kStaticRecipeBytes];

struct StaticLists {
    uint16_t w[kMaxListWords];
};

// Writes a call's row lists (passed by value) to the front of the array.
__global__ void put_static_lists(StaticLists lists, uint32_t n_words) {
    uint16_t* dst = reinterpret_cast<uint16_t*>(g_static_recipe);
    for (uint32_t i = threadIdx.x; i < n_words; i += blockDim.x) dst[i] = lists.w[i];
}

uint8_t* g_recipe_addr[kMaxDevices] = {};
std::mutex g_recipe_mu;

// Device address of g_static_recipe on the current device.  The first call on
// a device also runs the decode kernels' one-time set-up there (field tables
// for the planner, shared-memory limits), so no later call synchronises.
cudaError_t static_recipe_address(uint8_t** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_recipe_mu);
    if (!g_recipe_addr[dev]) {
        e = prepare_batch_kernels();
        if (e != cudaSuccess) return e;
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_static_recipe);
        if (e != cudaSuccess) return e;
        g_recipe_addr[dev] = static_cast<uint8_t*>(p);
    }
    *out = g_recipe_addr[dev];
    return cudaSuccess;
}

}  // namespace

extern "C" int32_t scrs_gf256_decode_static(int32_t engine, uint64_t k, uint64_t m, uint64_t L,
                                            const uint64_t* indices, const uint8_t* d_rows, uint64_t count,
                                            uint8_t* d_out, uint64_t out_len, void* stream, int32_t* d_status,
                                            scrs_error* err) {
    if (engine != SCRS_ENGINE_STANDARD_CAUCHY && engine != SCRS_ENGINE_GOOD_CAUCHY)
        return set_err(err, SCRS_ERR_BAD_ARGUMENT, 1);
    // Geometry rules of Profile::resolve (selector.rs:46-58).
    if (k == 0 || m == 0) return set_err(err, SCRS_CONFIG_ZERO_DIMENSION);
    if (L == 0) return set_err(err, SCRS_CONFIG_ZERO_SYMBOL_LEN);
    const uint64_t cap = engine == SCRS_ENGINE_STANDARD_CAUCHY ? 256 : 255;
    if (k > cap || m > cap || k + m > cap) return set_err(err, SCRS_CONFIG_TOO_MANY_SYMBOLS, cap);
    // Then the BatchCodec::decode_into_with order (batch/codec.rs:292-331).
    if (out_len != k * L) return set_err(err, SCRS_DECODE_WRONG_OUTPUT_LEN, k * L, out_len);
    if (count != k) return set_err(err, SCRS_DECODE_WRONG_COUNT, k, count);
    if (!indices || !d_rows || !d_out) return set_err(err, SCRS_ERR_NULL_ARGUMENT);
    const uint64_t n = k + m;
    uint16_t row_of[256];
    for (uint64_t i = 0; i < n; i++) row_of[i] = kNoRow;
    for (uint64_t q = 0; q < count; q++) {
        const uint64_t i = indices[q];
        if (i >= n) return set_err(err, SCRS_DECODE_INDEX_OUT_OF_RANGE, i, n);
        if (row_of[i] != kNoRow) return set_err(err, SCRS_DECODE_DUPLICATE_INDEX, i);
        row_of[i] = (uint16_t)q;
    }
    uint16_t missing[256], present[256], repairs[256];
    uint32_t r = 0, p = 0, t = 0;
    for (uint64_t i = 0; i < k; i++) {
        if (row_of[i] == kNoRow)
            missing[r++] = (uint16_t)i;
        else
            present[p++] = (uint16_t)i;
    }
    for (uint64_t j = 0; j < m; j++)
        if (row_of[k + j] != kNoRow) repairs[t++] = (uint16_t)j;
    const size_t list_words = 3 * (size_t)k + 3 * (size_t)r;
    const size_t coef_off = (list_words * 2 + 15) & ~(size_t)15;
    const size_t need = coef_off + (size_t)k * (r ? r : 1);
    if (need > kStaticRecipeBytes) return set_err(err, SCRS_ERR_CAPACITY, need, kStaticRecipeBytes);
    StaticLists lists;
    uint16_t* in_rows = lists.w;
    uint16_t* pass_rows = lists.w + k;
    uint16_t* out_rows = lists.w + 2 * k;
    uint16_t* l_missing = out_rows + r;
    uint16_t* l_repairs = l_missing + r;
    uint16_t* l_present = l_repairs + r;
    for (uint32_t x = 0; x < r; x++) {
        in_rows[x] = row_of[k + repairs[x]];
        pass_rows[x] = kNoRow;
        out_rows[x] = l_missing[x] = missing[x];
        l_repairs[x] = repairs[x];
    }
    for (uint32_t z = 0; z < p; z++) {
        in_rows[r + z] = row_of[present[z]];
        pass_rows[r + z] = present[z];
        l_present[z] = present[z];
    }
    uint8_t* base = nullptr;
    SCRS_CUDA(static_recipe_address(&base));
    cudaStream_t st = (cudaStream_t)stream;
    put_static_lists<<<1, 256, 0, st>>>(lists, (uint32_t)list_words);
    SCRS_CUDA(cudaGetLastError());
    const uint16_t* d_lists = reinterpret_cast<const uint16_t*>(base);
    uint8_t* d_coef = base + coef_off;
    if (r) {
        CauchyPlanTask P{};
        P.r = r;
        P.p = p;
        P.ld = r;
        P.engine = (uint32_t)engine;
        P.k = (uint32_t)k;
        P.missing = d_lists + 2 * k + r;
        P.repairs = d_lists + 2 * k + 2 * r;
        P.present = d_lists + 2 * k + 3 * r;
        P.coef = d_coef;
        SCRS_CUDA(launch_cauchy_plan_single(P, 0, st));
    }
    MxkTask T{};
    T.in = d_rows;
    T.out = d_out;
    T.coef = d_coef;
    T.in_rows = d_lists;
    T.pass_rows = d_lists + k;
    T.out_rows = d_lists + 2 * k;
    T.L = L;
    T.in_stride = L;
    T.out_stride = L;
    T.n_in = (uint32_t)k;
    T.n_out = r;
    T.ld = r ? r : 1;
    T.n_items = n_chunks(L, false);
    T.aligned = (L % 16 == 0 && aligned16(d_rows) && aligned16(d_out)) ? 1u : 0u;
    SCRS_CUDA(launch_mxk_single(T, 0, d_status, 0, st));
    return set_err(err, SCRS_OK);
}
