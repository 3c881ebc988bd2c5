// C ABI implementation of the SCRS trait surface on sm_100a
// (include/scrs_gpu.h).  Validation order follows the reference so error
// variants match; payload work runs in the multiply-XOR kernels
// (mxk_kernels.cu) and the additive-FFT kernels (afft_kernels.cu).
#include <stdlib.h>

#include <algorithm>
#include <memory>
#include <new>

#include "afft_engine.h"
#include "host_field.h"
#include "runtime.h"

using namespace scrs;

namespace {

bool is_gf16(int32_t engine) { return engine == SCRS_ENGINE_TOWER || engine == SCRS_ENGINE_AFFT; }

uint64_t engine_capacity(int32_t engine) {
    switch (engine) {
        case SCRS_ENGINE_STANDARD_CAUCHY: return 256;
        case SCRS_ENGINE_GOOD_CAUCHY: return 255;
        case SCRS_ENGINE_TOWER: return 65535;
        default: return 65536;
    }
}

// scrs/src/selector.rs:40-61
int32_t resolve(int32_t engine, uint64_t k, uint64_t m, uint64_t L, scrs_profile* out, scrs_error* err) {
    if (engine < 0 || engine > 3) return set_err(err, SCRS_ERR_BAD_ARGUMENT, 1, 0);
    if (k == 0 || m == 0) return set_err(err, SCRS_CONFIG_ZERO_DIMENSION);
    if (L == 0) return set_err(err, SCRS_CONFIG_ZERO_SYMBOL_LEN);
    if (is_gf16(engine) && (L % 2)) return set_err(err, SCRS_CONFIG_ODD_SYMBOL_LEN);
    uint64_t cap = engine_capacity(engine);
    if (k > cap || m > cap || k + m > cap) return set_err(err, SCRS_CONFIG_TOO_MANY_SYMBOLS, cap);
    if (out) *out = scrs_profile{engine, 0, k, m, L};
    return set_err(err, SCRS_OK);
}

int32_t check_profile(const scrs_profile* p, scrs_error* err) {
    if (!p) return set_err(err, SCRS_ERR_NULL_ARGUMENT);
    return resolve(p->engine, p->k, p->m, p->symbol_len, nullptr, err);
}

// Tower powers g^0..g^(n-1) on the device (x/y coordinates for the plan).
struct TowerTables {
    DevBuf powers;   // uint16[n]
    DevBuf coeffs;   // uint16[k*m] (encoders)
    std::vector<uint16_t> host_powers;
};

// Reduced-solve recipe buffers: lists for the plan kernel and the
// multiply-XOR task, plus the coefficient rows (received repairs first,
// then present data).  Coefficients are kept in a small device-resident LRU
// keyed by the erasure pattern (missing data indices + the repair columns
// used), as the reference's RecipeCache (decoder/cache.rs:15-100) keeps
// recipes: a repeated pattern skips the plan launch.  Every entry is sized
// for the largest erasure count (k * rmax elements, as the reference's
// decode scratch reserves k * max_r coefficients, tower/decoder.rs:53-78) in
// one arena allocated at scratch creation, with its key's capacity reserved,
// so a lookup never allocates, hit or miss (the zero-allocation contract of
// the *_with calls, tests/zero_alloc.rs:48-145).  Large codes get fewer
// entries: the arena holds at most kCacheArenaBytes or one entry.
struct RecipeBufs {
    struct Entry {
        std::vector<uint16_t> key;  // r, missing[r], repairs[r]
        void* coef = nullptr;       // elem[k * r] inside `arena`
        uint64_t last_use = 0;
        bool used = false;
    };
    static constexpr size_t kCacheEntries = 32;
    static constexpr size_t kCacheArenaBytes = 16u << 20;
    DevBuf lists;   // uint16: in_rows[k] pass_rows[k] out_rows[rmax] missing[rmax] repairs[rmax] present[k]
    DevBuf work;    // uint32[4*rmax] when rmax exceeds the shared-memory plan limit
    DevBuf arena;   // entries' coefficient buffers
    std::vector<uint16_t> host;  // same layout as `lists`
    std::vector<uint16_t> probe; // the key being looked up (capacity reserved at init)
    std::vector<Entry> cache;
    uint64_t clock = 0, hits = 0;
    uint32_t k = 0, rmax = 0, elem = 1;
    cudaError_t init(uint32_t k_, uint32_t rmax_, uint32_t elem_) {
        k = k_, rmax = rmax_, elem = elem_;
        host.assign((size_t)3 * k + 3 * rmax + 8, 0);
        probe.reserve(1 + 2 * (size_t)rmax);
        cudaError_t e = lists.ensure(host.size() * sizeof(uint16_t));
        if (e == cudaSuccess && rmax > kPlanSmemMaxR) e = work.ensure((size_t)4 * rmax * sizeof(uint32_t));
        if (e != cudaSuccess) return e;
        const size_t entry = ((size_t)k * std::max<uint32_t>(rmax, 1) * elem + 255) & ~(size_t)255;
        const size_t n = std::max<size_t>(1, std::min(kCacheEntries, kCacheArenaBytes / entry));
        e = arena.ensure(n * entry);
        if (e != cudaSuccess) return e;
        cache.resize(n);
        for (size_t i = 0; i < n; i++) {
            cache[i].key.reserve(1 + 2 * (size_t)rmax);
            cache[i].coef = arena.as<uint8_t>() + i * entry;
        }
        return cudaSuccess;
    }
    // Coefficient buffer for the pattern; *fresh says whether it must be
    // (re)computed.  A free entry is taken first, then the least recently
    // used one.  Reusing a buffer that a queued kernel may still read is
    // safe: its pattern's plan and multiply ran earlier on the same stream.
    cudaError_t lookup(const std::vector<uint16_t>& missing, const std::vector<uint16_t>& repairs, void** coef,
                       bool* fresh) {
        if (missing.size() > rmax || cache.empty()) return cudaErrorInvalidValue;
        std::vector<uint16_t>& key = probe;
        key.clear();
        key.push_back((uint16_t)missing.size());
        key.insert(key.end(), missing.begin(), missing.end());
        key.insert(key.end(), repairs.begin(), repairs.end());
        Entry* slot = nullptr;
        for (auto& e : cache) {
            if (e.used && e.key == key) {
                e.last_use = ++clock;
                hits++;
                *coef = e.coef;
                *fresh = false;
                return cudaSuccess;
            }
            if (!slot || (slot->used && (!e.used || e.last_use < slot->last_use))) slot = &e;
        }
        slot->key.assign(key.begin(), key.end());
        slot->used = true;
        slot->last_use = ++clock;
        *coef = slot->coef;
        *fresh = true;
        return cudaSuccess;
    }
    uint16_t* h_in() { return host.data(); }
    uint16_t* h_pass() { return host.data() + k; }
    uint16_t* h_out() { return host.data() + 2 * k; }
    uint16_t* h_missing() { return host.data() + 2 * k + rmax; }
    uint16_t* h_repairs() { return host.data() + 2 * k + 2 * rmax; }
    uint16_t* h_present() { return host.data() + 2 * k + 3 * rmax; }
    uint16_t* d(size_t off) const { return lists.as<uint16_t>() + off; }
};

// Build and run one reduced Cauchy reconstruction:
//   missing[r] data indices, repairs[r] repair columns, present[p] data indices;
//   source rows in `src` (row = codeword index via src_row()), output rows
//   in `out` (row = data index).
template <class SrcRow>
int32_t run_cauchy_recover(RecipeBufs& rb, int32_t engine, uint32_t k, const std::vector<uint16_t>& missing,
                           const std::vector<uint16_t>& repairs, const std::vector<uint16_t>& present,
                           SrcRow src_row, const uint8_t* src, uint64_t src_stride, uint8_t* out,
                           uint64_t L, const uint16_t* d_powers, int32_t* status, cudaStream_t s,
                           scrs_error* err) {
    const bool gf16 = is_gf16(engine);
    const uint32_t r = (uint32_t)missing.size(), p = (uint32_t)present.size();
    const uint32_t n_in = r + p;
    uint16_t* hin = rb.h_in();
    uint16_t* hpass = rb.h_pass();
    for (uint32_t t = 0; t < r; t++) {
        hin[t] = src_row(k + repairs[t]);
        hpass[t] = kNoRow;
    }
    for (uint32_t z = 0; z < p; z++) {
        hin[r + z] = src_row(present[z]);
        hpass[r + z] = present[z];
    }
    std::copy(missing.begin(), missing.end(), rb.h_out());
    std::copy(missing.begin(), missing.end(), rb.h_missing());
    std::copy(repairs.begin(), repairs.end(), rb.h_repairs());
    std::copy(present.begin(), present.end(), rb.h_present());
    SCRS_CUDA(cudaMemcpyAsync(rb.lists.p, rb.host.data(), rb.host.size() * sizeof(uint16_t),
                              cudaMemcpyHostToDevice, s));
    const uint32_t K = rb.k, R = rb.rmax;
    void* coef = nullptr;
    bool fresh = true;
    if (r) SCRS_CUDA(rb.lookup(missing, repairs, &coef, &fresh));
    if (r && fresh) {
        CauchyPlanTask P{};
        P.r = r;
        P.p = p;
        P.ld = r;
        P.engine = (uint32_t)engine;
        P.k = k;
        P.missing = rb.d(2 * K + R);
        P.repairs = rb.d(2 * K + 2 * R);
        P.present = rb.d(2 * K + 3 * R);
        P.powers = d_powers;
        P.coef = coef;
        P.work = r > kPlanSmemMaxR ? rb.work.as<uint32_t>() : nullptr;
        SCRS_CUDA(launch_cauchy_plan_single(P, gf16 ? 1 : 0, s));
    }
    MxkTask T{};
    T.in = src;
    T.out = out;
    T.coef = coef;
    T.in_rows = rb.d(0);
    T.out_rows = rb.d(2 * K);
    T.pass_rows = rb.d(K);
    T.L = L;
    T.in_stride = src_stride;
    T.out_stride = L;
    T.n_in = n_in;
    T.n_out = r;
    T.ld = std::max<uint32_t>(r, 1);
    T.n_items = n_chunks(L, gf16);
    T.aligned = (L % 16 == 0 && aligned16(src) && aligned16(out) && src_stride % 16 == 0) ? 1u : 0u;
    SCRS_CUDA(launch_mxk_single(T, gf16 ? 1 : 0, status, 0, s));
    return SCRS_OK;
}

}  // namespace

// ===========================================================================
// library
// ===========================================================================
extern "C" uint32_t scrs_abi_version(void) { return 0x00010000u; }

extern "C" uint64_t scrs_alloc_count(void) { return g_alloc_calls.load(std::memory_order_relaxed); }

extern "C" const char* scrs_status_name(int32_t code) {
    switch (code) {
        case SCRS_OK: return "Ok";
        case SCRS_CONFIG_ZERO_DIMENSION: return "ConfigError::ZeroDimension";
        case SCRS_CONFIG_TOO_MANY_SYMBOLS: return "ConfigError::TooManySymbols";
        case SCRS_CONFIG_ZERO_SYMBOL_LEN: return "ConfigError::ZeroSymbolLen";
        case SCRS_CONFIG_ODD_SYMBOL_LEN: return "ConfigError::OddSymbolLen";
        case SCRS_CONFIG_UNSUPPORTED_MODE: return "ConfigError::UnsupportedMode";
        case SCRS_ENCODE_WRONG_INPUT_LEN: return "EncodeError::WrongInputLen";
        case SCRS_ENCODE_INDEX_OUT_OF_RANGE: return "EncodeError::IndexOutOfRange";
        case SCRS_ENCODE_WRONG_PAYLOAD_LEN: return "EncodeError::WrongPayloadLen";
        case SCRS_ENCODE_DUPLICATE_DATA: return "EncodeError::DuplicateData";
        case SCRS_ENCODE_WRONG_OUTPUT_LEN: return "EncodeError::WrongOutputLen";
        case SCRS_ENCODE_SCRATCH_MISMATCH: return "EncodeError::ScratchMismatch";
        case SCRS_DECODE_WRONG_COUNT: return "DecodeError::WrongCount";
        case SCRS_DECODE_INDEX_OUT_OF_RANGE: return "DecodeError::IndexOutOfRange";
        case SCRS_DECODE_DUPLICATE_INDEX: return "DecodeError::DuplicateIndex";
        case SCRS_DECODE_WRONG_PAYLOAD_LEN: return "DecodeError::WrongPayloadLen";
        case SCRS_DECODE_TOO_MANY_SYMBOLS: return "DecodeError::TooManySymbols";
        case SCRS_DECODE_INSUFFICIENT_RANK: return "DecodeError::InsufficientRank";
        case SCRS_DECODE_WRONG_OUTPUT_LEN: return "DecodeError::WrongOutputLen";
        case SCRS_DECODE_SCRATCH_MISMATCH: return "DecodeError::ScratchMismatch";
        case SCRS_ERR_NULL_ARGUMENT: return "NullArgument";
        case SCRS_ERR_CUDA: return "Cuda";
        case SCRS_ERR_OUT_OF_MEMORY: return "OutOfMemory";
        case SCRS_ERR_NO_DEVICE: return "NoDevice";
        case SCRS_ERR_CAPACITY: return "Capacity";
        case SCRS_ERR_DEVICE_TIMEOUT: return "DeviceTimeout";
        case SCRS_ERR_BAD_ARGUMENT: return "BadArgument";
        case SCRS_ERR_JIT: return "Jit";
        default: return "Unknown";
    }
}

extern "C" int32_t scrs_profile_resolve(int32_t engine, uint64_t k, uint64_t m, uint64_t L, scrs_profile* out,
                                        scrs_error* err) {
    return resolve(engine, k, m, L, out, err);
}

extern "C" int32_t scrs_recommended_gf16_engine(uint64_t k, uint64_t m) {
    // lib.rs:85-93: large blocks (k+m > 256) or m >= k/3 pick the additive FFT.
    bool large = (k + m < k) || (k + m > 256);
    bool high = (m > UINT64_MAX / 3) || (m * 3 >= k);
    return (large || high) ? SCRS_ENGINE_AFFT : SCRS_ENGINE_TOWER;
}

extern "C" int32_t scrs_profile_recommended(int32_t field, uint64_t k, uint64_t m, uint64_t L,
                                            scrs_profile* out, scrs_error* err) {
    int32_t engine;
    if (field == SCRS_FIELD_GF256)  // selector.rs:73-80
        engine = (k + m <= 255) ? SCRS_ENGINE_GOOD_CAUCHY : SCRS_ENGINE_STANDARD_CAUCHY;
    else if (field == SCRS_FIELD_GF65536)
        engine = scrs_recommended_gf16_engine(k, m);
    else
        return set_err(err, SCRS_ERR_BAD_ARGUMENT, 1, 0);
    return resolve(engine, k, m, L, out, err);
}

// ===========================================================================
// BatchEncoder (selector.rs:435-529)
// ===========================================================================
struct scrs_batch_encoder {
    scrs_profile p{};
    OwnedStream stream;
    StatusWord status;
    DevBuf coef;  // GF(256): uint8[k*m]
    std::unique_ptr<AfftCodec> afft;
};

struct scrs_encode_scratch {
    int kind = 0;  // engine of the encoder that made it
    scrs_profile p{};
    DevBuf d_in, d_out;
    PinnedBuf h_in, h_out;
    std::unique_ptr<AfftWorkspace> afft;
};

extern "C" int32_t scrs_batch_encoder_create(const scrs_profile* p, scrs_batch_encoder** out, scrs_error* err) {
    int32_t st = check_profile(p, err);
    if (st) return st;
    if (!out) return set_err(err, SCRS_ERR_NULL_ARGUMENT);
    if (p->engine == SCRS_ENGINE_TOWER) return set_err(err, SCRS_CONFIG_UNSUPPORTED_MODE, (uint64_t)p->engine);
    std::unique_ptr<scrs_batch_encoder> e(new (std::nothrow) scrs_batch_encoder());
    if (!e) return set_err(err, SCRS_ERR_OUT_OF_MEMORY, sizeof(scrs_batch_encoder));
    e->p = *p;
    SCRS_CUDA(e->stream.init());
    SCRS_CUDA(e->status.init());
    if (p->engine == SCRS_ENGINE_AFFT) {
        e->afft.reset(new (std::nothrow) AfftCodec());
        if (!e->afft) return set_err(err, SCRS_ERR_OUT_OF_MEMORY, sizeof(AfftCodec));
        st = e->afft->init(p->k, p->m, p->symbol_len, err);
        if (st) return st;
    } else {
        std::vector<uint8_t> c((size_t)p->k * p->m);
        hf::gf8_coefficients(p->engine, (uint32_t)p->k, (uint32_t)p->m, c.data());
        SCRS_CUDA(e->coef.ensure(c.size()));
        SCRS_CUDA(upload_now(e->coef.p, c.data(), c.size(), e->stream.s));
    }
    *out = e.release();
    return set_err(err, SCRS_OK);
}

extern "C" void scrs_batch_encoder_destroy(scrs_batch_encoder* e) { delete e; }

extern "C" int32_t scrs_batch_encoder_profile(const scrs_batch_encoder* e, scrs_profile* out) {
    if (!e || !out) return SCRS_ERR_NULL_ARGUMENT;
    *out = e->p;
    return SCRS_OK;
}

extern "C" int32_t scrs_batch_encoder_scratch(const scrs_batch_encoder* e, scrs_encode_scratch** out,
                                              scrs_error* err) {
    if (!e || !out) return set_err(err, SCRS_ERR_NULL_ARGUMENT);
    std::unique_ptr<scrs_encode_scratch> s(new (std::nothrow) scrs_encode_scratch());
    if (!s) return set_err(err, SCRS_ERR_OUT_OF_MEMORY, sizeof(scrs_encode_scratch));
    s->kind = e->p.engine;
    s->p = e->p;
    const uint64_t k = e->p.k, m = e->p.m, L = e->p.symbol_len;
    SCRS_CUDA(s->d_in.ensure(k * L));
    SCRS_CUDA(s->d_out.ensure(m * L));
    SCRS_CUDA(s->h_in.ensure(k * L));
    SCRS_CUDA(s->h_out.ensure(m * L));
    if (e->afft) {
        s->afft.reset(new (std::nothrow) AfftWorkspace());
        if (!s->afft) return set_err(err, SCRS_ERR_OUT_OF_MEMORY, sizeof(AfftWorkspace));
        int32_t st = s->afft->init_encode(*e->afft, err);
        if (st) return st;
    }
    *out = s.release();
    return set_err(err, SCRS_OK);
}

extern "C" void scrs_encode_scratch_destroy(scrs_encode_scratch* s) { delete s; }

namespace {

bool encode_scratch_matches(const scrs_batch_encoder* e, const scrs_encode_scratch* s) {
    // selector.rs:516-527: GF(256) encoders take the unit scratch, AFFT its own.
    bool e_afft = e->p.engine == SCRS_ENGINE_AFFT, s_afft = s->kind == SCRS_ENGINE_AFFT;
    if (e_afft != s_afft) return false;
    // Device staging is sized per geometry.
    return s->p.k == e->p.k && s->p.m == e->p.m && s->p.symbol_len == e->p.symbol_len;
}

int32_t encode_device(const scrs_batch_encoder* e, const uint8_t* d_data, uint8_t* d_rep, scrs_encode_scratch* s,
                      cudaStream_t st, scrs_error* err) {
    const uint64_t k = e->p.k, m = e->p.m, L = e->p.symbol_len;
    if (e->afft) return e->afft->encode(d_data, d_rep, *s->afft, e->status.dev, st, err);
    MxkTask T{};
    T.in = d_data;
    T.out = d_rep;
    T.coef = e->coef.p;
    T.L = L;
    T.in_stride = L;
    T.out_stride = L;
    T.n_in = (uint32_t)k;
    T.n_out = (uint32_t)m;
    T.ld = (uint32_t)m;
    T.n_items = n_chunks(L, false);
    T.aligned = (L % 16 == 0 && aligned16(d_data) && aligned16(d_rep)) ? 1u : 0u;
    SCRS_CUDA(launch_mxk_single(T, 0, e->status.dev, 0, st));
    return SCRS_OK;
}

int32_t encode_host(const scrs_batch_encoder* e, const uint8_t* data, uint64_t dl, uint8_t* rep, uint64_t rl,
                    scrs_encode_scratch* s, scrs_error* err) {
    const uint64_t k = e->p.k, m = e->p.m, L = e->p.symbol_len;
    // batch/codec.rs:157-170, afft/encoder.rs:256-269
    if (dl != k * L) return set_err(err, SCRS_ENCODE_WRONG_INPUT_LEN, k * L, dl);
    if (rl != m * L) return set_err(err, SCRS_ENCODE_WRONG_OUTPUT_LEN, m * L, rl);
    if (!data || !rep) return set_err(err, SCRS_ERR_NULL_ARGUMENT);
    cudaStream_t st = e->stream.s;
    SCRS_CUDA(cudaMemcpyAsync(s->d_in.p, data, k * L, cudaMemcpyHostToDevice, st));
    int32_t r = encode_device(e, s->d_in.as<uint8_t>(), s->d_out.as<uint8_t>(), s, st, err);
    if (r) return r;
    SCRS_CUDA(cudaMemcpyAsync(rep, s->d_out.p, m * L, cudaMemcpyDeviceToHost, st));
    SCRS_CUDA(cudaStreamSynchronize(st));
    r = take_status(const_cast<scrs_batch_encoder*>(e)->status, err);
    if (r) return r;
    return set_err(err, SCRS_OK);
}

}  // namespace

extern "C" int32_t scrs_batch_encode_into_with(const scrs_batch_encoder* e, const uint8_t* data, uint64_t dl,
                                               uint8_t* rep, uint64_t rl, scrs_encode_scratch* s,
                                               scrs_error* err) {
    if (!e || !s) return set_err(err, SCRS_ERR_NULL_ARGUMENT);
    if (!encode_scratch_matches(e, s)) return set_err(err, SCRS_ENCODE_SCRATCH_MISMATCH);
    return encode_host(e, data, dl, rep, rl, s, err);
}

extern "C" int32_t scrs_batch_encode_into(const scrs_batch_encoder* e, const uint8_t* data, uint64_t dl,
                                          uint8_t* rep, uint64_t rl, scrs_error* err) {
    if (!e) return set_err(err, SCRS_ERR_NULL_ARGUMENT);
    const uint64_t k = e->p.k, m = e->p.m, L = e->p.symbol_len;
    if (dl != k * L) return set_err(err, SCRS_ENCODE_WRONG_INPUT_LEN, k * L, dl);
    if (rl != m * L) return set_err(err, SCRS_ENCODE_WRONG_OUTPUT_LEN, m * L, rl);
    scrs_encode_scratch* s = nullptr;
    int32_t st = scrs_batch_encoder_scratch(e, &s, err);
    if (st) return st;
    st = encode_host(e, data, dl, rep, rl, s, err);
    delete s;
    return st;
}

extern "C" int32_t scrs_batch_encode_into_with_device(const scrs_batch_encoder* e, const uint8_t* d_data,
                                                      uint64_t dl, uint8_t* d_rep, uint64_t rl,
                                                      scrs_encode_scratch* s, void* stream, scrs_error* err) {
    if (!e || !s) return set_err(err, SCRS_ERR_NULL_ARGUMENT);
    if (!encode_scratch_matches(e, s)) return set_err(err, SCRS_ENCODE_SCRATCH_MISMATCH);
    const uint64_t k = e->p.k, m = e->p.m, L = e->p.symbol_len;
    if (dl != k * L) return set_err(err, SCRS_ENCODE_WRONG_INPUT_LEN, k * L, dl);
    if (rl != m * L) return set_err(err, SCRS_ENCODE_WRONG_OUTPUT_LEN, m * L, rl);
    if (!d_data || !d_rep) return set_err(err, SCRS_ERR_NULL_ARGUMENT);
    int32_t r = encode_device(e, d_data, d_rep, s, (cudaStream_t)stream, err);
    if (r) return r;
    return set_err(err, SCRS_OK);
}

// ===========================================================================
// Decoder (lazy, every engine): decoder/streaming.rs, tower/decoder.rs,
// afft/decoder.rs.  push records the receipt and copies the payload (to
// pinned host staging for host payloads, device-to-device for device
// payloads); all payload arithmetic happens in finalize.
// ===========================================================================
struct scrs_decoder {
    scrs_profile p{};
    OwnedStream stream;
    StatusWord status;
    DevBuf payloads;       // n * L on the device
    PinnedBuf staging;     // n * L host staging for host pushes
    std::vector<uint8_t> have;      // receipt bitmap
    std::vector<uint8_t> on_host;   // payload row still in host staging
    uint64_t distinct = 0, received = 0;
    TowerTables tower;
    std::unique_ptr<AfftCodec> afft;
    // Stream order around the payload buffer.  Device pushes copy on the
    // caller's stream, chained on one stream at a time (push_stream; `pushed`
    // is recorded there when the chain moves or a finalize starts); a
    // finalize records `consumed` on its stream after the work that reads the
    // payloads, and the next writer of a payload row waits on it; host-staged
    // rows go up on the decoder's own stream (`uploaded`).
    cudaEvent_t uploaded = nullptr, pushed = nullptr, consumed = nullptr;
    cudaStream_t push_stream = nullptr, consumed_waited = nullptr;
    bool push_pending = false, consumed_pending = false, upload_inflight = false;
    ~scrs_decoder() {
        if (uploaded) cudaEventDestroy(uploaded);
        if (pushed) cudaEventDestroy(pushed);
        if (consumed) cudaEventDestroy(consumed);
    }
};

struct scrs_decode_scratch {
    int kind = 0;
    scrs_profile p{};
    RecipeBufs recipe;
    DevBuf d_out;  // k * L: host finalize lands here before the copy back
    std::unique_ptr<AfftWorkspace> afft;
    // per-call index lists, capacity reserved at creation (no allocation per call)
    std::vector<uint16_t> missing, present, repairs;
};

extern "C" int32_t scrs_decoder_create(const scrs_profile* p, scrs_decoder** out, scrs_error* err) {
    int32_t st = check_profile(p, err);
    if (st) return st;
    if (!out) return set_err(err, SCRS_ERR_NULL_ARGUMENT);
    std::unique_ptr<scrs_decoder> d(new (std::nothrow) scrs_decoder());
    if (!d) return set_err(err, SCRS_ERR_OUT_OF_MEMORY, sizeof(scrs_decoder));
    d->p = *p;
    const uint64_t n = p->k + p->m, L = p->symbol_len;
    SCRS_CUDA(d->stream.init());
    SCRS_CUDA(d->status.init());
    SCRS_CUDA(cudaEventCreateWithFlags(&d->uploaded, cudaEventDisableTiming));
    SCRS_CUDA(cudaEventCreateWithFlags(&d->pushed, cudaEventDisableTiming));
    SCRS_CUDA(cudaEventCreateWithFlags(&d->consumed, cudaEventDisableTiming));
    SCRS_CUDA(d->payloads.ensure(n * L));
    SCRS_CUDA(d->staging.ensure(n * L));
    d->have.assign(n, 0);
    d->on_host.assign(n, 0);
    if (p->engine == SCRS_ENGINE_TOWER) {
        d->tower.host_powers.resize(n);
        hf::tower_powers((uint32_t)n, d->tower.host_powers.data());
        SCRS_CUDA(d->tower.powers.ensure(n * 2));
        SCRS_CUDA(upload_now(d->tower.powers.p, d->tower.host_powers.data(), n * 2, d->stream.s));
    }
    if (p->engine == SCRS_ENGINE_AFFT) {
        d->afft.reset(new (std::nothrow) AfftCodec());
        if (!d->afft) return set_err(err, SCRS_ERR_OUT_OF_MEMORY, sizeof(AfftCodec));
        st = d->afft->init(p->k, p->m, p->symbol_len, err);
        if (st) return st;
    }
    *out = d.release();
    return set_err(err, SCRS_OK);
}

extern "C" void scrs_decoder_destroy(scrs_decoder* d) { delete d; }

extern "C" int32_t scrs_decoder_profile(const scrs_decoder* d, scrs_profile* out) {
    if (!d || !out) return SCRS_ERR_NULL_ARGUMENT;
    *out = d->p;
    return SCRS_OK;
}

extern "C" int32_t scrs_decoder_scratch(const scrs_decoder* d, scrs_decode_scratch** out, scrs_error* err) {
    if (!d || !out) return set_err(err, SCRS_ERR_NULL_ARGUMENT);
    std::unique_ptr<scrs_decode_scratch> s(new (std::nothrow) scrs_decode_scratch());
    if (!s) return set_err(err, SCRS_ERR_OUT_OF_MEMORY, sizeof(scrs_decode_scratch));
    s->kind = d->p.engine;
    s->p = d->p;
    const uint32_t k = (uint32_t)d->p.k, m = (uint32_t)d->p.m;
    s->missing.reserve(k);
    s->present.reserve(k);
    s->repairs.reserve(m);
    if (d->afft) {
        s->afft.reset(new (std::nothrow) AfftWorkspace());
        if (!s->afft) return set_err(err, SCRS_ERR_OUT_OF_MEMORY, sizeof(AfftWorkspace));
        int32_t st = s->afft->init_decode(*d->afft, err);
        if (st) return st;
    } else {
        SCRS_CUDA(s->recipe.init(k, std::min(k, m), is_gf16(d->p.engine) ? 2 : 1));
    }
    SCRS_CUDA(s->d_out.ensure((uint64_t)k * d->p.symbol_len));
    *out = s.release();
    return set_err(err, SCRS_OK);
}

extern "C" void scrs_decode_scratch_destroy(scrs_decode_scratch* s) { delete s; }

namespace {

// symbol_sink.rs:36-54 with the checks of decoder/streaming.rs:388-429.
int32_t push_common(scrs_decoder* d, uint64_t idx, const uint8_t* payload, uint64_t len, bool device,
                    cudaStream_t cs, scrs_push_outcome* outcome, scrs_error* err) {
    if (!d) return set_err(err, SCRS_ERR_NULL_ARGUMENT);
    const uint64_t n = d->p.k + d->p.m, L = d->p.symbol_len;
    if (idx >= n) return set_err(err, SCRS_DECODE_INDEX_OUT_OF_RANGE, idx, n);
    if (len != L) return set_err(err, SCRS_DECODE_WRONG_PAYLOAD_LEN, L, len);
    if (d->received >= n) return set_err(err, SCRS_DECODE_TOO_MANY_SYMBOLS, n, d->received);
    if (!payload) return set_err(err, SCRS_ERR_NULL_ARGUMENT);
    d->received++;
    scrs_push_outcome o{};
    if (d->distinct >= d->p.k || d->have[idx]) {
        o.kind = SCRS_PUSH_DEPENDENT;
    } else {
        if (device) {
            // after the last finalize's reads of the payload rows
            if (d->consumed_pending && d->consumed_waited != cs) {
                SCRS_CUDA(cudaStreamWaitEvent(cs, d->consumed, 0));
                d->consumed_waited = cs;
            }
            // the copies are chained on one stream at a time: moving to
            // another, it waits for the earlier stream's copies (so a row
            // pushed again after a reset lands last)
            if (d->push_pending && d->push_stream != cs) {
                SCRS_CUDA(cudaEventRecord(d->pushed, d->push_stream));
                SCRS_CUDA(cudaStreamWaitEvent(cs, d->pushed, 0));
            }
            SCRS_CUDA(cudaMemcpyAsync(d->payloads.as<uint8_t>() + idx * L, payload, L, cudaMemcpyDeviceToDevice, cs));
            d->push_stream = cs;
            d->push_pending = true;
            d->on_host[idx] = 0;
        } else {
            if (d->upload_inflight) {  // the staging rows of an earlier finalize may still be going up
                SCRS_CUDA(cudaStreamSynchronize(d->stream.s));
                d->upload_inflight = false;
            }
            memcpy(d->staging.as<uint8_t>() + idx * L, payload, L);
            d->on_host[idx] = 1;
        }
        d->have[idx] = 1;
        d->distinct++;
        if (d->distinct >= d->p.k) {
            o.kind = SCRS_PUSH_COMPLETE;
        } else {
            o.kind = SCRS_PUSH_ADVANCED;
            o.rank = d->distinct;
            o.received = d->received;
        }
    }
    if (outcome) *outcome = o;
    return set_err(err, SCRS_OK);
}

// Upload host-staged payload rows in contiguous runs.
int32_t upload_staged(scrs_decoder* d, scrs_error* err) {
    const uint64_t n = d->p.k + d->p.m, L = d->p.symbol_len;
    bool waited = false;
    uint64_t i = 0;
    while (i < n) {
        if (!(d->have[i] && d->on_host[i])) {
            i++;
            continue;
        }
        uint64_t j = i;
        while (j < n && d->have[j] && d->on_host[j]) j++;
        if (!waited && d->consumed_pending && d->consumed_waited != d->stream.s) {
            SCRS_CUDA(cudaStreamWaitEvent(d->stream.s, d->consumed, 0));  // after the last finalize's reads
            waited = true;
        }
        SCRS_CUDA(cudaMemcpyAsync(d->payloads.as<uint8_t>() + i * L, d->staging.as<uint8_t>() + i * L, (j - i) * L,
                                  cudaMemcpyHostToDevice, d->stream.s));
        for (uint64_t t = i; t < j; t++) d->on_host[t] = 0;
        d->upload_inflight = true;
        i = j;
    }
    return SCRS_OK;
}

int32_t finalize_enqueue(scrs_decoder* d, uint8_t* d_out, scrs_decode_scratch* s, cudaStream_t st,
                         scrs_error* err);

int32_t finalize_device(scrs_decoder* d, uint8_t* d_out, scrs_decode_scratch* s, cudaStream_t st,
                        scrs_error* err) {
    int32_t r = upload_staged(d, err);
    if (r) return r;
    if (st != d->stream.s) {  // order the payload uploads before the caller's stream
        SCRS_CUDA(cudaEventRecord(d->uploaded, d->stream.s));
        SCRS_CUDA(cudaStreamWaitEvent(st, d->uploaded, 0));
    }
    if (d->push_pending) {  // and the device pushes' copies
        if (d->push_stream != st) {
            SCRS_CUDA(cudaEventRecord(d->pushed, d->push_stream));
            SCRS_CUDA(cudaStreamWaitEvent(st, d->pushed, 0));
        }
        d->push_pending = false;
    }
    // an earlier finalize's reads on another stream: keep `consumed` covering them
    if (d->consumed_pending && d->consumed_waited != st) SCRS_CUDA(cudaStreamWaitEvent(st, d->consumed, 0));
    r = finalize_enqueue(d, d_out, s, st, err);
    if (r) return r;
    SCRS_CUDA(cudaEventRecord(d->consumed, st));  // the next writer of a payload row waits on this
    d->consumed_pending = true;
    d->consumed_waited = st;
    return SCRS_OK;
}

// The decode itself, enqueued on st once the payload rows are in place.
int32_t finalize_enqueue(scrs_decoder* d, uint8_t* d_out, scrs_decode_scratch* s, cudaStream_t st,
                         scrs_error* err) {
    const uint32_t k = (uint32_t)d->p.k, m = (uint32_t)d->p.m;
    const uint64_t L = d->p.symbol_len;
    if (d->afft) return d->afft->decode(d->payloads.as<uint8_t>(), d->have.data(), d_out, *s->afft,
                                        d->status.dev, st, err);
    // build_recipe (decoder/streaming.rs:163-194, tower/decoder.rs:218-247)
    std::vector<uint16_t>&missing = s->missing, &present = s->present, &repairs = s->repairs;
    missing.clear();
    present.clear();
    repairs.clear();
    for (uint32_t i = 0; i < k; i++) (d->have[i] ? present : missing).push_back((uint16_t)i);
    for (uint32_t j = 0; j < m && repairs.size() < missing.size(); j++)
        if (d->have[k + j]) repairs.push_back((uint16_t)j);
    if (repairs.size() != missing.size())
        return set_err(err, SCRS_DECODE_INSUFFICIENT_RANK, d->distinct, k);
    return run_cauchy_recover(
        s->recipe, d->p.engine, k, missing, repairs, present, [](uint32_t row) { return (uint16_t)row; },
        d->payloads.as<uint8_t>(), L, d_out, L, d->tower.powers.as<uint16_t>(), d->status.dev, st, err);
}

int32_t finalize_checks(scrs_decoder* d, uint64_t out_len, scrs_decode_scratch* s, scrs_error* err) {
    const uint64_t k = d->p.k, L = d->p.symbol_len;
    // ensure_complete, then output length (streaming.rs:495-502, tower/decoder.rs:205-212,
    // afft/decoder.rs:560-567), then scratch (selector.rs:239, tower/decoder.rs:219,
    // afft/decoder.rs:244).
    if (d->distinct < k) return set_err(err, SCRS_DECODE_INSUFFICIENT_RANK, d->distinct, k);
    if (out_len != k * L) return set_err(err, SCRS_DECODE_WRONG_OUTPUT_LEN, k * L, out_len);
    if (s) {
        bool s_cauchy = !is_gf16(s->kind), d_cauchy = !is_gf16(d->p.engine);
        if (s_cauchy != d_cauchy || (!d_cauchy && s->kind != d->p.engine))
            return set_err(err, SCRS_DECODE_SCRATCH_MISMATCH);
        if (s->p.k != d->p.k || s->p.m != d->p.m || s->p.symbol_len != d->p.symbol_len)
            return set_err(err, SCRS_DECODE_SCRATCH_MISMATCH);
    }
    return SCRS_OK;
}

int32_t finalize_host(scrs_decoder* d, uint8_t* out, uint64_t out_len, scrs_decode_scratch* s, scrs_error* err) {
    int32_t r = finalize_checks(d, out_len, s, err);
    if (r) return r;
    if (!out) return set_err(err, SCRS_ERR_NULL_ARGUMENT);
    uint8_t* d_out = s->d_out.as<uint8_t>();
    r = finalize_device(d, d_out, s, d->stream.s, err);
    if (r) return r;
    SCRS_CUDA(cudaMemcpyAsync(out, d_out, out_len, cudaMemcpyDeviceToHost, d->stream.s));
    SCRS_CUDA(cudaStreamSynchronize(d->stream.s));
    d->consumed_pending = d->upload_inflight = false;
    r = take_status(d->status, err);
    if (r) return r;
    return set_err(err, SCRS_OK);
}

}  // namespace

extern "C" int32_t scrs_dec_push(scrs_decoder* d, uint64_t idx, const uint8_t* payload, uint64_t len,
                                 scrs_push_outcome* outcome, scrs_error* err) {
    return push_common(d, idx, payload, len, false, nullptr, outcome, err);
}

extern "C" int32_t scrs_dec_push_device(scrs_decoder* d, uint64_t idx, const uint8_t* payload, uint64_t len,
                                        scrs_push_outcome* outcome, scrs_error* err) {
    return push_common(d, idx, payload, len, true, cudaStreamLegacy, outcome, err);
}

extern "C" int32_t scrs_dec_push_device_stream(scrs_decoder* d, uint64_t idx, const uint8_t* payload, uint64_t len,
                                               void* stream, scrs_push_outcome* outcome, scrs_error* err) {
    return push_common(d, idx, payload, len, true, (cudaStream_t)stream, outcome, err);
}

extern "C" int32_t scrs_dec_is_complete(const scrs_decoder* d) { return d && d->distinct >= d->p.k; }
extern "C" uint64_t scrs_dec_rank(const scrs_decoder* d) { return d ? d->distinct : 0; }
extern "C" uint64_t scrs_dec_received(const scrs_decoder* d) { return d ? d->received : 0; }
extern "C" void scrs_dec_reset(scrs_decoder* d) {
    if (!d) return;
    std::fill(d->have.begin(), d->have.end(), 0);
    std::fill(d->on_host.begin(), d->on_host.end(), 0);
    d->distinct = 0;
    d->received = 0;
}

extern "C" int32_t scrs_dec_finalize_into_with(scrs_decoder* d, uint8_t* out, uint64_t out_len,
                                               scrs_decode_scratch* s, scrs_error* err) {
    if (!d || !s) return set_err(err, SCRS_ERR_NULL_ARGUMENT);
    return finalize_host(d, out, out_len, s, err);
}

extern "C" int32_t scrs_dec_finalize_into(scrs_decoder* d, uint8_t* out, uint64_t out_len, scrs_error* err) {
    if (!d) return set_err(err, SCRS_ERR_NULL_ARGUMENT);
    int32_t r = finalize_checks(d, out_len, nullptr, err);
    if (r) return r;
    scrs_decode_scratch* s = nullptr;
    r = scrs_decoder_scratch(d, &s, err);
    if (r) return r;
    r = finalize_host(d, out, out_len, s, err);
    delete s;
    return r;
}

extern "C" int32_t scrs_dec_finalize_into_with_device(scrs_decoder* d, uint8_t* d_out, uint64_t out_len,
                                                      scrs_decode_scratch* s, void* stream, scrs_error* err) {
    if (!d || !s) return set_err(err, SCRS_ERR_NULL_ARGUMENT);
    int32_t r = finalize_checks(d, out_len, s, err);
    if (r) return r;
    if (!d_out) return set_err(err, SCRS_ERR_NULL_ARGUMENT);
    r = finalize_device(d, d_out, s, (cudaStream_t)stream, err);
    if (r) return r;
    return set_err(err, SCRS_OK);
}

// ===========================================================================
// BatchDecoder (selector.rs:247-352)
//   GF(256): BatchCodec::decode_into_with (batch/codec.rs:278-406)
//   Tower / AFFT: the blanket impl over the lazy decoder (codec.rs:203-239)
// ===========================================================================
struct scrs_batch_decoder {
    scrs_profile p{};
    OwnedStream stream;
    StatusWord status;
    scrs_decoder* lazy = nullptr;  // GF(65536) engines
    ~scrs_batch_decoder() { scrs_decoder_destroy(lazy); }
};

struct scrs_batch_decode_scratch {
    int kind = 0;
    scrs_profile p{};
    RecipeBufs recipe;          // GF(256)
    DevBuf d_rows, d_out;       // received rows / output (GF(256) host path)
    PinnedBuf h_rows;
    scrs_decode_scratch* lazy = nullptr;  // GF(65536)
    // per-call index lists, their capacity reserved here so that the calls
    // allocate nothing
    std::vector<uint16_t> missing, present, repairs, row_of;
    ~scrs_batch_decode_scratch() { scrs_decode_scratch_destroy(lazy); }
};

extern "C" int32_t scrs_batch_decoder_create(const scrs_profile* p, scrs_batch_decoder** out, scrs_error* err) {
    int32_t st = check_profile(p, err);
    if (st) return st;
    if (!out) return set_err(err, SCRS_ERR_NULL_ARGUMENT);
    std::unique_ptr<scrs_batch_decoder> b(new (std::nothrow) scrs_batch_decoder());
    if (!b) return set_err(err, SCRS_ERR_OUT_OF_MEMORY, sizeof(scrs_batch_decoder));
    b->p = *p;
    SCRS_CUDA(b->stream.init());
    SCRS_CUDA(b->status.init());
    if (is_gf16(p->engine)) {
        st = scrs_decoder_create(p, &b->lazy, err);
        if (st) return st;
    }
    *out = b.release();
    return set_err(err, SCRS_OK);
}

extern "C" void scrs_batch_decoder_destroy(scrs_batch_decoder* b) { delete b; }

extern "C" int32_t scrs_batch_decoder_profile(const scrs_batch_decoder* b, scrs_profile* out) {
    if (!b || !out) return SCRS_ERR_NULL_ARGUMENT;
    *out = b->p;
    return SCRS_OK;
}

extern "C" int32_t scrs_batch_decoder_scratch(const scrs_batch_decoder* b, scrs_batch_decode_scratch** out,
                                              scrs_error* err) {
    if (!b || !out) return set_err(err, SCRS_ERR_NULL_ARGUMENT);
    std::unique_ptr<scrs_batch_decode_scratch> s(new (std::nothrow) scrs_batch_decode_scratch());
    if (!s) return set_err(err, SCRS_ERR_OUT_OF_MEMORY, sizeof(scrs_batch_decode_scratch));
    s->kind = b->p.engine;
    s->p = b->p;
    const uint32_t k = (uint32_t)b->p.k, m = (uint32_t)b->p.m;
    const uint64_t L = b->p.symbol_len;
    s->missing.reserve(k);
    s->present.reserve(k);
    s->repairs.reserve(m);
    s->row_of.reserve((size_t)k + m);
    if (b->lazy) {
        int32_t st = scrs_decoder_scratch(b->lazy, &s->lazy, err);
        if (st) return st;
    } else {
        SCRS_CUDA(s->recipe.init(k, std::min(k, m), 1));
        SCRS_CUDA(s->d_rows.ensure((uint64_t)k * L));
        SCRS_CUDA(s->d_out.ensure((uint64_t)k * L));
        SCRS_CUDA(s->h_rows.ensure((uint64_t)k * L));
    }
    *out = s.release();
    return set_err(err, SCRS_OK);
}

extern "C" void scrs_batch_decode_scratch_destroy(scrs_batch_decode_scratch* s) { delete s; }

namespace {

// batch/codec.rs:289-343: scratch, output length, count, then per-symbol
// range / duplicate / payload-length checks in submission order.
int32_t gf8_batch_validate(const scrs_batch_decoder* b, const uint64_t* idx, const uint64_t* lens,
                           uint64_t count, uint64_t out_len, const scrs_batch_decode_scratch* s,
                           std::vector<uint16_t>& missing, std::vector<uint16_t>& present,
                           std::vector<uint16_t>& repairs, std::vector<uint16_t>& row_of, scrs_error* err) {
    const uint64_t k = b->p.k, m = b->p.m, n = k + m, L = b->p.symbol_len;
    if (is_gf16(s->kind) || s->p.k != k || s->p.m != m || s->p.symbol_len != L)
        return set_err(err, SCRS_DECODE_SCRATCH_MISMATCH);
    if (out_len != k * L) return set_err(err, SCRS_DECODE_WRONG_OUTPUT_LEN, k * L, out_len);
    if (count != k) return set_err(err, SCRS_DECODE_WRONG_COUNT, k, count);
    if (count && !idx) return set_err(err, SCRS_ERR_NULL_ARGUMENT);
    uint8_t seen[256] = {0};
    row_of.assign(n, kNoRow);
    missing.clear();
    present.clear();
    repairs.clear();
    for (uint64_t q = 0; q < count; q++) {
        uint64_t i = idx[q];
        if (i >= n) return set_err(err, SCRS_DECODE_INDEX_OUT_OF_RANGE, i, n);
        if (seen[i]) return set_err(err, SCRS_DECODE_DUPLICATE_INDEX, i);
        seen[i] = 1;
        if (lens && lens[q] != L) return set_err(err, SCRS_DECODE_WRONG_PAYLOAD_LEN, L, lens[q]);
        row_of[i] = (uint16_t)q;
    }
    for (uint64_t i = 0; i < k; i++) (seen[i] ? present : missing).push_back((uint16_t)i);
    for (uint64_t j = 0; j < m; j++)
        if (seen[k + j]) repairs.push_back((uint16_t)j);
    return SCRS_OK;
}

int32_t gf8_batch_run(scrs_batch_decoder* b, const std::vector<uint16_t>& missing,
                      const std::vector<uint16_t>& present, const std::vector<uint16_t>& repairs,
                      const std::vector<uint16_t>& row_of, const uint8_t* d_rows, uint8_t* d_out,
                      scrs_batch_decode_scratch* s, cudaStream_t st, scrs_error* err) {
    return run_cauchy_recover(
        s->recipe, b->p.engine, (uint32_t)b->p.k, missing, repairs, present,
        [&](uint32_t cw) { return row_of[cw]; }, d_rows, b->p.symbol_len, d_out, b->p.symbol_len, nullptr,
        b->status.dev, st, err);
}

}  // namespace

extern "C" int32_t scrs_batch_decode_into_with(scrs_batch_decoder* b, const uint64_t* idx,
                                               const uint8_t* const* pay, const uint64_t* lens, uint64_t count,
                                               uint8_t* out, uint64_t out_len, scrs_batch_decode_scratch* s,
                                               scrs_error* err) {
    if (!b || !s) return set_err(err, SCRS_ERR_NULL_ARGUMENT);
    if (b->lazy) {
        // codec.rs:219-238: count, reset, push each (Dependent -> DuplicateIndex), finalize.
        if (!s->lazy) return set_err(err, SCRS_DECODE_SCRATCH_MISMATCH);
        if (count != b->p.k) return set_err(err, SCRS_DECODE_WRONG_COUNT, b->p.k, count);
        if (count && (!idx || !pay || !lens)) return set_err(err, SCRS_ERR_NULL_ARGUMENT);
        scrs_dec_reset(b->lazy);
        for (uint64_t q = 0; q < count; q++) {
            scrs_push_outcome o;
            int32_t r = scrs_dec_push(b->lazy, idx[q], pay[q], lens[q], &o, err);
            if (r) return r;
            if (o.kind == SCRS_PUSH_DEPENDENT) return set_err(err, SCRS_DECODE_DUPLICATE_INDEX, idx[q]);
        }
        return scrs_dec_finalize_into_with(b->lazy, out, out_len, s->lazy, err);
    }
    if (s->lazy) return set_err(err, SCRS_DECODE_SCRATCH_MISMATCH);
    int32_t r = gf8_batch_validate(b, idx, lens, count, out_len, s, s->missing, s->present, s->repairs, s->row_of, err);
    if (r) return r;
    if (!out || (count && !pay)) return set_err(err, SCRS_ERR_NULL_ARGUMENT);
    const uint64_t L = b->p.symbol_len;
    uint8_t* h = s->h_rows.as<uint8_t>();
    for (uint64_t q = 0; q < count; q++) memcpy(h + q * L, pay[q], L);
    cudaStream_t st = b->stream.s;
    SCRS_CUDA(cudaMemcpyAsync(s->d_rows.p, h, count * L, cudaMemcpyHostToDevice, st));
    r = gf8_batch_run(b, s->missing, s->present, s->repairs, s->row_of, s->d_rows.as<uint8_t>(), s->d_out.as<uint8_t>(), s,
                      st, err);
    if (r) return r;
    SCRS_CUDA(cudaMemcpyAsync(out, s->d_out.p, out_len, cudaMemcpyDeviceToHost, st));
    SCRS_CUDA(cudaStreamSynchronize(st));
    r = take_status(b->status, err);
    if (r) return r;
    return set_err(err, SCRS_OK);
}

extern "C" int32_t scrs_batch_decode_into(scrs_batch_decoder* b, const uint64_t* idx, const uint8_t* const* pay,
                                          const uint64_t* lens, uint64_t count, uint8_t* out, uint64_t out_len,
                                          scrs_error* err) {
    scrs_batch_decode_scratch* s = nullptr;
    int32_t r = scrs_batch_decoder_scratch(b, &s, err);
    if (r) return r;
    r = scrs_batch_decode_into_with(b, idx, pay, lens, count, out, out_len, s, err);
    delete s;
    return r;
}

extern "C" int32_t scrs_batch_decode_into_with_device(scrs_batch_decoder* b, const uint64_t* idx,
                                                      const uint8_t* d_rows, uint64_t count, uint8_t* d_out,
                                                      uint64_t out_len, scrs_batch_decode_scratch* s,
                                                      void* stream, scrs_error* err) {
    if (!b || !s) return set_err(err, SCRS_ERR_NULL_ARGUMENT);
    const uint64_t L = b->p.symbol_len;
    cudaStream_t st = (cudaStream_t)stream;
    if (b->lazy) {
        // codec.rs:219-238 order: count, then each symbol as a push would
        // check it (range; Dependent -> DuplicateIndex), then finalize's checks.
        // The rows are read in place through a codeword-index -> row map.
        if (!s->lazy) return set_err(err, SCRS_DECODE_SCRATCH_MISMATCH);
        const uint64_t k = b->p.k, n = b->p.k + b->p.m;
        if (count != k) return set_err(err, SCRS_DECODE_WRONG_COUNT, k, count);
        if (count && (!idx || !d_rows)) return set_err(err, SCRS_ERR_NULL_ARGUMENT);
        scrs_decoder* d = b->lazy;
        scrs_dec_reset(d);
        std::vector<uint16_t>& row_of = s->row_of;
        row_of.assign(n, kNoRow);
        for (uint64_t q = 0; q < count; q++) {
            if (idx[q] >= n) return set_err(err, SCRS_DECODE_INDEX_OUT_OF_RANGE, idx[q], n);
            if (row_of[idx[q]] != kNoRow) return set_err(err, SCRS_DECODE_DUPLICATE_INDEX, idx[q]);
            row_of[idx[q]] = (uint16_t)q;
            d->have[idx[q]] = 1;
        }
        d->received = d->distinct = count;
        int32_t r = finalize_checks(d, out_len, s->lazy, err);
        if (r) return r;
        if (!d_out) return set_err(err, SCRS_ERR_NULL_ARGUMENT);
        if (d->afft) {
            r = d->afft->decode(d_rows, d->have.data(), d_out, *s->lazy->afft, d->status.dev, st, err,
                                row_of.data());
        } else {
            std::vector<uint16_t>&missing = s->missing, &present = s->present, &repairs = s->repairs;
            missing.clear();
            present.clear();
            repairs.clear();
            for (uint32_t i = 0; i < k; i++) (d->have[i] ? present : missing).push_back((uint16_t)i);
            for (uint32_t j = 0; j < b->p.m && repairs.size() < missing.size(); j++)
                if (d->have[k + j]) repairs.push_back((uint16_t)j);
            r = run_cauchy_recover(
                s->lazy->recipe, d->p.engine, (uint32_t)k, missing, repairs, present,
                [&](uint32_t cw) { return row_of[cw]; }, d_rows, L, d_out, L, d->tower.powers.as<uint16_t>(),
                d->status.dev, st, err);
        }
        if (r) return r;
        return set_err(err, SCRS_OK);
    }
    if (s->lazy) return set_err(err, SCRS_DECODE_SCRATCH_MISMATCH);
    int32_t r = gf8_batch_validate(b, idx, nullptr, count, out_len, s, s->missing, s->present, s->repairs, s->row_of,
                                   err);
    if (r) return r;
    if (!d_out || (count && !d_rows)) return set_err(err, SCRS_ERR_NULL_ARGUMENT);
    r = gf8_batch_run(b, s->missing, s->present, s->repairs, s->row_of, d_rows, d_out, s, st, err);
    if (r) return r;
    return set_err(err, SCRS_OK);
}

// ===========================================================================
// IncrementalEncoder (selector.rs:358-429): GF(256) Good Cauchy
// (encoder/streaming.rs) and Tower (tower/encoder.rs).  A feed records the
// data row (pinned staging or device copy); pending rows are folded into the
// device-resident repairs by one multiply-XOR launch before any repair read,
// so k feeds followed by reads cost one pass over the data.
// ===========================================================================
struct scrs_incremental_encoder {
    scrs_profile p{};
    OwnedStream stream;
    StatusWord status;
    DevBuf coef;       // [k][m] elements
    DevBuf repairs;    // m * L
    DevBuf data;       // k * L: fed rows awaiting the fold
    PinnedBuf staging; // k * L host staging
    DevBuf rows;       // uint16[k] pending row list
    std::vector<uint8_t> fed, pending_host, pending_dev;
    std::vector<uint16_t> pending;
    uint64_t fed_count = 0;
    // Device feeds copy on the caller's stream, chained on one stream at a
    // time (copy_stream); `copied` is recorded there when the chain moves or
    // a fold starts, and the fold waits on it.
    cudaEvent_t copied = nullptr;
    cudaStream_t copy_stream = nullptr;
    bool copy_pending = false;
    ~scrs_incremental_encoder() {
        if (copied) cudaEventDestroy(copied);
    }
};

extern "C" int32_t scrs_incremental_encoder_create(const scrs_profile* p, scrs_incremental_encoder** out,
                                                   scrs_error* err) {
    int32_t st = check_profile(p, err);
    if (st) return st;
    if (!out) return set_err(err, SCRS_ERR_NULL_ARGUMENT);
    if (p->engine != SCRS_ENGINE_GOOD_CAUCHY && p->engine != SCRS_ENGINE_TOWER)
        return set_err(err, SCRS_CONFIG_UNSUPPORTED_MODE, (uint64_t)p->engine);
    std::unique_ptr<scrs_incremental_encoder> e(new (std::nothrow) scrs_incremental_encoder());
    if (!e) return set_err(err, SCRS_ERR_OUT_OF_MEMORY, sizeof(scrs_incremental_encoder));
    e->p = *p;
    const uint64_t k = p->k, m = p->m, L = p->symbol_len;
    SCRS_CUDA(e->stream.init());
    SCRS_CUDA(e->status.init());
    SCRS_CUDA(cudaEventCreateWithFlags(&e->copied, cudaEventDisableTiming));
    if (p->engine == SCRS_ENGINE_TOWER) {
        std::vector<uint16_t> pw(k + m), c(k * m);
        hf::tower_powers((uint32_t)(k + m), pw.data());
        hf::tower_coefficients((uint32_t)k, (uint32_t)m, pw.data(), c.data());
        SCRS_CUDA(e->coef.ensure(c.size() * 2));
        SCRS_CUDA(upload_now(e->coef.p, c.data(), c.size() * 2, e->stream.s));
    } else {
        std::vector<uint8_t> c(k * m);
        hf::gf8_coefficients(p->engine, (uint32_t)k, (uint32_t)m, c.data());
        SCRS_CUDA(e->coef.ensure(c.size()));
        SCRS_CUDA(upload_now(e->coef.p, c.data(), c.size(), e->stream.s));
    }
    SCRS_CUDA(e->repairs.ensure(m * L));
    SCRS_CUDA(cudaMemset(e->repairs.p, 0, m * L));
    SCRS_CUDA(e->data.ensure(k * L));
    SCRS_CUDA(e->staging.ensure(k * L));
    SCRS_CUDA(e->rows.ensure(k * 2));
    e->fed.assign(k, 0);
    e->pending_host.assign(k, 0);
    e->pending_dev.assign(k, 0);
    e->pending.reserve(k);
    *out = e.release();
    return set_err(err, SCRS_OK);
}

extern "C" void scrs_incremental_encoder_destroy(scrs_incremental_encoder* e) { delete e; }

extern "C" int32_t scrs_incremental_encoder_profile(const scrs_incremental_encoder* e, scrs_profile* out) {
    if (!e || !out) return SCRS_ERR_NULL_ARGUMENT;
    *out = e->p;
    return SCRS_OK;
}

namespace {

int32_t feed_common(scrs_incremental_encoder* e, uint64_t idx, const uint8_t* data, uint64_t len, bool device,
                    cudaStream_t cs, scrs_error* err) {
    if (!e) return set_err(err, SCRS_ERR_NULL_ARGUMENT);
    const uint64_t k = e->p.k, m = e->p.m, L = e->p.symbol_len;
    // encoder/streaming.rs:163-177, tower/encoder.rs:90-104
    if (idx >= k) return set_err(err, SCRS_ENCODE_INDEX_OUT_OF_RANGE, idx, k + m);
    if (len != L) return set_err(err, SCRS_ENCODE_WRONG_PAYLOAD_LEN, L, len);
    if (e->fed[idx]) return set_err(err, SCRS_ENCODE_DUPLICATE_DATA, idx);
    if (!data) return set_err(err, SCRS_ERR_NULL_ARGUMENT);
    if (device) {
        // rows are written again only after a reset, which waits for the folds
        // that read them; chain this stream after an earlier one's copies
        if (e->copy_pending && e->copy_stream != cs) {
            SCRS_CUDA(cudaEventRecord(e->copied, e->copy_stream));
            SCRS_CUDA(cudaStreamWaitEvent(cs, e->copied, 0));
        }
        SCRS_CUDA(cudaMemcpyAsync(e->data.as<uint8_t>() + idx * L, data, L, cudaMemcpyDeviceToDevice, cs));
        e->copy_stream = cs;
        e->copy_pending = true;
        e->pending_dev[idx] = 1;
    } else {
        memcpy(e->staging.as<uint8_t>() + idx * L, data, L);
        e->pending_host[idx] = 1;
    }
    e->fed[idx] = 1;
    e->fed_count++;
    e->pending.push_back((uint16_t)idx);
    return set_err(err, SCRS_OK);
}

// Fold every pending data row into the repairs: repairs ^= C[i][.] * data_i.
int32_t flush(scrs_incremental_encoder* e, scrs_error* err) {
    if (e->pending.empty()) return SCRS_OK;
    const uint64_t k = e->p.k, m = e->p.m, L = e->p.symbol_len;
    const bool gf16 = e->p.engine == SCRS_ENGINE_TOWER;
    cudaStream_t st = e->stream.s;
    uint64_t i = 0;
    while (i < k) {  // host-staged rows in runs
        if (!e->pending_host[i]) {
            i++;
            continue;
        }
        uint64_t j = i;
        while (j < k && e->pending_host[j]) j++;
        SCRS_CUDA(cudaMemcpyAsync(e->data.as<uint8_t>() + i * L, e->staging.as<uint8_t>() + i * L, (j - i) * L,
                                  cudaMemcpyHostToDevice, st));
        i = j;
    }
    if (e->copy_pending) {  // the device feeds' copies
        SCRS_CUDA(cudaEventRecord(e->copied, e->copy_stream));
        SCRS_CUDA(cudaStreamWaitEvent(st, e->copied, 0));
        e->copy_pending = false;
    }
    std::sort(e->pending.begin(), e->pending.end());
    SCRS_CUDA(cudaMemcpyAsync(e->rows.p, e->pending.data(), e->pending.size() * 2, cudaMemcpyHostToDevice, st));
    MxkTask T{};
    T.in = e->data.as<uint8_t>();
    T.out = e->repairs.as<uint8_t>();
    T.coef = e->coef.p;
    T.in_rows = e->rows.as<uint16_t>();
    T.coef_rows = e->rows.as<uint16_t>();  // coefficient row = data index
    T.L = L;
    T.in_stride = L;
    T.out_stride = L;
    T.n_in = (uint32_t)e->pending.size();
    T.n_out = (uint32_t)m;
    T.ld = (uint32_t)m;
    T.n_items = n_chunks(L, gf16);
    T.aligned = (L % 16 == 0) ? 1u : 0u;
    T.accumulate = 1;
    SCRS_CUDA(launch_mxk_single(T, gf16 ? 1 : 0, e->status.dev, 0, st));
    e->pending.clear();
    std::fill(e->pending_host.begin(), e->pending_host.end(), 0);
    std::fill(e->pending_dev.begin(), e->pending_dev.end(), 0);
    // The pending-row list upload is pageable (staged before return), so the
    // host list can be reused immediately.
    return SCRS_OK;
}

}  // namespace

extern "C" int32_t scrs_inc_feed(scrs_incremental_encoder* e, uint64_t idx, const uint8_t* data, uint64_t len,
                                 scrs_error* err) {
    return feed_common(e, idx, data, len, false, nullptr, err);
}

extern "C" int32_t scrs_inc_feed_device(scrs_incremental_encoder* e, uint64_t idx, const uint8_t* data,
                                        uint64_t len, scrs_error* err) {
    return feed_common(e, idx, data, len, true, cudaStreamLegacy, err);
}

extern "C" int32_t scrs_inc_feed_device_stream(scrs_incremental_encoder* e, uint64_t idx, const uint8_t* data,
                                               uint64_t len, void* stream, scrs_error* err) {
    return feed_common(e, idx, data, len, true, (cudaStream_t)stream, err);
}

// encoder/streaming.rs:197-206, tower/encoder.rs:122-131
extern "C" int32_t scrs_inc_repair(const scrs_incremental_encoder* ce, uint64_t idx, uint8_t* dst,
                                   uint64_t dst_len, scrs_error* err) {
    if (!ce) return set_err(err, SCRS_ERR_NULL_ARGUMENT);
    scrs_incremental_encoder* e = const_cast<scrs_incremental_encoder*>(ce);
    const uint64_t k = e->p.k, m = e->p.m, L = e->p.symbol_len;
    if (idx >= m) return set_err(err, SCRS_ENCODE_INDEX_OUT_OF_RANGE, idx, k + m);
    if (dst_len != L) return set_err(err, SCRS_ENCODE_WRONG_OUTPUT_LEN, L, dst_len);
    if (!dst) return set_err(err, SCRS_ERR_NULL_ARGUMENT);
    int32_t r = flush(e, err);
    if (r) return r;
    SCRS_CUDA(cudaMemcpyAsync(dst, e->repairs.as<uint8_t>() + idx * L, L, cudaMemcpyDeviceToHost, e->stream.s));
    SCRS_CUDA(cudaStreamSynchronize(e->stream.s));
    r = take_status(e->status, err);
    if (r) return r;
    return set_err(err, SCRS_OK);
}

extern "C" int32_t scrs_inc_repair_device(const scrs_incremental_encoder* ce, uint64_t idx,
                                          const uint8_t** d_repair, scrs_error* err) {
    if (!ce || !d_repair) return set_err(err, SCRS_ERR_NULL_ARGUMENT);
    scrs_incremental_encoder* e = const_cast<scrs_incremental_encoder*>(ce);
    const uint64_t k = e->p.k, m = e->p.m, L = e->p.symbol_len;
    if (idx >= m) return set_err(err, SCRS_ENCODE_INDEX_OUT_OF_RANGE, idx, k + m);
    int32_t r = flush(e, err);
    if (r) return r;
    SCRS_CUDA(cudaStreamSynchronize(e->stream.s));
    r = take_status(e->status, err);
    if (r) return r;
    *d_repair = e->repairs.as<uint8_t>() + idx * L;
    return set_err(err, SCRS_OK);
}

extern "C" uint64_t scrs_inc_fed_count(const scrs_incremental_encoder* e) { return e ? e->fed_count : 0; }

extern "C" void scrs_inc_reset(scrs_incremental_encoder* e) {
    if (!e) return;
    cudaStreamSynchronize(e->stream.s);
    cudaMemsetAsync(e->repairs.p, 0, e->p.m * e->p.symbol_len, e->stream.s);
    std::fill(e->fed.begin(), e->fed.end(), 0);
    std::fill(e->pending_host.begin(), e->pending_host.end(), 0);
    std::fill(e->pending_dev.begin(), e->pending_dev.end(), 0);
    e->pending.clear();
    e->fed_count = 0;
}

// Self-test of the device-side failure path (include/scrs_gpu.h).
extern "C" int32_t scrs_selftest_wait_timeout(uint64_t limit_ns, scrs_error* err) {
    if (limit_ns == 0 || limit_ns > 100000000ull) return set_err(err, SCRS_ERR_BAD_ARGUMENT, 1);
    StatusWord sw;
    SCRS_CUDA(sw.init());
    OwnedStream st;
    SCRS_CUDA(st.init());
    SCRS_CUDA(launch_wait_selftest(sw.dev, limit_ns, st.s));
    SCRS_CUDA(cudaStreamSynchronize(st.s));
    return take_status(sw, err);
}

// Recipe-cache hits (repeated erasure patterns that skipped the plan launch).
extern "C" uint64_t scrs_decode_scratch_recipe_hits(const scrs_decode_scratch* s) {
    return s ? s->recipe.hits : 0;
}
extern "C" uint64_t scrs_batch_decode_scratch_recipe_hits(const scrs_batch_decode_scratch* s) {
    if (!s) return 0;
    return s->lazy ? s->lazy->recipe.hits : s->recipe.hits;
}

// Device-side status of a handle's last asynchronous work (used by the
// serving loop after its completion event fires).
namespace scrs {
int32_t internal_batch_encoder_status(scrs_batch_encoder* e, scrs_error* err) {
    return take_status(e->status, err);
}
int32_t internal_batch_decoder_status(scrs_batch_decoder* b, scrs_error* err) {
    int32_t r = take_status(b->status, err);
    if (!r && b->lazy) r = take_status(b->lazy->status, err);
    return r;
}
}  // namespace scrs
