// Serving loop: continuous batching of encode / decode requests of every
// engine on one GPU.
//
// Requests are submitted with device-resident inputs and outputs and admitted
// as slots and device memory free up: each slot is a stream with its own
// resident engines, so admitted work overlaps on the device.  GF(256)
// requests and small tower requests waiting in the queue are coalesced into
// one stripe batch (plan launches + one persistent drain per field) per slot;
// additive-FFT requests and large tower requests take a slot each.  Admission is first-come first-served under a device-memory budget
// that counts each admitted request's input and output bytes plus the
// resident engines' workspaces.  progress() polls the slots' completion
// events, returns finished requests and admits waiting ones; it never blocks
// on the device.
#include <algorithm>
#include <chrono>
#include <deque>
#include <map>
#include <memory>
#include <new>
#include <tuple>
#include <vector>

#include "host_field.h"
#include "runtime.h"

using namespace scrs;

namespace {

uint64_t now_ns() {
    return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
               std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

constexpr uint32_t kMaxSlots = 64;
constexpr uint32_t kMaxCoalesce = 4096;  // GF(256) requests per stripe batch
constexpr size_t kCachePerSlot = 8;      // resident engine profiles per slot

using ProfileKey = std::tuple<int32_t, uint64_t, uint64_t, uint64_t>;

bool is_gf256(int32_t engine) {
    return engine == SCRS_ENGINE_STANDARD_CAUCHY || engine == SCRS_ENGINE_GOOD_CAUCHY;
}

// Requests that run as stripes of the slot's stripe batch: GF(256) requests,
// and tower requests whose work per 2 KiB column chunk is bounded (at most 64
// inputs and 32 outputs: the persistent drain gives one CTA a whole chunk).
// Larger tower requests and additive-FFT requests take a slot each and use
// resident engines (a large tower request's multiply then splits its inputs
// over CTAs).
constexpr uint64_t kTowerBatchMaxK = 64, kTowerBatchMaxM = 32;
bool batchable(int32_t engine, uint64_t k, uint64_t m) {
    return is_gf256(engine) || (engine == SCRS_ENGINE_TOWER && k <= kTowerBatchMaxK && m <= kTowerBatchMaxM);
}

// Engines of one profile, resident on one slot.
struct Resident {
    scrs_profile p{};
    scrs_batch_encoder* enc = nullptr;  // AFFT
    scrs_encode_scratch* enc_s = nullptr;
    scrs_batch_decoder* dec = nullptr;  // tower, AFFT
    scrs_batch_decode_scratch* dec_s = nullptr;
    DevBuf tower_coef;                  // tower encode: uint16[k*m]
    uint64_t bytes = 0;                 // estimated device footprint
    uint64_t last_use = 0;
    ~Resident() {
        scrs_encode_scratch_destroy(enc_s);
        scrs_batch_encoder_destroy(enc);
        scrs_batch_decode_scratch_destroy(dec_s);
        scrs_batch_decoder_destroy(dec);
    }
};

// Estimated device bytes of the engines a request needs (admission only).
uint64_t resident_estimate(const scrs_profile& p, int32_t op) {
    const uint64_t k = p.k, m = p.m, L = p.symbol_len;
    if (p.engine == SCRS_ENGINE_TOWER) return op == SCRS_OP_ENCODE ? 2 * k * m : (k + m) * L + 4 * k * m + 64 * k;
    // AFFT: two bit-sliced work arrays of ts rows plus per-point tables
    uint64_t ts = 1;
    while (ts < k + m) ts <<= 1;
    return 2 * ts * ((L + 63) / 64) * 64 + 32 * ts;
}

struct Req {
    scrs_request d{};
    cudaEvent_t ready = nullptr;  // recorded on the caller's stream at submit
    uint64_t ticket = 0;
    uint64_t t_submit = 0;
    uint64_t bytes = 0;  // input + output
    std::vector<uint64_t> idx;
    std::vector<uint16_t> idx16;
};

struct Slot {
    OwnedStream stream;
    cudaEvent_t done = nullptr;
    StatusWord status;                 // direct launches (large tower encodes)
    scrs_stripe_batch* batch = nullptr;
    std::map<ProfileKey, std::unique_ptr<Resident>> cache;
    uint64_t cache_bytes = 0;
    std::vector<Req> running;
    std::vector<Resident*> used;
    bool used_batch = false;
    int32_t launch_code = 0;
    scrs_error launch_err{};
    std::vector<void*> seen_streams;  // scratch of admit()
    uint64_t held = 0;  // request bytes held while running
    bool busy = false;
    ~Slot() {
        if (done) cudaEventDestroy(done);
        scrs_stripe_batch_destroy(batch);
    }
};

}  // namespace

namespace scrs {
int32_t stripe_batch_set_impl(scrs_stripe_batch* b, const scrs_stripe_desc* descs, uint64_t count, bool async_stream,
                              cudaStream_t stream, scrs_error* err);
int32_t internal_batch_encoder_status(scrs_batch_encoder* e, scrs_error* err);
int32_t internal_batch_decoder_status(scrs_batch_decoder* b, scrs_error* err);
}  // namespace scrs

struct scrs_server {
    uint64_t budget = 0, in_use = 0, clock = 0, next_ticket = 1;
    std::vector<std::unique_ptr<Slot>> slots;
    std::deque<Req> queue;
    std::vector<scrs_completion> ready;  // finished but not yet returned
    std::vector<cudaEvent_t> free_events;  // input-ready events for reuse
    scrs_server_stats stats{};
    ~scrs_server() {
        for (cudaEvent_t e : free_events) cudaEventDestroy(e);
        for (const Req& r : queue) cudaEventDestroy(r.ready);
        for (auto& sl : slots)
            for (const Req& r : sl->running) cudaEventDestroy(r.ready);
    }
};

namespace {

uint64_t total_cache(const scrs_server* s) {
    uint64_t t = 0;
    for (auto& sl : s->slots) t += sl->cache_bytes;
    return t;
}

void finish(scrs_server* s, const Req& r, int32_t status, uint64_t t_done) {
    scrs_completion c{};
    c.ticket = r.ticket;
    c.tag = r.d.tag;
    c.status = status;
    c.submit_ns = r.t_submit;
    c.done_ns = t_done;
    s->ready.push_back(c);
    s->stats.completed++;
    if (status) s->stats.failed++;
}

// Get (or build) the resident engines of profile p for `op` on slot `sl`,
// evicting the slot's least recently used profiles to stay in budget.
int32_t resident(scrs_server* s, Slot& sl, const scrs_profile& p, int32_t op, Resident** out, scrs_error* err) {
    const ProfileKey key{p.engine, p.k, p.m, p.symbol_len};
    auto it = sl.cache.find(key);
    Resident* R = it == sl.cache.end() ? nullptr : it->second.get();
    const bool need_enc = op == SCRS_OP_ENCODE, need_dec = op == SCRS_OP_DECODE;
    const bool have = R && (need_enc ? (p.engine == SCRS_ENGINE_TOWER ? R->tower_coef.p != nullptr : R->enc != nullptr)
                                     : R->dec != nullptr);
    if (!have) {
        const uint64_t add = resident_estimate(p, op);
        while (!sl.cache.empty() && (sl.cache.size() >= kCachePerSlot || s->in_use + total_cache(s) + add > s->budget)) {
            auto victim = sl.cache.begin();
            for (auto v = sl.cache.begin(); v != sl.cache.end(); ++v)
                if (v->second->last_use < victim->second->last_use) victim = v;
            if (victim->first == key) break;
            sl.cache_bytes -= victim->second->bytes;
            sl.cache.erase(victim);
            it = sl.cache.find(key);
            R = it == sl.cache.end() ? nullptr : it->second.get();
        }
        if (!R) {
            std::unique_ptr<Resident> nr(new (std::nothrow) Resident());
            if (!nr) return set_err(err, SCRS_ERR_OUT_OF_MEMORY, sizeof(Resident));
            nr->p = p;
            R = nr.get();
            sl.cache[key] = std::move(nr);
        }
        int32_t rc = SCRS_OK;
        if (need_enc && p.engine == SCRS_ENGINE_TOWER) {
            std::vector<uint16_t> pw(p.k + p.m), c(p.k * p.m);
            hf::tower_powers((uint32_t)(p.k + p.m), pw.data());
            hf::tower_coefficients((uint32_t)p.k, (uint32_t)p.m, pw.data(), c.data());
            SCRS_CUDA(R->tower_coef.ensure(c.size() * 2));
            SCRS_CUDA(upload_now(R->tower_coef.p, c.data(), c.size() * 2, sl.stream.s));
        } else if (need_enc) {
            rc = scrs_batch_encoder_create(&p, &R->enc, err);
            if (!rc) rc = scrs_batch_encoder_scratch(R->enc, &R->enc_s, err);
        } else {
            rc = scrs_batch_decoder_create(&p, &R->dec, err);
            if (!rc) rc = scrs_batch_decoder_scratch(R->dec, &R->dec_s, err);
        }
        if (rc) {
            if (R->bytes == 0) sl.cache.erase(key);  // keep engines built earlier
            return rc;
        }
        R->bytes += add;
        sl.cache_bytes += add;
    }
    R->last_use = ++s->clock;
    *out = R;
    return SCRS_OK;
}

// Enqueue one large tower or additive-FFT request on the slot's stream.
int32_t launch_single(scrs_server* s, Slot& sl, Req& r, scrs_error* err) {
    scrs_profile p{};
    int32_t rc = scrs_profile_resolve(r.d.engine, r.d.k, r.d.m, r.d.symbol_len, &p, err);
    if (rc) return rc;
    Resident* R = nullptr;
    rc = resident(s, sl, p, r.d.op, &R, err);
    if (rc) return rc;
    const uint64_t k = p.k, m = p.m, L = p.symbol_len;
    cudaStream_t st = sl.stream.s;
    if (r.d.op == SCRS_OP_ENCODE && p.engine == SCRS_ENGINE_TOWER) {
        // Block encode of all k rows: repairs = C^T * data over GF((2^8)^2)
        // (the incremental tower encode of k in-order feeds, tower/encoder.rs:89-116).
        MxkTask T{};
        T.in = r.d.in;
        T.out = r.d.out;
        T.coef = R->tower_coef.p;
        T.L = L;
        T.in_stride = L;
        T.out_stride = L;
        T.n_in = (uint32_t)k;
        T.n_out = (uint32_t)m;
        T.ld = (uint32_t)m;
        T.n_items = n_chunks(L, true);
        T.aligned = (L % 16 == 0 && aligned16(r.d.in) && aligned16(r.d.out)) ? 1u : 0u;
        SCRS_CUDA(launch_mxk_single(T, 1, sl.status.dev, 0, st));
        return SCRS_OK;
    }
    sl.used.push_back(R);
    if (r.d.op == SCRS_OP_ENCODE)
        return scrs_batch_encode_into_with_device(R->enc, r.d.in, k * L, r.d.out, m * L, R->enc_s, st, err);
    return scrs_batch_decode_into_with_device(R->dec, r.idx.data(), r.d.in, k, r.d.out, k * L, R->dec_s, st, err);
}

// Enqueue a coalesced group of GF(256) requests as one stripe batch.
int32_t launch_group(Slot& sl, std::vector<Req>& group, scrs_error* err) {
    if (!sl.batch) {
        int32_t rc = scrs_stripe_batch_create(kMaxCoalesce, 0, &sl.batch, err);
        if (!rc) rc = scrs_stripe_batch_set_jit(sl.batch, 0, err);  // no compile inside a request's latency
        if (rc) return rc;
    }
    std::vector<scrs_stripe_desc> d(group.size());
    for (size_t q = 0; q < group.size(); q++) {
        const Req& r = group[q];
        d[q].op = r.d.op;
        d[q].engine = r.d.engine;
        d[q].k = (uint32_t)r.d.k;
        d[q].m = (uint32_t)r.d.m;
        d[q].symbol_len = r.d.symbol_len;
        d[q].in = r.d.in;
        d[q].out = r.d.out;
        d[q].indices = r.d.op == SCRS_OP_DECODE ? r.idx16.data() : nullptr;
    }
    // uploads enqueued on the slot's stream: the slot is idle, so its previous
    // run (which read the old batch contents) has finished
    int32_t rc = stripe_batch_set_impl(sl.batch, d.data(), d.size(), true, sl.stream.s, err);
    if (rc) return rc;
    sl.used_batch = true;
    return scrs_stripe_batch_run(sl.batch, sl.stream.s, 0, err);
}

// Check a finished slot and report its requests.
void retire(scrs_server* s, Slot& sl, uint64_t t_done) {
    int32_t status = sl.launch_code;
    scrs_error e{};
    if (!status && sl.used_batch) status = scrs_stripe_batch_check(sl.batch, &e);
    for (Resident* R : sl.used) {
        if (status) break;
        if (R->enc) status = internal_batch_encoder_status(R->enc, &e);
        if (!status && R->dec) status = internal_batch_decoder_status(R->dec, &e);
    }
    if (!status) status = take_status(sl.status, &e);
    for (const Req& r : sl.running) {
        finish(s, r, status, t_done);
        s->free_events.push_back(r.ready);  // its wait has run: reusable
    }
    s->in_use -= sl.held;
    sl.held = 0;
    sl.running.clear();
    sl.used.clear();
    sl.used_batch = false;
    sl.launch_code = 0;
    sl.busy = false;
}

// Make the slot's stream wait for the work that wrote its requests' inputs:
// one wait per distinct caller stream, on the event of that stream's latest
// request (events recorded later on a stream cover the earlier ones).
int32_t wait_inputs(Slot& sl) {
    std::vector<void*>& seen = sl.seen_streams;
    seen.clear();
    for (size_t q = sl.running.size(); q-- > 0;) {
        const Req& r = sl.running[q];
        if (std::find(seen.begin(), seen.end(), r.d.stream) != seen.end()) continue;
        seen.push_back(r.d.stream);
        const cudaError_t e = cudaStreamWaitEvent(sl.stream.s, r.ready, 0);
        if (e != cudaSuccess) return set_err(&sl.launch_err, SCRS_ERR_CUDA, (uint64_t)e, (uint64_t)__LINE__);
    }
    return SCRS_OK;
}

// Admit waiting requests into idle slots (first come, first served).  A tower
// or AFFT request goes to an idle slot that already holds its profile's
// engines when there is one (building engines allocates device memory).
void admit(scrs_server* s) {
    for (;;) {
        if (s->queue.empty()) return;
        Req& head = s->queue.front();
        if (s->in_use + head.bytes > s->budget) return;  // wait for memory
        Slot* pick = nullptr;
        const bool batch = batchable(head.d.engine, head.d.k, head.d.m);
        for (auto& slp : s->slots) {
            if (slp->busy) continue;
            if (!pick) pick = slp.get();
            if (batch) break;
            const ProfileKey key{head.d.engine, head.d.k, head.d.m, head.d.symbol_len};
            if (slp->cache.count(key)) {
                pick = slp.get();
                break;
            }
        }
        if (!pick) return;  // every slot busy
        Slot& sl = *pick;
        std::vector<Req> group;
        uint64_t held = 0;
        if (batch) {
            // coalesce every waiting GF(256) and tower request that fits, in arrival order
            for (auto it = s->queue.begin(); it != s->queue.end() && group.size() < kMaxCoalesce;) {
                if (!batchable(it->d.engine, it->d.k, it->d.m)) {
                    ++it;
                    continue;
                }
                if (s->in_use + held + it->bytes > s->budget) break;
                held += it->bytes;
                group.push_back(std::move(*it));
                it = s->queue.erase(it);
            }
        } else {
            held = head.bytes;
            group.push_back(std::move(head));
            s->queue.pop_front();
        }
        s->in_use += held;
        sl.held = held;
        sl.busy = true;
        sl.running = std::move(group);
        // the inputs' producers first: one wait per distinct caller stream
        // (the latest request of a stream covers the earlier ones)
        int32_t rc = wait_inputs(sl);
        if (!rc && batch) {
            rc = launch_group(sl, sl.running, &sl.launch_err);
            s->stats.batches++;
        } else if (!rc) {
            rc = launch_single(s, sl, sl.running[0], &sl.launch_err);
        }
        s->stats.admitted += sl.running.size();
        if (rc) sl.launch_code = rc;
        if (cudaEventRecord(sl.done, sl.stream.s) != cudaSuccess && !sl.launch_code) sl.launch_code = SCRS_ERR_CUDA;
    }
}

}  // namespace

extern "C" int32_t scrs_server_create(uint64_t memory_budget, uint32_t n_slots, scrs_server** out, scrs_error* err) {
    if (!out) return set_err(err, SCRS_ERR_NULL_ARGUMENT);
    if (n_slots == 0 || n_slots > kMaxSlots) return set_err(err, SCRS_ERR_BAD_ARGUMENT, 2);
    if (memory_budget == 0) return set_err(err, SCRS_ERR_BAD_ARGUMENT, 1);
    std::unique_ptr<scrs_server> s(new (std::nothrow) scrs_server());
    if (!s) return set_err(err, SCRS_ERR_OUT_OF_MEMORY, sizeof(scrs_server));
    s->budget = memory_budget;
    for (uint32_t i = 0; i < n_slots; i++) {
        std::unique_ptr<Slot> sl(new (std::nothrow) Slot());
        if (!sl) return set_err(err, SCRS_ERR_OUT_OF_MEMORY, sizeof(Slot));
        SCRS_CUDA(sl->stream.init());
        SCRS_CUDA(sl->status.init());
        SCRS_CUDA(cudaEventCreateWithFlags(&sl->done, cudaEventDisableTiming));
        s->slots.push_back(std::move(sl));
    }
    *out = s.release();
    return set_err(err, SCRS_OK);
}

extern "C" void scrs_server_destroy(scrs_server* s) {
    if (!s) return;
    for (auto& sl : s->slots)
        if (sl->busy) cudaEventSynchronize(sl->done);
    delete s;
}

extern "C" int32_t scrs_server_submit(scrs_server* s, const scrs_request* rq, uint64_t* ticket, scrs_error* err) {
    if (!s || !rq) return set_err(err, SCRS_ERR_NULL_ARGUMENT);
    if (rq->op != SCRS_OP_ENCODE && rq->op != SCRS_OP_DECODE) return set_err(err, SCRS_ERR_BAD_ARGUMENT, 1);
    scrs_profile p{};
    int32_t rc = scrs_profile_resolve(rq->engine, rq->k, rq->m, rq->symbol_len, &p, err);
    if (rc) return rc;
    if (!rq->in || !rq->out) return set_err(err, SCRS_ERR_NULL_ARGUMENT);
    const uint64_t k = p.k, m = p.m, L = p.symbol_len, n = k + m;
    Req r;
    r.d = *rq;
    r.d.indices = nullptr;
    if (rq->op == SCRS_OP_DECODE) {
        // batch/codec.rs:289-343: count, then range and duplicates in order
        if (!rq->indices) return set_err(err, SCRS_ERR_NULL_ARGUMENT);
        std::vector<uint8_t> seen(n, 0);
        r.idx.assign(rq->indices, rq->indices + k);
        r.idx16.resize(k);
        for (uint64_t q = 0; q < k; q++) {
            const uint64_t i = r.idx[q];
            if (i >= n) return set_err(err, SCRS_DECODE_INDEX_OUT_OF_RANGE, i, n);
            if (seen[i]) return set_err(err, SCRS_DECODE_DUPLICATE_INDEX, i);
            seen[i] = 1;
            r.idx16[q] = (uint16_t)i;
        }
    }
    r.bytes = k * L + (rq->op == SCRS_OP_ENCODE ? m : k) * L;
    const uint64_t need = r.bytes + (batchable(p.engine, p.k, p.m) ? 0 : resident_estimate(p, rq->op));
    if (need > s->budget) return set_err(err, SCRS_ERR_CAPACITY, need, s->budget);
    if (s->free_events.empty()) {
        cudaEvent_t e = nullptr;
        SCRS_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        s->free_events.push_back(e);
    }
    r.d.stream = rq->stream ? rq->stream : (void*)cudaStreamLegacy;
    SCRS_CUDA(cudaEventRecord(s->free_events.back(), (cudaStream_t)r.d.stream));
    r.ready = s->free_events.back();
    s->free_events.pop_back();
    r.ticket = s->next_ticket++;
    r.t_submit = now_ns();
    if (ticket) *ticket = r.ticket;
    s->queue.push_back(std::move(r));
    s->stats.submitted++;
    admit(s);
    return set_err(err, SCRS_OK);
}

extern "C" int32_t scrs_server_progress(scrs_server* s, scrs_completion* done, uint32_t capacity, uint32_t* n_done,
                                        scrs_error* err) {
    if (!s || !n_done || (capacity && !done)) return set_err(err, SCRS_ERR_NULL_ARGUMENT);
    for (auto& slp : s->slots) {
        Slot& sl = *slp;
        if (!sl.busy) continue;
        cudaError_t q = cudaEventQuery(sl.done);
        if (q == cudaErrorNotReady) continue;
        if (q != cudaSuccess && !sl.launch_code) sl.launch_code = SCRS_ERR_CUDA;
        retire(s, sl, now_ns());
    }
    admit(s);
    const uint32_t n = (uint32_t)std::min<size_t>(capacity, s->ready.size());
    std::copy(s->ready.begin(), s->ready.begin() + n, done);
    s->ready.erase(s->ready.begin(), s->ready.begin() + n);
    *n_done = n;
    return set_err(err, SCRS_OK);
}

extern "C" int32_t scrs_server_reserve(scrs_server* s, int32_t op, int32_t engine, uint64_t k, uint64_t m,
                                       uint64_t symbol_len, scrs_error* err) {
    if (!s) return set_err(err, SCRS_ERR_NULL_ARGUMENT);
    if (op != SCRS_OP_ENCODE && op != SCRS_OP_DECODE) return set_err(err, SCRS_ERR_BAD_ARGUMENT, 2);
    scrs_profile p{};
    int32_t rc = scrs_profile_resolve(engine, k, m, symbol_len, &p, err);
    if (rc) return rc;
    for (auto& sl : s->slots)  // engines in use must not be evicted
        if (sl->busy) return set_err(err, SCRS_ERR_BAD_ARGUMENT, 3);
    if (is_gf256(p.engine)) return set_err(err, SCRS_ERR_BAD_ARGUMENT, 1);
    if (batchable(p.engine, p.k, p.m)) return set_err(err, SCRS_OK);  // runs in the stripe batch: nothing to build
    for (auto& sl : s->slots) {
        Resident* R = nullptr;
        rc = resident(s, *sl, p, op, &R, err);
        if (rc) return rc;
    }
    return set_err(err, SCRS_OK);
}

extern "C" uint64_t scrs_server_pending(const scrs_server* s) {
    if (!s) return 0;
    uint64_t n = s->queue.size() + s->ready.size();
    for (auto& sl : s->slots) n += sl->running.size();
    return n;
}

extern "C" int32_t scrs_server_get_stats(const scrs_server* s, scrs_server_stats* out) {
    if (!s || !out) return SCRS_ERR_NULL_ARGUMENT;
    *out = s->stats;
    out->memory_in_use = s->in_use;
    out->resident_bytes = total_cache(s);
    return SCRS_OK;
}
