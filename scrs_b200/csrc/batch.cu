// Batched GF(256) stripes: many independent BatchCodec::encode_into
// (batch/codec.rs:156) and decode_into_with (batch/codec.rs:278) calls of
// uneven geometry, run as one device work queue.
//
//   set():  validate descriptors, build per-stripe tasks and the decode
//           lists on the host, upload everything in one copy;
//   run():  one plan launch builds every decode matrix on the device (the
//           closed-form reduced Cauchy solve), one persistent launch drains
//           the (stripe, chunk) work queue; optionally replayed as a graph;
//   run_plain(): the same work as one plan + one multiply-XOR launch per
//           stripe, the baseline the persistent form is measured against.
//
// Host-buffer mode (set_host): the stripes are cut into up to kMaxPieces
// pieces of about equal input bytes; piece p's host->device copies, its plan
// and drain launches and its device->host copies run on three streams, so the
// copies of one piece overlap the compute of the previous one and both copy
// directions run at once.  A decode stripe's present data rows are already
// in the caller's input rows: the device computes only the missing rows and
// copies them back (compact) into pinned staging, and host worker threads
// copy the present rows from the input rows into `out` while the GPU runs,
// then each piece's missing rows from the staging once that piece is back.
// The link then carries k*L in and r*L out per decode stripe instead of
// k*L each way.
#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <thread>
#include <tuple>
#if defined(__SSE2__)
#include <emmintrin.h>
#endif

#include "host_field.h"
#include "jit.h"
#include "runtime.h"
#include "tune.h"

using namespace scrs;

namespace {

// Host worker threads of a host-buffer batch.  run(f) calls f(w) on every
// worker w and returns when all have finished.
class HostPool {
   public:
    ~HostPool() {
        {
            std::lock_guard<std::mutex> g(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto& t : threads_) t.join();
    }
    int size() const { return (int)threads_.size(); }
    bool start(int n) {
        if (!threads_.empty()) return true;
        try {
            for (int w = 0; w < n; w++) threads_.emplace_back([this, w] { loop(w); });
        } catch (...) {
            return !threads_.empty();
        }
        return true;
    }
    void run(const std::function<void(int)>& f) {
        std::unique_lock<std::mutex> g(mu_);
        work_ = &f;
        remaining_ = (int)threads_.size();
        gen_++;
        cv_.notify_all();
        done_cv_.wait(g, [this] { return remaining_ == 0; });
        work_ = nullptr;
    }

   private:
    void loop(int w) {
        uint64_t seen = 0;
        for (;;) {
            const std::function<void(int)>* f;
            {
                std::unique_lock<std::mutex> g(mu_);
                cv_.wait(g, [&] { return stop_ || gen_ != seen; });
                if (stop_) return;
                seen = gen_;
                f = work_;
            }
            (*f)(w);
            std::lock_guard<std::mutex> g(mu_);
            if (--remaining_ == 0) done_cv_.notify_one();
        }
    }
    std::vector<std::thread> threads_;
    std::mutex mu_;
    std::condition_variable cv_, done_cv_;
    const std::function<void(int)>* work_ = nullptr;
    uint64_t gen_ = 0;
    int remaining_ = 0;
    bool stop_ = false;
};

}  // namespace

struct scrs_stripe_batch {
    uint64_t max_stripes = 0, max_items = 0;
    StatusWord status;
    DevBuf d_tasks, d_plans, d_counter, d_arena, d_item_task;
    std::vector<uint32_t> item_task;
    std::vector<MxkTask> tasks;
    std::vector<CauchyPlanTask> plans;    // GF(256) decode plans, then (from plans16_lo) the tower ones
    std::vector<uint8_t> task_gf16;       // per task: a tower stripe
    std::vector<uint8_t> arena;
    uint32_t total_items = 0, max_in = 1, max_plan_r = 0;
    // Tower stripes (GF((2^8)^2)) take the items [gen_hi, total_items) and
    // their own persistent drain; their plans are plans[plans16_lo, end).
    uint32_t gen_hi = 0, max_in16 = 1, max_plan_r16 = 0, plans16_lo = 0;
    int shape16 = kShapeAny;
    std::map<std::pair<uint32_t, uint32_t>, std::vector<uint16_t>> tower_coef;  // host tables by (k, m)
    std::vector<uint16_t> l_row_of, l_missing, l_present, l_repairs;  // per-stripe list scratch
    std::vector<uint8_t> l_seen;
    scrs_tune_key key{};  // geometry key of the current GF(256) descriptors (autotuner table)
    // Encode groups of one (engine, k, m) run through a kernel specialised to
    // their matrix (jit.cu): items [item_lo, item_hi) each; the generic drain
    // takes items [gen_lo, gen_hi).
    struct SpecRun {
        JitKernel jk;
        uint32_t item_lo, item_hi;
        uint64_t stripes;
    };
    bool jit = true;
    std::vector<SpecRun> spec;
    uint32_t gen_lo = 0;
    cudaGraphExec_t graph = nullptr;
    uint64_t graph_version = 0;   // autotuner table version the graph was captured under
    uint64_t graph_launches = 0;  // kernels in the captured graph
    uint64_t last_launches = 0;
    int sm_count = 0;
    std::vector<uint32_t> plan_begin;  // plans of stripes before stripe s
    PinnedBuf upload;                  // staging of asynchronous set uploads
    // host-buffer mode
    struct Copy {
        const void* src;
        void* dst;
        size_t bytes;
        uint32_t part_lo, part_hi;  // the stripes' own copies this one merges
        bool split;                 // the driver refused the merged form
    };
    struct Piece {
        uint32_t item_lo, item_hi, plan_lo, plan_hi;
        size_t h2d_lo, h2d_hi, d2h_lo, d2h_hi;
    };
    bool host_mode = false;
    // decode stripes of a host-buffer batch (see the top of this file)
    struct RowCopy {
        const uint8_t* src;
        uint8_t* dst;
        size_t bytes;
    };
    bool compact_decode = false;            // set_impl builds compact decode tasks (set_host)
    PinnedBuf h_missing;                    // the missing rows, compact, as the device returns them
    std::vector<RowCopy> present_copies;    // caller's input row -> caller's output row
    std::vector<RowCopy> missing_copies;    // h_missing row -> caller's output row, by piece
    std::vector<size_t> missing_at;         // first missing copy of each piece, then the total
    std::unique_ptr<HostPool> pool;
    DevBuf stage_in, stage_out;
    std::vector<Copy> h2d, d2h;              // merged copies
    std::vector<Copy> h2d_parts, d2h_parts;  // one per stripe
    std::vector<Piece> pieces;
    cudaStream_t s_in = nullptr, s_out = nullptr;
    std::vector<cudaEvent_t> events;  // start, end, per piece: copied in, computed; then per piece: copied out
    // recorded on a run's stream after its work: the next set waits for it
    // before it rewrites the device descriptors and staging that run reads
    cudaEvent_t ran = nullptr;
    bool ran_pending = false;
    // branch of a run for the specialised drains (see enqueue_batch)
    cudaStream_t s_fork = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    int shape = kShapeAny;  // kShapeAligned / kShapeWhole when every task satisfies it (launch_gf256_mxk)
    ~scrs_stripe_batch() {
        if (ran) cudaEventDestroy(ran);
        if (ev_fork) cudaEventDestroy(ev_fork);
        if (ev_join) cudaEventDestroy(ev_join);
        if (s_fork) cudaStreamDestroy(s_fork);
        if (graph) cudaGraphExecDestroy(graph);
        for (cudaEvent_t e : events) cudaEventDestroy(e);
        if (s_in) cudaStreamDestroy(s_in);
        if (s_out) cudaStreamDestroy(s_out);
    }
};

namespace {
constexpr size_t kMaxPieces = 64;  // one work counter each in d_counter
constexpr size_t kMaxSpecRuns = 4;  // specialised groups per batch (counters 1..4)
constexpr size_t kTowerCounter = 1 + kMaxSpecRuns;  // work counter of the tower drain

// g^i for i < 65535 (tower/cauchy.rs:44-49) on the current device: the x and
// y coordinates every tower decode plan reads.  Uploaded once per device.
cudaError_t tower_powers_table(const uint16_t** out) {
    static std::mutex mu;
    static std::map<int, std::unique_ptr<DevBuf>> tables;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(mu);
    auto it = tables.find(dev);
    if (it == tables.end()) {
        std::vector<uint16_t> pw(65535);
        hf::tower_powers(65535, pw.data());
        std::unique_ptr<DevBuf> t(new (std::nothrow) DevBuf());
        if (!t) return cudaErrorMemoryAllocation;
        if ((e = t->ensure(65535 * 2)) != cudaSuccess || (e = upload_now(t->p, pw.data(), 65535 * 2)) != cudaSuccess)
            return e;
        it = tables.emplace(dev, std::move(t)).first;
    }
    *out = it->second->as<uint16_t>();
    return cudaSuccess;
}
// A group is specialised when it has at least one persistent grid of items
// (this many CTAs per SM on every SM).
constexpr uint64_t kJitMinCtasPerSm = 8;
}

extern "C" int32_t scrs_stripe_batch_create(uint64_t max_stripes, uint64_t max_items, scrs_stripe_batch** out,
                                            scrs_error* err) {
    if (!out) return set_err(err, SCRS_ERR_NULL_ARGUMENT);
    if (max_stripes == 0 || max_stripes > (1u << 24) || max_items > 0xFFFFFFFFull)
        return set_err(err, SCRS_ERR_BAD_ARGUMENT, 1);
    std::unique_ptr<scrs_stripe_batch> b(new (std::nothrow) scrs_stripe_batch());
    if (!b) return set_err(err, SCRS_ERR_OUT_OF_MEMORY, sizeof(scrs_stripe_batch));
    b->max_stripes = max_stripes;
    b->max_items = max_items ? max_items : 0xFFFFFFFFull;
    int dev = 0;
    SCRS_CUDA(cudaGetDevice(&dev));
    SCRS_CUDA(cudaDeviceGetAttribute(&b->sm_count, cudaDevAttrMultiProcessorCount, dev));
    SCRS_CUDA(b->status.init());
    SCRS_CUDA(cudaEventCreateWithFlags(&b->ran, cudaEventDisableTiming));
    SCRS_CUDA(cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming));
    SCRS_CUDA(cudaEventCreateWithFlags(&b->ev_join, cudaEventDisableTiming));
    SCRS_CUDA(cudaStreamCreateWithFlags(&b->s_fork, cudaStreamNonBlocking));
    SCRS_CUDA(b->d_tasks.ensure(max_stripes * sizeof(MxkTask)));
    SCRS_CUDA(b->d_plans.ensure(max_stripes * sizeof(CauchyPlanTask)));
    SCRS_CUDA(b->d_counter.ensure(kMaxPieces * sizeof(uint32_t)));
    b->tasks.reserve(max_stripes);
    b->plans.reserve(max_stripes);
    *out = b.release();
    return set_err(err, SCRS_OK);
}

extern "C" void scrs_stripe_batch_destroy(scrs_stripe_batch* b) { delete b; }

extern "C" uint64_t scrs_stripe_batch_last_launches(const scrs_stripe_batch* b) {
    return b ? b->last_launches : 0;
}

namespace scrs {
// set() with the uploads either synchronous (async_stream == false) or staged
// through pinned memory and enqueued on `stream` (the serving loop's form:
// no host wait; the batch must not be set again before that stream has run
// the uploads).
int32_t stripe_batch_set_impl(scrs_stripe_batch* b, const scrs_stripe_desc* descs, uint64_t count, bool async_stream,
                              cudaStream_t stream, scrs_error* err);
}  // namespace scrs

extern "C" int32_t scrs_stripe_batch_set(scrs_stripe_batch* b, const scrs_stripe_desc* descs, uint64_t count,
                                         scrs_error* err) {
    return stripe_batch_set_impl(b, descs, count, false, nullptr, err);
}

namespace {

// Wait (on the host, or on `stream` for the staged form) for the last run's
// reads of the device descriptors and staging before they are rewritten.
int32_t wait_last_run(scrs_stripe_batch* b, bool async_stream, cudaStream_t stream, scrs_error* err) {
    if (!b->ran_pending) return SCRS_OK;
    if (async_stream)
        SCRS_CUDA(cudaStreamWaitEvent(stream, b->ran, 0));
    else
        SCRS_CUDA(cudaEventSynchronize(b->ran));
    b->ran_pending = false;
    return SCRS_OK;
}

// Shape flags of a generic drain launch staging seg_rows rows per segment:
// the batch's set-time flags, plus kShapeOneSeg when every generic task fits
// one segment (batch tasks never accumulate).
int drain_shape(const scrs_stripe_batch* b, int seg_rows) {
    return b->shape | ((int)b->max_in <= seg_rows ? kShapeOneSeg : 0);
}

// The end of a run on `st`: record it for the next set.
int32_t ran_on(scrs_stripe_batch* b, cudaStream_t st, scrs_error* err) {
    SCRS_CUDA(cudaEventRecord(b->ran, st));
    b->ran_pending = true;
    return set_err(err, SCRS_OK);
}

}  // namespace

int32_t scrs::stripe_batch_set_impl(scrs_stripe_batch* b, const scrs_stripe_desc* descs, uint64_t count,
                                    bool async_stream, cudaStream_t stream, scrs_error* err) {
    if (!b || (count && !descs)) return set_err(err, SCRS_ERR_NULL_ARGUMENT);
    if (count > b->max_stripes) return set_err(err, SCRS_ERR_CAPACITY, count, b->max_stripes);
    int32_t rw = wait_last_run(b, async_stream, stream, err);
    if (rw) return rw;
    // ---- validate and size the arena: [encode coefficient tables][decode slots]
    size_t coef_bytes = 0, slot_bytes = 0;
    std::map<std::tuple<int, uint32_t, uint32_t>, size_t> coef_off;
    uint64_t items = 0, n_tower = 0;
    auto align16 = [](size_t x) { return (x + 15) & ~(size_t)15; };
    for (uint64_t s = 0; s < count; s++) {
        const scrs_stripe_desc& d = descs[s];
        if (d.op != SCRS_OP_ENCODE && d.op != SCRS_OP_DECODE) return set_err(err, SCRS_ERR_BAD_ARGUMENT, 1, s);
        const bool gf16 = d.engine == SCRS_ENGINE_TOWER;
        if (d.engine != SCRS_ENGINE_STANDARD_CAUCHY && d.engine != SCRS_ENGINE_GOOD_CAUCHY && !gf16)
            return set_err(err, SCRS_ERR_BAD_ARGUMENT, 2, s);
        if (d.k == 0 || d.m == 0) return set_err(err, SCRS_CONFIG_ZERO_DIMENSION, 0, s);
        if (d.symbol_len == 0) return set_err(err, SCRS_CONFIG_ZERO_SYMBOL_LEN, 0, s);
        if (gf16 && d.symbol_len % 2) return set_err(err, SCRS_CONFIG_ODD_SYMBOL_LEN, 0, s);
        const uint64_t cap = d.engine == SCRS_ENGINE_STANDARD_CAUCHY ? 256 : gf16 ? 65535 : 255;
        if ((uint64_t)d.k + d.m > cap) return set_err(err, SCRS_CONFIG_TOO_MANY_SYMBOLS, cap, s);
        if (!d.in || !d.out) return set_err(err, SCRS_ERR_NULL_ARGUMENT, 0, s);
        const size_t elem = gf16 ? 2 : 1;
        n_tower += gf16;
        items += n_chunks(d.symbol_len, gf16);
        if (d.op == SCRS_OP_ENCODE) {
            auto key = std::make_tuple(d.engine, d.k, d.m);
            if (!coef_off.count(key)) {
                coef_off[key] = coef_bytes;
                coef_bytes = align16(coef_bytes + (size_t)d.k * d.m * elem);
            }
        } else {
            if (!d.indices) return set_err(err, SCRS_ERR_NULL_ARGUMENT, 0, s);
            const uint32_t n = d.k + d.m;
            std::vector<uint8_t>& seen = b->l_seen;
            seen.assign(n, 0);
            uint32_t r = 0;
            for (uint32_t q = 0; q < d.k; q++) {
                uint32_t i = d.indices[q];
                if (i >= n) return set_err(err, SCRS_DECODE_INDEX_OUT_OF_RANGE, i, n);
                if (seen[i]) return set_err(err, SCRS_DECODE_DUPLICATE_INDEX, i, s);
                seen[i] = 1;
                if (i >= d.k) r++;
            }
            // lists: in_rows[k] pass_rows[k] out_rows[r] missing[r] repairs[r] present[k-r]; coef[k*r]
            slot_bytes = align16(slot_bytes + 2 * ((size_t)3 * d.k + 3 * r));
            slot_bytes = align16(slot_bytes + (size_t)d.k * std::max<uint32_t>(r, 1) * elem);
        }
    }
    if (items > b->max_items || items > 0xFFFFFFFFull) return set_err(err, SCRS_ERR_CAPACITY, items, b->max_items);
    if (n_tower && b->compact_decode) return set_err(err, SCRS_ERR_BAD_ARGUMENT, 2);  // host-buffer batches: GF(256)
    const uint16_t* d_powers = nullptr;
    if (n_tower) SCRS_CUDA(tower_powers_table(&d_powers));
    const size_t arena_bytes = coef_bytes + slot_bytes;
    b->arena.assign(arena_bytes + 16, 0);
    SCRS_CUDA(b->d_arena.ensure_grow(b->arena.size()));
    uint8_t* dbase = b->d_arena.as<uint8_t>();
    for (auto& kv : coef_off) {
        const int engine = std::get<0>(kv.first);
        const uint32_t k = std::get<1>(kv.first), m = std::get<2>(kv.first);
        if (engine == SCRS_ENGINE_TOWER) {  // tower/cauchy.rs:69-106, cached per geometry
            std::vector<uint16_t>& t = b->tower_coef[std::make_pair(k, m)];
            if (t.empty()) {
                std::vector<uint16_t> pw(k + m);
                hf::tower_powers(k + m, pw.data());
                t.resize((size_t)k * m);
                hf::tower_coefficients(k, m, pw.data(), t.data());
            }
            memcpy(b->arena.data() + kv.second, t.data(), t.size() * 2);
        } else {
            hf::gf8_coefficients(engine, k, m, b->arena.data() + kv.second);
        }
    }
    // ---- tasks (tower plans are kept apart, then appended after the GF(256) ones)
    b->tasks.clear();
    b->task_gf16.clear();
    b->plans.clear();
    std::vector<CauchyPlanTask> plans16;
    b->plan_begin.assign(count + 1, 0);
    size_t off = coef_bytes;  // decode slots follow the coefficient tables
    uint32_t max_r = 0, max_r16 = 0;
    for (uint64_t s = 0; s < count; s++) {
        const scrs_stripe_desc& d = descs[s];
        const bool gf16 = d.engine == SCRS_ENGINE_TOWER;
        const size_t elem = gf16 ? 2 : 1;
        b->plan_begin[s] = (uint32_t)b->plans.size();
        MxkTask T{};
        T.in = d.in;
        T.out = d.out;
        T.L = d.symbol_len;
        T.in_stride = d.symbol_len;
        T.out_stride = d.symbol_len;
        T.n_in = d.k;
        T.n_items = n_chunks(d.symbol_len, gf16);
        T.aligned = (d.symbol_len % 16 == 0 && aligned16(d.in) && aligned16(d.out)) ? 1u : 0u;
        if (d.op == SCRS_OP_ENCODE) {
            T.coef = dbase + coef_off[std::make_tuple(d.engine, d.k, d.m)];
            T.n_out = d.m;
            T.ld = d.m;
        } else {
            const uint32_t k = d.k, n = d.k + d.m;
            std::vector<uint16_t>&row_of = b->l_row_of, &missing = b->l_missing, &present = b->l_present,
                                 &repairs = b->l_repairs;
            row_of.assign(n, kNoRow);
            missing.clear();
            present.clear();
            repairs.clear();
            for (uint32_t q = 0; q < k; q++) row_of[d.indices[q]] = (uint16_t)q;
            for (uint32_t i = 0; i < k; i++) (row_of[i] != kNoRow ? present : missing).push_back((uint16_t)i);
            for (uint32_t j = 0; j < d.m; j++)
                if (row_of[k + j] != kNoRow) repairs.push_back((uint16_t)j);
            const uint32_t r = (uint32_t)missing.size(), p = (uint32_t)present.size();
            uint16_t* L16 = reinterpret_cast<uint16_t*>(b->arena.data() + off);
            uint16_t* in_rows = L16;
            uint16_t* pass_rows = L16 + k;
            uint16_t* out_rows = L16 + 2 * k;
            uint16_t* l_missing = out_rows + r;
            uint16_t* l_repairs = l_missing + r;
            uint16_t* l_present = l_repairs + r;
            for (uint32_t t = 0; t < r; t++) in_rows[t] = row_of[k + repairs[t]], pass_rows[t] = kNoRow;
            for (uint32_t z = 0; z < p; z++) in_rows[r + z] = row_of[present[z]], pass_rows[r + z] = present[z];
            std::copy(missing.begin(), missing.end(), out_rows);
            std::copy(missing.begin(), missing.end(), l_missing);
            std::copy(repairs.begin(), repairs.end(), l_repairs);
            std::copy(present.begin(), present.end(), l_present);
            const size_t dl = (size_t)(reinterpret_cast<uint8_t*>(L16) - b->arena.data());
            uint16_t* dL16 = reinterpret_cast<uint16_t*>(dbase + dl);
            off = align16(off + 2 * ((size_t)3 * k + 3 * r));
            uint8_t* dcoef = dbase + off;
            off = align16(off + (size_t)k * std::max<uint32_t>(r, 1) * elem);
            T.in_rows = dL16;
            // compact (host-buffer batches): the r missing rows only, as rows
            // 0..r-1 of `out`; the present rows never leave the host
            T.pass_rows = b->compact_decode ? nullptr : dL16 + k;
            T.out_rows = b->compact_decode ? nullptr : dL16 + 2 * k;
            T.coef = dcoef;
            T.n_out = r;
            T.ld = std::max<uint32_t>(r, 1);
            if (r) {
                CauchyPlanTask P{};
                P.r = r;
                P.p = p;
                P.ld = r;
                P.engine = (uint32_t)d.engine;
                P.k = k;
                P.missing = dL16 + 2 * k + r;
                P.repairs = dL16 + 2 * k + 2 * r;
                P.present = dL16 + 2 * k + 3 * r;
                P.powers = gf16 ? d_powers : nullptr;
                P.coef = dcoef;
                if (gf16) {
                    plans16.push_back(P);
                    max_r16 = std::max(max_r16, r);
                } else {
                    b->plans.push_back(P);
                    max_r = std::max(max_r, r);
                }
            }
        }
        b->tasks.push_back(T);
        b->task_gf16.push_back(gf16 ? 1 : 0);
    }
    b->plan_begin[count] = (uint32_t)b->plans.size();
    b->plans16_lo = (uint32_t)b->plans.size();
    b->plans.insert(b->plans.end(), plans16.begin(), plans16.end());
    b->max_plan_r = max_r;
    b->max_plan_r16 = max_r16;
    if (n_tower) {  // the autotuner's key describes the GF(256) stripes (the drain it tunes)
        std::vector<scrs_stripe_desc> gf8;
        for (uint64_t s = 0; s < count; s++)
            if (descs[s].engine != SCRS_ENGINE_TOWER) gf8.push_back(descs[s]);
        b->key = tune_key_of(gf8.data(), gf8.size());
    } else {
        b->key = tune_key_of(descs, count);
    }
    // ---- items: specialised GF(256) encode groups, the generic GF(256)
    // drain's tasks, then the tower tasks (each task in stripe order)
    b->spec.clear();
    std::vector<char> in_spec(count, 0);
    uint32_t next = 0;
    if (b->jit) {
        std::map<std::tuple<int, uint32_t, uint32_t>, std::vector<uint32_t>> groups;
        std::vector<std::tuple<int, uint32_t, uint32_t>> order;  // first appearance
        for (uint64_t s = 0; s < count; s++) {
            const scrs_stripe_desc& d = descs[s];
            if (d.op != SCRS_OP_ENCODE || d.engine == SCRS_ENGINE_TOWER || !jit_eligible(d.k, d.m)) continue;
            auto key = std::make_tuple(d.engine, d.k, d.m);
            auto& g = groups[key];
            if (g.empty()) order.push_back(key);
            g.push_back((uint32_t)s);
        }
        for (auto& key : order) {
            if (b->spec.size() == kMaxSpecRuns) break;
            auto& g = groups[key];
            uint64_t n = 0;
            for (uint32_t t : g) n += b->tasks[t].n_items;
            JitKernel jk{};
            scrs_error je{};
            if (n < kJitMinCtasPerSm * (uint64_t)b->sm_count ||
                jit_kernel(std::get<0>(key), std::get<1>(key), std::get<2>(key), true, &jk, &je) != SCRS_OK)
                continue;  // too small to fill the GPU, or not compiled: the generic drain runs it
            const uint32_t lo = next;
            for (uint32_t t : g) {
                b->tasks[t].item_begin = next;
                next += b->tasks[t].n_items;
                in_spec[t] = 1;
            }
            b->spec.push_back({jk, lo, next, (uint64_t)g.size()});
        }
    }
    b->gen_lo = next;
    uint32_t max_in = 1, max_in16 = 1;
    for (int pass = 0; pass < 2; pass++) {
        for (uint64_t t = 0; t < count; t++) {
            if (in_spec[t] || b->task_gf16[t] != pass) continue;
            b->tasks[t].item_begin = next;
            next += b->tasks[t].n_items;
            uint32_t& mx = pass ? max_in16 : max_in;
            mx = std::max(mx, b->tasks[t].n_in);
        }
        if (pass == 0) b->gen_hi = next;
    }
    b->total_items = next;
    b->max_in = max_in;
    b->max_in16 = max_in16;
    auto shape_of = [&](uint8_t gf16) {
        bool all_aligned = true, all_whole = true;
        for (size_t t = 0; t < b->tasks.size(); t++) {
            if (b->task_gf16[t] != gf16) continue;
            all_aligned &= b->tasks[t].aligned != 0;
            all_whole &= b->tasks[t].L % FieldGeom<0>::kChunk == 0;
        }
        return !all_aligned ? kShapeAny : all_whole ? (kShapeAligned | kShapeWhole) : kShapeAligned;
    };
    b->shape = shape_of(0);
    b->shape16 = shape_of(1);
    b->item_task.resize(next);
    for (size_t t = 0; t < b->tasks.size(); t++)
        std::fill(b->item_task.begin() + b->tasks[t].item_begin,
                  b->item_task.begin() + b->tasks[t].item_begin + b->tasks[t].n_items, (uint32_t)t);
    SCRS_CUDA(b->d_item_task.ensure_grow((size_t)next * 4));
    if (off > arena_bytes) return set_err(err, SCRS_ERR_CAPACITY, off, arena_bytes);  // layout invariant
    struct Up {
        void* dst;
        const void* src;
        size_t bytes;
    } ups[4] = {{b->d_item_task.p, b->item_task.data(), (size_t)next * 4},
                {b->d_arena.p, b->arena.data(), b->arena.size()},
                {b->d_tasks.p, b->tasks.data(), b->tasks.size() * sizeof(MxkTask)},
                {b->d_plans.p, b->plans.data(), b->plans.size() * sizeof(CauchyPlanTask)}};
    if (async_stream) {
        size_t total = 0;
        for (auto& u : ups) total += (u.bytes + 15) & ~(size_t)15;
        if (total > b->upload.bytes) SCRS_CUDA(b->upload.ensure(total + total / 2));
        uint8_t* h = b->upload.as<uint8_t>();
        for (auto& u : ups) {
            if (!u.bytes) continue;
            memcpy(h, u.src, u.bytes);
            SCRS_CUDA(cudaMemcpyAsync(u.dst, h, u.bytes, cudaMemcpyHostToDevice, stream));
            h += (u.bytes + 15) & ~(size_t)15;
        }
    } else {
        for (auto& u : ups) SCRS_CUDA(upload_now(u.dst, u.src, u.bytes));
    }
    b->host_mode = false;  // scrs_stripe_batch_set_host re-enables it after this call
    if (b->graph) {  // geometry changed: the captured graph no longer applies
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    return set_err(err, SCRS_OK);
}

extern "C" int32_t scrs_stripe_batch_set_host(scrs_stripe_batch* b, const scrs_stripe_desc* descs,
                                              uint64_t count, scrs_error* err) {
    if (!b || (count && !descs)) return set_err(err, SCRS_ERR_NULL_ARGUMENT);
    if (count > b->max_stripes) return set_err(err, SCRS_ERR_CAPACITY, count, b->max_stripes);
    int32_t rw = wait_last_run(b, false, nullptr, err);  // the staging below may be reallocated
    if (rw) return rw;
    // Output rows per stripe on the device: m repairs, or the r missing data
    // rows of a decode (indices are validated by the set below; a bad list
    // only sizes the staging here).
    auto rows_out = [](const scrs_stripe_desc& d) -> uint64_t {
        if (d.op != SCRS_OP_DECODE) return d.m;
        uint64_t r = 0;
        for (uint32_t q = 0; q < d.k; q++) r += d.indices[q] >= d.k;
        return r;
    };
    size_t in_bytes = 0, out_bytes = 0, miss_bytes = 0;
    for (uint64_t s = 0; s < count; s++) {
        const scrs_stripe_desc& d = descs[s];
        if (!d.in || !d.out || (d.op == SCRS_OP_DECODE && !d.indices))
            return set_err(err, SCRS_ERR_NULL_ARGUMENT, 0, s);
        const uint64_t ob = rows_out(d) * d.symbol_len;
        in_bytes += (((uint64_t)d.k * d.symbol_len) + 15) & ~15ull;
        out_bytes += (ob + 15) & ~15ull;
        if (d.op == SCRS_OP_DECODE) miss_bytes += (ob + 15) & ~15ull;
    }
    SCRS_CUDA(b->stage_in.ensure(in_bytes));
    SCRS_CUDA(b->stage_out.ensure(out_bytes));
    SCRS_CUDA(b->h_missing.ensure(miss_bytes));
    std::vector<scrs_stripe_desc> dev(descs, descs + count);
    b->h2d.clear();
    b->d2h.clear();
    b->h2d_parts.clear();
    b->d2h_parts.clear();
    b->present_copies.clear();
    b->missing_copies.clear();
    b->missing_at.clear();
    // piece boundaries: about equal input bytes per piece
    const size_t n_pieces = std::min<size_t>(kMaxPieces, std::max<uint64_t>(count, 1));
    std::vector<uint64_t> cut;  // first stripe of each piece, then count
    size_t oi = 0, oo = 0, om = 0, acc = 0;
    for (uint64_t s = 0; s < count; s++) {
        const size_t ib = (size_t)descs[s].k * descs[s].symbol_len;
        if (cut.empty() || (acc * n_pieces >= in_bytes * cut.size() && cut.size() < n_pieces)) cut.push_back(s);
        acc += (ib + 15) & ~(size_t)15;
    }
    cut.push_back(count);
    std::vector<size_t> h2d_at, d2h_at;  // copy-list positions of each piece
    size_t piece = 0;
    for (uint64_t s = 0; s < count; s++) {
        const scrs_stripe_desc& d = descs[s];
        const bool first = s == cut[piece];
        if (first) {
            h2d_at.push_back(b->h2d.size());
            d2h_at.push_back(b->d2h.size());
            b->missing_at.push_back(b->missing_copies.size());
        }
        const uint64_t L = d.symbol_len;
        const size_t ib = (size_t)d.k * L, ob = (size_t)rows_out(d) * L;
        uint8_t* din = b->stage_in.as<uint8_t>() + oi;
        uint8_t* dout = b->stage_out.as<uint8_t>() + oo;
        // device outputs land in the caller's buffer (repairs) or in the
        // missing-row staging (decodes)
        uint8_t* hout = d.op == SCRS_OP_DECODE ? b->h_missing.as<uint8_t>() + om : d.out;
        dev[s].in = din;
        dev[s].out = dout;
        if (d.op == SCRS_OP_DECODE) {
            const uint32_t k = d.k;
            uint16_t row_of[256];
            std::fill(row_of, row_of + std::min<uint32_t>(k, 256), kNoRow);
            for (uint32_t q = 0; q < k; q++)
                if (d.indices[q] < k && d.indices[q] < 256) row_of[d.indices[q]] = (uint16_t)q;
            uint32_t t = 0;
            for (uint32_t i = 0; i < k && i < 256; i++) {
                if (row_of[i] != kNoRow)
                    b->present_copies.push_back({d.in + (size_t)row_of[i] * L, d.out + (size_t)i * L, L});
                else
                    b->missing_copies.push_back({hout + (size_t)(t++) * L, d.out + (size_t)i * L, L});
            }
        }
        // merge with the previous copy of the same piece when both sides are
        // contiguous (the stripe's own copy is kept in case the driver refuses
        // a merged copy whose host side spans two allocations)
        const uint32_t part = (uint32_t)b->h2d_parts.size();
        b->h2d_parts.push_back({d.in, din, ib, part, part + 1, false});
        b->d2h_parts.push_back({dout, hout, ob, part, part + 1, false});
        if (!first && (const uint8_t*)b->h2d.back().src + b->h2d.back().bytes == d.in &&
            (uint8_t*)b->h2d.back().dst + b->h2d.back().bytes == din) {
            b->h2d.back().bytes += ib;
            b->h2d.back().part_hi = part + 1;
        } else {
            b->h2d.push_back({d.in, din, ib, part, part + 1, false});
        }
        if (ob) {
            const bool joins = b->d2h.size() > d2h_at.back() &&
                               (const uint8_t*)b->d2h.back().src + b->d2h.back().bytes == dout &&
                               (uint8_t*)b->d2h.back().dst + b->d2h.back().bytes == hout;
            if (joins) {
                b->d2h.back().bytes += ob;
                b->d2h.back().part_hi = part + 1;
            } else {
                b->d2h.push_back({dout, hout, ob, part, part + 1, false});
            }
        }
        oi += (ib + 15) & ~(size_t)15;
        oo += (ob + 15) & ~(size_t)15;
        if (d.op == SCRS_OP_DECODE) om += (ob + 15) & ~(size_t)15;
        if (s + 1 == cut[piece + 1]) piece++;
    }
    b->missing_at.push_back(b->missing_copies.size());
    const bool jit = b->jit;  // pieces are stripe ranges: keep the items in stripe order
    b->jit = false;
    b->compact_decode = true;
    int32_t r = scrs_stripe_batch_set(b, dev.data(), count, err);
    b->jit = jit;
    b->compact_decode = false;
    if (r) return r;
    b->pieces.clear();
    for (size_t q = 0; q + 1 < cut.size(); q++) {
        const uint64_t s0 = cut[q], s1 = cut[q + 1];
        scrs_stripe_batch::Piece P{};
        P.item_lo = b->tasks[s0].item_begin;
        P.item_hi = s1 < count ? b->tasks[s1].item_begin : b->total_items;
        P.plan_lo = b->plan_begin[s0];
        P.plan_hi = b->plan_begin[s1];
        P.h2d_lo = h2d_at[q];
        P.h2d_hi = q + 1 < h2d_at.size() ? h2d_at[q + 1] : b->h2d.size();
        P.d2h_lo = d2h_at[q];
        P.d2h_hi = q + 1 < d2h_at.size() ? d2h_at[q + 1] : b->d2h.size();
        b->pieces.push_back(P);
    }
    if (!b->s_in) SCRS_CUDA(cudaStreamCreateWithFlags(&b->s_in, cudaStreamNonBlocking));
    if (!b->s_out) SCRS_CUDA(cudaStreamCreateWithFlags(&b->s_out, cudaStreamNonBlocking));
    while (b->events.size() < 2 + 3 * kMaxPieces) {
        cudaEvent_t e;
        SCRS_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        b->events.push_back(e);
    }
    if (!b->pool) {
        b->pool.reset(new (std::nothrow) HostPool());
        if (!b->pool) return set_err(err, SCRS_ERR_OUT_OF_MEMORY, sizeof(HostPool));
        const unsigned hw = std::thread::hardware_concurrency();
        b->pool->start((int)std::max(1u, std::min(8u, hw ? hw / 2 : 1u)));
        if (b->pool->size() == 0) return set_err(err, SCRS_ERR_OUT_OF_MEMORY, sizeof(std::thread));
    }
    b->host_mode = true;
    return set_err(err, SCRS_OK);
}

namespace {

// Enqueue merged copy `c` on `st`.  Host buffers of consecutive stripes may
// touch without being one allocation; the driver refuses a copy spanning
// two (cudaErrorInvalidValue, nothing enqueued), and such a copy is split
// into its stripes' own copies, now and on every later run.
int32_t issue_copy(scrs_stripe_batch::Copy& c, const std::vector<scrs_stripe_batch::Copy>& parts,
                   cudaMemcpyKind kind, cudaStream_t st, scrs_error* err) {
    if (!c.split) {
        const cudaError_t e = cudaMemcpyAsync(c.dst, c.src, c.bytes, kind, st);
        if (e == cudaSuccess) return SCRS_OK;
        if (e != cudaErrorInvalidValue || c.part_hi - c.part_lo < 2) return set_err(err, SCRS_ERR_CUDA, e, __LINE__);
        cudaGetLastError();
        c.split = true;
    }
    for (uint32_t q = c.part_lo; q < c.part_hi; q++)
        SCRS_CUDA(cudaMemcpyAsync(parts[q].dst, parts[q].src, parts[q].bytes, kind, st));
    return SCRS_OK;
}

int32_t copy_in(scrs_stripe_batch* b, cudaStream_t st, scrs_error* err) {
    if (!b->host_mode) return SCRS_OK;
    for (auto& c : b->h2d) {
        int32_t r = issue_copy(c, b->h2d_parts, cudaMemcpyHostToDevice, st, err);
        if (r) return r;
    }
    return SCRS_OK;
}

int32_t copy_out(scrs_stripe_batch* b, cudaStream_t st, scrs_error* err) {
    if (!b->host_mode) return SCRS_OK;
    for (auto& c : b->d2h) {
        int32_t r = issue_copy(c, b->d2h_parts, cudaMemcpyDeviceToHost, st, err);
        if (r) return r;
    }
    return SCRS_OK;
}

// Drain launch parameters: the autotuner's entry for the batch's key, else
// min(largest k, 16) rows per segment and the most CTAs per SM that fit.
struct DrainCfg {
    int seg_rows, ctas_per_sm, grid;
};

DrainCfg drain_cfg(const scrs_stripe_batch* b) {
    DrainCfg c{mxk_default_seg((int)b->max_in), 0, 0};
    scrs_tune_params p{};
    if (tune_lookup(b->key, &p)) {
        c.seg_rows = std::max(1, std::min({(int)p.seg_rows, (int)b->max_in, FieldGeom<0>::kSegMax}));
        c.ctas_per_sm = (int)p.ctas_per_sm;
    }
    const int fit = mxk_ctas_per_sm(c.seg_rows, drain_shape(b, c.seg_rows));
    if (c.ctas_per_sm <= 0 || c.ctas_per_sm > fit) c.ctas_per_sm = fit;
    const uint32_t items = b->gen_hi - b->gen_lo;
    c.grid = std::max(1, std::min<int>(b->sm_count * c.ctas_per_sm, (int)std::max<uint32_t>(items, 1)));
    return c;
}

// The tower stripes' drain: all their inputs per segment up to 16 rows, the
// most CTAs per SM that fit.
DrainCfg drain_cfg16(const scrs_stripe_batch* b) {
    DrainCfg c{std::max(1, std::min((int)b->max_in16, FieldGeom<1>::kSegMax)), 0, 0};
    const int shape = b->shape16 | ((int)b->max_in16 <= c.seg_rows ? kShapeOneSeg : 0);
    c.ctas_per_sm = mxk_ctas_per_sm(c.seg_rows, shape, 1);
    const uint32_t items = b->total_items - b->gen_hi;
    c.grid = std::max(1, std::min<int>(b->sm_count * c.ctas_per_sm, (int)std::max<uint32_t>(items, 1)));
    return c;
}

// The drains of a device-resident run: the specialised groups' kernels, then
// the generic drain (work counter q + 1 for group q, 0 for the generic one).
int32_t enqueue_drains(scrs_stripe_batch* b, cudaStream_t st, scrs_error* err, bool run_spec = true,
                       bool run_generic = true) {
    for (size_t q = 0; run_spec && q < b->spec.size(); q++) {
        const scrs_stripe_batch::SpecRun& R = b->spec[q];
        SCRS_CUDA(launch_jit(R.jk, b->d_tasks.as<MxkTask>(), b->d_item_task.as<uint32_t>(), R.item_lo, R.item_hi,
                             b->d_counter.as<uint32_t>() + 1 + q, b->status.dev, b->sm_count * R.jk.ctas_per_sm, st));
        b->last_launches++;
    }
    if (run_generic && b->gen_hi > b->gen_lo) {
        const DrainCfg c = drain_cfg(b);
        SCRS_CUDA(launch_gf256_mxk(b->d_tasks.as<MxkTask>(), b->d_item_task.as<uint32_t>(), b->gen_lo, b->gen_hi,
                                   b->d_counter.as<uint32_t>(), b->status.dev, c.seg_rows, c.grid, st,
                                   drain_shape(b, c.seg_rows)));
        b->last_launches++;
    }
    if (run_generic && b->total_items > b->gen_hi) {
        const DrainCfg c = drain_cfg16(b);
        const int shape = b->shape16 | ((int)b->max_in16 <= c.seg_rows ? kShapeOneSeg : 0);
        SCRS_CUDA(launch_gf256_mxk(b->d_tasks.as<MxkTask>(), b->d_item_task.as<uint32_t>(), b->gen_hi,
                                   b->total_items, b->d_counter.as<uint32_t>() + kTowerCounter, b->status.dev,
                                   c.seg_rows, c.grid, st, shape, 1));
        b->last_launches++;
    }
    return SCRS_OK;
}

// The decode plans: GF(256) ones, then tower ones.
int32_t enqueue_plans(scrs_stripe_batch* b, cudaStream_t st, scrs_error* err) {
    if (b->plans16_lo) {
        SCRS_CUDA(launch_cauchy_plan(b->d_plans.as<CauchyPlanTask>(), b->plans16_lo, 0, b->max_plan_r, st));
        b->last_launches++;
    }
    if (b->plans.size() > b->plans16_lo) {
        SCRS_CUDA(launch_cauchy_plan(b->d_plans.as<CauchyPlanTask>() + b->plans16_lo,
                                     (uint32_t)b->plans.size() - b->plans16_lo, 1, b->max_plan_r16, st));
        b->last_launches++;
    }
    return SCRS_OK;
}

// One run on st.  With specialised drains and a generic one, the specialised
// drains go on a branch (s_fork, joined back before the run ends), so that
// they overlap the plan launch and the generic drain's CTAs take the SMs the
// specialised drains' tails leave idle; the drains touch disjoint items and
// outputs.  Under graph capture the fork and join become graph edges.
int32_t enqueue_batch(scrs_stripe_batch* b, cudaStream_t st, scrs_error* err) {
    SCRS_CUDA(cudaMemsetAsync(b->d_counter.p, 0, (kTowerCounter + 1) * sizeof(uint32_t), st));
    b->last_launches = 0;
    const bool fork = !b->spec.empty() && b->total_items > b->gen_lo;
    if (fork) {
        SCRS_CUDA(cudaEventRecord(b->ev_fork, st));
        SCRS_CUDA(cudaStreamWaitEvent(b->s_fork, b->ev_fork, 0));
        int32_t r = enqueue_drains(b, b->s_fork, err, true, false);
        if (r) return r;
    }
    int32_t rp = enqueue_plans(b, st, err);
    if (rp) return rp;
    if (!fork) return enqueue_drains(b, st, err);
    int32_t r = enqueue_drains(b, st, err, false, true);
    if (r) return r;
    SCRS_CUDA(cudaEventRecord(b->ev_join, b->s_fork));
    SCRS_CUDA(cudaStreamWaitEvent(st, b->ev_join, 0));
    return SCRS_OK;
}

// Row copy on a host worker that leaves the destination out of the caches:
// the rows are 4 KiB or so, below the size where memcpy itself switches to
// non-temporal stores, and a regular store first reads the destination line
// from host memory, which the copy engines are reading and writing at the
// same time.  16-byte aligned rows of whole 16-byte units take the streaming
// stores (the caller fences once after its copies); anything else memcpy.
void copy_row_streaming(uint8_t* dst, const uint8_t* src, size_t bytes) {
#if defined(__SSE2__)
    if (((reinterpret_cast<uintptr_t>(dst) | reinterpret_cast<uintptr_t>(src) | bytes) & 15) == 0) {
        __m128i* d = reinterpret_cast<__m128i*>(dst);
        const __m128i* s = reinterpret_cast<const __m128i*>(src);
        size_t n = bytes / 16, i = 0;
        for (; i + 4 <= n; i += 4) {
            const __m128i a = _mm_load_si128(s + i), b = _mm_load_si128(s + i + 1);
            const __m128i c = _mm_load_si128(s + i + 2), e = _mm_load_si128(s + i + 3);
            _mm_stream_si128(d + i, a);
            _mm_stream_si128(d + i + 1, b);
            _mm_stream_si128(d + i + 2, c);
            _mm_stream_si128(d + i + 3, e);
        }
        for (; i < n; i++) _mm_stream_si128(d + i, _mm_load_si128(s + i));
        return;
    }
#endif
    memcpy(dst, src, bytes);
}

void fence_streaming_stores() {
#if defined(__SSE2__)
    _mm_sfence();
#endif
}

// The host side of a host-buffer run's decode stripes, on the worker
// threads: first every present row (caller's input row -> output row), then
// piece by piece, once the piece's device->host copies are done (its event,
// or nothing to wait for when `pieces_done`), the missing rows from the
// staging.  Each worker takes a contiguous share of each list.
int32_t host_copies(scrs_stripe_batch* b, bool pieces_done, scrs_error* err) {
    if (b->present_copies.empty() && b->missing_copies.empty()) return SCRS_OK;
    std::atomic<int> failed{0};
    const int W = b->pool->size();
    const std::function<void(int)> work = [&](int w) {
        auto share = [&](size_t lo, size_t hi, int part) {
            const size_t n = hi - lo;
            return std::make_pair(lo + n * (size_t)part / (size_t)W, lo + n * (size_t)(part + 1) / (size_t)W);
        };
        const auto pr = share(0, b->present_copies.size(), w);
        for (size_t i = pr.first; i < pr.second; i++)
            copy_row_streaming(b->present_copies[i].dst, b->present_copies[i].src, b->present_copies[i].bytes);
        for (size_t q = 0; q + 1 < b->missing_at.size(); q++) {
            const auto mr = share(b->missing_at[q], b->missing_at[q + 1], w);
            if (mr.first == mr.second) continue;
            if (!pieces_done) {
                const cudaError_t e = cudaEventSynchronize(b->events[2 + 2 * kMaxPieces + q]);
                if (e != cudaSuccess) {
                    failed.store((int)e);
                    fence_streaming_stores();
                    return;
                }
            }
            for (size_t i = mr.first; i < mr.second; i++)
                copy_row_streaming(b->missing_copies[i].dst, b->missing_copies[i].src, b->missing_copies[i].bytes);
        }
        fence_streaming_stores();  // the stores are visible to the caller once run() returns
    };
    b->pool->run(work);
    if (failed.load()) return set_err(err, SCRS_ERR_CUDA, (uint64_t)failed.load(), __LINE__);
    return SCRS_OK;
}

// Host-buffer run: copies and compute of consecutive pieces overlap (see
// top).  Returns once the outputs are in the caller's buffers (the host
// copies of the decode stripes' rows are part of the run).
int32_t run_host(scrs_stripe_batch* b, cudaStream_t st, scrs_error* err) {
    cudaEvent_t ev_start = b->events[0], ev_end = b->events[1];
    SCRS_CUDA(cudaEventRecord(ev_start, st));
    SCRS_CUDA(cudaStreamWaitEvent(b->s_in, ev_start, 0));
    SCRS_CUDA(cudaStreamWaitEvent(b->s_out, ev_start, 0));
    SCRS_CUDA(cudaMemsetAsync(b->d_counter.p, 0, kMaxPieces * sizeof(uint32_t), st));
    const DrainCfg c = drain_cfg(b);
    b->last_launches = 0;
    for (size_t q = 0; q < b->pieces.size(); q++) {
        const scrs_stripe_batch::Piece& P = b->pieces[q];
        cudaEvent_t ev_in = b->events[2 + 2 * q], ev_done = b->events[3 + 2 * q];
        for (size_t i = P.h2d_lo; i < P.h2d_hi; i++) {
            int32_t r = issue_copy(b->h2d[i], b->h2d_parts, cudaMemcpyHostToDevice, b->s_in, err);
            if (r) return r;
        }
        SCRS_CUDA(cudaEventRecord(ev_in, b->s_in));
        SCRS_CUDA(cudaStreamWaitEvent(st, ev_in, 0));
        if (P.plan_hi > P.plan_lo) {
            SCRS_CUDA(launch_cauchy_plan(b->d_plans.as<CauchyPlanTask>() + P.plan_lo, P.plan_hi - P.plan_lo, 0,
                                         b->max_plan_r, st));
            b->last_launches++;
        }
        if (P.item_hi > P.item_lo) {
            SCRS_CUDA(launch_gf256_mxk(b->d_tasks.as<MxkTask>(), b->d_item_task.as<uint32_t>(), P.item_lo, P.item_hi,
                                       b->d_counter.as<uint32_t>() + q, b->status.dev, c.seg_rows, c.grid, st,
                                       drain_shape(b, c.seg_rows)));
            b->last_launches++;
        }
        SCRS_CUDA(cudaEventRecord(ev_done, st));
        SCRS_CUDA(cudaStreamWaitEvent(b->s_out, ev_done, 0));
        for (size_t i = P.d2h_lo; i < P.d2h_hi; i++) {
            int32_t r = issue_copy(b->d2h[i], b->d2h_parts, cudaMemcpyDeviceToHost, b->s_out, err);
            if (r) return r;
        }
        SCRS_CUDA(cudaEventRecord(b->events[2 + 2 * kMaxPieces + q], b->s_out));
    }
    SCRS_CUDA(cudaEventRecord(ev_end, b->s_out));
    SCRS_CUDA(cudaStreamWaitEvent(st, ev_end, 0));
    int32_t r = host_copies(b, false, err);
    if (r) return r;
    return ran_on(b, st, err);
}

}  // namespace

extern "C" int32_t scrs_stripe_batch_run(scrs_stripe_batch* b, void* stream, int32_t use_graph, scrs_error* err) {
    if (!b) return set_err(err, SCRS_ERR_NULL_ARGUMENT);
    cudaStream_t st = (cudaStream_t)stream;
    if (b->host_mode) return run_host(b, st, err);  // pipelined copies; no graph
    int32_t r0 = copy_in(b, st, err);
    if (r0) return r0;
    if (!use_graph) {
        int32_t r = enqueue_batch(b, st, err);
        if (r) return r;
        r = copy_out(b, st, err);
        if (r) return r;
        return ran_on(b, st, err);
    }
    if (b->graph && b->graph_version != tune_version()) {  // launch parameters may have changed
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    if (!b->graph) {
        SCRS_CUDA(prepare_batch_kernels());  // its one-time set-up cannot run inside the capture
        // Capture on a private stream so the legacy default stream can be used by callers.
        cudaStream_t cap;
        SCRS_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
        int32_t r = SCRS_OK;
        if (e == cudaSuccess) {
            r = enqueue_batch(b, cap, err);
            e = cudaStreamEndCapture(cap, &g);
        }
        cudaStreamDestroy(cap);
        if (r) {
            if (g) cudaGraphDestroy(g);
            return r;
        }
        SCRS_CUDA(e);
        b->graph_launches = b->last_launches;
        b->graph_version = tune_version();
        e = cudaGraphInstantiate(&b->graph, g, 0);
        cudaGraphDestroy(g);
        SCRS_CUDA(e);
    }
    SCRS_CUDA(cudaGraphLaunch(b->graph, st));
    b->last_launches = b->graph_launches;
    r0 = copy_out(b, st, err);
    if (r0) return r0;
    return ran_on(b, st, err);
}

extern "C" int32_t scrs_stripe_batch_run_plain(scrs_stripe_batch* b, void* stream, scrs_error* err) {
    if (!b) return set_err(err, SCRS_ERR_NULL_ARGUMENT);
    cudaStream_t st = (cudaStream_t)stream;
    int32_t r0 = copy_in(b, st, err);
    if (r0) return r0;
    b->last_launches = 0;
    size_t pi[2] = {0, b->plans16_lo};  // next plan of each field
    const size_t pend[2] = {b->plans16_lo, b->plans.size()};
    for (size_t t = 0; t < b->tasks.size(); t++) {
        const MxkTask& T = b->tasks[t];
        const int f = b->task_gf16[t];
        // decode stripes carry row lists (encodes none); with erasures they have a plan
        if (T.in_rows && T.n_out && pi[f] < pend[f]) {
            SCRS_CUDA(launch_cauchy_plan_single(b->plans[pi[f]++], f, st));
            b->last_launches++;
        }
        SCRS_CUDA(launch_mxk_single(T, f, b->status.dev, 0, st));
        b->last_launches++;
    }
    r0 = copy_out(b, st, err);
    if (r0) return r0;
    if (b->host_mode) {  // the decode stripes' rows on the host, after the copies back
        SCRS_CUDA(cudaStreamSynchronize(st));
        r0 = host_copies(b, true, err);
        if (r0) return r0;
    }
    return ran_on(b, st, err);
}

extern "C" int32_t scrs_stripe_batch_run_timed(scrs_stripe_batch* b, void* stream, float* plan_ms,
                                               float* drain_ms, scrs_error* err) {
    float spec = 0, gen = 0;
    int32_t rc = scrs_stripe_batch_run_timed_drains(b, stream, plan_ms, &spec, &gen, err);
    if (!rc && drain_ms) *drain_ms = spec + gen;
    return rc;
}

extern "C" int32_t scrs_stripe_batch_run_timed_drains(scrs_stripe_batch* b, void* stream, float* plan_ms,
                                                      float* spec_ms, float* generic_ms, scrs_error* err) {
    if (!b) return set_err(err, SCRS_ERR_NULL_ARGUMENT);
    cudaStream_t st = (cudaStream_t)stream;
    cudaEvent_t ev[4];
    for (auto& e : ev) SCRS_CUDA(cudaEventCreate(&e));
    SCRS_CUDA(cudaMemsetAsync(b->d_counter.p, 0, (kTowerCounter + 1) * sizeof(uint32_t), st));
    b->last_launches = 0;
    cudaEventRecord(ev[0], st);
    int32_t rp = enqueue_plans(b, st, err);
    if (rp) return rp;
    cudaEventRecord(ev[1], st);
    int32_t rc = enqueue_drains(b, st, err, false, true);
    if (rc) return rc;
    cudaEventRecord(ev[2], st);
    rc = enqueue_drains(b, st, err, true, false);
    if (rc) return rc;
    cudaEventRecord(ev[3], st);
    SCRS_CUDA(cudaEventSynchronize(ev[3]));
    float t[3] = {0, 0, 0};
    for (int i = 0; i < 3; i++) cudaEventElapsedTime(&t[i], ev[i], ev[i + 1]);
    for (auto& e : ev) cudaEventDestroy(e);
    if (plan_ms) *plan_ms = t[0];
    if (generic_ms) *generic_ms = t[1];
    if (spec_ms) *spec_ms = t[2];
    return set_err(err, SCRS_OK);
}

extern "C" int32_t scrs_stripe_batch_check(scrs_stripe_batch* b, scrs_error* err) {
    if (!b) return set_err(err, SCRS_ERR_NULL_ARGUMENT);
    int32_t r = take_status(b->status, err);
    if (r) return r;
    return set_err(err, SCRS_OK);
}

extern "C" int32_t scrs_stripe_batch_tune_key(const scrs_stripe_batch* b, scrs_tune_key* key, scrs_error* err) {
    if (!b || !key) return set_err(err, SCRS_ERR_NULL_ARGUMENT);
    *key = b->key;
    return set_err(err, SCRS_OK);
}

extern "C" int32_t scrs_stripe_batch_launch_params(const scrs_stripe_batch* b, scrs_tune_params* params,
                                                   scrs_error* err) {
    if (!b || !params) return set_err(err, SCRS_ERR_NULL_ARGUMENT);
    const DrainCfg c = drain_cfg(b);
    *params = scrs_tune_params{(uint32_t)c.seg_rows, (uint32_t)c.ctas_per_sm, 0.0f, 0};
    return set_err(err, SCRS_OK);
}

namespace {

// Median device time of `reps` drain launches (after one untimed launch).
int32_t time_drain(scrs_stripe_batch* b, cudaStream_t st, int seg_rows, int grid, uint32_t reps, cudaEvent_t e0,
                   cudaEvent_t e1, float* median_ms, scrs_error* err) {
    std::vector<float> t;
    for (uint32_t rep = 0; rep <= reps; rep++) {
        SCRS_CUDA(cudaMemsetAsync(b->d_counter.p, 0, 4, st));
        SCRS_CUDA(cudaEventRecord(e0, st));
        SCRS_CUDA(launch_gf256_mxk(b->d_tasks.as<MxkTask>(), b->d_item_task.as<uint32_t>(), b->gen_lo, b->gen_hi,
                                   b->d_counter.as<uint32_t>(), b->status.dev, seg_rows, grid, st,
                                   drain_shape(b, seg_rows)));
        SCRS_CUDA(cudaEventRecord(e1, st));
        SCRS_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        SCRS_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        if (rep) t.push_back(ms);
    }
    std::sort(t.begin(), t.end());
    *median_ms = t[t.size() / 2];
    return SCRS_OK;
}

}  // namespace

extern "C" int32_t scrs_stripe_batch_autotune(scrs_stripe_batch* b, void* stream, uint32_t reps,
                                              scrs_tune_params* chosen, scrs_error* err) {
    if (!b || !chosen) return set_err(err, SCRS_ERR_NULL_ARGUMENT);
    if (reps > 100) return set_err(err, SCRS_ERR_BAD_ARGUMENT, 3, reps);
    if (reps == 0) reps = 5;
    cudaStream_t st = (cudaStream_t)stream;
    if (b->gen_hi <= b->gen_lo) return scrs_stripe_batch_launch_params(b, chosen, err);
    // inputs on the device and decode matrices built before any drain
    if (b->host_mode) {
        int32_t r = run_host(b, st, err);
        if (r) return r;
    } else {
        int32_t r = enqueue_plans(b, st, err);
        if (r) return r;
    }
    const int max_seg = std::min<int>((int)b->max_in, FieldGeom<0>::kSegMax);
    const int def_seg = mxk_default_seg((int)b->max_in);
    std::vector<int> segs{def_seg};
    for (int s : {8, 12, 16, 24, 32, max_seg}) {
        s = std::min(s, max_seg);
        if (std::find(segs.begin(), segs.end(), s) == segs.end()) segs.push_back(s);
    }
    cudaEvent_t e0, e1;
    SCRS_CUDA(cudaEventCreate(&e0));
    SCRS_CUDA(cudaEventCreate(&e1));
    scrs_tune_params best{};
    int32_t rc = SCRS_OK;
    for (int seg : segs) {
        const int fit = mxk_ctas_per_sm(seg, drain_shape(b, seg));
        std::vector<int> ctas{fit};
        for (int c : {(3 * fit + 3) / 4, (fit + 1) / 2}) {
            c = std::max(1, c);
            if (std::find(ctas.begin(), ctas.end(), c) == ctas.end()) ctas.push_back(c);
        }
        for (int c : ctas) {
            const int grid = std::max(1, std::min<int>(b->sm_count * c, (int)(b->gen_hi - b->gen_lo)));
            float ms = 0;
            rc = time_drain(b, st, seg, grid, reps, e0, e1, &ms, err);
            if (rc) break;
            // the default (first candidate) holds unless beaten by 1 %
            if (best.seg_rows == 0 || ms < 0.99f * best.drain_ms)
                best = scrs_tune_params{(uint32_t)seg, (uint32_t)c, ms, 0};
        }
        if (rc) break;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    rc = take_status(b->status, err);  // a drain that gave up on a wait
    if (rc) return rc;
    tune_store(b->key, best);
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    *chosen = best;
    return set_err(err, SCRS_OK);
}

extern "C" int32_t scrs_stripe_batch_set_jit(scrs_stripe_batch* b, int32_t enable, scrs_error* err) {
    if (!b) return set_err(err, SCRS_ERR_NULL_ARGUMENT);
    b->jit = enable != 0;
    return set_err(err, SCRS_OK);
}

extern "C" uint64_t scrs_stripe_batch_jit_stripes(const scrs_stripe_batch* b) {
    uint64_t n = 0;
    if (b)
        for (auto& R : b->spec) n += R.stripes;
    return n;
}
