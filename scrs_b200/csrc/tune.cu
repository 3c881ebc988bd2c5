// Autotuner table (host only): see tune.h and include/scrs_gpu.h.
#include "tune.h"

#include <atomic>
#include <map>
#include <mutex>
#include <tuple>

#include "runtime.h"

namespace scrs {
namespace {

using KeyTuple = std::tuple<uint32_t, uint32_t, uint32_t, uint32_t>;

KeyTuple tie_key(const scrs_tune_key& k) { return KeyTuple(k.field, k.k_bucket, k.m_bucket, k.l_bucket); }

struct Table {
    std::mutex mu;
    std::map<KeyTuple, scrs_tune_params> entries;
    std::atomic<uint64_t> version{0};
};

Table& table() {
    static Table t;
    return t;
}

uint32_t ceil_log2(uint64_t v) {
    uint32_t b = 0;
    while (b < 63 && (1ull << b) < v) b++;
    return b;
}

uint32_t floor_log2(uint64_t v) {
    uint32_t b = 0;
    while (v > 1) v >>= 1, b++;
    return b;
}

bool valid_params(const scrs_tune_params& p) {
    return p.seg_rows >= 1 && p.seg_rows <= (uint32_t)FieldGeom<0>::kSegMax && p.ctas_per_sm >= 1 &&
           p.ctas_per_sm <= 32;
}

}  // namespace

scrs_tune_key tune_key_of(const scrs_stripe_desc* descs, uint64_t count) {
    uint64_t max_k = 1, outs = 0, bytes = 0;
    for (uint64_t s = 0; s < count; s++) {
        const scrs_stripe_desc& d = descs[s];
        max_k = d.k > max_k ? d.k : max_k;
        bytes += d.symbol_len;
        if (d.op == SCRS_OP_ENCODE) {
            outs += d.m;
        } else if (d.indices) {
            uint64_t present = 0;
            for (uint32_t q = 0; q < d.k; q++) present += d.indices[q] < d.k;
            outs += d.k - (present < d.k ? present : d.k);
        }
    }
    const uint64_t n = count ? count : 1;
    scrs_tune_key key{};
    key.field = 0;
    key.k_bucket = ceil_log2(max_k);
    key.m_bucket = ceil_log2((outs + n - 1) / n);
    key.l_bucket = floor_log2(bytes / n);
    return key;
}

bool tune_lookup(const scrs_tune_key& key, scrs_tune_params* out) {
    Table& t = table();
    std::lock_guard<std::mutex> g(t.mu);
    auto it = t.entries.find(tie_key(key));
    if (it == t.entries.end()) return false;
    *out = it->second;
    return true;
}

void tune_store(const scrs_tune_key& key, const scrs_tune_params& p) {
    Table& t = table();
    std::lock_guard<std::mutex> g(t.mu);
    t.entries[tie_key(key)] = p;
    t.version++;
}

uint64_t tune_version() { return table().version.load(); }

}  // namespace scrs

using namespace scrs;

extern "C" int32_t scrs_tune_key_of(const scrs_stripe_desc* descs, uint64_t count, scrs_tune_key* key,
                                    scrs_error* err) {
    if (!key || (count && !descs)) return set_err(err, SCRS_ERR_NULL_ARGUMENT);
    *key = tune_key_of(descs, count);
    return set_err(err, SCRS_OK);
}

extern "C" uint64_t scrs_tune_table_size(void) {
    Table& t = table();
    std::lock_guard<std::mutex> g(t.mu);
    return t.entries.size();
}

extern "C" int32_t scrs_tune_table_entry(uint64_t i, scrs_tune_key* key, scrs_tune_params* params, scrs_error* err) {
    if (!key || !params) return set_err(err, SCRS_ERR_NULL_ARGUMENT);
    Table& t = table();
    std::lock_guard<std::mutex> g(t.mu);
    if (i >= t.entries.size()) return set_err(err, SCRS_ERR_BAD_ARGUMENT, 1, i);
    auto it = t.entries.begin();
    std::advance(it, (long)i);
    key->field = std::get<0>(it->first);
    key->k_bucket = std::get<1>(it->first);
    key->m_bucket = std::get<2>(it->first);
    key->l_bucket = std::get<3>(it->first);
    *params = it->second;
    return set_err(err, SCRS_OK);
}

extern "C" int32_t scrs_tune_table_set(const scrs_tune_key* key, const scrs_tune_params* params, scrs_error* err) {
    if (!key || !params) return set_err(err, SCRS_ERR_NULL_ARGUMENT);
    if (key->field != 0) return set_err(err, SCRS_ERR_BAD_ARGUMENT, 1, key->field);
    if (!valid_params(*params)) return set_err(err, SCRS_ERR_BAD_ARGUMENT, 2, params->seg_rows);
    tune_store(*key, *params);
    return set_err(err, SCRS_OK);
}

extern "C" void scrs_tune_table_clear(void) {
    Table& t = table();
    std::lock_guard<std::mutex> g(t.mu);
    t.entries.clear();
    t.version++;
}
