// Autotuner table for the persistent stripe-batch drain (include/scrs_gpu.h
// scrs_tune_*): geometry key -> (seg_rows, ctas_per_sm), process-wide.
#pragma once

#include <stdint.h>

#include "../../include/scrs_gpu.h"

namespace scrs {

// Key of a descriptor list; descriptors are not validated here beyond what
// the key needs (a decode stripe without indices counts as no output rows).
scrs_tune_key tune_key_of(const scrs_stripe_desc* descs, uint64_t count);
// The entry for `key`, if any.
bool tune_lookup(const scrs_tune_key& key, scrs_tune_params* out);
void tune_store(const scrs_tune_key& key, const scrs_tune_params& p);
// Incremented by every change of the table (graphs captured before a change
// are re-captured).
uint64_t tune_version();

}  // namespace scrs
