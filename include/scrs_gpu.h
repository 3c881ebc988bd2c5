/*
 * scrs_gpu.h — C ABI of the B200 (sm_100a) erasure-coding engines.
 *
 * The surface mirrors the SCRS Rust trait family one-to-one so that a Rust
 * (or any FFI) caller can drop the GPU engines in beside the CPU ones:
 *
 *   Profile::resolve / Profile::recommended      scrs/src/selector.rs:40,67
 *   recommended_gf16_engine                      scrs/src/lib.rs:85
 *   batch_encoder + BatchEncoder                 scrs/src/selector.rs:457, codec.rs:136-151
 *   batch_decoder + BatchDecoder                 scrs/src/selector.rs:270, codec.rs:157-175
 *   incremental_encoder + IncrementalEncoder     scrs/src/selector.rs:370, codec.rs:122-131
 *   decoder + Decoder + SymbolSink               scrs/src/selector.rs:117, codec.rs:180-201,
 *                                                scrs/src/transport/symbol_sink.rs:36-54
 *   ConfigError / EncodeError / DecodeError      scrs/src/error.rs:12-126
 *
 * Conventions
 *  - Every fallible call returns an int32 status: SCRS_OK (0) or one of the
 *    SCRS_* codes below.  When `err` is non-NULL it receives the code and
 *    the variant's detail fields (see scrs_error).
 *  - Buffers passed to the plain entry points are HOST memory; the library
 *    copies them to the device, runs the kernels and copies results back
 *    before returning.  The *_device entry points take device pointers and
 *    a CUDA stream (passed as void*) and return after enqueueing the work.
 *  - Handles own their device memory.  After *_create / *_scratch, the
 *    *_with calls perform no device or host allocation (the contract of
 *    scrs/tests/zero_alloc.rs:103-145).
 *  - Handles are not thread safe, as the reference engines are &mut-exclusive.
 *  - Sizes are uint64_t; indices are uint64_t codeword positions.
 */
#ifndef SCRS_GPU_H
#define SCRS_GPU_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define SCRS_API __attribute__((visibility("default")))
#else
#define SCRS_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- vocabulary: scrs/src/codec.rs:20-39 ------------------------------ */
enum {
    SCRS_ENGINE_STANDARD_CAUCHY = 0, /* GF(256), k+m <= 256            */
    SCRS_ENGINE_GOOD_CAUCHY = 1,     /* GF(256), k+m <= 255            */
    SCRS_ENGINE_TOWER = 2,           /* GF((2^8)^2), k+m <= 65535      */
    SCRS_ENGINE_AFFT = 3             /* GF(2^16) additive FFT, <= 65536 */
};
enum { SCRS_FIELD_GF256 = 0, SCRS_FIELD_GF65536 = 1 };

/* ---- status codes: scrs/src/error.rs ----------------------------------- */
enum {
    SCRS_OK = 0,
    /* ConfigError (error.rs:12-31); detail a = cap / engine */
    SCRS_CONFIG_ZERO_DIMENSION = 101,
    SCRS_CONFIG_TOO_MANY_SYMBOLS = 102, /* a = cap                        */
    SCRS_CONFIG_ZERO_SYMBOL_LEN = 103,
    SCRS_CONFIG_ODD_SYMBOL_LEN = 104,
    SCRS_CONFIG_UNSUPPORTED_MODE = 105, /* a = engine                     */
    /* EncodeError (error.rs:35-71) */
    SCRS_ENCODE_WRONG_INPUT_LEN = 201,    /* a = expected, b = got        */
    SCRS_ENCODE_INDEX_OUT_OF_RANGE = 202, /* a = index, b = n             */
    SCRS_ENCODE_WRONG_PAYLOAD_LEN = 203,  /* a = expected, b = got        */
    SCRS_ENCODE_DUPLICATE_DATA = 204,     /* a = index                    */
    SCRS_ENCODE_WRONG_OUTPUT_LEN = 205,   /* a = expected, b = got        */
    SCRS_ENCODE_SCRATCH_MISMATCH = 206,
    /* DecodeError (error.rs:75-126) */
    SCRS_DECODE_WRONG_COUNT = 301,        /* a = expected, b = got        */
    SCRS_DECODE_INDEX_OUT_OF_RANGE = 302, /* a = index, b = n             */
    SCRS_DECODE_DUPLICATE_INDEX = 303,    /* a = index                    */
    SCRS_DECODE_WRONG_PAYLOAD_LEN = 304,  /* a = expected, b = got        */
    SCRS_DECODE_TOO_MANY_SYMBOLS = 305,   /* a = cap, b = received        */
    SCRS_DECODE_INSUFFICIENT_RANK = 306,  /* a = rank, b = k              */
    SCRS_DECODE_WRONG_OUTPUT_LEN = 307,   /* a = expected, b = got        */
    SCRS_DECODE_SCRATCH_MISMATCH = 308,
    /* Runtime errors with no counterpart in the reference (a CPU library
     * cannot meet them): bad pointers, CUDA failures, device limits. */
    SCRS_ERR_NULL_ARGUMENT = 901,
    SCRS_ERR_CUDA = 902,          /* a = cudaError_t value                 */
    SCRS_ERR_OUT_OF_MEMORY = 903, /* a = bytes requested                   */
    SCRS_ERR_NO_DEVICE = 904,
    SCRS_ERR_CAPACITY = 905,      /* a = requested, b = limit              */
    SCRS_ERR_DEVICE_TIMEOUT = 906,/* a bounded device-side wait expired    */
    SCRS_ERR_BAD_ARGUMENT = 907,  /* a = argument position                 */
    SCRS_ERR_JIT = 908            /* a = nvrtcResult of a failed run-time compile */
};

/* PushOutcome (symbol_sink.rs:11-26) */
enum { SCRS_PUSH_ADVANCED = 0, SCRS_PUSH_COMPLETE = 1, SCRS_PUSH_DEPENDENT = 2 };

typedef struct scrs_profile {
    int32_t engine;
    int32_t reserved;
    uint64_t k;
    uint64_t m;
    uint64_t symbol_len;
} scrs_profile;

typedef struct scrs_error {
    int32_t code;
    int32_t reserved;
    uint64_t a;
    uint64_t b;
} scrs_error;

typedef struct scrs_push_outcome {
    int32_t kind; /* SCRS_PUSH_* */
    int32_t reserved;
    uint64_t rank;     /* valid for SCRS_PUSH_ADVANCED */
    uint64_t received; /* valid for SCRS_PUSH_ADVANCED */
} scrs_push_outcome;

typedef struct scrs_batch_encoder scrs_batch_encoder;
typedef struct scrs_encode_scratch scrs_encode_scratch;
typedef struct scrs_batch_decoder scrs_batch_decoder;
typedef struct scrs_batch_decode_scratch scrs_batch_decode_scratch;
typedef struct scrs_incremental_encoder scrs_incremental_encoder;
typedef struct scrs_decoder scrs_decoder;
typedef struct scrs_decode_scratch scrs_decode_scratch;
typedef struct scrs_stripe_batch scrs_stripe_batch;

/* ---- library ------------------------------------------------------------ */
/* ABI version (major << 16 | minor). No reference counterpart. */
SCRS_API uint32_t scrs_abi_version(void);
/* Human-readable name of a status code. No reference counterpart. */
SCRS_API const char* scrs_status_name(int32_t code);
/* Device and pinned-host allocations (cudaMalloc, cudaHostAlloc) the library
 * has made since it was loaded, from every thread.  The zero-allocation
 * contract of the *_with calls (scrs/tests/zero_alloc.rs:48-145 counts heap
 * allocations with a counting global allocator) is checked by reading this
 * before and after steady-state calls. */
SCRS_API uint64_t scrs_alloc_count(void);

/* ---- profiles: selector.rs:40-88, lib.rs:85-93 -------------------------- */
SCRS_API int32_t scrs_profile_resolve(int32_t engine, uint64_t k, uint64_t m,
                             uint64_t symbol_len, scrs_profile* out,
                             scrs_error* err);
SCRS_API int32_t scrs_profile_recommended(int32_t field, uint64_t k, uint64_t m,
                                 uint64_t symbol_len, scrs_profile* out,
                                 scrs_error* err);
/* Returns SCRS_ENGINE_TOWER or SCRS_ENGINE_AFFT (lib.rs:85). */
SCRS_API int32_t scrs_recommended_gf16_engine(uint64_t k, uint64_t m);

/* ---- BatchEncoder: selector.rs:457-529, codec.rs:136-151 ---------------- */
/* UnsupportedMode for Tower (selector.rs:465). */
SCRS_API int32_t scrs_batch_encoder_create(const scrs_profile* profile,
                                  scrs_batch_encoder** out, scrs_error* err);
SCRS_API void scrs_batch_encoder_destroy(scrs_batch_encoder* enc);
SCRS_API int32_t scrs_batch_encoder_profile(const scrs_batch_encoder* enc,
                                   scrs_profile* out);
/* BatchEncoder::scratch (codec.rs:140). */
SCRS_API int32_t scrs_batch_encoder_scratch(const scrs_batch_encoder* enc,
                                   scrs_encode_scratch** out, scrs_error* err);
SCRS_API void scrs_encode_scratch_destroy(scrs_encode_scratch* scratch);
/* BatchEncoder::encode_into (codec.rs:143): throwaway scratch. */
SCRS_API int32_t scrs_batch_encode_into(const scrs_batch_encoder* enc,
                               const uint8_t* data, uint64_t data_len,
                               uint8_t* repairs, uint64_t repairs_len,
                               scrs_error* err);
/* BatchEncoder::encode_into_with (codec.rs:145): host buffers. */
SCRS_API int32_t scrs_batch_encode_into_with(const scrs_batch_encoder* enc,
                                    const uint8_t* data, uint64_t data_len,
                                    uint8_t* repairs, uint64_t repairs_len,
                                    scrs_encode_scratch* scratch,
                                    scrs_error* err);
/* Device-resident form of encode_into_with: d_data / d_repairs are device
 * pointers; enqueued on `stream` (a cudaStream_t, NULL = legacy default). */
SCRS_API int32_t scrs_batch_encode_into_with_device(const scrs_batch_encoder* enc,
                                           const uint8_t* d_data,
                                           uint64_t data_len,
                                           uint8_t* d_repairs,
                                           uint64_t repairs_len,
                                           scrs_encode_scratch* scratch,
                                           void* stream, scrs_error* err);

/* ---- BatchDecoder: selector.rs:270-352, codec.rs:157-175 ---------------- */
SCRS_API int32_t scrs_batch_decoder_create(const scrs_profile* profile,
                                  scrs_batch_decoder** out, scrs_error* err);
SCRS_API void scrs_batch_decoder_destroy(scrs_batch_decoder* dec);
SCRS_API int32_t scrs_batch_decoder_profile(const scrs_batch_decoder* dec,
                                   scrs_profile* out);
SCRS_API int32_t scrs_batch_decoder_scratch(const scrs_batch_decoder* dec,
                                   scrs_batch_decode_scratch** out,
                                   scrs_error* err);
SCRS_API void scrs_batch_decode_scratch_destroy(scrs_batch_decode_scratch* scratch);
/* BatchDecoder::decode_into_with (codec.rs:169).  The Rust slice of
 * (index, payload) pairs is passed as three parallel arrays of `count`
 * entries: indices[i], payloads[i] (host pointer), payload_lens[i]. */
SCRS_API int32_t scrs_batch_decode_into_with(scrs_batch_decoder* dec,
                                    const uint64_t* indices,
                                    const uint8_t* const* payloads,
                                    const uint64_t* payload_lens,
                                    uint64_t count, uint8_t* out,
                                    uint64_t out_len,
                                    scrs_batch_decode_scratch* scratch,
                                    scrs_error* err);
/* BatchDecoder::decode_into (codec.rs:163): throwaway scratch. */
SCRS_API int32_t scrs_batch_decode_into(scrs_batch_decoder* dec,
                               const uint64_t* indices,
                               const uint8_t* const* payloads,
                               const uint64_t* payload_lens, uint64_t count,
                               uint8_t* out, uint64_t out_len,
                               scrs_error* err);
/* Device-resident form: payloads are `count` rows of symbol_len bytes at
 * d_payloads (row i belongs to indices[i], indices in HOST memory); d_out is
 * k*symbol_len device bytes. Enqueued on `stream`. */
SCRS_API int32_t scrs_batch_decode_into_with_device(scrs_batch_decoder* dec,
                                           const uint64_t* indices,
                                           const uint8_t* d_payloads,
                                           uint64_t count, uint8_t* d_out,
                                           uint64_t out_len,
                                           scrs_batch_decode_scratch* scratch,
                                           void* stream, scrs_error* err);

/* Self-test of the device-side failure path (no reference counterpart):
 * launches one bounded wait that nothing completes and returns the status it
 * reports, SCRS_ERR_DEVICE_TIMEOUT after about limit_ns (1 ns .. 100 ms);
 * the context stays usable.  Every wait in the kernels is bounded the same
 * way (2 s) and reports through the same status word. */
SCRS_API int32_t scrs_selftest_wait_timeout(uint64_t limit_ns, scrs_error* err);

/* Decode recipes (the reduced inverse's coefficients) are kept in a small
 * device-resident LRU per decode scratch, keyed by the erasure pattern, as
 * the reference's RecipeCache (decoder/cache.rs:15-100): a repeated pattern
 * skips the plan launch.  Returns how many decodes hit it.  A scratch's
 * device work must stay ordered on one stream (the reference's scratch is
 * exclusively borrowed). */
SCRS_API uint64_t scrs_batch_decode_scratch_recipe_hits(const scrs_batch_decode_scratch* scratch);
SCRS_API uint64_t scrs_decode_scratch_recipe_hits(const scrs_decode_scratch* scratch);

/* GF(256) batch decode that allocates nothing (no counterpart in the
 * reference).  For callers that cannot call cudaMalloc: the allocation may
 * synchronise the device, which a latency-bound receive loop cannot afford,
 * and a process that reserved its device memory at start-up has no headroom
 * for per-codec buffers.  Same inputs, outputs and validation as
 * scrs_batch_decode_into_with_device, without a decoder handle or scratch:
 * the reconstruction recipe lives in one fixed 16 KiB device array built into
 * the library.  Decodes whose recipe exceeds it (2*(3k+3r) + k*r bytes for
 * r erased data symbols) fail with SCRS_ERR_CAPACITY (a = needed, b = 16384).
 * Calls share that array: calls whose device work overlaps race and must be
 * ordered on one stream.  The first call on a device does the one-time
 * set-up there (the array's address, the decode kernels' tables and limits;
 * it synchronises); make it before any stream capture on that device.
 * The call returns before its device work runs, so a bounded device wait
 * that runs out is reported through d_status, an optional caller-owned
 * device int32 (NULL: not reported): the kernels store
 * SCRS_ERR_DEVICE_TIMEOUT there and never clear it, so zero it before the
 * first call and read it after synchronising `stream`. */
SCRS_API int32_t scrs_gf256_decode_static(int32_t engine, uint64_t k,
                                          uint64_t m, uint64_t symbol_len,
                                          const uint64_t* indices,
                                          const uint8_t* d_rows, uint64_t count,
                                          uint8_t* d_out, uint64_t out_len,
                                          void* stream, int32_t* d_status,
                                          scrs_error* err);

/* ---- IncrementalEncoder: selector.rs:370-429, codec.rs:122-131 ---------- */
/* UnsupportedMode for Standard Cauchy and AFFT (selector.rs:379). */
SCRS_API int32_t scrs_incremental_encoder_create(const scrs_profile* profile,
                                        scrs_incremental_encoder** out,
                                        scrs_error* err);
SCRS_API void scrs_incremental_encoder_destroy(scrs_incremental_encoder* enc);
SCRS_API int32_t scrs_incremental_encoder_profile(const scrs_incremental_encoder* enc,
                                         scrs_profile* out);
/* IncrementalEncoder::feed (codec.rs:124): host payload. */
SCRS_API int32_t scrs_inc_feed(scrs_incremental_encoder* enc, uint64_t index,
                      const uint8_t* data, uint64_t data_len,
                      scrs_error* err);
/* Device-resident feed: d_data is a device pointer.  The row is copied on
 * `stream`, so the copy follows the caller's earlier work on that stream and
 * the caller may overwrite d_data with work enqueued there afterwards; later
 * calls on this handle wait for the copy (through an event recorded on
 * `stream` when they start, so `stream` must stay valid until the next
 * repair read or reset). */
SCRS_API int32_t scrs_inc_feed_device_stream(scrs_incremental_encoder* enc, uint64_t index,
                                    const uint8_t* d_data, uint64_t data_len,
                                    void* stream, scrs_error* err);
/* scrs_inc_feed_device_stream on the legacy default stream (which orders
 * the copy with the work of every blocking stream of the context). */
SCRS_API int32_t scrs_inc_feed_device(scrs_incremental_encoder* enc, uint64_t index,
                             const uint8_t* d_data, uint64_t data_len,
                             scrs_error* err);
/* IncrementalEncoder::repair (codec.rs:126).  The Rust call borrows the
 * repair; across the ABI the repair is copied into `dst` (host). */
SCRS_API int32_t scrs_inc_repair(const scrs_incremental_encoder* enc, uint64_t index,
                        uint8_t* dst, uint64_t dst_len, scrs_error* err);
/* Borrow form: device address of repair `index`, complete when the call
 * returns.  The address stays valid until destroy; the bytes there change
 * with the next reset or fold of new feeds. */
SCRS_API int32_t scrs_inc_repair_device(const scrs_incremental_encoder* enc,
                               uint64_t index, const uint8_t** d_repair,
                               scrs_error* err);
SCRS_API uint64_t scrs_inc_fed_count(const scrs_incremental_encoder* enc);
SCRS_API void scrs_inc_reset(scrs_incremental_encoder* enc);

/* ---- Decoder + SymbolSink: selector.rs:117-242, codec.rs:180-201 -------- */
SCRS_API int32_t scrs_decoder_create(const scrs_profile* profile, scrs_decoder** out,
                            scrs_error* err);
SCRS_API void scrs_decoder_destroy(scrs_decoder* dec);
SCRS_API int32_t scrs_decoder_profile(const scrs_decoder* dec, scrs_profile* out);
SCRS_API int32_t scrs_decoder_scratch(const scrs_decoder* dec,
                             scrs_decode_scratch** out, scrs_error* err);
SCRS_API void scrs_decode_scratch_destroy(scrs_decode_scratch* scratch);
/* SymbolSink::push (symbol_sink.rs:42): host payload, copied to the
 * device-resident payload buffer (no payload arithmetic). */
SCRS_API int32_t scrs_dec_push(scrs_decoder* dec, uint64_t index,
                      const uint8_t* payload, uint64_t payload_len,
                      scrs_push_outcome* outcome, scrs_error* err);
/* Device-resident push: d_payload is a device pointer, copied on `stream`
 * into the decoder's payload buffer (after the caller's earlier work on
 * `stream`; the caller may overwrite d_payload with work enqueued there
 * afterwards).  The copy also waits for the reads of the last finalize, so
 * a reset decoder can be refilled while that decode still runs.  The next
 * finalize waits for the copy through an event it records on `stream`, so
 * `stream` must stay valid until then. */
SCRS_API int32_t scrs_dec_push_device_stream(scrs_decoder* dec, uint64_t index,
                                    const uint8_t* d_payload, uint64_t payload_len,
                                    void* stream, scrs_push_outcome* outcome,
                                    scrs_error* err);
/* scrs_dec_push_device_stream on the legacy default stream. */
SCRS_API int32_t scrs_dec_push_device(scrs_decoder* dec, uint64_t index,
                             const uint8_t* d_payload, uint64_t payload_len,
                             scrs_push_outcome* outcome, scrs_error* err);
SCRS_API int32_t scrs_dec_is_complete(const scrs_decoder* dec);
SCRS_API uint64_t scrs_dec_rank(const scrs_decoder* dec);
SCRS_API uint64_t scrs_dec_received(const scrs_decoder* dec);
SCRS_API void scrs_dec_reset(scrs_decoder* dec);
/* Decoder::finalize_into (codec.rs:194): throwaway scratch. */
SCRS_API int32_t scrs_dec_finalize_into(scrs_decoder* dec, uint8_t* out,
                               uint64_t out_len, scrs_error* err);
/* Decoder::finalize_into_with (codec.rs:196): host output. */
SCRS_API int32_t scrs_dec_finalize_into_with(scrs_decoder* dec, uint8_t* out,
                                    uint64_t out_len,
                                    scrs_decode_scratch* scratch,
                                    scrs_error* err);
/* Device-resident finalize into d_out (device), enqueued on `stream` after
 * the pushes' copies; returns without waiting.  Later pushes (after a reset)
 * and host uploads wait on the device for this decode's reads of the
 * payload buffer; a host push after a reset waits on the host for the
 * upload of the staged rows. */
SCRS_API int32_t scrs_dec_finalize_into_with_device(scrs_decoder* dec, uint8_t* d_out,
                                           uint64_t out_len,
                                           scrs_decode_scratch* scratch,
                                           void* stream, scrs_error* err);

/* ---- Batched GF(256) and tower stripes in one persistent launch ---------
 * No single reference counterpart: this runs many independent
 * BatchCodec::encode_into (batch/codec.rs:156) and
 * BatchCodec::decode_into_with (batch/codec.rs:278) calls of uneven
 * geometry as one device work queue, and tower stripes likewise: a tower
 * encode gives the repairs of k in-order feeds (tower/encoder.rs:89-131), a
 * tower decode the lazy decoder's reconstruction (tower/decoder.rs:218-546).
 * Per-stripe decode matrices are built on the device; GF(256) and tower
 * stripes drain through one persistent kernel per field.  All pointers in a
 * stripe descriptor are device pointers except `indices`, which is host
 * memory read during submit. */
enum { SCRS_OP_ENCODE = 0, SCRS_OP_DECODE = 1 };

typedef struct scrs_stripe_desc {
    int32_t op;     /* SCRS_OP_ENCODE or SCRS_OP_DECODE                     */
    int32_t engine; /* SCRS_ENGINE_STANDARD_CAUCHY, _GOOD_CAUCHY or _TOWER     */
    uint32_t k;
    uint32_t m;
    uint64_t symbol_len;
    /* encode: k*symbol_len data, row i at in + i*symbol_len.
     * decode: k received symbols, row i at in + i*symbol_len. */
    const uint8_t* in;
    /* encode: m*symbol_len repairs.  decode: k*symbol_len data.  The
     * stripes' outputs must not overlap one another or any input: a stripe
     * with more inputs than one staged segment accumulates partial sums in
     * its output. */
    uint8_t* out;
    /* decode only: k codeword indices of the received rows (host memory). */
    const uint16_t* indices;
} scrs_stripe_desc;

/* Capacity is fixed at creation so that submit allocates nothing. */
SCRS_API int32_t scrs_stripe_batch_create(uint64_t max_stripes, uint64_t max_work_items,
                                 scrs_stripe_batch** out, scrs_error* err);
SCRS_API void scrs_stripe_batch_destroy(scrs_stripe_batch* batch);
/* Validate and upload `count` descriptors (the host part of a submit).
 * Errors carry the first offending stripe position in `err->b` when the
 * variant has no second detail field. */
SCRS_API int32_t scrs_stripe_batch_set(scrs_stripe_batch* batch,
                              const scrs_stripe_desc* descs, uint64_t count,
                              scrs_error* err);
/* Host-buffer form of scrs_stripe_batch_set: every `in` / `out` pointer is
 * HOST memory (pinned memory gives asynchronous copies).  The batch owns
 * device staging sized at this call.  Each run cuts the stripes into up to
 * 64 pieces of about equal input bytes and pipelines them: the inputs of
 * piece p+1 are copied in and the outputs of piece p-1 copied out (on two
 * internal streams) while piece p computes; the run's stream waits for the
 * last copy.  Copies of stripes that are contiguous in host memory are
 * merged; a merged copy the driver refuses (host buffers that touch but are
 * separate allocations) is issued stripe by stripe instead.  A decode
 * stripe's present data rows are copied on the host, by the batch's worker
 * threads, from its input rows into `out` while the GPU runs; the device
 * computes and copies back only the missing rows (through pinned staging the
 * batch owns), so the link carries k*L bytes in and r*L out per decode
 * stripe with r data symbols erased (BatchCodec writes the present rows into
 * the output the same way, batch/codec.rs:323-324).  In this mode
 * scrs_stripe_batch_run returns once every output is in its host buffer, and
 * use_graph is ignored.  Host-buffer batches take GF(256) stripes only (a
 * tower stripe: SCRS_ERR_BAD_ARGUMENT, a = 2). */
SCRS_API int32_t scrs_stripe_batch_set_host(scrs_stripe_batch* batch,
                                            const scrs_stripe_desc* descs,
                                            uint64_t count, scrs_error* err);
/* Run the uploaded stripes on `stream`: one device-side plan kernel builds
 * every decode matrix, one persistent kernel drains the work queue.  With
 * use_graph != 0 the pair is captured once into a CUDA graph and replayed. */
SCRS_API int32_t scrs_stripe_batch_run(scrs_stripe_batch* batch, void* stream,
                              int32_t use_graph, scrs_error* err);
/* Baseline form of the same work: one plan launch and one kernel launch per
 * stripe (the plain one-call-per-stripe GPU form). */
SCRS_API int32_t scrs_stripe_batch_run_plain(scrs_stripe_batch* batch, void* stream,
                                    scrs_error* err);
/* Number of kernels the last run launched (for launch accounting). */
SCRS_API uint64_t scrs_stripe_batch_last_launches(const scrs_stripe_batch* batch);
/* Measurement form of scrs_stripe_batch_run (no graph): brackets the plan
 * launch and the persistent drain launch with CUDA events on `stream`,
 * synchronises, and reports each launch's device time in milliseconds. */
SCRS_API int32_t scrs_stripe_batch_run_timed(scrs_stripe_batch* batch, void* stream,
                                             float* plan_ms, float* drain_ms,
                                             scrs_error* err);
/* As scrs_stripe_batch_run_timed, with the drain split: the kernels
 * specialised to encode matrices (spec_ms, 0 when there are none) and the
 * generic drain (generic_ms); drain_ms above is their sum. */
SCRS_API int32_t scrs_stripe_batch_run_timed_drains(scrs_stripe_batch* batch, void* stream,
                                                    float* plan_ms, float* spec_ms,
                                                    float* generic_ms, scrs_error* err);
/* After the run's stream has synchronised: SCRS_OK, or the device-side
 * failure a kernel recorded (SCRS_ERR_DEVICE_TIMEOUT). */
SCRS_API int32_t scrs_stripe_batch_check(scrs_stripe_batch* batch, scrs_error* err);

/* ---- Autotuner for the persistent drain ----------------------------------
 * No reference counterpart.  Two launch parameters of the drain kernel are
 * tuned per batch geometry:
 *   seg_rows     input rows staged in shared memory per segment (1..32).
 *                Stripes with more inputs than this pass over their output
 *                rows once per segment; more rows cost shared memory per CTA
 *                and so CTAs per SM.
 *   ctas_per_sm  CTAs of the persistent grid per SM (with the SM count this
 *                fixes the grid, hence the stripes each CTA drains).
 * A process-wide table maps a geometry key to chosen parameters, and every
 * scrs_stripe_batch_run consults it; a batch whose key has no entry stages
 * min(largest k, 16) rows and runs the most CTAs per SM that fit.  Changing
 * the table re-captures graphs on their next run. */
typedef struct scrs_tune_key {
    uint32_t field;    /* 0: GF(256) stripe batches                          */
    uint32_t k_bucket; /* ceil(log2(largest k))                              */
    uint32_t m_bucket; /* ceil(log2(mean output rows per stripe)), 0 if <= 1 */
    uint32_t l_bucket; /* floor(log2(mean symbol_len))                       */
} scrs_tune_key;

typedef struct scrs_tune_params {
    uint32_t seg_rows;    /* 1..32                                          */
    uint32_t ctas_per_sm; /* 1..32; capped by what fits at run time         */
    float drain_ms;       /* the winner's measured drain time (informative) */
    uint32_t reserved;
} scrs_tune_params;

/* Key of a descriptor list (host only; no device work). */
SCRS_API int32_t scrs_tune_key_of(const scrs_stripe_desc* descs, uint64_t count,
                                  scrs_tune_key* key, scrs_error* err);
/* Key of the batch's current descriptors. */
SCRS_API int32_t scrs_stripe_batch_tune_key(const scrs_stripe_batch* batch, scrs_tune_key* key,
                                            scrs_error* err);
/* The seg_rows and ctas_per_sm a run of the batch would use now. */
SCRS_API int32_t scrs_stripe_batch_launch_params(const scrs_stripe_batch* batch,
                                                 scrs_tune_params* params, scrs_error* err);
/* Time the drain of the batch's current stripes on `stream` under each
 * candidate (seg_rows in {8, 12, 16, 24, 32, largest k} capped at the
 * largest k; ctas_per_sm in {most that fit, 3/4 of it, 1/2 of it}), one
 * untimed and `reps` timed launches each (0 means 5, at most 100), keep the
 * fastest median (the default must be beaten by 1 %), store it in the table
 * under the batch's key and return it.  Outputs are rewritten with the same
 * values by every launch; a host-buffer batch first runs once to stage its
 * inputs.  Synchronises `stream`. */
SCRS_API int32_t scrs_stripe_batch_autotune(scrs_stripe_batch* batch, void* stream, uint32_t reps,
                                            scrs_tune_params* chosen, scrs_error* err);
/* ---- Encode kernels specialised to one coefficient matrix ------------------
 * No reference counterpart.  Encode stripes of a GF(256) engine with
 * k <= 32 and k*m <= 64 run, inside stripe batches, through a drain kernel
 * generated for their (engine, k, m) matrix (every coefficient's XOR network
 * inlined) and compiled for sm_100a by NVRTC on first use; the kernel is
 * cached for the life of the process.  scrs_jit_prepare compiles (and, with
 * load != 0, loads for the current device) ahead of time, so the first
 * batch does not pay the compile; without load it needs no device.
 * SCRS_ERR_BAD_ARGUMENT for an engine or geometry that is not specialised,
 * SCRS_ERR_JIT (a = nvrtcResult) when the compile fails or NVRTC cannot be
 * loaded (it is opened on first use; without it every stripe stays on the
 * precompiled kernels). */
SCRS_API int32_t scrs_jit_prepare(int32_t engine, uint32_t k, uint32_t m, int32_t load,
                                  uint64_t* cubin_bytes, scrs_error* err);
/* Whether scrs_stripe_batch_set specialises eligible encode stripes (1, the
 * default) or runs every stripe through the generic drain (0).  Takes
 * effect at the next set. */
SCRS_API int32_t scrs_stripe_batch_set_jit(scrs_stripe_batch* batch, int32_t enable, scrs_error* err);
/* Stripes of the current descriptors that run through specialised kernels. */
SCRS_API uint64_t scrs_stripe_batch_jit_stripes(const scrs_stripe_batch* batch);

/* The table (for saving and loading it): entries 0..size-1, set, clear. */
SCRS_API uint64_t scrs_tune_table_size(void);
SCRS_API int32_t scrs_tune_table_entry(uint64_t i, scrs_tune_key* key, scrs_tune_params* params,
                                       scrs_error* err);
SCRS_API int32_t scrs_tune_table_set(const scrs_tune_key* key, const scrs_tune_params* params,
                                     scrs_error* err);
SCRS_API void scrs_tune_table_clear(void);

/* ---- Serving loop (continuous batching) ----------------------------------
 * No reference counterpart: a request loop over the engines above.  Requests
 * of every engine are submitted with device-resident inputs and outputs and
 * admitted first come, first served as one of `slots` streams and the device
 * memory budget free up; admitted work overlaps on the device.  Waiting
 * GF(256) requests and tower requests of at most 64 inputs and 32 outputs
 * are coalesced into one stripe batch per slot; additive-FFT requests and
 * larger tower requests take a slot each and use engines kept resident per
 * slot (least recently used profiles are evicted).  The budget counts every
 * admitted request's input and output bytes plus estimated resident engine
 * workspaces.  Results are identical to running each request alone. */
typedef struct scrs_server scrs_server;
typedef struct scrs_request {
    int32_t op;          /* SCRS_OP_ENCODE or SCRS_OP_DECODE                    */
    int32_t engine;      /* SCRS_ENGINE_*                                       */
    uint64_t k, m, symbol_len;
    const uint8_t* in;   /* device: encode k*L data; decode k received rows,
                            row q holding codeword index indices[q]             */
    uint8_t* out;        /* device: encode m*L repairs; decode k*L data        */
    const uint64_t* indices; /* host, decode only: k indices (copied at submit) */
    uint64_t tag;        /* returned with the completion                       */
    void* stream;        /* the stream `in` was written on (NULL: the legacy
                            default stream): the request's device work waits
                            for the work enqueued there before the submit      */
} scrs_request;
typedef struct scrs_completion {
    uint64_t ticket, tag;
    int32_t status;      /* SCRS_OK or the request's error                      */
    int32_t reserved;
    uint64_t submit_ns, done_ns; /* host steady clock: submit, completion seen */
} scrs_completion;
typedef struct scrs_server_stats {
    uint64_t submitted, admitted, completed, failed, batches;
    uint64_t memory_in_use, resident_bytes;
} scrs_server_stats;
/* memory_budget in bytes; 1 <= slots <= 64. */
SCRS_API int32_t scrs_server_create(uint64_t memory_budget, uint32_t slots,
                                    scrs_server** out, scrs_error* err);
/* Waits for in-flight work, then frees everything. */
SCRS_API void scrs_server_destroy(scrs_server* server);
/* Validates (profile, decode indices, budget: SCRS_ERR_CAPACITY when the
 * request alone exceeds it), queues, and admits what fits.  Buffers must
 * stay valid until the request's completion is returned; `out` is complete
 * on the device when it is.  Requests in flight at the same time must not
 * share an output buffer (they may be coalesced into one stripe batch).  The input is read after the work enqueued on
 * req->stream before this call. */
SCRS_API int32_t scrs_server_submit(scrs_server* server, const scrs_request* req,
                                    uint64_t* ticket, scrs_error* err);
/* Non-blocking: retires finished slots, admits waiting requests and returns
 * up to `capacity` completions in `done` (count in *n_done). */
SCRS_API int32_t scrs_server_progress(scrs_server* server, scrs_completion* done,
                                      uint32_t capacity, uint32_t* n_done,
                                      scrs_error* err);
/* Build the resident engines of one additive-FFT or large tower profile for `op`
 * on every slot, so that no request of that profile pays the build (device
 * allocations, which stall the whole device) on its way through.  For
 * start-up: SCRS_ERR_BAD_ARGUMENT (a = 3) while any slot is running
 * requests, (a = 1) for a GF(256) engine (its stripe batches need no
 * resident engines); SCRS_OK with nothing built for a tower profile of at
 * most 64 inputs and 32 outputs (those run in the stripe batches too).  Resident engines count against
 * the memory budget and
 * each slot keeps at most 8 profiles, least recently used evicted first. */
SCRS_API int32_t scrs_server_reserve(scrs_server* server, int32_t op, int32_t engine,
                                     uint64_t k, uint64_t m, uint64_t symbol_len,
                                     scrs_error* err);
/* Requests queued, running or completed but not yet returned. */
SCRS_API uint64_t scrs_server_pending(const scrs_server* server);
SCRS_API int32_t scrs_server_get_stats(const scrs_server* server, scrs_server_stats* out);

#ifdef __cplusplus
}
#endif
#endif /* SCRS_GPU_H */
