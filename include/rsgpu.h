/*
 * rsgpu.h -- C ABI of the B200 erasure-coding library (librsgpu.so).
 *
 * The library replaces the encode / reconstruct / verify hot path of
 * rustfs-erasure-codec 9.1.0 (a Rust crate with no C ABI of its own).  Every
 * entry point below names the reference API it stands in for (file:line in
 * the reference crate); a Rust binding maps each `ReedSolomon` method onto one
 * call through an `extern "C"` block with these signatures.
 *
 * Conventions
 *  - Return value: 0 on success, otherwise the reference `Error` discriminant
 *    + 1 (src/errors.rs:3-21, values 1..16 below), or a device/runtime code
 *    (>= 100).  Every argument check runs on the host before any launch, so a
 *    call that fails validation writes nothing.
 *  - Shards are passed as arrays of pointers plus an array of per-shard byte
 *    lengths, the flat equivalent of the reference's `&[T: AsRef<[u8]>]`.
 *    `mem` says where the bytes live: RSGPU_MEM_HOST (pageable or pinned host
 *    memory; the library stages it through device memory and the call returns
 *    once results are back in host memory) or RSGPU_MEM_DEVICE (device memory
 *    of the codec's GPU; work is queued on `stream` and the call returns
 *    without waiting, except where a host-visible result such as a verify
 *    flag is returned).
 *  - `stream` is a cudaStream_t passed as void* (NULL = the legacy default
 *    stream).
 *  - A codec handle may be shared by threads; its caches are internally
 *    locked.  Workspaces belong to one caller at a time.
 */
#ifndef RSGPU_H
#define RSGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- error codes (src/errors.rs:3-21, discriminant + 1) ---- */
enum {
  RSGPU_OK = 0,
  RSGPU_ERR_TOO_FEW_SHARDS = 1,
  RSGPU_ERR_TOO_MANY_SHARDS = 2,
  RSGPU_ERR_TOO_FEW_DATA_SHARDS = 3,
  RSGPU_ERR_TOO_MANY_DATA_SHARDS = 4,
  RSGPU_ERR_TOO_FEW_PARITY_SHARDS = 5,
  RSGPU_ERR_TOO_MANY_PARITY_SHARDS = 6,
  RSGPU_ERR_TOO_FEW_BUFFER_SHARDS = 7,
  RSGPU_ERR_TOO_MANY_BUFFER_SHARDS = 8,
  RSGPU_ERR_INCORRECT_SHARD_SIZE = 9,
  RSGPU_ERR_TOO_FEW_SHARDS_PRESENT = 10,
  RSGPU_ERR_EMPTY_SHARD = 11,
  RSGPU_ERR_INVALID_SHARD_FLAGS = 12,
  RSGPU_ERR_INVALID_INDEX = 13,
  RSGPU_ERR_INVALID_CUSTOM_MATRIX = 14,
  RSGPU_ERR_UNSUPPORTED_CODEC_FAMILY = 15,
  RSGPU_ERR_UNSUPPORTED_LEOPARD_PROTOTYPE = 16,
  /* device / runtime conditions with no reference counterpart */
  RSGPU_ERR_CUDA = 100,
  RSGPU_ERR_OUT_OF_MEMORY = 101,
  RSGPU_ERR_INVALID_ARGUMENT = 102,
  RSGPU_ERR_DEVICE_TIMEOUT = 103,
  RSGPU_ERR_NO_DEVICE = 104,
  RSGPU_ERR_SCRATCH_LIMIT = 105,
  RSGPU_ERR_STREAM_IO = 106, /* a stream read/write callback failed (see rsgpu_stream_status) */
};

enum { RSGPU_MEM_HOST = 0, RSGPU_MEM_DEVICE = 1 };

/* src/core/options.rs:14-82 */
enum { RSGPU_FAMILY_CLASSIC = 0, RSGPU_FAMILY_LEOPARD_GF8 = 1, RSGPU_FAMILY_LEOPARD_GF16 = 2 };
enum {
  RSGPU_LEOPARD_DISABLED = 0,
  RSGPU_LEOPARD_AS_NEEDED = 1,
  RSGPU_LEOPARD_PREFER_GF16 = 2,
  RSGPU_LEOPARD_PREFER_LEOPARD = 3
};
enum {
  RSGPU_MATRIX_VANDERMONDE = 0,
  RSGPU_MATRIX_CAUCHY = 1,
  RSGPU_MATRIX_JERASURE_LIKE = 2,
  RSGPU_MATRIX_CUSTOM = 3
};
/* src/core/recovery_plan.rs:11-16 (ReconstructionGoal) */
enum { RSGPU_GOAL_ALL = 0, RSGPU_GOAL_DATA = 1, RSGPU_GOAL_REQUIRED = 2 };
/* Field of a classic codec: galois_8 (bytes) or galois_16 (2-byte tower). */
enum { RSGPU_FIELD_GF8 = 0, RSGPU_FIELD_GF16_TOWER = 1 };

/* src/core/options.rs:97-146 (CodecOptions).  Zero means "automatic" exactly
 * as in the reference. */
typedef struct rsgpu_options {
  int32_t fast_one_parity;
  int32_t inversion_cache;
  size_t inversion_cache_capacity;
  size_t inversion_cache_max_bytes;
  int32_t codec_family;
  int32_t leopard_mode;
  int32_t matrix_mode;
  size_t max_parallel_jobs;
} rsgpu_options;

typedef struct rsgpu_codec rsgpu_codec;
typedef struct rsgpu_verify_ws rsgpu_verify_ws;
typedef struct rsgpu_reconstruct_ws rsgpu_reconstruct_ws;

/* Cache statistics (src/core/metrics.rs:105-215, ReconstructionCacheStats). */
typedef struct rsgpu_cache_stats {
  uint64_t requests, hits, misses, inserts, evictions;
  uint64_t entries, retained_bytes;
} rsgpu_cache_stats;

/* ------------------------------------------------------------ construction */
/* src/core/options.rs:134-146 (CodecOptions::default). */
void rsgpu_options_default(rsgpu_options *out);

/* src/core/codec.rs:264-349 (ReedSolomon::new / with_options), galois_8. */
int32_t rsgpu_codec_new(size_t data_shards, size_t parity_shards, const rsgpu_options *opts,
                        rsgpu_codec **out);
/* src/core/codec.rs:546-615 (with_custom_matrix); rows = parity_shards rows
 * of data_shards coefficients, row-major. */
int32_t rsgpu_codec_with_custom_matrix(size_t data_shards, size_t parity_shards,
                                       const uint8_t *rows, const rsgpu_options *opts,
                                       rsgpu_codec **out);
/* src/galois_16.rs:605 (galois_16::ReedSolomon::new): classic codec over the
 * GF((2^8)^2) tower field; shard lengths count bytes and must be even. */
int32_t rsgpu_codec_new_gf16(size_t data_shards, size_t parity_shards, rsgpu_codec **out);
/* galois_16::ReedSolomon::with_custom_matrix (src/core/codec.rs:546-615):
 * rows = parity_shards x data_shards tower elements, 2 bytes each
 * ([X coefficient, constant]). */
int32_t rsgpu_codec_gf16_with_custom_matrix(size_t data_shards, size_t parity_shards, const uint8_t *rows,
                                            rsgpu_codec **out);
void rsgpu_codec_free(rsgpu_codec *codec);

/* src/core/codec.rs:353-380 (data_shard_count, parity_shard_count, ...) */
size_t rsgpu_data_shard_count(const rsgpu_codec *codec);
size_t rsgpu_parity_shard_count(const rsgpu_codec *codec);
size_t rsgpu_total_shard_count(const rsgpu_codec *codec);
int32_t rsgpu_codec_family(const rsgpu_codec *codec);
/* Classic encoding matrix, (k+m)*k coefficients (2 bytes each for the tower
 * field); src/core/format.rs matrix rows.  Returns
 * RSGPU_ERR_UNSUPPORTED_CODEC_FAMILY for Leopard codecs. */
int32_t rsgpu_encoding_matrix(const rsgpu_codec *codec, uint8_t *out, size_t out_len);

/* ------------------------------------------------------------ per-call API */
/* src/core/encode.rs:935-947 (encode): shards[0..k) are read, shards[k..k+m)
 * are written. */
int32_t rsgpu_encode(const rsgpu_codec *codec, uint8_t *const *shards, const size_t *lens,
                     size_t n_shards, int32_t mem, void *stream);
/* src/core/encode.rs:950-972 (encode_sep). */
int32_t rsgpu_encode_sep(const rsgpu_codec *codec, const uint8_t *const *data,
                         const size_t *data_lens, size_t n_data, uint8_t *const *parity,
                         const size_t *parity_lens, size_t n_parity, int32_t mem, void *stream);
/* src/core/reconstruct.rs:731-790 (reconstruct / reconstruct_data /
 * reconstruct_some).  present[i] == 0 marks shard i missing; a missing shard
 * must still point at a writable buffer of the common length when it is a
 * target.  `lens[i]` is ignored for missing shards.  For
 * RSGPU_GOAL_REQUIRED, `required` holds n_required flags (k or k+m). */
int32_t rsgpu_reconstruct(const rsgpu_codec *codec, uint8_t *const *shards, const size_t *lens,
                          const uint8_t *present, size_t n_shards, int32_t goal,
                          const uint8_t *required, size_t n_required, int32_t mem,
                          void *stream);
/* src/core/verify.rs:72-94 (verify).  *ok receives 1 or 0. */
int32_t rsgpu_verify(const rsgpu_codec *codec, const uint8_t *const *shards, const size_t *lens,
                     size_t n_shards, int32_t *ok, int32_t mem, void *stream);

/* src/core/workspace.rs:16-69 (VerifyWorkspace) and src/core/verify.rs:96-115
 * (verify_with_workspace).  The workspace keeps the device staging and the
 * mismatch flag between calls. */
int32_t rsgpu_verify_ws_new(const rsgpu_codec *codec, size_t shard_len, rsgpu_verify_ws **out);
void rsgpu_verify_ws_free(rsgpu_verify_ws *ws);
int32_t rsgpu_verify_with_workspace(const rsgpu_codec *codec, const uint8_t *const *shards,
                                    const size_t *lens, size_t n_shards, rsgpu_verify_ws *ws,
                                    int32_t *ok, int32_t mem, void *stream);

/* src/core/verify.rs:157-176 (verify_with_buffer) and :180-200
 * (verify_with_buffer_par): the parity recomputed from shards[0..k) is
 * written into buffer[0..m) (n_buffer == m buffers of the shard length, in
 * `mem` like the shards) and *ok receives 1 when it equals shards[k..k+m).
 * Leopard codecs as verify_leopard_with_buffer (src/core/verify.rs:35-57).
 * Errors: piece count, then TooFew/TooManyBufferShards, then shard sizes. */
int32_t rsgpu_verify_with_buffer(const rsgpu_codec *codec, const uint8_t *const *shards, const size_t *lens,
                                 size_t n_shards, uint8_t *const *buffer, const size_t *buffer_lens,
                                 size_t n_buffer, int32_t *ok, int32_t mem, void *stream);

/* src/galois_8/policy.rs:543-700 (decode_idx): progressive recovery into
 * caller-initialised destinations.  NULL entries of dst / input stand for
 * None; both arrays hold k+m entries.  With expect_input (n_expect == k+m
 * flags), its first k expected indices are the decoding inputs and each call
 * adds (XOR) into every non-NULL dst the contributions of the inputs it
 * supplies, so calls over disjoint input batches accumulate the recovered
 * shards (zero the destinations before the first call).  With expect_input ==
 * NULL (merge mode), dst[i] ^= input[i] for every supplied input.  The whole
 * layout is validated before anything is written.  Classic GF(2^8) codecs
 * only (others: RSGPU_ERR_UNSUPPORTED_CODEC_FAMILY).  dst and input buffers
 * must not overlap. */
int32_t rsgpu_decode_idx(const rsgpu_codec *codec, uint8_t *const *dst, const size_t *dst_lens, size_t n_dst,
                         const uint8_t *expect_input, size_t n_expect, const uint8_t *const *input,
                         const size_t *input_lens, size_t n_input, int32_t mem, void *stream);

/* src/core/reconstruct.rs:539-726 (prepare_reconstruct_workspace /
 * reconstruct_with_workspace): a reusable plan for one erasure pattern.
 * Classic codecs only, as in the reference (Leopard:
 * RSGPU_ERR_UNSUPPORTED_CODEC_FAMILY).  Preparing builds (or takes from the
 * cache) the pattern's decode tables and keeps a private device copy, so a
 * singular custom matrix fails at prepare time and running the plan does no
 * cache lookup.  Reuse checks, in order: piece count, family, the codec's
 * shard counts and encoding format (InvalidCustomMatrix on a different
 * format), present shard lengths, the same missing pattern
 * (InvalidShardFlags), the same length (IncorrectShardSize). */
int32_t rsgpu_prepare_reconstruct_ws(const rsgpu_codec *codec, const uint8_t *present,
                                     size_t n_shards, size_t shard_len, int32_t goal,
                                     const uint8_t *required, size_t n_required,
                                     rsgpu_reconstruct_ws **out);
void rsgpu_reconstruct_ws_free(rsgpu_reconstruct_ws *ws);
/* Targets of a prepared plan (src/core/workspace.rs:92-112). */
size_t rsgpu_reconstruct_ws_targets(const rsgpu_reconstruct_ws *ws, size_t *out, size_t cap);
int32_t rsgpu_reconstruct_with_ws(const rsgpu_codec *codec, rsgpu_reconstruct_ws *ws,
                                  uint8_t *const *shards, const size_t *lens,
                                  const uint8_t *present, size_t n_shards, int32_t mem,
                                  void *stream);

/* ------------------------------------------------------------ batched API */
/* Many stripes of one codec and one shard length in a single launch (no
 * reference counterpart: the reference codes one stripe per call).
 * shard_ptrs holds n_stripes * (k+m) pointers, stripe-major, all in `mem`.
 * src/core/encode.rs:950-972 semantics per stripe. */
int32_t rsgpu_encode_batch(const rsgpu_codec *codec, size_t n_stripes, uint8_t *const *shard_ptrs,
                           size_t shard_len, int32_t mem, void *stream);
/* Per-stripe erasure patterns: present holds n_stripes * (k+m) flags.
 * src/core/reconstruct.rs:731-790 semantics per stripe. */
int32_t rsgpu_reconstruct_batch(const rsgpu_codec *codec, size_t n_stripes,
                                uint8_t *const *shard_ptrs, const uint8_t *present,
                                size_t shard_len, int32_t goal, int32_t mem, void *stream);
/* ok receives n_stripes flags (host memory).  src/core/verify.rs:72-94. */
int32_t rsgpu_verify_batch(const rsgpu_codec *codec, size_t n_stripes,
                           const uint8_t *const *shard_ptrs, size_t shard_len, uint8_t *ok,
                           int32_t mem, void *stream);

/* ------------------------------------------------------------ prepared batches */
/* A prepared batch holds the plans, decode tables and job/pointer tables of
 * one batched operation in device memory, so that running it again is a bare
 * kernel launch: it allocates nothing and never synchronizes, and can
 * therefore be captured in a CUDA graph.  Shard pointers must be device
 * pointers that stay valid for the life of the batch.  No reference
 * counterpart (the reference re-plans every call; its closest analogue is
 * the reusable ReconstructWorkspace, src/core/workspace.rs:70-112). */
enum { RSGPU_OP_ENCODE = 0, RSGPU_OP_RECONSTRUCT = 1, RSGPU_OP_VERIFY = 2 };
typedef struct rsgpu_batch rsgpu_batch;
int32_t rsgpu_batch_prepare(const rsgpu_codec *codec, int32_t op, size_t n_stripes,
                            uint8_t *const *shard_ptrs, const uint8_t *present, size_t shard_len,
                            int32_t goal, rsgpu_batch **out);
/* Queue the batch on `stream` (for verify: clear flags, then compare). */
int32_t rsgpu_batch_launch(rsgpu_batch *batch, void *stream);
/* Verify batches only: wait for `stream`, then write n_stripes flags. */
int32_t rsgpu_batch_verify_result(rsgpu_batch *batch, uint8_t *ok, void *stream);
/* Kernels one launch of this batch issues. */
uint32_t rsgpu_batch_kernel_count(const rsgpu_batch *batch);
void rsgpu_batch_free(rsgpu_batch *batch);

/* ------------------------------------------------------------ incremental parity, layout, format */
/* encode_single (src/core/encode.rs:889-909): data shard i_data's
 * contribution to the parity; i_data == 0 overwrites the parity (c * d_0),
 * later shards add to it, so calls for i = 0..k-1 in order give the full
 * parity.  `shards` holds k + m buffers; only shard i_data is read and only
 * the parity is written.  Leopard codecs: RSGPU_ERR_UNSUPPORTED_CODEC_FAMILY. */
int32_t rsgpu_encode_single(const rsgpu_codec *codec, size_t i_data, uint8_t *const *shards, const size_t *lens,
                            size_t n, int32_t mem, void *stream);
/* encode_single_sep (src/core/encode.rs:912-930). */
int32_t rsgpu_encode_single_sep(const rsgpu_codec *codec, size_t i_data, const uint8_t *data, size_t data_len,
                                uint8_t *const *parity, const size_t *parity_lens, size_t n_parity, int32_t mem,
                                void *stream);
/* update (src/core/encode.rs:1048-1120): parity += sum over changed data
 * shards j of c[j] * (old_j + new_j); new_data[j] = NULL marks an unchanged
 * shard (its new_lens entry is ignored). */
int32_t rsgpu_update(const rsgpu_codec *codec, const uint8_t *const *old_data, const size_t *old_lens, size_t n_old,
                     const uint8_t *const *new_data, const size_t *new_lens, size_t n_new, uint8_t *const *parity,
                     const size_t *parity_lens, size_t n_parity, int32_t mem, void *stream);
/* split / join (src/core/codec.rs:476-538), host memory, no device work:
 * split writes k shards of rsgpu_split_shard_len(data_len) bytes back to back
 * into `out` (zero-padded; Leopard rounds to a non-zero multiple of 64 bytes;
 * lengths count bytes, 2 per element for galois_16); join concatenates the k
 * data shards and keeps min(out_len, k * shard_len) bytes. */
size_t rsgpu_split_shard_len(const rsgpu_codec *codec, size_t data_len);
int32_t rsgpu_split(const rsgpu_codec *codec, const uint8_t *data, size_t data_len, uint8_t *out, size_t out_len);
int32_t rsgpu_join(const rsgpu_codec *codec, const uint8_t *const *shards, const size_t *lens, size_t n,
                   uint8_t *out, size_t out_len, size_t *written);
/* EncodingFormat::stable_id_bytes (src/core/format.rs:168-220), version 1:
 * *len = the identity's size; with out != NULL (cap >= *len) the bytes. */
int32_t rsgpu_format_id(const rsgpu_codec *codec, uint8_t *out, size_t cap, size_t *len);

/* ------------------------------------------------------------ block streaming */
/* src/core/stream.rs:650-1000 (encode_stream, verify_stream,
 * reconstruct_stream_from) over callbacks instead of Read / Write objects.
 * A read callback fills up to `cap` bytes of shard `shard` and returns the
 * count (0 at the end of that stream) or a negative error; the library retries
 * short reads until the block is full or the stream ends.  A write callback
 * writes all `len` bytes and returns >= 0, or a negative error.  Block size is
 * clamped to [1 KiB, 16 MiB] (default 4 MiB).  Classic GF(2^8) codecs only;
 * others get RSGPU_ERR_UNSUPPORTED_CODEC_FAMILY, like the reference.  On an
 * I/O failure the call returns RSGPU_ERR_STREAM_IO and `status` names the
 * shard and the callback's code; codec errors return their code with the
 * shard index in `status` (e.g. IncorrectShardSize for a short stream).
 * Every output block before a failing block has been written. */
typedef int64_t (*rsgpu_read_fn)(void *ctx, size_t shard, uint8_t *buf, size_t cap);
typedef int64_t (*rsgpu_write_fn)(void *ctx, size_t shard, const uint8_t *buf, size_t len);
typedef struct rsgpu_stream_options {
  size_t block_size;
} rsgpu_stream_options;
enum { RSGPU_STREAM_OK = 0, RSGPU_STREAM_CODEC = 1, RSGPU_STREAM_READ = 2, RSGPU_STREAM_WRITE = 3 };
typedef struct rsgpu_stream_status {
  int32_t kind;       /* RSGPU_STREAM_* */
  int32_t code;       /* codec: RSGPU_ERR_*; read / write: the callback's return value */
  size_t shard_index;
} rsgpu_stream_status;
void rsgpu_stream_options_default(rsgpu_stream_options *out);
/* encode_stream: n_data readers (data shards 0..k), n_parity writers (parity
 * shards k..k+m, passed as shard indices k..k+m to the callback).  Shorter data
 * streams are zero-padded to the block's longest one. */
int32_t rsgpu_encode_stream(const rsgpu_codec *codec, size_t n_data, rsgpu_read_fn read, void *read_ctx,
                            size_t n_parity, rsgpu_write_fn write, void *write_ctx, const rsgpu_stream_options *opts,
                            rsgpu_stream_status *status);
/* verify_stream: *ok = 1 when every block verifies. */
int32_t rsgpu_verify_stream(const rsgpu_codec *codec, size_t n_shards, rsgpu_read_fn read, void *read_ctx,
                            const rsgpu_stream_options *opts, int32_t *ok, rsgpu_stream_status *status);
/* reconstruct_stream_from: has_reader[i] / has_writer[i] mark the present
 * and the missing shards (exactly one of the two per index, else
 * InvalidShardFlags); every missing shard is rebuilt and written. */
int32_t rsgpu_reconstruct_stream_from(const rsgpu_codec *codec, size_t n_shards, const uint8_t *has_reader,
                                      rsgpu_read_fn read, void *read_ctx, const uint8_t *has_writer,
                                      rsgpu_write_fn write, void *write_ctx, const rsgpu_stream_options *opts,
                                      rsgpu_stream_status *status);

/* ------------------------------------------------------------ mixed batches */
/* A mixed batch runs many stripes of different codecs (classic GF(2^8),
 * Leopard GF(2^8) / GF(2^16)), shard lengths and operations in ONE persistent
 * kernel over a device work queue of column tiles, optionally launched
 * through a captured CUDA graph.  Like a prepared batch it is planned once and
 * launched any number of times without allocating or synchronizing; shard
 * pointers are device pointers that must stay valid, and every codec must
 * outlive the batch.  Each operation gets a plan (algorithm, tile); every plan
 * writes the same bytes, so the plan only changes the speed.  No reference
 * counterpart: the reference serves one stripe per call
 * (src/core/encode.rs:935-972, src/core/reconstruct.rs:731-790,
 * src/core/verify.rs:14-174), and these batches are the many-call form of
 * exactly those operations.  Tower-field (galois_16) codecs are not accepted
 * (RSGPU_ERR_UNSUPPORTED_CODEC_FAMILY). */
typedef struct rsgpu_mix rsgpu_mix;
typedef struct rsgpu_mix_op {
  const rsgpu_codec *codec;
  int32_t op;              /* RSGPU_OP_* */
  int32_t goal;            /* reconstruct: RSGPU_GOAL_ALL or RSGPU_GOAL_DATA */
  uint8_t *const *shards;  /* k + m device pointers */
  const uint8_t *present;  /* reconstruct: k + m flags (ignored otherwise) */
  size_t shard_len;
} rsgpu_mix_op;

/* Algorithms: RSGPU_ALGO_APPLY = the K1 table kernel over the operation's
 * coefficient matrix (classic; for Leopard GF(2^8) the FFT pipeline written
 * out as a dense matrix over the Leopard field); tile 0 = 8 KiB of columns and
 * four outputs per pass over the inputs, 1 = 4 KiB and four, 2 = 4 KiB and
 * eight.  RSGPU_ALGO_FFT = the Leopard transform, tile
 * t = 2^t 64-byte column blocks per work item (t = 1..3; transforms of at
 * most 16 lanes run in registers on 1 KiB of columns whatever t is). */
enum { RSGPU_ALGO_APPLY = 0, RSGPU_ALGO_FFT = 1 };
typedef struct rsgpu_plan {
  int32_t algo;
  int32_t tile;
} rsgpu_plan;

/* Planners: FIXED = a fixed rule per family; TABLE = the measured autotuner
 * table (FIXED where it has no entry); MODEL = the learned cost model, with
 * the table as its fallback.  Order: SUBMIT keeps the operations' order in the
 * queue; COST puts the most expensive work items first. */
enum { RSGPU_PLANNER_FIXED = 0, RSGPU_PLANNER_TABLE = 1, RSGPU_PLANNER_MODEL = 2 };
enum { RSGPU_ORDER_SUBMIT = 0, RSGPU_ORDER_COST = 1 };
typedef struct rsgpu_mix_options {
  int32_t planner;     /* RSGPU_PLANNER_* */
  int32_t order;       /* RSGPU_ORDER_* */
  int32_t graph;       /* nonzero: launch through a captured CUDA graph */
  int32_t ctas_per_sm; /* resident CTAs per SM (0: as many as fit) */
} rsgpu_mix_options;

typedef struct rsgpu_mix_info {
  size_t n_ops, n_jobs, n_items, n_classes;
  uint64_t algorithmic_bytes; /* bytes read + written by one launch */
  size_t device_bytes;        /* device memory the batch holds */
  uint32_t grid, smem_bytes, kernels_per_launch, pad;
} rsgpu_mix_info;

void rsgpu_mix_options_default(rsgpu_mix_options *out);
int32_t rsgpu_mix_prepare(const rsgpu_mix_op *ops, size_t n_ops, const rsgpu_mix_options *opts, rsgpu_mix **out);
/* As rsgpu_mix_prepare with an explicit plan per operation (the autotuner's
 * sweep uses it); RSGPU_ERR_INVALID_ARGUMENT for a plan the codec cannot run. */
int32_t rsgpu_mix_prepare_planned(const rsgpu_mix_op *ops, size_t n_ops, const rsgpu_plan *plans,
                                  const rsgpu_mix_options *opts, rsgpu_mix **out);
int32_t rsgpu_mix_launch(rsgpu_mix *mix, void *stream);
/* Wait for `stream`, then write one flag per operation: verify operations 1
 * when the parity matched, 0 otherwise; other operations 1. */
int32_t rsgpu_mix_results(rsgpu_mix *mix, uint8_t *ok, void *stream);
int32_t rsgpu_mix_get_info(const rsgpu_mix *mix, rsgpu_mix_info *out);
/* The plan chosen for each operation. */
int32_t rsgpu_mix_get_plans(const rsgpu_mix *mix, rsgpu_plan *out, size_t n_ops);
void rsgpu_mix_free(rsgpu_mix *mix);

/* ------------------------------------------------------------ autotuner and cost model */
/* The plan of a mixed-batch operation is chosen from measurements.
 *
 * Autotuner: rsgpu_tune measures every valid plan for each distinct class
 * among `ops` (class = family, k, m, operation, erasure-count bucket,
 * shard-length bucket), each on synthetic device stripes of the class's own
 * shape, and keeps the fastest in a process-wide table (the
 * RSGPU_PLANNER_TABLE planner).  Every measurement is also kept as a sample.
 *
 * Cost model: a small MLP (RSGPU_MODEL_FEATURES inputs, two hidden layers of
 * RSGPU_MODEL_HIDDEN ReLU units, one output per plan: predicted log2 GB/s)
 * trained and evaluated by the library's own CUDA kernels on the tuner's
 * samples (the RSGPU_PLANNER_MODEL planner; a class the table has measured
 * keeps its measured plan).  Plans never change bytes, so neither can change
 * an output.  Features of an operation (rsgpu_plan_features): classic GF(2^8),
 * Leopard GF(2^8), Leopard GF(2^16) indicators; log2 k / 16; log2 m / 16;
 * (log2 shard_len - 12) / 10; encode, reconstruct, verify indicators;
 * erased / m; erased data shards / max(erased, 1).  Plan order of the model's
 * outputs (rsgpu_plan_index): APPLY tiles 0, 1, 2, then FFT tiles 1, 2, 3.
 * No reference counterpart. */
#define RSGPU_MODEL_FEATURES 11
#define RSGPU_MODEL_PLANS 6
#define RSGPU_MODEL_HIDDEN 32
typedef struct rsgpu_tune_options {
  size_t target_bytes; /* shard bytes per measured batch (0: 256 MiB) */
  int32_t repeats;     /* timed launches per plan, best kept (0: 3) */
  int32_t pad;
} rsgpu_tune_options;
typedef struct rsgpu_tune_sample {
  float features[RSGPU_MODEL_FEATURES];
  rsgpu_plan plan;
  float gbps; /* algorithmic bytes / second / 1e9 */
} rsgpu_tune_sample;
int32_t rsgpu_plan_features(const rsgpu_mix_op *op, float *out);
/* Index of `plan` among the model's outputs, or -1. */
int32_t rsgpu_plan_index(rsgpu_plan plan);
int32_t rsgpu_tune(const rsgpu_mix_op *ops, size_t n_ops, const rsgpu_tune_options *opts, size_t *classes_tuned);
size_t rsgpu_tuner_samples(rsgpu_tune_sample *out, size_t cap);
size_t rsgpu_tuner_table_size(void);
/* Best measured plan of the class `op` belongs to (0), or RSGPU_ERR_INVALID_INDEX. */
int32_t rsgpu_tuner_lookup(const rsgpu_mix_op *op, rsgpu_plan *out);
int32_t rsgpu_tuner_save(const char *path);
int32_t rsgpu_tuner_load(const char *path);
void rsgpu_tuner_clear(void);

typedef struct rsgpu_train_options {
  int32_t epochs;   /* full-batch Adam steps (0: 2000) */
  float lr;         /* (0: 3e-3) */
  uint64_t seed;    /* weight initialization */
} rsgpu_train_options;
/* Parameters: W1 (F x H), b1 (H), W2 (H x H), b2 (H), W3 (H x P), b3 (P),
 * row-major, in that order. */
size_t rsgpu_model_param_count(void);
int32_t rsgpu_model_get_params(float *out, size_t n);
int32_t rsgpu_model_set_params(const float *in, size_t n);
/* Train on n rows: features (n x F), targets (n x P, log2 GB/s) and mask
 * (n x P, 1 where the target was measured).  Loss = mean over masked entries
 * of the squared error.  Installs the trained model for the planner. */
int32_t rsgpu_model_train(const float *features, const float *targets, const uint8_t *mask, size_t n,
                          const rsgpu_train_options *opts, float *final_loss);
/* The same, on the tuner's samples (best of repeated measurements per class
 * and plan). */
int32_t rsgpu_model_train_from_tuner(const rsgpu_train_options *opts, float *final_loss);
/* Forward pass on the GPU: out = n x P predictions. */
int32_t rsgpu_model_predict(const float *features, size_t n, float *out);
/* One forward and backward pass with `params` on the GPU (no update): the
 * loss and its gradient with respect to every parameter. */
int32_t rsgpu_model_gradients(const float *params, const float *features, const float *targets, const uint8_t *mask,
                              size_t n, float *loss, float *grads);
int32_t rsgpu_model_ready(void);

/* ------------------------------------------------------------ request server */
/* Continuous batching of encode / reconstruct / verify requests onto the GPU.
 * Submit from any thread; a worker thread admits pending requests in arrival
 * order while a request slot and the device-memory budget allow (a request
 * holds (k + m) * shard_len bytes while admitted), runs everything admitted
 * since the last launch as ONE mixed batch (plans from `planner`) on the next
 * free of `streams` launch streams, and reports completions.  Launches overlap
 * on the device; requests arriving meanwhile join the next launch.
 * Host-memory requests (pinned memory recommended) are staged through device
 * memory: inputs in, outputs (parity, rebuilt shards) back into the caller's
 * buffers; device-memory requests (shards resident in HBM) run in place.
 * The planner reads the cost model's picks from a grid of predictions over
 * quantized features (made by one batched GPU forward pass per operation kind
 * and weight set), and a Leopard GF(2^8) rebuild pattern whose dense map has
 * become due runs the FFT decode while the server derives the map on a side
 * stream, so building a batch never waits for the GPU.  Codecs must outlive
 * the server (a map derivation may still use one after its requests are
 * done).
 * Shard buffers must stay untouched until the request completes.  Results
 * are byte-identical to the per-call entry points whatever else is in the
 * batch.  No reference counterpart: the reference is called once per stripe
 * by the storage node's own request handlers. */
typedef struct rsgpu_server rsgpu_server;
typedef struct rsgpu_server_options {
  size_t device_budget;  /* bytes admitted requests may hold (0: half of free memory) */
  uint32_t max_inflight; /* requests admitted at once (0: 4096) */
  uint32_t max_batch;    /* requests per launch (0: 64) */
  uint32_t streams;      /* launches in flight at once (0: 3) */
  int32_t planner;       /* RSGPU_PLANNER_* (default MODEL) */
} rsgpu_server_options;
typedef struct rsgpu_request {
  const rsgpu_codec *codec;
  int32_t op;              /* RSGPU_OP_* */
  int32_t goal;            /* reconstruct: RSGPU_GOAL_ALL or _DATA */
  uint8_t *const *shards;  /* k + m pointers (copied at submit) */
  const uint8_t *present;  /* reconstruct: k + m flags (copied at submit) */
  size_t shard_len;
  int32_t mem;             /* RSGPU_MEM_HOST or RSGPU_MEM_DEVICE */
  int32_t pad;
  uint64_t tag;            /* returned with the completion */
} rsgpu_request;
typedef struct rsgpu_completion {
  uint64_t tag;
  int32_t status;  /* 0 or an error code */
  int32_t ok;      /* verify: 1 when the parity matched, 0 otherwise; others 1 */
  double submit_s, admit_s, done_s; /* seconds since the server started */
} rsgpu_completion;
typedef struct rsgpu_server_stats {
  uint64_t submitted, completed, launches;
  size_t pending, inflight, budget_bytes, reserved_bytes, max_reserved_bytes;
  uint32_t max_concurrent_launches, pad;
  double prepare_seconds; /* worker time spent planning, building and launching batches */
  double max_prepare_seconds;  /* the longest single build-and-launch of a batch */
  double max_loop_gap_seconds; /* the longest time between two passes of the worker loop */
} rsgpu_server_stats;
void rsgpu_server_options_default(rsgpu_server_options *out);
int32_t rsgpu_server_new(const rsgpu_server_options *opts, rsgpu_server **out);
/* Validation errors (reference precedence) return immediately; a request
 * larger than the whole budget gets RSGPU_ERR_OUT_OF_MEMORY. */
int32_t rsgpu_server_submit(rsgpu_server *s, const rsgpu_request *r);
/* Up to `cap` completions; waits up to timeout_ms (-1: until one arrives). */
size_t rsgpu_server_poll(rsgpu_server *s, rsgpu_completion *out, size_t cap, int32_t timeout_ms);
int32_t rsgpu_server_get_stats(rsgpu_server *s, rsgpu_server_stats *out);
/* Finishes every submitted request, then stops. */
void rsgpu_server_free(rsgpu_server *s);

/* ------------------------------------------------------------ no-allocation path */
/* Leopard reconstruction (every missing shard, like rsgpu_reconstruct with
 * RSGPU_GOAL_ALL and RSGPU_MEM_DEVICE) that allocates no memory at all.  It
 * has no counterpart in the reference.
 *
 * Who needs it: callers that must not allocate device memory while serving,
 * for example a storage node that reserved the GPU's memory for its shard
 * buffers at start-up, or a process held to a fixed device-memory quota.
 * For them a cudaMalloc can fail when the memory is already spoken for, and
 * it can also synchronize the device, stalling the other streams mid-request.
 * The regular entry points allocate job tables, decode plans and, for codes
 * too wide for shared memory, the work rows; this one uses fixed buffers in
 * static device memory instead (about 16.3 MiB per GPU, held by every GPU that
 * loads the library until the process exits).
 *
 * Limits: the codec must be Leopard (GF(2^8) or GF(2^16)) with at most
 * RSGPU_NOALLOC_MAX_LANES transform lanes (next power of two of
 * next_pow2(parity) + data); larger codes get RSGPU_ERR_SCRATCH_LIMIT.
 * Shard pointers are device pointers.
 *
 * Usage rules: the first call on a device looks up the static buffers'
 * device addresses (cudaGetSymbolAddress); make that first call before any
 * stream capture.  The work is queued on `stream` and the call returns
 * without waiting.  Every call shares the same static buffers, which keep the
 * previous call's contents (each call rewrites everything it reads before
 * reading it): two calls whose work overlaps on the GPU, for example on two
 * streams, race and produce garbage. */
#define RSGPU_NOALLOC_MAX_LANES 16384u
#define RSGPU_NOALLOC_SCRATCH_BYTES (16u << 20)
int32_t rsgpu_leopard_reconstruct_noalloc(const rsgpu_codec *codec, uint8_t *const *shards, const size_t *lens,
                                          const uint8_t *present, size_t n_shards, void *stream);

/* ------------------------------------------------------------ introspection */
/* src/core/codec.rs:412-414 (reconstruction_cache_stats): device decode-table
 * cache of a classic codec; for Leopard codecs, the error-locator cache (one
 * entry per erasure pattern, least recently used patterns evicted beyond
 * 32 MiB or 64 patterns, whichever is larger; the reference bounds its
 * decode-plan cache the same way, src/core/leopard_gf16/decode.rs:268-305). */
int32_t rsgpu_get_cache_stats(const rsgpu_codec *codec, rsgpu_cache_stats *out);
/* Number of kernels this process launched through the library so far. */
uint64_t rsgpu_kernel_launch_count(void);
/* Human-readable text for a return code. */
const char *rsgpu_error_string(int32_t code);
/* Library build identification ("rsgpu <version> sm_100a"). */
const char *rsgpu_version(void);

#ifdef __cplusplus
}
#endif
#endif /* RSGPU_H */
