// batch.cu -- mixed batches: many stripes of different codecs, shard lengths
// and operations in one persistent kernel over a device work queue.
//
// The reference runs one call per stripe (src/core/encode.rs:935-972,
// src/core/reconstruct.rs:731-790, src/core/verify.rs:14-174), each over its
// own rayon pool; a storage node that serves many small, uneven stripes pays
// a launch, a plan and a tail per stripe.  Here the host turns every
// operation of a batch into column tiles ("items") once, ahead of time:
//
//   item  = (job, tile)             8 bytes, ordered by the planner
//   job   = one stripe's operation  (class, shard length, K1 descriptor or
//                                    index of its Leopard descriptor)
//   class = one kernel body         (K1 tile of 8 or 4 KiB columns, write or
//                                    verify; Leopard FFT encode / verify /
//                                    decode over GF(2^8) or GF(2^16) with its
//                                    codec's geometry and tile width)
//
// and k_mix, launched with one resident CTA set per SM, pulls items from a
// global counter until the queue is empty.  Memory-bound K1 tiles and
// compute-bound Leopard tiles of different stripes therefore share every SM
// at once, small stripes cost no launch of their own, and the queue order
// (heaviest items first) keeps the tail short.  Preparing resolves decode
// tables (K3), error locators (K7a) and dense maps once, copies every
// per-pattern table into memory the batch owns, and can capture the launch
// (counter reset + kernel) in a CUDA graph; launching allocates nothing and
// never synchronizes.
//
// Plans.  Every operation gets a plan (algorithm, tile):
//   RSGPU_ALGO_APPLY  the K1 table kernel over the operation's coefficient
//                     matrix: the classic matrix, or for Leopard GF(2^8) the
//                     FFT pipeline written out as a dense matrix over the
//                     Leopard field (exact: the pipeline is linear); tile 0 =
//                     8 KiB of columns per item, 1 = 4 KiB;
//   RSGPU_ALGO_FFT    the Leopard transform tile, 2^tile 64-byte blocks per
//                     item.
// Every plan writes the same bytes; plans only change the speed.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <numeric>
#include <string>
#include <tuple>
#include <vector>

#include "apply_tile.cuh"
#include "batch.hpp"
#include "codec.hpp"
#include "handles.hpp"
#include "launch_cfg.hpp"
#include "leo_fft.cuh"
#include "leopard.hpp"

namespace rsgpu {

#define RS_CUDA(expr)                              \
  do {                                             \
    cudaError_t e_ = (expr);                       \
    if (e_ != cudaSuccess) return cuda_status(e_); \
  } while (0)

namespace {

constexpr int kMixThreads = 256;
// Resident k_mix CTAs per SM when shared memory allows (80 registers).  Three
// rather than two (128 registers) ran the bench's mixed workload 11% faster
// (791.7 against 710.9 GB/s; its fixed-plan, transform-heavy batches 15%)
// although the transform tiles then spill; the K1 tiles do not.  Four (64
// registers) spilled more and gained 3%.
constexpr int kMixBlocks = 3;
constexpr uint32_t kTailTile = 0xFFFFFFFFu;

// K1 kinds: bits 0..1 = tile (0: 8 KiB of columns, 4 outputs per pass over
// the inputs; 1: 4 KiB, 4; 2: 4 KiB, 8), bit 2 = verify.
enum MixKind : uint32_t {
  MK_APPLY = 0,
  MK_APPLY_VERIFY = 4,
  MK_LEO8_ENC = 8,
  MK_LEO8_VERIFY = 9,
  MK_LEO8_DEC = 10,
  MK_LEO16_ENC = 16,
  MK_LEO16_VERIFY = 17,
  MK_LEO16_DEC = 18,
};

struct MixItem {
  uint32_t job;
  uint32_t tile;  // tile index within the job, or kTailTile (K1 byte tail)
};

struct MixJob {
  uint32_t cls;
  uint32_t sub;  // Leopard: index into the LeoJob array
  uint64_t len;  // bytes per shard
  JobDesc d;     // K1 jobs
};
static_assert(sizeof(MixJob) == 48, "MixJob layout");

struct MixClass {
  uint32_t kind;
  uint32_t global_work;  // Leopard: work rows in the per-CTA scratch slab
  uint32_t tile_bytes;   // Leopard: columns per work item
  uint32_t pad;
  LeoArgs leo;           // Leopard: geometry, tables, stage plans, nb
};

struct MixArgs {
  const MixItem *items;
  const MixJob *jobs;
  const MixClass *classes;
  const uint8_t *const *ptrs;
  uint32_t *flags;
  uint32_t *counter;
  uint32_t *scratch;       // per-CTA Leopard work rows (wide codes)
  uint64_t scratch_words;  // words per CTA
  uint32_t n_items;
};

__global__ void __launch_bounds__(kMixThreads, kMixBlocks) k_mix(MixArgs a) {
  extern __shared__ __align__(16) uint32_t smem[];
  __shared__ uint32_t s_item, s_bad;
  __shared__ LeoArgs s_leo;
  uint32_t *gwork = a.scratch ? a.scratch + size_t(blockIdx.x) * a.scratch_words : nullptr;
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(a.counter, 1u);
    __syncthreads();
    const uint32_t it = s_item;
    if (it >= a.n_items) break;  // CTA-uniform
    const MixItem item = a.items[it];
    const MixJob &job = a.jobs[item.job];
    const MixClass &cls = a.classes[job.cls];
    const uint32_t kind = cls.kind;
    if (kind < MK_LEO8_ENC) {
      const JobDesc d = job.d;
      if (item.tile == kTailTile) {
        const bool verify = kind & MK_APPLY_VERIFY;
        bool bad = false;
        for (uint64_t col = d.vec_len + threadIdx.x; col < job.len; col += kMixThreads)
          bad |= verify ? apply_column<true>(a.ptrs, d, col) : apply_column<false>(a.ptrs, d, col);
        if (bad) atomicOr(a.flags + d.flag_idx, 1u);
      } else {
        const uint64_t t = item.tile;
        switch (kind) {
          case 0: apply_tile<1, 2, 4, 0, false>(a.ptrs, a.flags, d, t * (2 * kApplyTile)); break;
          case 1: apply_tile<1, 1, 4, 0, false>(a.ptrs, a.flags, d, t * kApplyTile); break;
          case 2: apply_tile<2, 1, 4, 0, false>(a.ptrs, a.flags, d, t * kApplyTile); break;
          case 4: apply_tile<1, 2, 4, 0, true>(a.ptrs, a.flags, d, t * (2 * kApplyTile)); break;
          case 5: apply_tile<1, 1, 4, 0, true>(a.ptrs, a.flags, d, t * kApplyTile); break;
          default: apply_tile<2, 1, 4, 0, true>(a.ptrs, a.flags, d, t * kApplyTile); break;
        }
      }
    } else {
      // The class's Leopard arguments go to shared memory once per item, so
      // the transform loops read them without global loads.
      constexpr int kWords = sizeof(LeoArgs) / 4;
      if (threadIdx.x < kWords)
        reinterpret_cast<uint32_t *>(&s_leo)[threadIdx.x] = reinterpret_cast<const uint32_t *>(&cls.leo)[threadIdx.x];
      __syncthreads();
      const LeoJob jd = s_leo.jobs[job.sub];
      uint32_t *W = cls.global_work ? gwork : smem;
      const uint64_t col0 = uint64_t(item.tile) * cls.tile_bytes;
      switch (kind) {
        case MK_LEO8_ENC: fft_encode_tile<8, false, kMixThreads>(W, s_leo, jd, col0, job.len, &s_bad); break;
        case MK_LEO8_VERIFY: fft_encode_tile<8, true, kMixThreads>(W, s_leo, jd, col0, job.len, &s_bad); break;
        case MK_LEO8_DEC: fft_decode_tile<8, kMixThreads, false>(W, s_leo, jd, col0, job.len); break;
        case MK_LEO16_ENC: fft_encode_tile<16, false, kMixThreads>(W, s_leo, jd, col0, job.len, &s_bad); break;
        case MK_LEO16_VERIFY: fft_encode_tile<16, true, kMixThreads>(W, s_leo, jd, col0, job.len, &s_bad); break;
        default: fft_decode_tile<16, kMixThreads, false>(W, s_leo, jd, col0, job.len); break;
      }
    }
    __syncthreads();  // every thread is done with s_item / s_leo before the next grab
  }
}

// Largest shared-memory work area of a transform tile; a batch that uses it
// runs two CTAs per SM, one whose tiles need at most ~72 KiB runs kMixBlocks.
constexpr size_t kMixSmem = 96 * 1024;

size_t align256(size_t n) { return (n + 255) & ~size_t(255); }

int sm_count() {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  }
  return sms;
}

bool is_leopard(const Codec &c) { return c.family != RSGPU_FAMILY_CLASSIC; }

// Resident k_mix CTAs per SM for a dynamic shared-memory size (the limit is
// raised to the largest size a batch can ask for the first time it is
// needed).
cudaError_t mix_shape(size_t smem, int *per_sm) {
  const void *fn = reinterpret_cast<const void *>(k_mix);
  if (smem > 48 * 1024 - 1024) {
    cudaError_t e = ensure_smem_limit(fn, std::max(smem, kMixSmem + (8 << 10)));
    if (e != cudaSuccess) return e;
  }
  return blocks_per_sm(fn, kMixThreads, smem, per_sm);
}
bool is_tower(const Codec &c) { return c.family == RSGPU_FAMILY_CLASSIC && c.field != RSGPU_FIELD_GF8; }

// Transform lanes of one column (m for encode / verify, n for decode); at
// most 16 run in registers with no work rows.
uint32_t fft_reg_lanes(const LeoGeometry &g, int op) { return op == RSGPU_OP_RECONSTRUCT ? g.n : g.m; }
// Work rows of a tile in shared (or global) memory: IFFT scratch plus
// accumulator (2m) for encode, n for decode; none in registers-only mode.
uint32_t fft_rows(const LeoGeometry &g, int op) {
  if (fft_reg_lanes(g, op) <= 16) return 0;
  return op == RSGPU_OP_RECONSTRUCT ? g.n : 2 * g.m;
}
uint64_t fft_item_bytes(const LeoGeometry &g, int op, uint32_t nb) {
  return fft_reg_lanes(g, op) <= 16 ? uint64_t(4 * kMixThreads) : uint64_t(64) * nb;
}

}  // namespace

// ------------------------------------------------------------------ planning
bool mix_plan_valid(const Codec &c, int op, const rsgpu_plan &p) {
  (void)op;
  if (!is_leopard(c)) return p.algo == RSGPU_ALGO_APPLY && p.tile >= 0 && p.tile <= 2;
  if (p.algo == RSGPU_ALGO_FFT) return p.tile >= 1 && p.tile <= 3;
  // Dense maps exist for the byte field only.
  return p.algo == RSGPU_ALGO_APPLY && c.family == RSGPU_FAMILY_LEOPARD_GF8 && p.tile >= 0 && p.tile <= 2;
}

bool mix_fft_in_registers(Codec &c, int op) {
  if (!is_leopard(c)) return false;
  LeoGeometry g{};
  leopard_geometry(c, &g);
  return fft_reg_lanes(g, op) <= 16;
}

rsgpu_plan mix_default_plan(Codec &c, int op, size_t len) {
  rsgpu_plan p{};
  if (!is_leopard(c)) {
    p.algo = RSGPU_ALGO_APPLY;
    p.tile = len >= 2 * kApplyTile ? 0 : 1;
    return p;
  }
  LeoGeometry g{};
  leopard_geometry(c, &g);
  const uint32_t rows = fft_rows(g, op);
  int t = 1;  // 2^t 64-byte blocks per item (ignored in registers-only mode)
  while (t < 3 && size_t(rows) * (size_t(64) << (t + 1)) <= kMixSmem && (size_t(64) << (t + 1)) <= len) ++t;
  p.algo = RSGPU_ALGO_FFT;
  p.tile = t;
  return p;
}

namespace {

// The plan table prices each class on batches that fill the GPU, where wider
// Leopard transform tiles (more 64-byte blocks per work item) win.  A batch
// with fewer work items than k_mix has resident CTAs leaves SMs idle, and there
// the finest tile is the fastest: more items run side by side.  Measured on one
// B200, a lone GF(2^16) 2048+1024 rebuild of 8 KiB shards takes 2.38 ms at
// 4 blocks per item and 1.17 ms at 2 (1024+512 at 16 KiB: 1.12 -> 0.53 ms).
// Every tile produces the same bytes.
void refine_small_batch(const rsgpu_mix_op *ops, size_t n_ops, std::vector<rsgpu_plan> &plans) {
  const uint64_t slots = uint64_t(kMixBlocks) * sm_count();
  uint64_t items = 0;
  bool coarse = false;
  for (size_t i = 0; i < n_ops && items < slots; ++i) {
    const size_t len = ops[i].shard_len;
    uint64_t tile;
    if (plans[i].algo == RSGPU_ALGO_FFT) {
      LeoGeometry g{};
      leopard_geometry(const_cast<rsgpu_codec *>(ops[i].codec)->c, &g);
      tile = fft_item_bytes(g, ops[i].op, 1u << plans[i].tile);
      coarse = coarse || plans[i].tile > 1;
    } else {
      tile = plans[i].tile == 0 ? 2 * kApplyTile : kApplyTile;
    }
    items += (len + tile - 1) / tile;
  }
  if (!coarse || items >= slots) return;
  for (size_t i = 0; i < n_ops; ++i)
    if (plans[i].algo == RSGPU_ALGO_FFT && plans[i].tile > 1) plans[i].tile = 1;
}

}  // namespace

// ------------------------------------------------------------------ the batch
struct MixBatch {
  std::vector<rsgpu_plan> plans;
  size_t n_ops = 0;
  void *d_blob = nullptr;
  uint32_t *d_flags = nullptr;
  uint32_t *d_counter = nullptr;
  uint32_t *d_scratch = nullptr;
  uint16_t *d_locs = nullptr;     // the batch's copies of its Leopard error locators
  bool scratch_borrowed = false;  // d_scratch belongs to the caller's ScratchSlot
  MixArgs args{};
  size_t smem = 0;
  int grid = 0;
  bool any_verify = false;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  rsgpu_mix_info info{};
  std::vector<uint32_t *> owned_tables;  // private copies of classic decode tables
  // One-shot batches: wide Leopard reconstructions run by their codec's own
  // decode kernel, launched on the batch's stream after k_mix.
  std::vector<std::shared_ptr<LeoLaunch>> side;
  uint32_t mix_kernels = 0;  // k_mix launches per launch (0 or 1)
  std::vector<void *> ordered_bufs;  // one-shot batches: dense maps derived on the stream
  // Stream-ordered batches (one-shot launches of the request server): device
  // memory comes from cudaMallocAsync on `stream` and goes back with
  // cudaFreeAsync after the work queued there, so neither building nor
  // freeing the batch synchronizes the device.
  cudaStream_t stream = nullptr;
  bool stream_ordered = false;
  ~MixBatch() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (stream_ordered) {
      for (void *p : {(void *)d_blob, (void *)d_flags, (void *)d_counter, (void *)d_locs})
        if (p) cudaFreeAsync(p, stream);
      for (void *p : ordered_bufs) cudaFreeAsync(p, stream);
      if (d_scratch && !scratch_borrowed) cudaFreeAsync(d_scratch, stream);
      return;
    }
    if (d_blob || d_flags || d_counter || d_scratch || d_locs) cudaDeviceSynchronize();
    if (d_locs) cudaFree(d_locs);
    if (d_blob) cudaFree(d_blob);
    if (d_flags) cudaFree(d_flags);
    if (d_counter) cudaFree(d_counter);
    if (d_scratch) cudaFree(d_scratch);
    for (uint32_t *t : owned_tables) cudaFree(t);
  }
  template <class T>
  cudaError_t alloc(T **p, size_t bytes) {
    return stream_ordered ? cudaError_t(lib_malloc_async(reinterpret_cast<void **>(p), bytes, stream))
                          : cudaMalloc(reinterpret_cast<void **>(p), bytes);
  }

  int enqueue(cudaStream_t s) const {
    RS_CUDA(cudaMemsetAsync(d_counter, 0, sizeof(uint32_t), s));
    if (any_verify) RS_CUDA(cudaMemsetAsync(d_flags, 0, std::max<size_t>(n_ops, 1) * 4, s));
    if (args.n_items) {
      k_mix<<<grid, kMixThreads, smem, s>>>(args);
      RS_CUDA(cudaGetLastError());
    }
    for (const auto &L : side) {
      const int rc = leo_launch(*L, s);
      if (rc) return rc;
    }
    return RSGPU_OK;
  }
};

namespace {

int validate_op(const rsgpu_mix_op &o, int device) {
  if (!o.codec || !o.shards) return RSGPU_ERR_INVALID_ARGUMENT;
  if (o.op < RSGPU_OP_ENCODE || o.op > RSGPU_OP_VERIFY) return RSGPU_ERR_INVALID_ARGUMENT;
  const Codec &c = o.codec->c;
  if (c.device != device) return RSGPU_ERR_INVALID_ARGUMENT;
  if (is_tower(c)) return RSGPU_ERR_UNSUPPORTED_CODEC_FAMILY;
  if (o.shard_len == 0) return RSGPU_ERR_EMPTY_SHARD;
  if (is_leopard(c) && (o.shard_len % 64)) return RSGPU_ERR_INCORRECT_SHARD_SIZE;
  const size_t total = c.k + c.m;
  for (size_t i = 0; i < total; ++i)
    if (!o.shards[i]) return RSGPU_ERR_INVALID_ARGUMENT;
  if (o.op == RSGPU_OP_RECONSTRUCT) {
    if (!o.present || (o.goal != RSGPU_GOAL_ALL && o.goal != RSGPU_GOAL_DATA)) return RSGPU_ERR_INVALID_SHARD_FLAGS;
    size_t np = 0;
    for (size_t i = 0; i < total; ++i) np += o.present[i] ? 1 : 0;
    if (np < c.k) return RSGPU_ERR_TOO_FEW_SHARDS_PRESENT;
    // Leopard recovers at most m missing shards (src/core/leopard_gf16/decode.rs:744-748).
    if (is_leopard(c) && total - np > c.m) return RSGPU_ERR_TOO_FEW_SHARDS_PRESENT;
  }
  return RSGPU_OK;
}

// Host image of the batch before upload.
struct MixBuild {
  std::vector<MixClass> classes;
  std::map<std::tuple<const Codec *, uint32_t, uint32_t>, uint32_t> leo_class;  // (codec, kind, nb) -> class
  std::vector<MixJob> jobs;
  std::vector<LeoJob> leo_jobs;
  std::vector<const uint8_t *> ptrs;
  std::vector<uint8_t> roles;
  std::vector<size_t> role_of_leo_job;  // offset into roles, or SIZE_MAX
  std::vector<uint32_t> tables;         // host-packed K1 tables (dense Leopard maps)
  std::vector<size_t> table_of_job;     // word offset into tables (SIZE_MAX: none)
  std::vector<double> job_cost;         // relative cost per item
  uint32_t apply_class[8] = {UINT32_MAX, UINT32_MAX, UINT32_MAX, UINT32_MAX,
                             UINT32_MAX, UINT32_MAX, UINT32_MAX, UINT32_MAX};
  uint64_t scratch_words = 0;
  size_t smem = 0;
  uint64_t algorithmic_bytes = 0;

  uint32_t apply_cls(uint32_t kind) {
    if (apply_class[kind] == UINT32_MAX) {
      MixClass c{};
      c.kind = kind;
      apply_class[kind] = uint32_t(classes.size());
      classes.push_back(c);
    }
    return apply_class[kind];
  }

  void push_job(MixJob j, size_t table_word, double cost) {
    jobs.push_back(j);
    table_of_job.push_back(table_word);
    job_cost.push_back(cost);
  }
};

// Grows a stream's work-row buffer to `need` bytes (with headroom), in the
// stream's order: the old buffer is freed behind the work queued before.
cudaError_t grow_slot(ScratchSlot &slot, size_t need, cudaStream_t s) {
  if (slot.bytes >= need) return cudaSuccess;
  if (slot.ptr) {
    cudaError_t e = cudaFreeAsync(slot.ptr, s);
    if (e != cudaSuccess) return e;
  }
  slot.ptr = nullptr;
  slot.bytes = 0;
  const size_t want = need + need / 4;
  cudaError_t e = cudaError_t(lib_malloc_async(&slot.ptr, want, s));
  if (e != cudaSuccess) return e;
  slot.bytes = want;
  return cudaSuccess;
}

// Relative cost of one item: bytes it moves times a per-algorithm factor.
// Only the order of the queue depends on it; the cost model refines it.
double item_cost(uint64_t tile_bytes, size_t shards, double factor) { return double(tile_bytes) * shards * factor; }

int add_apply_job(MixBuild &B, const rsgpu_plan &plan, bool verify, size_t n_in, size_t n_out, size_t ptr_off,
                  size_t len, uint32_t flag_idx, const uint32_t *dev_tbl, size_t host_tbl) {
  const uint32_t kind = uint32_t(plan.tile) | (verify ? MK_APPLY_VERIFY : 0u);
  MixJob j{};
  j.cls = B.apply_cls(kind);
  j.len = len;
  j.d.ptr_off = uint32_t(ptr_off);
  j.d.n_in = uint16_t(n_in);
  j.d.n_out = uint16_t(n_out);
  j.d.flag_idx = flag_idx;
  j.d.tbl = dev_tbl;
  bool aligned = true;
  for (size_t i = 0; i < n_in + n_out; ++i) aligned &= (reinterpret_cast<uintptr_t>(B.ptrs[ptr_off + i]) & 15) == 0;
  j.d.vec_len = aligned ? (len & ~uint64_t(15)) : 0;
  const double passes = double((n_out + 3) / 4);
  B.push_job(j, host_tbl, item_cost(1, n_in + n_out, 1.0 + 0.1 * passes * n_in / 16.0));
  return RSGPU_OK;
}

}  // namespace

int mix_build(const rsgpu_mix_op *ops, size_t n_ops, const rsgpu_plan *forced, const rsgpu_mix_options &opt,
              MixPtr &out, cudaStream_t ordered, ScratchSlot *scratch, std::vector<DenseWant> *deferred) {
  int device = 0;
  RS_CUDA(cudaGetDevice(&device));
  for (size_t i = 0; i < n_ops; ++i) {
    int rc = validate_op(ops[i], device);
    if (rc) return rc;
  }
  MixPtr batch(new MixBatch());
  MixBatch &b = *batch;
  if (ordered) {
    if (opt.graph) return RSGPU_ERR_INVALID_ARGUMENT;
    b.stream = ordered;
    b.stream_ordered = true;
  }
  b.n_ops = n_ops;
  b.plans.resize(n_ops);
  for (size_t i = 0; i < n_ops; ++i) {
    Codec &c = const_cast<rsgpu_codec *>(ops[i].codec)->c;
    b.plans[i] = forced ? forced[i] : mix_default_plan(c, ops[i].op, ops[i].shard_len);
  }
  if (!forced) {
    int rc = mix_plan_batch(ops, n_ops, opt.planner, b.plans);
    if (rc) return rc;
    // A one-shot batch (the request server's) runs a Leopard GF(2^8)
    // rebuild through its dense map only when the per-call rule says so:
    // the plan table prices launches, and deriving a new pattern's map (a
    // small FFT launch, a wait and host packing) is host time that a batch
    // run once cannot amortise.  Prepared batches keep the planner's choice.
    if (b.stream_ordered)
      for (size_t i = 0; i < n_ops; ++i) {
        Codec &c = const_cast<rsgpu_codec *>(ops[i].codec)->c;
        if (ops[i].op != RSGPU_OP_RECONSTRUCT || c.family != RSGPU_FAMILY_LEOPARD_GF8 ||
            b.plans[i].algo != RSGPU_ALGO_APPLY)
          continue;
        if (!leopard_dense_due(c, ops[i].present, ops[i].goal, ops[i].shard_len)) {
          b.plans[i] = mix_default_plan(c, ops[i].op, ops[i].shard_len);
        } else if (deferred && !leopard_dense_cached(c, ops[i].present, ops[i].goal)) {
          b.plans[i] = mix_default_plan(c, ops[i].op, ops[i].shard_len);
          deferred->push_back(DenseWant{ops[i].codec,
                                        std::string(reinterpret_cast<const char *>(ops[i].present), c.k + c.m),
                                        ops[i].goal});
        }
      }
    refine_small_batch(ops, n_ops, b.plans);
  }
  for (size_t i = 0; i < n_ops; ++i) {
    Codec &c = const_cast<rsgpu_codec *>(ops[i].codec)->c;
    if (!mix_plan_valid(c, ops[i].op, b.plans[i])) return RSGPU_ERR_INVALID_ARGUMENT;
  }
  // One-shot batches (the request server's) route Leopard reconstructions
  // whose k_mix work rows would not fit shared memory (GF(2^16) codes of
  // 2048 lanes and more) to the codec's own decode kernel: one 1024-thread
  // CTA per SM keeps a single work-row slab per SM in L2, where three k_mix
  // CTAs per SM keep three.  Measured on a B200, GF(2^16) 2048+1024 at
  // 8 KiB: 0.41 against 1.05 ms for one stripe, 3.08 against 5.03 ms for 16,
  // 9.2 against 13.7 ms for 48 (k_mix at its fastest tile).  Encodes stay
  // in k_mix: there the two are on par.  Same bytes either way.
  std::vector<char> routed(n_ops, 0);
  if (b.stream_ordered)
    for (size_t i = 0; i < n_ops; ++i) {
      Codec &c = const_cast<rsgpu_codec *>(ops[i].codec)->c;
      if (!is_leopard(c) || ops[i].op != RSGPU_OP_RECONSTRUCT || b.plans[i].algo != RSGPU_ALGO_FFT) continue;
      LeoGeometry g{};
      int rc = leopard_geometry(c, &g);
      if (rc) return rc;
      routed[i] = size_t(fft_rows(g, ops[i].op)) * 2 * 64 > kMixSmem;
    }
  // One-shot batches run large Leopard GF(2^8) rebuilds whose dense map is
  // not cached through a map derived on the batch's stream (the FFT decode
  // of unit vectors, then a packing kernel; no host wait) instead of the FFT
  // decode.  One B200, one stripe of 4 MiB shards, k_mix: 128+64 rebuilds in
  // 1.53 ms through the map against 4.95 ms by the FFT (5.14 ms by the
  // codec's decode kernel), 32+16 in 0.12 against 1.02 ms; deriving costs
  // two small launches.  Same bytes: the map is the decode's own.
  constexpr uint64_t kInlineDenseBytes = uint64_t(32) << 20;
  std::vector<char> inline_dense(n_ops, 0);
  if (b.stream_ordered)
    for (size_t i = 0; i < n_ops; ++i) {
      Codec &c = const_cast<rsgpu_codec *>(ops[i].codec)->c;
      if (c.family != RSGPU_FAMILY_LEOPARD_GF8 || ops[i].op != RSGPU_OP_RECONSTRUCT ||
          b.plans[i].algo != RSGPU_ALGO_FFT || routed[i])
        continue;
      inline_dense[i] = uint64_t(c.k + c.m) * ops[i].shard_len >= kInlineDenseBytes;
    }

  MixBuild B;
  // Decode tables and locators are built on the batch's stream when it has
  // one, so they precede its launch in stream order.
  cudaStream_t s = b.stream_ordered ? b.stream : nullptr;
  // ---- classic reconstructions: plans and decode tables per codec, in one
  // K3 launch per codec.
  std::map<const Codec *, std::vector<size_t>> classic_rec;
  std::map<const Codec *, std::vector<size_t>> leo_dense_rec;
  std::map<const Codec *, std::vector<size_t>> leo_fft_rec;
  for (size_t i = 0; i < n_ops; ++i) {
    const Codec &c = ops[i].codec->c;
    if (ops[i].op != RSGPU_OP_RECONSTRUCT || routed[i] || inline_dense[i]) continue;
    if (!is_leopard(c))
      classic_rec[&c].push_back(i);
    else if (b.plans[i].algo == RSGPU_ALGO_APPLY)
      leo_dense_rec[&c].push_back(i);
    else
      leo_fft_rec[&c].push_back(i);
  }
  std::vector<ClassicPlan> cplans(n_ops);
  std::vector<const uint32_t *> ctbl(n_ops, nullptr);
  for (auto &kv : classic_rec) {
    Codec &c = const_cast<Codec &>(*kv.first);
    std::vector<const ClassicPlan *> pp;
    for (size_t i : kv.second) {
      int rc = c.plan_classic(ops[i].present, ops[i].goal, nullptr, 0, cplans[i]);
      if (rc) return rc;
      pp.push_back(&cplans[i]);
    }
    std::vector<const uint32_t *> tbls;
    int rc;
    if (b.stream_ordered) {
      // A one-shot batch may use the cache's blocks in place: an evicted
      // block is recycled only after a device-wide synchronization, which
      // cannot happen before this launch has finished.
      rc = c.decode_tables_shared(pp, tbls, s);
    } else {
      uint32_t *owned = nullptr;
      rc = c.decode_tables_copy(pp, tbls, &owned, s);
      if (owned) b.owned_tables.push_back(owned);
    }
    if (rc) return rc;
    for (size_t x = 0; x < kv.second.size(); ++x) ctbl[kv.second[x]] = tbls[x];
  }
  // ---- Leopard FFT reconstructions: error locators per codec.
  std::vector<const uint16_t *> lerr(n_ops, nullptr);
  std::vector<uint32_t> lin(n_ops, 0);
  // The batch keeps its own copies of the locators (one device buffer for
  // all its patterns), so the codec's cache may evict them meanwhile.
  size_t loc_words = 0;
  for (auto &kv : leo_fft_rec) {
    LeoGeometry g{};
    int rc = leopard_geometry(const_cast<Codec &>(*kv.first), &g);
    if (rc) return rc;
    loc_words += kv.second.size() * size_t(g.n);
  }
  if (loc_words) RS_CUDA(b.alloc(&b.d_locs, loc_words * 2));
  size_t loc_used = 0;
  for (auto &kv : leo_fft_rec) {
    Codec &c = const_cast<Codec &>(*kv.first);
    const size_t total = c.k + c.m;
    LeoGeometry g{};
    leopard_geometry(c, &g);
    std::vector<uint8_t> pres(kv.second.size() * total);
    for (size_t x = 0; x < kv.second.size(); ++x) std::memcpy(&pres[x * total], ops[kv.second[x]].present, total);
    std::vector<const uint16_t *> err(kv.second.size());
    std::vector<uint32_t> ic(kv.second.size());
    int rc = leopard_locators(c, kv.second.size(), pres.data(), b.d_locs + loc_used, err.data(), ic.data(), s,
                              b.stream_ordered);
    if (rc) return rc;
    loc_used += kv.second.size() * size_t(g.n);
    for (size_t x = 0; x < kv.second.size(); ++x) {
      lerr[kv.second[x]] = err[x];
      lin[kv.second[x]] = ic[x];
    }
  }
  // ---- Leopard dense reconstructions: maps per codec (goal is per op, so
  // group by goal as well).
  std::vector<LeoDenseMap> dmaps(n_ops);
  for (auto &kv : leo_dense_rec) {
    Codec &c = const_cast<Codec &>(*kv.first);
    const size_t total = c.k + c.m;
    for (int goal : {RSGPU_GOAL_ALL, RSGPU_GOAL_DATA}) {
      std::vector<size_t> idx;
      for (size_t i : kv.second)
        if (ops[i].goal == goal) idx.push_back(i);
      if (idx.empty()) continue;
      // One map per distinct presence pattern.
      std::map<std::string, size_t> uniq;
      std::vector<size_t> which(idx.size());
      std::vector<uint8_t> pres;
      for (size_t x = 0; x < idx.size(); ++x) {
        std::string key(reinterpret_cast<const char *>(ops[idx[x]].present), total);
        auto it = uniq.find(key);
        if (it == uniq.end()) {
          it = uniq.emplace(key, uniq.size()).first;
          pres.insert(pres.end(), key.begin(), key.end());
        }
        which[x] = it->second;
      }
      std::vector<LeoDenseMap> maps;
      int rc = leopard_dense_decode(c, uniq.size(), pres.data(), goal, maps, s);
      if (rc) return rc;
      for (size_t x = 0; x < idx.size(); ++x) dmaps[idx[x]] = maps[which[x]];
    }
  }
  // ---- dense encode tables per Leopard GF(2^8) codec (host-packed once).
  std::map<const Codec *, size_t> dense_enc_tbl;  // word offset into B.tables
  for (size_t i = 0; i < n_ops; ++i) {
    const Codec &c = ops[i].codec->c;
    if (!is_leopard(c) || b.plans[i].algo != RSGPU_ALGO_APPLY || ops[i].op == RSGPU_OP_RECONSTRUCT) continue;
    if (dense_enc_tbl.count(&c)) continue;
    std::vector<uint8_t> rows;
    int rc = leopard_dense_encode(const_cast<Codec &>(c), rows);
    if (rc) return rc;
    const size_t off = B.tables.size();
    B.tables.resize(off + packed_table_words(c.m, c.k));
    pack_tables_with(leopard_mul8(), rows.data(), c.m, c.k, B.tables.data() + off);
    dense_enc_tbl[&c] = off;
  }

  // ---- inline dense maps (one-shot batches): derived on the stream now
  struct InlineMap {
    std::vector<uint16_t> inputs, targets;
    const uint32_t *tbl = nullptr;
  };
  std::vector<InlineMap> imaps(n_ops);
  for (size_t i = 0; i < n_ops; ++i) {
    if (!inline_dense[i]) continue;
    Codec &c = const_cast<rsgpu_codec *>(ops[i].codec)->c;
    uint8_t *img = nullptr;
    RS_CUDA(b.alloc(&img, leopard_dense_inline_bytes(c, ops[i].present, ops[i].goal)));
    b.ordered_bufs.push_back(img);
    size_t nt = 0, ni = 0;
    for (size_t x = 0; x < c.k + c.m; ++x) {
      ni += ops[i].present[x] ? 1 : 0;
      nt += !ops[i].present[x] && (ops[i].goal == RSGPU_GOAL_ALL || x < c.k);
    }
    uint32_t *tbl = nullptr;
    RS_CUDA(b.alloc(&tbl, std::max<size_t>(packed_table_words(nt, ni), 1) * 4));
    b.ordered_bufs.push_back(tbl);
    int rc = leopard_dense_inline(c, ops[i].present, ops[i].goal, img, tbl, imaps[i].inputs, imaps[i].targets,
                                  b.stream);
    if (rc) return rc;
    imaps[i].tbl = tbl;
    b.plans[i] = rsgpu_plan{RSGPU_ALGO_APPLY, imaps[i].targets.size() > 4 ? 2 : 0};
  }

  // ---- routed reconstructions: one launch per (codec, shard length, goal).
  // Their work rows go to the stream's own buffer (the caller's ScratchSlot,
  // shared with k_mix's wide tiles, which run before them on the stream),
  // sized below for the larger of the two users.
  size_t routed_scratch = 0;
  {
    std::map<std::tuple<const Codec *, size_t, int>, std::vector<size_t>> groups;
    for (size_t i = 0; i < n_ops; ++i)
      if (routed[i]) groups[std::make_tuple(&ops[i].codec->c, ops[i].shard_len, ops[i].goal)].push_back(i);
    for (auto &kv : groups) {
      Codec &c = const_cast<Codec &>(*std::get<0>(kv.first));
      const size_t total = c.k + c.m, len = std::get<1>(kv.first);
      std::vector<uint8_t *> sh;
      std::vector<uint8_t> pres;
      for (size_t i : kv.second) {
        sh.insert(sh.end(), ops[i].shards, ops[i].shards + total);
        pres.insert(pres.end(), ops[i].present, ops[i].present + total);
        size_t np = 0, nt = 0;
        for (size_t x = 0; x < total; ++x) {
          np += ops[i].present[x] ? 1 : 0;
          nt += !ops[i].present[x] && (ops[i].goal == RSGPU_GOAL_ALL || x < c.k);
        }
        if (nt) B.algorithmic_bytes += uint64_t(np + nt) * len;
      }
      std::shared_ptr<LeoLaunch> L;
      const size_t want = scratch ? leo_reconstruct_scratch_bytes(c) : 0;
      if (want) {
        RS_CUDA(grow_slot(*scratch, want, b.stream));
        routed_scratch = std::max(routed_scratch, want);
      }
      int rc = prepare_leo_reconstruct_once(c, kv.second.size(), sh.data(), pres.data(), len, std::get<2>(kv.first),
                                            b.stream, want ? scratch->ptr : nullptr, L);
      if (rc) return rc;
      b.side.push_back(L);
    }
  }

  // ---- jobs
  for (size_t i = 0; i < n_ops; ++i) {
    if (routed[i]) continue;
    const rsgpu_mix_op &o = ops[i];
    if (inline_dense[i]) {
      const InlineMap &mp = imaps[i];
      if (mp.targets.empty()) continue;
      const size_t off = B.ptrs.size();
      for (uint16_t x : mp.inputs) B.ptrs.push_back(o.shards[x]);
      for (uint16_t t : mp.targets) B.ptrs.push_back(o.shards[t]);
      add_apply_job(B, b.plans[i], false, mp.inputs.size(), mp.targets.size(), off, o.shard_len, 0, mp.tbl, SIZE_MAX);
      B.algorithmic_bytes += uint64_t(mp.inputs.size() + mp.targets.size()) * o.shard_len;
      continue;
    }
    Codec &c = const_cast<rsgpu_codec *>(o.codec)->c;
    const size_t total = c.k + c.m, len = o.shard_len;
    const rsgpu_plan &p = b.plans[i];
    const bool verify = o.op == RSGPU_OP_VERIFY;
    if (verify) b.any_verify = true;
    if (!is_leopard(c) || p.algo == RSGPU_ALGO_APPLY) {
      // ---- K1 job
      if (o.op == RSGPU_OP_RECONSTRUCT) {
        if (!is_leopard(c)) {
          const ClassicPlan &cp = cplans[i];
          if (cp.all_present || cp.targets.empty()) continue;
          const size_t off = B.ptrs.size();
          for (uint16_t sv : cp.survivors) B.ptrs.push_back(o.shards[sv]);
          for (uint16_t t : cp.targets) B.ptrs.push_back(o.shards[t]);
          add_apply_job(B, p, false, c.k, cp.targets.size(), off, len, 0, ctbl[i], SIZE_MAX);
          B.algorithmic_bytes += uint64_t(c.k + cp.targets.size()) * len;
        } else {
          const LeoDenseMap &mp = dmaps[i];
          if (mp.targets.empty()) continue;
          const size_t off = B.ptrs.size();
          for (uint16_t x : mp.inputs) B.ptrs.push_back(o.shards[x]);
          for (uint16_t t : mp.targets) B.ptrs.push_back(o.shards[t]);
          const size_t toff = B.tables.size();
          B.tables.insert(B.tables.end(), mp.packed->begin(), mp.packed->end());  // packed once per pattern
          add_apply_job(B, p, false, mp.inputs.size(), mp.targets.size(), off, len, 0, nullptr, toff);
          B.algorithmic_bytes += uint64_t(mp.inputs.size() + mp.targets.size()) * len;
        }
      } else {
        const size_t off = B.ptrs.size();
        for (size_t x = 0; x < total; ++x) B.ptrs.push_back(o.shards[x]);
        if (!is_leopard(c))
          add_apply_job(B, p, verify, c.k, c.m, off, len, uint32_t(i), c.d_enc_tbl, SIZE_MAX);
        else
          add_apply_job(B, p, verify, c.k, c.m, off, len, uint32_t(i), nullptr, dense_enc_tbl[&c]);
        B.algorithmic_bytes += uint64_t(total) * len;
      }
      continue;
    }
    // ---- Leopard FFT job
    LeoGeometry g{};
    leopard_geometry(c, &g);
    const uint32_t rows = fft_rows(g, o.op);
    const uint32_t nb = 1u << p.tile;
    const size_t work = size_t(rows) * nb * 64;
    const bool b16 = g.bits == 16;
    uint32_t kind = o.op == RSGPU_OP_ENCODE ? MK_LEO8_ENC : verify ? MK_LEO8_VERIFY : MK_LEO8_DEC;
    if (b16) kind += MK_LEO16_ENC - MK_LEO8_ENC;
    auto key = std::make_tuple(static_cast<const Codec *>(&c), kind, nb);
    uint32_t cls;
    auto it = B.leo_class.find(key);
    if (it != B.leo_class.end()) {
      cls = it->second;
    } else {
      MixClass mc{};
      mc.kind = kind;
      mc.global_work = work > kMixSmem;
      mc.tile_bytes = uint32_t(fft_item_bytes(g, o.op, nb));
      LeoArgs &a = mc.leo;
      a.skew = g.skew;
      a.bank = g.bank;
      a.kbank = g.kbank;
      a.sktab = g.sktab;
      a.st_ienc = g.st_ienc;
      a.st_fenc = g.st_fenc;
      a.st_idec = g.st_idec;
      a.st_fdec = g.st_fdec;
      a.n_ienc = g.n_ienc;
      a.n_fenc = g.n_fenc;
      a.n_idec = g.n_idec;
      a.n_fdec = g.n_fdec;
      a.k = g.k;
      a.p = g.p;
      a.m = g.m;
      a.n = g.n;
      a.mtrunc = g.mtrunc;
      a.last = g.last;
      a.mod = g.mod;
      a.nb = nb;
      a.lanes = rows;
      if (mc.global_work)
        B.scratch_words = std::max<uint64_t>(B.scratch_words, uint64_t(rows) * nb * kRowWords);
      else
        B.smem = std::max(B.smem, work);
      cls = uint32_t(B.classes.size());
      B.classes.push_back(mc);
      B.leo_class.emplace(key, cls);
    }
    LeoJob lj{};
    lj.ptr_off = uint32_t(B.ptrs.size());
    lj.flag_idx = uint32_t(i);
    for (size_t x = 0; x < total; ++x) B.ptrs.push_back(o.shards[x]);
    size_t role_off = SIZE_MAX;
    uint64_t bytes = uint64_t(total) * len;
    if (o.op == RSGPU_OP_RECONSTRUCT) {
      role_off = B.roles.size();
      size_t np = 0, nt = 0;
      for (size_t x = 0; x < total; ++x) {
        const bool want = o.goal == RSGPU_GOAL_ALL || x < c.k;
        const uint8_t role = o.present[x] ? 1 : (want ? 2 : 0);
        np += role == 1;
        nt += role == 2;
        B.roles.push_back(role);
      }
      if (nt == 0) {
        B.roles.resize(role_off);
        B.ptrs.resize(lj.ptr_off);
        continue;
      }
      lj.err = lerr[i];
      lj.input_count = lin[i];
      bytes = uint64_t(np + nt) * len;
    }
    MixJob j{};
    j.cls = cls;
    j.sub = uint32_t(B.leo_jobs.size());
    j.len = len;
    B.leo_jobs.push_back(lj);
    B.role_of_leo_job.push_back(role_off);
    const double factor = (b16 ? 12.0 : 6.0) * (o.op == RSGPU_OP_RECONSTRUCT ? 2.5 : 1.0);
    B.push_job(j, SIZE_MAX, item_cost(1, std::max<uint32_t>(rows, 32), factor));
    B.algorithmic_bytes += bytes;
  }

  // ---- items, heaviest first.  A job's items come in runs of equal cost
  // (its full tiles, a short last tile, the unaligned tail), so a stable sort
  // of the runs yields exactly the order a stable sort of the items would, in
  // O(runs log runs) host time: ~0.3 ms instead of ~5 ms for a batch of 160k
  // items, which the request server pays on every batch it builds.
  struct ItemRun {
    double cost;
    uint32_t job, t0, count;
  };
  std::vector<ItemRun> runs;
  uint64_t n_items = 0;
  auto add_run = [&](double c, size_t ji, uint64_t t0, uint64_t count) {
    if (!count) return;
    runs.push_back(ItemRun{c, uint32_t(ji), uint32_t(t0), uint32_t(count)});
    n_items += count;
  };
  for (size_t ji = 0; ji < B.jobs.size(); ++ji) {
    const MixJob &j = B.jobs[ji];
    const MixClass &mc = B.classes[j.cls];
    if (mc.kind < MK_LEO8_ENC) {
      const uint32_t t = mc.kind & 3;
      const uint64_t tile = t == 0 ? 2 * kApplyTile : kApplyTile;
      const uint64_t full = j.d.vec_len / tile, rest = j.d.vec_len % tile;
      add_run(B.job_cost[ji] * double(tile), ji, 0, full);
      if (rest) add_run(B.job_cost[ji] * double(rest), ji, full, 1);
      if (j.d.vec_len < j.len) add_run(B.job_cost[ji] * double(j.len - j.d.vec_len) * 16.0, ji, kTailTile, 1);
    } else {
      const uint64_t tile = mc.tile_bytes;
      add_run(B.job_cost[ji] * double(tile) * (mc.global_work ? 2.0 : 1.0), ji, 0, (j.len + tile - 1) / tile);
    }
  }
  if (n_items >= UINT32_MAX) return RSGPU_ERR_INVALID_ARGUMENT;
  if (opt.order == RSGPU_ORDER_COST)
    std::stable_sort(runs.begin(), runs.end(), [](const ItemRun &x, const ItemRun &y) { return x.cost > y.cost; });
  std::vector<MixItem> items;
  items.reserve(n_items);
  for (const ItemRun &r : runs) {
    if (r.t0 == kTailTile) {
      items.push_back(MixItem{r.job, kTailTile});
      continue;
    }
    for (uint32_t t = 0; t < r.count; ++t) items.push_back(MixItem{r.job, r.t0 + t});
  }

  // ---- upload: classes | jobs | items | ptrs | leo jobs | roles | tables
  const size_t o_cls = 0;
  const size_t o_jobs = align256(o_cls + B.classes.size() * sizeof(MixClass));
  const size_t o_items = align256(o_jobs + B.jobs.size() * sizeof(MixJob));
  const size_t o_ptrs = align256(o_items + items.size() * sizeof(MixItem));
  const size_t o_leo = align256(o_ptrs + B.ptrs.size() * sizeof(void *));
  const size_t o_roles = align256(o_leo + B.leo_jobs.size() * sizeof(LeoJob));
  const size_t o_tbl = align256(o_roles + B.roles.size());
  const size_t total_bytes = o_tbl + B.tables.size() * 4 + 256;
  RS_CUDA(b.alloc(&b.d_blob, total_bytes));
  RS_CUDA(b.alloc(&b.d_flags, std::max<size_t>(n_ops, 1) * 4));
  RS_CUDA(b.alloc(&b.d_counter, 256));
  if (b.stream_ordered)
    RS_CUDA(cudaMemsetAsync(b.d_flags, 0, std::max<size_t>(n_ops, 1) * 4, b.stream));
  else
    RS_CUDA(cudaMemset(b.d_flags, 0, std::max<size_t>(n_ops, 1) * 4));
  uint8_t *base = static_cast<uint8_t *>(b.d_blob);
  const uint32_t *tbl_base = reinterpret_cast<const uint32_t *>(base + o_tbl);
  for (size_t ji = 0; ji < B.jobs.size(); ++ji) {
    MixJob &j = B.jobs[ji];
    if (B.table_of_job[ji] != SIZE_MAX) j.d.tbl = tbl_base + B.table_of_job[ji];
  }
  for (size_t x = 0; x < B.leo_jobs.size(); ++x)
    if (B.role_of_leo_job[x] != SIZE_MAX) B.leo_jobs[x].role = base + o_roles + B.role_of_leo_job[x];
  // Every device pointer a Leopard tile reads from its class arguments: jobs,
  // pointer table, verify flags (skew and bank were set per codec above; the
  // work rows come from the kernel, not from args.scratch).
  for (MixClass &mc : B.classes) {
    mc.leo.jobs = reinterpret_cast<const LeoJob *>(base + o_leo);
    mc.leo.ptrs = reinterpret_cast<const uint8_t *const *>(base + o_ptrs);
    mc.leo.flags = b.d_flags;
  }
  std::vector<uint8_t> host(o_tbl + B.tables.size() * 4, 0);
  std::memcpy(host.data() + o_cls, B.classes.data(), B.classes.size() * sizeof(MixClass));
  std::memcpy(host.data() + o_jobs, B.jobs.data(), B.jobs.size() * sizeof(MixJob));
  std::memcpy(host.data() + o_items, items.data(), items.size() * sizeof(MixItem));
  std::memcpy(host.data() + o_ptrs, B.ptrs.data(), B.ptrs.size() * sizeof(void *));
  std::memcpy(host.data() + o_leo, B.leo_jobs.data(), B.leo_jobs.size() * sizeof(LeoJob));
  std::memcpy(host.data() + o_roles, B.roles.data(), B.roles.size());
  std::memcpy(host.data() + o_tbl, B.tables.data(), B.tables.size() * 4);
  if (b.stream_ordered) {  // through pinned memory: never waits for the stream's earlier work
    const int rc = upload_to(b.d_blob, host.data(), host.size(), b.stream);
    if (rc) return rc;
  } else
    RS_CUDA(cudaMemcpy(b.d_blob, host.data(), host.size(), cudaMemcpyHostToDevice));

  // ---- launch shape
  b.smem = B.smem;
  int per_sm = 0;
  RS_CUDA(mix_shape(b.smem, &per_sm));
  per_sm = std::max(per_sm, 1);
  if (opt.ctas_per_sm > 0) per_sm = std::min(per_sm, int(opt.ctas_per_sm));
  b.grid = int(std::max<uint64_t>(1, std::min<uint64_t>(items.size(), uint64_t(per_sm) * sm_count())));
  if (B.scratch_words || routed_scratch) {
    const size_t need = std::max(size_t(b.grid) * B.scratch_words * 4, routed_scratch);
    if (scratch && b.stream_ordered) {
      RS_CUDA(grow_slot(*scratch, need, b.stream));
      b.d_scratch = static_cast<uint32_t *>(scratch->ptr);
      b.scratch_borrowed = true;
      for (const auto &L : b.side) leo_set_scratch(*L, scratch->ptr);  // the buffer may have moved
    } else {
      RS_CUDA(b.alloc(&b.d_scratch, need));
    }
  }
  MixArgs &a = b.args;
  a.items = reinterpret_cast<const MixItem *>(base + o_items);
  a.jobs = reinterpret_cast<const MixJob *>(base + o_jobs);
  a.classes = reinterpret_cast<const MixClass *>(base + o_cls);
  a.ptrs = reinterpret_cast<const uint8_t *const *>(base + o_ptrs);
  a.flags = b.d_flags;
  a.counter = b.d_counter;
  a.scratch = b.d_scratch;
  a.scratch_words = B.scratch_words;
  a.n_items = uint32_t(items.size());

  b.info.n_ops = n_ops;
  b.info.n_jobs = B.jobs.size();
  b.info.n_items = items.size();
  b.info.n_classes = B.classes.size();
  b.info.grid = uint32_t(b.grid);
  b.info.smem_bytes = uint32_t(b.smem);
  b.info.device_bytes = total_bytes + size_t(b.grid) * B.scratch_words * 4;
  b.info.algorithmic_bytes = B.algorithmic_bytes;
  b.mix_kernels = items.empty() ? 0 : 1;
  b.info.kernels_per_launch = b.mix_kernels;
  for (const auto &L : b.side) b.info.kernels_per_launch += leo_kernel_count(*L);

  if (opt.graph) {
    cudaStream_t cs = nullptr;
    RS_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    int rc = e == cudaSuccess ? b.enqueue(cs) : cuda_status(e);
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(cs, &g);
    if (rc == RSGPU_OK && e != cudaSuccess) rc = cuda_status(e);
    b.graph = g;
    if (rc == RSGPU_OK) rc = cuda_status(cudaGraphInstantiate(&b.exec, g, 0));
    cudaStreamDestroy(cs);
    if (rc) return rc;
  }
  if (!b.stream_ordered) RS_CUDA(cudaDeviceSynchronize());
  out = std::move(batch);
  return RSGPU_OK;
}

int mix_launch(MixBatch &b, cudaStream_t s) {
  if (b.exec) {
    RS_CUDA(cudaGraphLaunch(b.exec, s));
  } else {
    int rc = b.enqueue(s);
    if (rc) return rc;
  }
  launch_counter_add(b.mix_kernels);  // the routed launches count themselves
  return RSGPU_OK;
}

int mix_results(MixBatch &b, uint8_t *ok, cudaStream_t s) {
  std::vector<uint32_t> f(std::max<size_t>(b.n_ops, 1));
  RS_CUDA(cudaMemcpyAsync(f.data(), b.d_flags, f.size() * 4, cudaMemcpyDeviceToHost, s));
  RS_CUDA(cudaStreamSynchronize(s));
  for (size_t i = 0; i < b.n_ops; ++i) ok[i] = f[i] ? 0 : 1;
  return RSGPU_OK;
}

const rsgpu_mix_info &mix_info(const MixBatch &b) { return b.info; }
const std::vector<rsgpu_plan> &mix_plans(const MixBatch &b) { return b.plans; }
void MixDeleter::operator()(MixBatch *b) const { delete b; }
int mix_validate(const rsgpu_mix_op &o, int device) { return validate_op(o, device); }
const uint32_t *mix_flags(const MixBatch &b) { return b.d_flags; }

}  // namespace rsgpu

// ====================================================================== C ABI
struct rsgpu_mix {
  rsgpu::MixPtr b;
};

namespace {
int mix_prepare(const rsgpu_mix_op *ops, size_t n_ops, const rsgpu_plan *plans, const rsgpu_mix_options *opts,
                rsgpu_mix **out) {
  if (!out || (!ops && n_ops)) return RSGPU_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  rsgpu_mix_options o;
  rsgpu_mix_options_default(&o);
  if (opts) o = *opts;
  std::unique_ptr<rsgpu_mix> h(new (std::nothrow) rsgpu_mix());
  if (!h) return RSGPU_ERR_OUT_OF_MEMORY;
  int rc = rsgpu::mix_build(ops, n_ops, plans, o, h->b);
  if (rc) return rc;
  *out = h.release();
  return RSGPU_OK;
}
}  // namespace

extern "C" {

void rsgpu_mix_options_default(rsgpu_mix_options *out) {
  if (!out) return;
  std::memset(out, 0, sizeof(*out));
  out->planner = RSGPU_PLANNER_FIXED;
  out->order = RSGPU_ORDER_COST;
  out->graph = 1;
}

int32_t rsgpu_mix_prepare(const rsgpu_mix_op *ops, size_t n_ops, const rsgpu_mix_options *opts, rsgpu_mix **out) {
  return mix_prepare(ops, n_ops, nullptr, opts, out);
}

int32_t rsgpu_mix_prepare_planned(const rsgpu_mix_op *ops, size_t n_ops, const rsgpu_plan *plans,
                                  const rsgpu_mix_options *opts, rsgpu_mix **out) {
  if (!plans && n_ops) return RSGPU_ERR_INVALID_ARGUMENT;
  return mix_prepare(ops, n_ops, plans, opts, out);
}

int32_t rsgpu_mix_launch(rsgpu_mix *mix, void *stream) {
  if (!mix || !mix->b) return RSGPU_ERR_INVALID_ARGUMENT;
  return rsgpu::mix_launch(*mix->b, static_cast<cudaStream_t>(stream));
}

int32_t rsgpu_mix_results(rsgpu_mix *mix, uint8_t *ok, void *stream) {
  if (!mix || !mix->b || !ok) return RSGPU_ERR_INVALID_ARGUMENT;
  return rsgpu::mix_results(*mix->b, ok, static_cast<cudaStream_t>(stream));
}

int32_t rsgpu_mix_get_info(const rsgpu_mix *mix, rsgpu_mix_info *out) {
  if (!mix || !mix->b || !out) return RSGPU_ERR_INVALID_ARGUMENT;
  *out = rsgpu::mix_info(*mix->b);
  return RSGPU_OK;
}

int32_t rsgpu_mix_get_plans(const rsgpu_mix *mix, rsgpu_plan *out, size_t n_ops) {
  if (!mix || !mix->b || (!out && n_ops)) return RSGPU_ERR_INVALID_ARGUMENT;
  const auto &p = rsgpu::mix_plans(*mix->b);
  if (n_ops != p.size()) return RSGPU_ERR_INVALID_ARGUMENT;
  std::copy(p.begin(), p.end(), out);
  return RSGPU_OK;
}

void rsgpu_mix_free(rsgpu_mix *mix) { delete mix; }

}  // extern "C"
