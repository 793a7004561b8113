// codec.cpp -- classic codec runtime: construction, validation, recovery
// planning, the HBM-resident decode-table cache and K1/K3 submission.
#include "codec.hpp"

#include <algorithm>
#include <atomic>
#include <cstring>
#include <map>
#include <mutex>

namespace rsgpu {

static std::atomic<uint64_t> g_launches{0};
uint64_t launch_counter_add(uint64_t n) { return g_launches.fetch_add(n) + n; }
uint64_t launch_counter() { return g_launches.load(); }

int cuda_status(cudaError_t e) {
  if (e == cudaSuccess) return RSGPU_OK;
  if (e == cudaErrorMemoryAllocation) return RSGPU_ERR_OUT_OF_MEMORY;
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return RSGPU_ERR_NO_DEVICE;
  return RSGPU_ERR_CUDA;
}

#define RS_CUDA(expr)                          \
  do {                                         \
    cudaError_t e_ = (expr);                   \
    if (e_ != cudaSuccess) return cuda_status(e_); \
  } while (0)

// ------------------------------------------------------------------ uploads
namespace {
struct UploadSlot {
  void *host = nullptr;
  size_t cap = 0;
  cudaEvent_t done = nullptr;
  ~UploadSlot() {
    if (done) cudaEventDestroy(done);
    if (host) cudaFreeHost(host);
  }
};
// Bounce buffers per thread.  A buffer is reused once the copy last issued
// from it has completed (an event query, never a wait), else another buffer
// is taken or a new one allocated: the copies are stream-ordered, and a
// stream may wait a long time behind other streams' persistent kernels.
// Buffers are not freed while the thread runs (freeing pinned memory
// synchronizes the device), except when the pool is full and no free buffer
// is large enough, which a steady workload reaches only while warming up.
constexpr size_t kUploadSlots = 64;
struct UploadPool {
  std::vector<std::unique_ptr<UploadSlot>> slots;
  size_t next = 0;
};
thread_local UploadPool t_upload;

}  // namespace

int lib_pool(void **out) {
  static std::mutex mu;
  static std::map<int, cudaMemPool_t> pools;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return int(e);
  std::lock_guard<std::mutex> g(mu);
  auto it = pools.find(dev);
  if (it == pools.end()) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t p = nullptr;
    if ((e = cudaMemPoolCreate(&p, &props)) != cudaSuccess) return int(e);
    uint64_t keep = 2ull << 30;
    if ((e = cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep)) != cudaSuccess) return int(e);
    it = pools.emplace(dev, p).first;
  }
  *out = it->second;
  return int(cudaSuccess);
}

int lib_malloc_async(void **p, size_t bytes, void *stream) {
  void *pool = nullptr;
  int e = lib_pool(&pool);
  if (e != int(cudaSuccess)) return e;
  return int(cudaMallocFromPoolAsync(p, bytes, static_cast<cudaMemPool_t>(pool), static_cast<cudaStream_t>(stream)));
}

namespace {

}  // namespace

// Copies `bytes` of host data to device memory `dst`, stream-ordered on s,
// through a pinned, event-guarded bounce buffer.  A copy from pageable memory
// could instead block the calling thread until the stream reached it (the
// driver stages large pageable copies in a bounded buffer), i.e. behind
// whatever the stream waits for.
int upload_to(void *dst, const void *src, size_t bytes, void *stream) {
  if (!bytes) return RSGPU_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  UploadPool &pool = t_upload;
  UploadSlot *u = nullptr, *small = nullptr;
  const size_t n = pool.slots.size();
  for (size_t i = 0; i < n && !u; ++i) {  // first fit, starting after the last slot used
    UploadSlot *x = pool.slots[(pool.next + i) % n].get();
    if (cudaEventQuery(x->done) == cudaErrorNotReady) continue;
    if (x->cap >= bytes) {
      u = x;
      pool.next = (pool.next + i + 1) % n;
    } else if (!small) {
      small = x;
    }
  }
  cudaGetLastError();  // a not-ready query is not an error
  if (!u) {
    size_t cap = size_t(1) << 20;
    while (cap < bytes) cap <<= 1;
    if (pool.slots.size() < kUploadSlots) {
      pool.slots.emplace_back(new UploadSlot());
      u = pool.slots.back().get();
      RS_CUDA(cudaEventCreateWithFlags(&u->done, cudaEventDisableTiming));
    } else {
      u = small ? small : pool.slots[pool.next].get();
      RS_CUDA(cudaEventSynchronize(u->done));  // every buffer is in flight: wait for one
      if (u->cap < bytes) {
        cudaFreeHost(u->host);
        u->host = nullptr;
        u->cap = 0;
      }
    }
    if (!u->host) {
      RS_CUDA(cudaHostAlloc(&u->host, cap, cudaHostAllocDefault));
      u->cap = cap;
    }
  }
  std::memcpy(u->host, src, bytes);
  RS_CUDA(cudaMemcpyAsync(dst, u->host, bytes, cudaMemcpyHostToDevice, s));
  RS_CUDA(cudaEventRecord(u->done, s));
  return RSGPU_OK;
}

// Gives the calling thread's bounce-buffer pool at least `n` free buffers of
// `bytes` each, so that its first uploads of up to that size allocate no
// pinned memory (cudaHostAlloc of megabytes took tens of milliseconds on a
// request path).
int upload_prewarm(size_t n, size_t bytes) {
  UploadPool &pool = t_upload;
  size_t have = 0;
  for (auto &x : pool.slots) have += x->cap >= bytes ? 1 : 0;
  while (have < n && pool.slots.size() < kUploadSlots) {
    pool.slots.emplace_back(new UploadSlot());
    UploadSlot *u = pool.slots.back().get();
    RS_CUDA(cudaEventCreateWithFlags(&u->done, cudaEventDisableTiming));
    RS_CUDA(cudaHostAlloc(&u->host, bytes, cudaHostAllocDefault));
    u->cap = bytes;
    ++have;
  }
  return RSGPU_OK;
}

namespace {
// Copies `bytes` of host data to a fresh stream-ordered device allocation
// (upload_to).  The device block is freed stream-ordered by the caller.
int upload(const void *src, size_t bytes, void **dev, cudaStream_t s) {
  RS_CUDA(cudaError_t(lib_malloc_async(dev, std::max<size_t>(bytes, 16), s)));
  return upload_to(*dev, src, bytes, s);
}
}  // namespace

// ------------------------------------------------------------------ table pool
TablePool::~TablePool() {
  for (void *p : slabs_) cudaFree(p);
}

uint32_t *TablePool::get() {
  if (free_.empty()) {
    void *slab = nullptr;
    if (cudaMalloc(&slab, kSlab) != cudaSuccess) return nullptr;
    slabs_.push_back(slab);
    const size_t n = kSlab / block_;
    for (size_t i = 0; i < n; ++i) free_.push_back(reinterpret_cast<uint32_t *>(static_cast<char *>(slab) + i * block_));
  }
  uint32_t *p = free_.back();
  free_.pop_back();
  return p;
}

// ------------------------------------------------------------------ setup
Codec::~Codec() {
  cudaDeviceSynchronize();
  pool_.reset();
  if (d_matrix) cudaFree(d_matrix);
  if (d_log) cudaFree(d_log);
  if (d_exp) cudaFree(d_exp);
  if (d_enc_tbl) cudaFree(d_enc_tbl);
  if (d_status) cudaFree(d_status);
}

int Codec::take_device_status(cudaStream_t s) {
  if (!d_status) return RSGPU_OK;
  uint32_t v = 0;
  RS_CUDA(cudaMemcpyAsync(&v, d_status, 4, cudaMemcpyDeviceToHost, s));
  RS_CUDA(cudaStreamSynchronize(s));
  if (!v) return RSGPU_OK;
  RS_CUDA(cudaMemsetAsync(d_status, 0, 4, s));
  RS_CUDA(cudaStreamSynchronize(s));
  return RSGPU_ERR_DEVICE_TIMEOUT;
}

int Codec::init_classic(const uint8_t *custom_rows) {
  int rc = build_encoding_matrix(k, m, opts.matrix_mode, opts.fast_one_parity != 0, custom_rows, matrix);
  if (rc != RSGPU_OK) return rc;
  RS_CUDA(cudaGetDevice(&device));
  const Gf8 &f = gf8();
  RS_CUDA(cudaMalloc(&d_matrix, matrix.size()));
  RS_CUDA(cudaMemcpy(d_matrix, matrix.data(), matrix.size(), cudaMemcpyHostToDevice));
  RS_CUDA(cudaMalloc(&d_log, 256));
  RS_CUDA(cudaMemcpy(d_log, f.log, 256, cudaMemcpyHostToDevice));
  RS_CUDA(cudaMalloc(&d_exp, 510));
  RS_CUDA(cudaMemcpy(d_exp, f.exp, 510, cudaMemcpyHostToDevice));
  std::vector<uint32_t> packed(packed_table_words(m, k));
  pack_tables(&matrix[k * k], m, k, packed.data());
  RS_CUDA(cudaMalloc(&d_enc_tbl, packed.size() * 4));
  RS_CUDA(cudaMemcpy(d_enc_tbl, packed.data(), packed.size() * 4, cudaMemcpyHostToDevice));
  RS_CUDA(cudaMalloc(&d_status, 4));
  RS_CUDA(cudaMemset(d_status, 0, 4));
  pool_.reset(new TablePool(std::max<size_t>(256, packed_table_words(m, k) * 4)));
  // Distinct patterns are unbounded in number, but decode tables are small:
  // keep up to 65536 resident unless the caller set an explicit capacity.
  capacity_ = opts.inversion_cache_capacity ? opts.inversion_cache_capacity : 65536;
  return RSGPU_OK;
}

// ------------------------------------------------------------------ validation
// check_piece_count!(all) + check_slices!(multi) (src/macros.rs:142-245).
int Codec::check_all(const size_t *lens, size_t n, size_t *shard_len) const {
  if (n < k + m) return RSGPU_ERR_TOO_FEW_SHARDS;
  if (n > k + m) return RSGPU_ERR_TOO_MANY_SHARDS;
  const size_t len = lens[0];
  if (len == 0) return RSGPU_ERR_EMPTY_SHARD;
  for (size_t i = 0; i < n; ++i)
    if (lens[i] != len) return RSGPU_ERR_INCORRECT_SHARD_SIZE;
  *shard_len = len;
  return RSGPU_OK;
}

// src/core/recovery_plan.rs:262-517: survivors are the first k present shards;
// targets are the missing shards the goal asks for; an inverse is needed only
// when a missing data shard feeds some requested output.
int Codec::plan_classic(const uint8_t *present, int goal, const uint8_t *required, size_t n_required,
                        ClassicPlan &p) const {
  p = ClassicPlan{};
  const size_t total = k + m;
  if (goal == RSGPU_GOAL_REQUIRED && n_required != k && n_required != total)
    return p.status = RSGPU_ERR_INVALID_SHARD_FLAGS;
  size_t n_present = 0, missing_data = 0;
  for (size_t i = 0; i < total; ++i) {
    if (present[i]) {
      ++n_present;
      if (p.survivors.size() < k) p.survivors.push_back(uint16_t(i));
    } else if (i < k) {
      ++missing_data;
    }
  }
  if (n_present == total) {
    p.all_present = true;
    return RSGPU_OK;
  }
  if (n_present < k) return p.status = RSGPU_ERR_TOO_FEW_SHARDS_PRESENT;
  for (size_t i = 0; i < total; ++i) {
    if (present[i]) continue;
    bool want = goal == RSGPU_GOAL_ALL || (goal == RSGPU_GOAL_DATA && i < k) ||
                (goal == RSGPU_GOAL_REQUIRED && i < n_required && required[i]);
    if (!want) continue;
    p.targets.push_back(uint16_t(i));
    if (i < k) ++p.n_data_targets;
  }
  p.needs_inverse = missing_data > 0 && !p.targets.empty();
  return RSGPU_OK;
}

// ------------------------------------------------------------------ decode cache
static PatternKey key_of(const ClassicPlan &p, size_t k) {
  PatternKey key;
  // Survivors determine the inverse; targets determine the composed rows.
  for (uint16_t s : p.survivors) key.present[s >> 6] |= 1ull << (s & 63);
  for (uint16_t t : p.targets) key.targets[t >> 6] |= 1ull << (t & 63);
  (void)k;
  return key;
}

int Codec::decode_tables(const std::vector<const ClassicPlan *> &plans, std::vector<const uint32_t *> &tbls,
                         cudaStream_t s) {
  tbls.assign(plans.size(), nullptr);
  std::vector<DecodeTask> tasks;
  std::vector<size_t> task_of_plan(plans.size(), SIZE_MAX);
  std::unordered_map<PatternKey, size_t, PatternKeyHash> pending;  // new key -> task index
  const bool use_cache = opts.inversion_cache != 0;
  std::vector<uint32_t *> transient;  // blocks for uncached builds
  for (size_t i = 0; i < plans.size(); ++i) {
    const ClassicPlan &p = *plans[i];
    if (p.all_present || p.targets.empty()) continue;
    // A table block holds the rows of at most m outputs over k inputs.
    if (p.targets.size() > m || p.survivors.size() != k) return RSGPU_ERR_INVALID_ARGUMENT;
    PatternKey key = key_of(p, k);
    ++stats_.requests;
    if (use_cache) {
      auto it = cache_.find(key);
      if (it != cache_.end()) {
        ++stats_.hits;
        lru_.splice(lru_.end(), lru_, it->second.lru);
        tbls[i] = it->second.tbl;
        continue;
      }
    }
    auto pit = pending.find(key);
    if (pit != pending.end()) {
      task_of_plan[i] = pit->second;
      continue;
    }
    ++stats_.misses;
    DecodeTask t;
    std::memset(&t, 0, sizeof(t));
    for (size_t x = 0; x < p.survivors.size(); ++x) t.survivors[x] = uint8_t(p.survivors[x]);
    for (size_t x = 0; x < p.targets.size(); ++x) t.targets[x] = uint8_t(p.targets[x]);
    t.n_out = uint32_t(p.targets.size());
    t.needs_inverse = p.needs_inverse;
    uint32_t *blk = pool_->get();
    if (!blk) return RSGPU_ERR_OUT_OF_MEMORY;
    t.tbl_out = blk;
    task_of_plan[i] = tasks.size();
    pending.emplace(key, tasks.size());
    tasks.push_back(t);
    if (use_cache) {
      if (cache_.size() >= capacity_) {
        // Evict the least recently used entry; its block is recycled only
        // after a device-wide sync, so no queued kernel can still read it.
        PatternKey victim = lru_.front();
        lru_.pop_front();
        auto vit = cache_.find(victim);
        retire_.push_back(vit->second.tbl);
        cache_.erase(vit);
        ++stats_.evictions;
      }
      DecodeEntry e;
      e.tbl = blk;
      e.survivors = p.survivors;
      e.targets = p.targets;
      lru_.push_back(key);
      e.lru = std::prev(lru_.end());
      cache_.emplace(key, std::move(e));
      ++stats_.inserts;
    } else {
      transient.push_back(blk);
    }
  }
  if (!tasks.empty()) {
    void *d_tasks = nullptr;
    int rc = upload(tasks.data(), tasks.size() * sizeof(DecodeTask), &d_tasks, s);
    if (rc) return rc;
    int *d_status = nullptr;
    RS_CUDA(cudaError_t(lib_malloc_async(reinterpret_cast<void **>(&d_status), tasks.size() * sizeof(int), s)));
    DecodeTableArgs a;
    a.tasks = static_cast<const DecodeTask *>(d_tasks);
    a.matrix = d_matrix;
    a.gf_log = d_log;
    a.gf_exp = d_exp;
    a.status = d_status;
    a.k = int(k);
    int max_out = 0;
    for (auto &t : tasks) max_out = std::max<int>(max_out, int(t.n_out));
    RS_CUDA(launch_decode_tables(a, int(tasks.size()), max_out, s));
    // Vandermonde and Cauchy constructions are MDS: every k x k survivor
    // system is invertible, so their outputs can follow without a round trip.
    // Other matrices must report a singular system before any output is
    // written (validate-before-write), which needs the status on the host.
    const bool mds = opts.matrix_mode == RSGPU_MATRIX_VANDERMONDE || opts.matrix_mode == RSGPU_MATRIX_CAUCHY ||
                     (opts.fast_one_parity && m == 1);
    int bad = 0;
    if (!mds) {
      std::vector<int> st(tasks.size());
      RS_CUDA(cudaMemcpyAsync(st.data(), d_status, st.size() * sizeof(int), cudaMemcpyDeviceToHost, s));
      RS_CUDA(cudaStreamSynchronize(s));
      for (int v : st) bad |= v;
    }
    RS_CUDA(cudaFreeAsync(d_status, s));
    RS_CUDA(cudaFreeAsync(d_tasks, s));
    if (bad) {
      // Drop every entry built by this call: a singular pattern must not stay cached.
      for (auto &kv : pending) {
        auto it = cache_.find(kv.first);
        if (it != cache_.end()) {
          lru_.erase(it->second.lru);
          retire_.push_back(it->second.tbl);
          cache_.erase(it);
        }
      }
      for (uint32_t *b : transient) retire_.push_back(b);
      return RSGPU_ERR_INVALID_CUSTOM_MATRIX;
    }
  }
  for (size_t i = 0; i < plans.size(); ++i)
    if (task_of_plan[i] != SIZE_MAX) tbls[i] = tasks[task_of_plan[i]].tbl_out;
  for (uint32_t *b : transient) retire_.push_back(b);
  if (retire_.size() >= 1024) {
    RS_CUDA(cudaDeviceSynchronize());
    for (uint32_t *b : retire_) pool_->put(b);
    retire_.clear();
  }
  return RSGPU_OK;
}

int Codec::decode_tables_shared(const std::vector<const ClassicPlan *> &plans, std::vector<const uint32_t *> &tbls,
                                cudaStream_t s) {
  std::lock_guard<std::mutex> g(mu_);
  return decode_tables(plans, tbls, s);
}

int Codec::decode_tables_copy(const std::vector<const ClassicPlan *> &plans, std::vector<const uint32_t *> &tbls,
                              uint32_t **owned, cudaStream_t s) {
  *owned = nullptr;
  std::lock_guard<std::mutex> g(mu_);
  int rc = decode_tables(plans, tbls, s);
  if (rc) return rc;
  std::unordered_map<const uint32_t *, size_t> slot;
  for (const uint32_t *t : tbls)
    if (t && !slot.count(t)) slot.emplace(t, slot.size());
  if (slot.empty()) return RSGPU_OK;
  const size_t words = (pool_->block_bytes() + 3) / 4;
  RS_CUDA(cudaMalloc(reinterpret_cast<void **>(owned), slot.size() * words * 4));
  for (auto &kv : slot)
    RS_CUDA(cudaMemcpyAsync(*owned + kv.second * words, kv.first, words * 4, cudaMemcpyDeviceToDevice, s));
  RS_CUDA(cudaStreamSynchronize(s));
  for (auto &t : tbls)
    if (t) t = *owned + slot[t] * words;
  return RSGPU_OK;
}

void Codec::stats(rsgpu_cache_stats *out) {
  std::lock_guard<std::mutex> g(mu_);
  *out = stats_;
  out->entries = cache_.size();
  out->retained_bytes = cache_.size() * (pool_ ? pool_->block_bytes() : 0);
}

// ------------------------------------------------------------------ K1 submission
int ApplyLaunch::build(std::vector<JobDesc> &jobs, const std::vector<const uint8_t *> &ptrs, size_t len, bool vfy,
                       uint32_t *flags, cudaStream_t s, bool persistent, bool accumulate) {
  verify = vfy;
  max_tail = 0;
  uint32_t max_out = 0;
  int any_vec = 0;
  int tbl_stage = 0;
  for (auto &j : jobs) {
    tbl_stage |= j.tbl != jobs[0].tbl;
    bool aligned = true;
    const uint32_t n_ptr = uint32_t(j.n_in) + j.n_out * (j.verify_store ? 2u : 1u);
    for (uint32_t i = 0; i < n_ptr; ++i)
      aligned &= (reinterpret_cast<uintptr_t>(ptrs[j.ptr_off + i]) & 15) == 0;
    j.vec_len = aligned ? (len & ~uint64_t(15)) : 0;
    max_tail = std::max<uint64_t>(max_tail, len - j.vec_len);
    max_out = std::max<uint32_t>(max_out, j.n_out);
    any_vec |= j.vec_len > 0;
  }
  const size_t jb = jobs.size() * sizeof(JobDesc);
  std::vector<uint8_t> blob(jb + ptrs.size() * sizeof(void *));
  std::memcpy(blob.data(), jobs.data(), jb);
  std::memcpy(blob.data() + jb, ptrs.data(), ptrs.size() * sizeof(void *));
  owned = persistent;
  if (persistent) {
    RS_CUDA(cudaMalloc(&d_blob, std::max<size_t>(blob.size(), 16)));
    RS_CUDA(cudaMemcpy(d_blob, blob.data(), blob.size(), cudaMemcpyHostToDevice));
  } else {
    int rc = upload(blob.data(), blob.size(), &d_blob, s);
    if (rc) return rc;
  }
  args.jobs = static_cast<const JobDesc *>(d_blob);
  args.ptrs = reinterpret_cast<const uint8_t *const *>(static_cast<char *>(d_blob) + jb);
  args.flags = flags;
  args.len = len;
  args.n_jobs = uint32_t(jobs.size());
  args.max_out = max_out;
  args.any_vec = any_vec;
  args.tbl_stage = tbl_stage;
  args.accumulate = accumulate ? 1 : 0;
  return RSGPU_OK;
}

int ApplyLaunch::launch(cudaStream_t s) const {
  if (args.n_jobs == 0) return RSGPU_OK;
  return cuda_status(launch_apply(args, verify, max_tail, s));
}

void ApplyLaunch::release(cudaStream_t s) {
  if (!d_blob) return;
  if (owned)
    cudaFree(d_blob);
  else
    cudaFreeAsync(d_blob, s);
  d_blob = nullptr;
}

int Codec::run_apply(std::vector<JobDesc> &jobs, std::vector<const uint8_t *> &ptrs, size_t len, bool verify,
                     uint32_t *flags_dev, cudaStream_t s, bool accumulate) {
  if (jobs.empty()) return RSGPU_OK;
  ApplyLaunch l;
  int rc = l.build(jobs, ptrs, len, verify, flags_dev, s, false, accumulate);
  if (rc) return rc;
  l.args.stall = d_status;
  rc = l.launch(s);
  l.release(s);
  return rc;
}

int Codec::encode_jobs(size_t n_stripes, uint8_t *const *shards, std::vector<JobDesc> &jobs,
                       std::vector<const uint8_t *> &ptrs, bool verify) {
  jobs.assign(n_stripes, JobDesc{});
  ptrs.assign(shards, shards + n_stripes * (k + m));
  for (size_t i = 0; i < n_stripes; ++i) {
    JobDesc &j = jobs[i];
    j.ptr_off = uint32_t(i * (k + m));
    j.n_in = uint16_t(k);
    j.n_out = uint16_t(m);
    j.flag_idx = verify ? uint32_t(i) : 0;
    j.tbl = d_enc_tbl;
  }
  return RSGPU_OK;
}

int Codec::encode_dev(size_t n_stripes, uint8_t *const *shards, size_t len, cudaStream_t s) {
  std::vector<JobDesc> jobs;
  std::vector<const uint8_t *> ptrs;
  encode_jobs(n_stripes, shards, jobs, ptrs, false);
  return run_apply(jobs, ptrs, len, false, nullptr, s);
}

int Codec::verify_dev(size_t n_stripes, const uint8_t *const *shards, size_t len, uint8_t *ok_host, cudaStream_t s,
                      const uint32_t *tbl) {
  std::vector<JobDesc> jobs;
  std::vector<const uint8_t *> ptrs;
  encode_jobs(n_stripes, const_cast<uint8_t *const *>(shards), jobs, ptrs, true);
  if (tbl)
    for (auto &j : jobs) j.tbl = tbl;
  uint32_t *flags = nullptr;
  RS_CUDA(cudaError_t(lib_malloc_async(reinterpret_cast<void **>(&flags), n_stripes * 4, s)));
  RS_CUDA(cudaMemsetAsync(flags, 0, n_stripes * 4, s));
  int rc = run_apply(jobs, ptrs, len, true, flags, s);
  if (rc) return rc;
  std::vector<uint32_t> f(n_stripes);
  RS_CUDA(cudaMemcpyAsync(f.data(), flags, n_stripes * 4, cudaMemcpyDeviceToHost, s));
  RS_CUDA(cudaFreeAsync(flags, s));
  if ((rc = take_device_status(s))) return rc;  // also waits for s
  for (size_t i = 0; i < n_stripes; ++i) ok_host[i] = f[i] ? 0 : 1;
  return RSGPU_OK;
}

int Codec::apply_parity_columns(const std::vector<const uint8_t *> &inputs, const std::vector<size_t> &cols,
                                uint8_t *const *parity, size_t len, bool accumulate, cudaStream_t s) {
  if (inputs.empty()) return RSGPU_OK;
  const size_t n_in = inputs.size();
  std::vector<uint8_t> rows(m * n_in);
  for (size_t r = 0; r < m; ++r)
    for (size_t j = 0; j < n_in; ++j) rows[r * n_in + j] = matrix[(k + r) * k + cols[j]];
  std::vector<uint32_t> tbl(packed_table_words(m, n_in));
  pack_tables(rows.data(), m, n_in, tbl.data());
  void *d_tbl = nullptr;
  int rc = upload(tbl.data(), tbl.size() * 4, &d_tbl, s);
  if (rc) return rc;
  std::vector<JobDesc> jobs(1);
  jobs[0].ptr_off = 0;
  jobs[0].n_in = uint16_t(n_in);
  jobs[0].n_out = uint16_t(m);
  jobs[0].tbl = static_cast<const uint32_t *>(d_tbl);
  std::vector<const uint8_t *> ptrs(inputs);
  for (size_t r = 0; r < m; ++r) ptrs.push_back(parity[r]);
  rc = run_apply(jobs, ptrs, len, false, nullptr, s, accumulate);
  RS_CUDA(cudaFreeAsync(d_tbl, s));
  return rc;
}

int Codec::apply_with_tables(std::vector<JobDesc> &jobs, const std::vector<size_t> &tbl_off,
                             std::vector<const uint8_t *> &ptrs, const std::vector<uint32_t> &tables, size_t len,
                             cudaStream_t s) {
  if (jobs.empty()) return RSGPU_OK;
  void *d = nullptr;
  int rc = upload(tables.data(), tables.size() * 4, &d, s);
  if (rc) return rc;
  for (size_t i = 0; i < jobs.size(); ++i) jobs[i].tbl = static_cast<const uint32_t *>(d) + tbl_off[i];
  rc = run_apply(jobs, ptrs, len, false, nullptr, s);
  RS_CUDA(cudaFreeAsync(d, s));
  return rc;
}

int Codec::verify_dev_async(size_t n_stripes, uint8_t *const *shards, size_t len, uint32_t *flags_dev,
                            cudaStream_t s) {
  std::vector<JobDesc> jobs;
  std::vector<const uint8_t *> ptrs;
  encode_jobs(n_stripes, shards, jobs, ptrs, true);
  return run_apply(jobs, ptrs, len, true, flags_dev, s);
}

int Codec::verify_with_buffer_dev(uint8_t *const *ptrs3, size_t len, uint8_t *ok_host, cudaStream_t s) {
  std::vector<JobDesc> jobs(1);
  jobs[0].ptr_off = 0;
  jobs[0].n_in = uint16_t(k);
  jobs[0].n_out = uint16_t(m);
  jobs[0].verify_store = 1;
  jobs[0].tbl = d_enc_tbl;
  std::vector<const uint8_t *> ptrs(ptrs3, ptrs3 + k + 2 * m);
  uint32_t *flags = nullptr;
  RS_CUDA(cudaError_t(lib_malloc_async(reinterpret_cast<void **>(&flags), 4, s)));
  RS_CUDA(cudaMemsetAsync(flags, 0, 4, s));
  int rc = run_apply(jobs, ptrs, len, true, flags, s);
  if (rc) return rc;
  uint32_t f = 0;
  RS_CUDA(cudaMemcpyAsync(&f, flags, 4, cudaMemcpyDeviceToHost, s));
  RS_CUDA(cudaFreeAsync(flags, s));
  if ((rc = take_device_status(s))) return rc;  // also waits for s
  *ok_host = f ? 0 : 1;
  return RSGPU_OK;
}

int run_pairs(const std::vector<PairOp> &pairs, int mode, uint8_t *ok_host, cudaStream_t s) {
  if (pairs.empty()) {
    if (ok_host) *ok_host = 1;
    return RSGPU_OK;
  }
  uint64_t max_len = 0;
  for (const PairOp &p : pairs) max_len = std::max<uint64_t>(max_len, p.len);
  void *d_pairs = nullptr;
  int rc = upload(pairs.data(), pairs.size() * sizeof(PairOp), &d_pairs, s);
  if (rc) return rc;
  uint32_t *flag = nullptr;
  if (ok_host) {
    RS_CUDA(cudaError_t(lib_malloc_async(reinterpret_cast<void **>(&flag), 4, s)));
    RS_CUDA(cudaMemsetAsync(flag, 0, 4, s));
  }
  RS_CUDA(launch_pairs(static_cast<const PairOp *>(d_pairs), uint32_t(pairs.size()), max_len, mode, flag, s));
  RS_CUDA(cudaFreeAsync(d_pairs, s));
  if (ok_host) {
    uint32_t f = 0;
    RS_CUDA(cudaMemcpyAsync(&f, flag, 4, cudaMemcpyDeviceToHost, s));
    RS_CUDA(cudaFreeAsync(flag, s));
    RS_CUDA(cudaStreamSynchronize(s));
    *ok_host = f ? 0 : 1;
  }
  return RSGPU_OK;
}

int Codec::decode_idx_dev(const std::vector<uint16_t> &selected, const std::vector<uint16_t> &outs,
                          const std::vector<uint16_t> &cols, uint8_t *const *dst, const uint8_t *const *input,
                          size_t len, cudaStream_t s) {
  // A decode-table block holds the packed rows of at most m outputs, so the
  // destinations go in chunks of m, one table and one K1 job per chunk.
  bool identity = true;  // the selected inputs are the data shards in order
  for (size_t i = 0; i < k; ++i) identity &= selected[i] == i;
  std::vector<ClassicPlan> plans;
  for (size_t o0 = 0; o0 < outs.size(); o0 += m) {
    ClassicPlan p;
    p.survivors = selected;
    p.targets.assign(outs.begin() + o0, outs.begin() + std::min(outs.size(), o0 + m));
    for (uint16_t o : p.targets) p.n_data_targets += o < k ? 1 : 0;
    p.needs_inverse = !identity;
    plans.push_back(std::move(p));
  }
  std::vector<const ClassicPlan *> pp;
  for (const ClassicPlan &p : plans) pp.push_back(&p);
  std::vector<const uint32_t *> tbls;
  int rc;
  {
    std::lock_guard<std::mutex> g(mu_);
    rc = decode_tables(pp, tbls, s);
  }
  if (rc) return rc;
  const size_t n_sel = cols.size();
  // Only some of the selected inputs arrive in this call: gather their
  // columns of each chunk's rows into tables of their own.
  uint32_t *reduced = nullptr;
  std::vector<size_t> red_off(plans.size(), 0);
  if (n_sel != k) {
    size_t words = 0;
    for (size_t c = 0; c < plans.size(); ++c) {
      red_off[c] = words;
      words += packed_table_words(plans[c].targets.size(), n_sel);
    }
    RS_CUDA(cudaError_t(lib_malloc_async(reinterpret_cast<void **>(&reduced), words * 4, s)));
    GatherCols gc{};
    for (size_t j = 0; j < n_sel; ++j) gc.cols[j] = uint8_t(cols[j]);
    for (size_t c = 0; c < plans.size(); ++c) {
      const uint32_t groups = uint32_t((plans[c].targets.size() + 3) / 4);
      RS_CUDA(launch_gather_tables(tbls[c], reduced + red_off[c], gc, groups, uint32_t(k), uint32_t(n_sel), s));
    }
  }
  std::vector<JobDesc> jobs(plans.size());
  std::vector<const uint8_t *> ptrs;
  for (size_t c = 0; c < plans.size(); ++c) {
    jobs[c].ptr_off = uint32_t(ptrs.size());
    jobs[c].n_in = uint16_t(n_sel);
    jobs[c].n_out = uint16_t(plans[c].targets.size());
    jobs[c].tbl = reduced ? reduced + red_off[c] : tbls[c];
    for (uint16_t col : cols) ptrs.push_back(input[selected[col]]);
    for (uint16_t o : plans[c].targets) ptrs.push_back(dst[o]);
  }
  rc = run_apply(jobs, ptrs, len, false, nullptr, s, true);
  if (reduced) RS_CUDA(cudaFreeAsync(reduced, s));
  return rc;
}

int Codec::reconstruct_jobs(size_t n_stripes, uint8_t *const *shards, const uint8_t *present, int goal,
                            const uint8_t *required, size_t n_required, std::vector<JobDesc> &jobs,
                            std::vector<const uint8_t *> &ptrs, cudaStream_t s, uint32_t **owned) {
  const size_t total = k + m;
  std::vector<ClassicPlan> plans(n_stripes);
  for (size_t i = 0; i < n_stripes; ++i) {
    int rc = plan_classic(present + i * total, goal, required, n_required, plans[i]);
    if (rc) return rc;
  }
  std::vector<const ClassicPlan *> pp(n_stripes);
  for (size_t i = 0; i < n_stripes; ++i) pp[i] = &plans[i];
  std::vector<const uint32_t *> tbls;
  int rc;
  if (owned) {
    rc = decode_tables_copy(pp, tbls, owned, s);
  } else {
    std::lock_guard<std::mutex> g(mu_);
    rc = decode_tables(pp, tbls, s);
  }
  if (rc) return rc;
  jobs.clear();
  ptrs.clear();
  jobs.reserve(n_stripes);
  ptrs.reserve(n_stripes * total);
  for (size_t i = 0; i < n_stripes; ++i) {
    const ClassicPlan &p = plans[i];
    if (p.all_present || p.targets.empty()) continue;
    JobDesc j{};
    j.ptr_off = uint32_t(ptrs.size());
    j.n_in = uint16_t(k);
    j.n_out = uint16_t(p.targets.size());
    j.tbl = tbls[i];
    for (uint16_t sv : p.survivors) ptrs.push_back(shards[i * total + sv]);
    for (uint16_t t : p.targets) ptrs.push_back(shards[i * total + t]);
    jobs.push_back(j);
  }
  return RSGPU_OK;
}

int Codec::reconstruct_dev(size_t n_stripes, uint8_t *const *shards, const uint8_t *present, size_t len, int goal,
                           const uint8_t *required, size_t n_required, cudaStream_t s) {
  std::vector<JobDesc> jobs;
  std::vector<const uint8_t *> ptrs;
  int rc = reconstruct_jobs(n_stripes, shards, present, goal, required, n_required, jobs, ptrs, s);
  if (rc) return rc;
  return run_apply(jobs, ptrs, len, false, nullptr, s);
}

}  // namespace rsgpu
