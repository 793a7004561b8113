// server.cpp -- the request server: continuous batching of encode /
// reconstruct / verify requests of any codec and size onto the GPU.
//
// The reference is a library called once per stripe from the storage node's
// own request handlers (src/core/encode.rs:935-972,
// src/core/reconstruct.rs:731-790, src/core/verify.rs:14-174).  This server is
// the GPU-side loop such a node feeds: requests are submitted from any thread
// and complete asynchronously.  One worker thread runs the loop (and between
// its passes, the dense-map derivations of step 4):
//
//   1. retire: every launch whose completion event has fired finishes its
//      requests (verify flags read from pinned memory), frees their device
//      staging and gives back their slots and device-memory reservation;
//   2. admit: while a launch slot (stream) is free, take pending requests in
//      arrival order as long as a request slot and the device-memory budget
//      allow (a request reserves its stripe bytes: (k + m) * shard_len);
//   3. launch: copy the admitted host-memory requests' inputs into
//      stream-ordered device staging, build ONE mixed batch for all admitted
//      requests (plans from the planner: measured table / cost model), run it
//      in the persistent kernel, copy outputs back, record an event.
//
//   4. derive: a Leopard GF(2^8) rebuild pattern whose dense map has become
//      due runs the FFT decode in its batch, and its map is derived on a side
//      stream (queued, never waited for: a wait there queues behind the
//      persistent batches of the launch streams); a finished derivation adds
//      the map to its codec's cache, where later batches find it.
//
// Up to `streams` launches are in flight at once, so requests that arrive
// while others run are admitted into the next launch and their work overlaps
// the running ones on the device.  Decode tables and error locators stay
// cached in HBM by their codecs; device-memory requests (shards resident in
// HBM) are used in place.  Every step of a launch is stream-ordered, so the
// loop never synchronizes the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <future>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <thread>
#include <vector>

#include <set>
#include <string>

#include "batch.hpp"
#include "codec.hpp"
#include "handles.hpp"
#include "leopard.hpp"
#include "rsgpu.h"

namespace rsgpu {

#define SV_CUDA(expr)                              \
  do {                                             \
    cudaError_t e_ = (expr);                       \
    if (e_ != cudaSuccess) return cuda_status(e_); \
  } while (0)

namespace {

using Clock = std::chrono::steady_clock;

struct Req {
  rsgpu_request r{};
  std::vector<uint8_t *> shards;  // caller's pointers
  std::vector<uint8_t> present;
  std::vector<uint8_t *> dev;     // device pointers the batch uses
  uint8_t *staging = nullptr;     // device staging of a host-memory request
  size_t reserve = 0;             // budget bytes held while admitted
  double t_submit = 0, t_admit = 0;
};

struct Flight {
  std::vector<Req *> reqs;
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  uint32_t *h_flags = nullptr;  // pinned, one word per request
  size_t h_cap = 0;
  ScratchSlot scratch;  // work rows of this flight's batches
  bool busy = false;
};

// Work-row buffers of stopped servers, by device, for the next server to
// take: a buffer grows to the widest batch it has served (hundreds of MB for
// wide GF(2^16) decodes), and growing it again in every new server put that
// allocation, which can block for up to hundreds of milliseconds, on some
// request's path.  Buffers are returned only after their stream has
// finished, so a later stream may use them at once.
std::mutex g_slots_mu;
std::map<int, std::vector<ScratchSlot>> g_slots;

ScratchSlot take_slot(int device) {
  std::lock_guard<std::mutex> g(g_slots_mu);
  auto &v = g_slots[device];
  if (v.empty()) return ScratchSlot{};
  auto best = std::max_element(v.begin(), v.end(), [](const ScratchSlot &x, const ScratchSlot &y) {
    return x.bytes < y.bytes;
  });
  ScratchSlot out = *best;
  v.erase(best);
  return out;
}

void return_slot(int device, const ScratchSlot &s) {
  if (!s.ptr) return;
  std::lock_guard<std::mutex> g(g_slots_mu);
  g_slots[device].push_back(s);
}

}  // namespace

class Server {
 public:
  explicit Server(const rsgpu_server_options &o) : opt_(o) {}
  ~Server() { stop(); }

  int start() {
    SV_CUDA(cudaGetDevice(&device_));
    if (opt_.device_budget == 0) {
      size_t free_b = 0, total_b = 0;
      SV_CUDA(cudaMemGetInfo(&free_b, &total_b));
      opt_.device_budget = free_b / 2;
    }
    if (opt_.max_inflight == 0) opt_.max_inflight = 4096;
    // 64 requests per launch: on the bench's serving stream at 800 GB/s
    // offered (B200), 64 gave 334-346 GB/s with p50 42-47 ms and p99 75-81 ms,
    // 512 gave 326-344 GB/s with p50 60-64 ms and p99 85-100 ms (32: as 64,
    // with more host time per byte).  Smaller launches let the streams
    // overlap and shorten the last launch of a burst.
    if (opt_.max_batch == 0) opt_.max_batch = 64;
    if (opt_.streams == 0) opt_.streams = 3;
    flights_.resize(opt_.streams);
    for (auto &f : flights_) {
      SV_CUDA(cudaStreamCreateWithFlags(&f.stream, cudaStreamNonBlocking));
      SV_CUDA(cudaEventCreateWithFlags(&f.done, cudaEventDisableTiming));
      f.scratch = take_slot(device_);
    }
    // Every stream starts with a work-row buffer as large as the largest one
    // handed over, so that no stream grows its own (a pool allocation of up
    // to a few hundred MB) under its first wide batch, on a request's path.
    // Best effort: a stream whose allocation fails starts empty and grows its
    // buffer when a batch needs it, as it would without this step.
    size_t widest = 0;
    for (auto &f : flights_) widest = std::max(widest, f.scratch.bytes);
    for (auto &f : flights_) {
      if (f.scratch.bytes >= widest) continue;
      if (f.scratch.ptr) SV_CUDA(cudaFreeAsync(f.scratch.ptr, f.stream));
      f.scratch = ScratchSlot{};
      void *p = nullptr;
      if (cudaError_t(lib_malloc_async(&p, widest, f.stream)) == cudaSuccess) {
        f.scratch.ptr = p;
        f.scratch.bytes = widest;
      } else {
        cudaGetLastError();  // an out-of-memory here is not sticky
      }
    }
    // Memory the first batches would otherwise map on a request's path:
    // growing the library's device pool (work rows, batch blobs) mapped fresh
    // device memory for 15-100 ms in the first batches of a server.  A block
    // allocated and freed here stays in the pool, which keeps up to 2 GiB of
    // freed memory.  Best effort, like the buffers above.
    {
      void *p = nullptr;
      if (cudaError_t(lib_malloc_async(&p, kPoolReserve, flights_[0].stream)) == cudaSuccess) {
        cudaFreeAsync(p, flights_[0].stream);
        cudaStreamSynchronize(flights_[0].stream);
      } else {
        cudaGetLastError();
      }
    }
    t0_ = Clock::now();
    // The worker's bounce buffers (batch blobs go through them) are
    // allocated before start returns: cudaHostAlloc of tens of megabytes at
    // the top of the loop delayed a new server's first requests by ~30 ms.
    std::promise<void> warm;
    std::future<void> warmed = warm.get_future();
    worker_ = std::thread([this, &warm] {
      cudaSetDevice(device_);
      upload_prewarm(kUploadWarmBuffers, kUploadWarmBytes);
      warm.set_value();
      loop();
    });
    warmed.wait();
    return RSGPU_OK;
  }

  void stop() {
    {
      std::lock_guard<std::mutex> g(mu_);
      if (stopping_) return;
      stopping_ = true;
    }
    cv_.notify_all();
    if (worker_.joinable()) worker_.join();
    if (dstream_) {
      cudaStreamSynchronize(dstream_);
      poll_derivations();
      cudaStreamDestroy(dstream_);
      dstream_ = nullptr;
    }
    for (auto &p : pinned_pool_) cudaFreeHost(p.first);
    pinned_pool_.clear();
    for (auto &f : flights_) {
      if (f.stream) cudaStreamSynchronize(f.stream);
      return_slot(device_, f.scratch);  // its stream has finished
      f.scratch = ScratchSlot{};
      if (f.done) cudaEventDestroy(f.done);
      if (f.stream) cudaStreamDestroy(f.stream);
      if (f.h_flags) cudaFreeHost(f.h_flags);
    }
    flights_.clear();
  }

  int submit(const rsgpu_request &r) {
    if (!r.codec || !r.shards) return RSGPU_ERR_INVALID_ARGUMENT;
    if (r.mem != RSGPU_MEM_HOST && r.mem != RSGPU_MEM_DEVICE) return RSGPU_ERR_INVALID_ARGUMENT;
    const Codec &c = r.codec->c;
    const size_t total = c.k + c.m;
    std::unique_ptr<Req> q(new (std::nothrow) Req());
    if (!q) return RSGPU_ERR_OUT_OF_MEMORY;
    q->r = r;
    q->shards.assign(r.shards, r.shards + total);
    if (r.op == RSGPU_OP_RECONSTRUCT && r.present) q->present.assign(r.present, r.present + total);
    rsgpu_mix_op op = as_op(*q, q->shards.data());
    int rc = mix_validate(op, device_);
    if (rc) return rc;
    const size_t stripe = total * r.shard_len;
    if (stripe > opt_.device_budget) return RSGPU_ERR_OUT_OF_MEMORY;
    q->reserve = stripe;
    q->t_submit = now();
    {
      std::lock_guard<std::mutex> g(mu_);
      if (stopping_) return RSGPU_ERR_INVALID_ARGUMENT;
      pending_.push_back(q.release());
      ++submitted_;
    }
    cv_.notify_all();
    return RSGPU_OK;
  }

  size_t poll(rsgpu_completion *out, size_t cap, int32_t timeout_ms) {
    std::unique_lock<std::mutex> g(mu_);
    if (done_.empty() && timeout_ms != 0) {
      auto pred = [&] { return !done_.empty(); };
      if (timeout_ms < 0)
        done_cv_.wait(g, pred);
      else
        done_cv_.wait_for(g, std::chrono::milliseconds(timeout_ms), pred);
    }
    const size_t n = std::min(cap, done_.size());
    for (size_t i = 0; i < n; ++i) {
      out[i] = done_.front();
      done_.pop_front();
    }
    return n;
  }

  void stats(rsgpu_server_stats *s) {
    std::lock_guard<std::mutex> g(mu_);
    s->submitted = submitted_;
    s->completed = completed_;
    s->launches = launches_;
    s->pending = pending_.size();
    s->inflight = inflight_;
    s->budget_bytes = opt_.device_budget;
    s->reserved_bytes = reserved_;
    s->max_reserved_bytes = max_reserved_;
    s->max_concurrent_launches = max_concurrent_;
    s->prepare_seconds = prepare_s_;
    s->max_prepare_seconds = max_prepare_s_;
    s->max_loop_gap_seconds = max_gap_s_;
  }

 private:
  static constexpr size_t kPoolReserve = size_t(1) << 30;
  static constexpr size_t kUploadWarmBuffers = 4;
  static constexpr size_t kUploadWarmBytes = size_t(16) << 20;
  rsgpu_server_options opt_;
  int device_ = 0;
  std::thread worker_;
  std::mutex mu_;
  std::condition_variable cv_, done_cv_;
  std::deque<Req *> pending_;
  std::deque<rsgpu_completion> done_;
  std::vector<Flight> flights_;
  bool stopping_ = false;
  uint64_t submitted_ = 0, completed_ = 0, launches_ = 0;
  size_t inflight_ = 0, reserved_ = 0, max_reserved_ = 0;
  uint32_t max_concurrent_ = 0;
  double prepare_s_ = 0;  // worker time spent building and launching batches
  double max_prepare_s_ = 0;  // longest single build-and-launch
  double max_gap_s_ = 0;      // longest time between two passes of the worker loop
  Clock::time_point t0_;
  // Dense-map derivations in flight on their own stream (step 4), and the
  // pinned buffers they use (kept until the server stops: freeing pinned
  // memory synchronizes the device).
  struct Deriving {
    DenseDerivation d;
    std::pair<uint8_t *, size_t> pinned;
    std::string key;
  };
  static constexpr size_t kMaxDerivations = 8;
  cudaStream_t dstream_ = nullptr;
  std::vector<Deriving> deriving_;
  std::vector<DenseWant> wants_;  // filled by mix_build, drained after each launch
  std::set<std::string> deriving_keys_;
  std::vector<std::pair<uint8_t *, size_t>> pinned_pool_;
  uint64_t derived_ = 0;

  // Step 4: queue the derivation of maps that batches found due.
  void start_derivations(const std::vector<DenseWant> &wants) {
    for (const DenseWant &w : wants) {
      if (deriving_.size() >= kMaxDerivations) break;
      std::string key(reinterpret_cast<const char *>(&w.codec), sizeof(w.codec));
      key += w.pattern;
      key += char(w.goal);
      if (deriving_keys_.count(key)) continue;
      Codec &c = const_cast<rsgpu_codec *>(w.codec)->c;
      const uint8_t *pres = reinterpret_cast<const uint8_t *>(w.pattern.data());
      const size_t need = leopard_dense_derive_bytes(c, pres, w.goal);
      if (!dstream_ && cudaStreamCreateWithFlags(&dstream_, cudaStreamNonBlocking) != cudaSuccess) return;
      std::pair<uint8_t *, size_t> buf{nullptr, 0};
      for (size_t i = 0; i < pinned_pool_.size(); ++i)
        if (pinned_pool_[i].second >= need) {
          buf = pinned_pool_[i];
          pinned_pool_.erase(pinned_pool_.begin() + long(i));
          break;
        }
      if (!buf.first) {
        if (cudaMallocHost(reinterpret_cast<void **>(&buf.first), need) != cudaSuccess) return;
        buf.second = need;
      }
      Deriving dv;
      dv.pinned = buf;
      dv.key = key;
      if (leopard_dense_derive_start(c, pres, w.goal, buf.first, dstream_, dv.d) != RSGPU_OK) {
        // The batch already runs this pattern through the FFT decode; only
        // the map is missing.  Settle the side stream before its buffer is
        // reused.
        cudaStreamSynchronize(dstream_);
        if (dv.d.done) cudaEventDestroy(dv.d.done);
        pinned_pool_.push_back(buf);
        continue;
      }
      deriving_keys_.insert(key);
      deriving_.push_back(std::move(dv));
    }
  }

  // Finishes the derivations whose work is done.  Returns true on progress.
  bool poll_derivations() {
    bool any = false;
    for (size_t i = 0; i < deriving_.size();) {
      Deriving &dv = deriving_[i];
      if (cudaEventQuery(dv.d.done) == cudaErrorNotReady) {
        ++i;
        continue;
      }
      leopard_dense_derive_finish(dv.d);
      ++derived_;
      pinned_pool_.push_back(dv.pinned);
      deriving_keys_.erase(dv.key);
      deriving_.erase(deriving_.begin() + long(i));
      any = true;
    }
    return any;
  }

  double now() const { return std::chrono::duration<double>(Clock::now() - t0_).count(); }

  static rsgpu_mix_op as_op(const Req &q, uint8_t *const *ptrs) {
    rsgpu_mix_op o{};
    o.codec = q.r.codec;
    o.op = q.r.op;
    o.goal = q.r.goal;
    o.shards = ptrs;
    o.present = q.present.empty() ? nullptr : q.present.data();
    o.shard_len = q.r.shard_len;
    return o;
  }

  // Shards a request reads (input) and writes (output).
  static void roles(const Req &q, std::vector<size_t> &in, std::vector<size_t> &out) {
    const Codec &c = q.r.codec->c;
    const size_t total = c.k + c.m;
    in.clear();
    out.clear();
    for (size_t i = 0; i < total; ++i) {
      if (q.r.op == RSGPU_OP_ENCODE) {
        (i < c.k ? in : out).push_back(i);
      } else if (q.r.op == RSGPU_OP_VERIFY) {
        in.push_back(i);
      } else if (q.present[i]) {
        in.push_back(i);
      } else if (q.r.goal == RSGPU_GOAL_ALL || i < c.k) {
        out.push_back(i);
      }
    }
  }

  void finish(Req *q, int status, int ok) {
    rsgpu_completion c{};
    c.tag = q->r.tag;
    c.status = status;
    c.ok = ok;
    c.submit_s = q->t_submit;
    c.admit_s = q->t_admit;
    c.done_s = now();
    {
      std::lock_guard<std::mutex> g(mu_);
      done_.push_back(c);
      ++completed_;
    }
    done_cv_.notify_all();
    delete q;
  }

  // Step 1.  Returns true when a launch finished.
  bool retire() {
    bool any = false;
    for (auto &f : flights_) {
      if (!f.busy || cudaEventQuery(f.done) == cudaErrorNotReady) continue;
      const cudaError_t e = cudaEventQuery(f.done);
      const int status = e == cudaSuccess ? RSGPU_OK : cuda_status(e);
      size_t freed = 0;
      for (size_t i = 0; i < f.reqs.size(); ++i) {
        Req *q = f.reqs[i];
        freed += q->reserve;
        finish(q, status, f.h_flags[i] ? 0 : 1);
      }
      {
        std::lock_guard<std::mutex> g(mu_);
        inflight_ -= f.reqs.size();
        reserved_ -= freed;
      }
      f.reqs.clear();
      f.busy = false;
      any = true;
    }
    return any;
  }

  // Steps 2 and 3 on one free launch slot.  Returns true when it launched.
  bool admit_and_launch(Flight &f) {
    std::vector<Req *> take;
    {
      std::lock_guard<std::mutex> g(mu_);
      while (!pending_.empty() && take.size() < opt_.max_batch && inflight_ + take.size() < opt_.max_inflight) {
        Req *q = pending_.front();
        if (reserved_ + q->reserve > opt_.device_budget) break;  // wait for memory (arrival order)
        reserved_ += q->reserve;
        max_reserved_ = std::max(max_reserved_, reserved_);
        pending_.pop_front();
        take.push_back(q);
      }
      inflight_ += take.size();
    }
    if (take.empty()) return false;
    const double t = now();
    struct Timer {  // adds this call's host time to prepare_s_ on every return path
      Server *sv;
      double t0;
      ~Timer() {
        const double dt = sv->now() - t0;
        std::lock_guard<std::mutex> g(sv->mu_);
        sv->prepare_s_ += dt;
        sv->max_prepare_s_ = std::max(sv->max_prepare_s_, dt);
      }
    } timer{this, t};
    std::vector<size_t> in, out;
    std::vector<rsgpu_mix_op> ops(take.size());
    int rc = RSGPU_OK;
    for (size_t i = 0; i < take.size() && rc == RSGPU_OK; ++i) {
      Req *q = take[i];
      q->t_admit = t;
      const Codec &c = q->r.codec->c;
      const size_t total = c.k + c.m, len = q->r.shard_len;
      if (q->r.mem == RSGPU_MEM_DEVICE) {
        q->dev = q->shards;
      } else {
        if (cudaError_t(lib_malloc_async(reinterpret_cast<void **>(&q->staging), total * len, f.stream)) != cudaSuccess) {
          rc = RSGPU_ERR_OUT_OF_MEMORY;
          break;
        }
        q->dev.resize(total);
        for (size_t j = 0; j < total; ++j) q->dev[j] = q->staging + j * len;
        roles(*q, in, out);
        for (size_t j : in)
          if (cudaMemcpyAsync(q->dev[j], q->shards[j], len, cudaMemcpyHostToDevice, f.stream) != cudaSuccess)
            rc = RSGPU_ERR_CUDA;
      }
      ops[i] = as_op(*q, q->dev.data());
    }
    MixPtr b;
    if (rc == RSGPU_OK) {
      rsgpu_mix_options mo;
      rsgpu_mix_options_default(&mo);
      mo.planner = opt_.planner;
      mo.graph = 0;
      rc = mix_build(ops.data(), ops.size(), nullptr, mo, b, f.stream, &f.scratch, &wants_);
    }
    if (rc == RSGPU_OK) rc = mix_launch(*b, f.stream);
    if (!wants_.empty()) {
      start_derivations(wants_);
      wants_.clear();
    }
    if (rc == RSGPU_OK) {
      for (Req *q : take) {
        if (q->r.mem != RSGPU_MEM_HOST) continue;
        roles(*q, in, out);
        for (size_t j : out)
          cudaMemcpyAsync(q->shards[j], q->dev[j], q->r.shard_len, cudaMemcpyDeviceToHost, f.stream);
      }
      if (f.h_cap < take.size()) {
        if (f.h_flags) cudaFreeHost(f.h_flags);
        f.h_cap = std::max<size_t>(take.size(), 1024);
        if (cudaMallocHost(&f.h_flags, f.h_cap * 4) != cudaSuccess) rc = RSGPU_ERR_OUT_OF_MEMORY;
      }
      if (rc == RSGPU_OK)
        cudaMemcpyAsync(f.h_flags, mix_flags(*b), take.size() * 4, cudaMemcpyDeviceToHost, f.stream);
    }
    b.reset();  // stream-ordered: its memory is released after the queued work
    for (Req *q : take)
      if (q->staging) cudaFreeAsync(q->staging, f.stream);
    if (rc != RSGPU_OK) {
      cudaStreamSynchronize(f.stream);
      size_t freed = 0;
      for (Req *q : take) {
        freed += q->reserve;
        finish(q, rc, 0);
      }
      std::lock_guard<std::mutex> g(mu_);
      inflight_ -= take.size();
      reserved_ -= freed;
      return true;
    }
    cudaEventRecord(f.done, f.stream);
    f.reqs = std::move(take);
    f.busy = true;
    uint32_t busy = 0;
    for (auto &x : flights_) busy += x.busy ? 1 : 0;
    std::lock_guard<std::mutex> g(mu_);
    ++launches_;
    max_concurrent_ = std::max(max_concurrent_, busy);
    return true;
  }

  void loop() {
    double last = now();
    for (;;) {
      const double t_pass = now();
      const double gap = t_pass - last;
      last = t_pass;
      bool progress = retire();
      for (auto &f : flights_)
        if (!f.busy) progress |= admit_and_launch(f);
      if (!deriving_.empty()) progress |= poll_derivations();
      bool idle_exit = false;
      {
        std::unique_lock<std::mutex> g(mu_);
        max_gap_s_ = std::max(max_gap_s_, gap);
        bool any_busy = false;
        for (auto &f : flights_) any_busy |= f.busy;
        if (stopping_ && pending_.empty() && !any_busy) idle_exit = true;
        else if (!progress)
          // Nothing to do until a submission or a launch finishes: short
          // waits keep completion latency low without spinning a core.
          cv_.wait_for(g, std::chrono::microseconds(any_busy ? 20 : 500));
      }
      if (idle_exit) break;
    }
  }
};

}  // namespace rsgpu

struct rsgpu_server {
  std::unique_ptr<rsgpu::Server> s;
};

extern "C" {

void rsgpu_server_options_default(rsgpu_server_options *out) {
  if (!out) return;
  std::memset(out, 0, sizeof(*out));
  out->planner = RSGPU_PLANNER_MODEL;
}

int32_t rsgpu_server_new(const rsgpu_server_options *opts, rsgpu_server **out) {
  if (!out) return RSGPU_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  int dev_count = 0;
  if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count == 0) return RSGPU_ERR_NO_DEVICE;
  rsgpu_server_options o;
  rsgpu_server_options_default(&o);
  if (opts) o = *opts;
  std::unique_ptr<rsgpu_server> h(new (std::nothrow) rsgpu_server());
  if (!h) return RSGPU_ERR_OUT_OF_MEMORY;
  h->s.reset(new (std::nothrow) rsgpu::Server(o));
  if (!h->s) return RSGPU_ERR_OUT_OF_MEMORY;
  int rc = h->s->start();
  if (rc) return rc;
  *out = h.release();
  return RSGPU_OK;
}

int32_t rsgpu_server_submit(rsgpu_server *s, const rsgpu_request *r) {
  if (!s || !r) return RSGPU_ERR_INVALID_ARGUMENT;
  return s->s->submit(*r);
}

size_t rsgpu_server_poll(rsgpu_server *s, rsgpu_completion *out, size_t cap, int32_t timeout_ms) {
  if (!s || (!out && cap)) return 0;
  return s->s->poll(out, cap, timeout_ms);
}

int32_t rsgpu_server_get_stats(rsgpu_server *s, rsgpu_server_stats *out) {
  if (!s || !out) return RSGPU_ERR_INVALID_ARGUMENT;
  s->s->stats(out);
  return RSGPU_OK;
}

void rsgpu_server_free(rsgpu_server *s) { delete s; }

}  // extern "C"
