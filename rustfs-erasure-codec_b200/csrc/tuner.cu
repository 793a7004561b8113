// tuner.cu -- plan selection for mixed batches: the measured autotuner table
// and the planner that consults it and the learned cost model (model.cu).
//
// A class is (family, k, m, operation, goal, erasure-count bucket, shard
// length bucket).  rsgpu_tune measures every plan valid for a class on
// synthetic device stripes of that shape, in a mixed batch of that class
// alone, and records the best; every measurement is also kept as a training
// sample for the cost model.  Buckets: erasures e -> 0 for e = 0, else
// 1 + floor(log2 e); shard length -> round(log2 length).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <tuple>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "batch.hpp"
#include "codec.hpp"
#include "handles.hpp"
#include "model.hpp"

namespace rsgpu {

#define RS_CUDA(expr)                              \
  do {                                             \
    cudaError_t e_ = (expr);                       \
    if (e_ != cudaSuccess) return cuda_status(e_); \
  } while (0)

namespace {

constexpr int F = RSGPU_MODEL_FEATURES;
constexpr int P = RSGPU_MODEL_PLANS;

struct TuneKey {
  uint8_t family, op, goal, ebucket, lbucket;
  uint16_t k, m;
  bool operator<(const TuneKey &o) const {
    return std::tie(family, op, goal, ebucket, lbucket, k, m) <
           std::tie(o.family, o.op, o.goal, o.ebucket, o.lbucket, o.k, o.m);
  }
};

struct TuneEntry {
  rsgpu_plan best{};
  float gbps[P] = {};
  uint8_t measured[P] = {};
  float features[F] = {};
};

struct Tuner {
  std::mutex mu;
  std::map<TuneKey, TuneEntry> table;
  std::vector<rsgpu_tune_sample> samples;
};
Tuner &tuner() {
  static Tuner t;
  return t;
}

int ilog2_floor(uint64_t v) {
  int b = -1;
  while (v) {
    v >>= 1;
    ++b;
  }
  return b;
}

size_t erased(const rsgpu_mix_op &o, size_t *data_erased) {
  const Codec &c = o.codec->c;
  size_t e = 0, d = 0;
  if (o.op == RSGPU_OP_RECONSTRUCT && o.present)
    for (size_t i = 0; i < c.k + c.m; ++i)
      if (!o.present[i]) {
        ++e;
        d += i < c.k;
      }
  if (data_erased) *data_erased = d;
  return e;
}

TuneKey key_of(const rsgpu_mix_op &o) {
  const Codec &c = o.codec->c;
  TuneKey k{};
  k.family = uint8_t(c.family);
  k.op = uint8_t(o.op);
  k.goal = uint8_t(o.op == RSGPU_OP_RECONSTRUCT ? o.goal : 0);
  const size_t e = erased(o, nullptr);
  k.ebucket = uint8_t(e == 0 ? 0 : 1 + ilog2_floor(e));
  k.lbucket = uint8_t(std::lround(std::log2(double(std::max<size_t>(o.shard_len, 1)))));
  k.k = uint16_t(c.k);
  k.m = uint16_t(c.m);
  return k;
}

std::vector<rsgpu_plan> candidates(Codec &c, int op, size_t len) {
  std::vector<rsgpu_plan> out;
  for (int i = 0; i < P; ++i) {
    rsgpu_plan p = i < 3 ? rsgpu_plan{RSGPU_ALGO_APPLY, i} : rsgpu_plan{RSGPU_ALGO_FFT, i - 2};
    if (!mix_plan_valid(c, op, p)) continue;
    // Transforms of at most 16 lanes ignore the FFT tile: measure one.
    if (p.algo == RSGPU_ALGO_FFT && p.tile > 1 && mix_fft_in_registers(c, op)) continue;
    if (p.algo == RSGPU_ALGO_FFT && (size_t(64) << p.tile) > std::max<size_t>(len, 128)) continue;
    out.push_back(p);
  }
  return out;
}

}  // namespace

int plan_index(const rsgpu_plan &p) {
  if (p.algo == RSGPU_ALGO_APPLY && p.tile >= 0 && p.tile <= 2) return p.tile;
  if (p.algo == RSGPU_ALGO_FFT && p.tile >= 1 && p.tile <= 3) return 2 + p.tile;
  return -1;
}

rsgpu_plan plan_of_index(int i) { return i < 3 ? rsgpu_plan{RSGPU_ALGO_APPLY, i} : rsgpu_plan{RSGPU_ALGO_FFT, i - 2}; }

int plan_features(const rsgpu_mix_op &o, float *f) {
  if (!o.codec) return RSGPU_ERR_INVALID_ARGUMENT;
  const Codec &c = o.codec->c;
  size_t d = 0;
  const size_t e = erased(o, &d);
  for (int i = 0; i < F; ++i) f[i] = 0.f;
  f[0] = c.family == RSGPU_FAMILY_CLASSIC ? 1.f : 0.f;
  f[1] = c.family == RSGPU_FAMILY_LEOPARD_GF8 ? 1.f : 0.f;
  f[2] = c.family == RSGPU_FAMILY_LEOPARD_GF16 ? 1.f : 0.f;
  f[3] = float(std::log2(double(c.k)) / 16.0);
  f[4] = float(std::log2(double(c.m)) / 16.0);
  f[5] = float((std::log2(double(std::max<size_t>(o.shard_len, 1))) - 12.0) / 10.0);
  f[6] = o.op == RSGPU_OP_ENCODE ? 1.f : 0.f;
  f[7] = o.op == RSGPU_OP_RECONSTRUCT ? 1.f : 0.f;
  f[8] = o.op == RSGPU_OP_VERIFY ? 1.f : 0.f;
  f[9] = float(double(e) / double(c.m));
  f[10] = float(double(d) / double(std::max<size_t>(e, 1)));
  return RSGPU_OK;
}

bool table_lookup(const rsgpu_mix_op &o, rsgpu_plan *out) {
  Tuner &t = tuner();
  std::lock_guard<std::mutex> g(t.mu);
  auto it = t.table.find(key_of(o));
  if (it == t.table.end()) return false;
  *out = it->second.best;
  return true;
}

namespace {

// The model's pick over a grid of quantized features, per (family, k, m,
// operation, goal): shard length in quarter octaves from 64 B, erased / m in
// 64ths, erased data / erased in 16ths.  A grid is one batched forward pass
// on the GPU, made the first time an operation of its kind needs the model
// (and again after the weights change); planning a batch then reads it on the
// host, so a request path never waits for an inference launch, which would
// queue behind the persistent batches other streams keep on the device.
constexpr int kGridLen = 97, kGridErased = 65, kGridData = 17;

struct GridKey {
  int family, k, m, op, goal;
  bool operator<(const GridKey &o) const {
    return std::tie(family, k, m, op, goal) < std::tie(o.family, o.k, o.m, o.op, o.goal);
  }
};
struct Grid {
  uint64_t version = 0;
  std::vector<int8_t> best;  // plan index per cell, -1 where no plan is valid
};
std::mutex grid_mu;
std::map<GridKey, Grid> &grids() {
  static std::map<GridKey, Grid> g;
  return g;
}

int grid_cells(int op) { return op == RSGPU_OP_RECONSTRUCT ? kGridLen * kGridErased * kGridData : kGridLen; }

// Cell of an operation, and the features the grid evaluates at that cell.
int grid_cell(const rsgpu_mix_op &o) {
  const Codec &c = o.codec->c;
  const double lg = std::log2(double(std::max<size_t>(o.shard_len, 1)));
  const int lq = int(std::min<long>(kGridLen - 1, std::max<long>(0, std::lround((lg - 6.0) * 4.0))));
  if (o.op != RSGPU_OP_RECONSTRUCT) return lq;
  size_t d = 0;
  const size_t e = erased(o, &d);
  const int eq = int(std::lround(64.0 * double(e) / double(c.m)));
  const int dq = int(std::lround(16.0 * double(d) / double(std::max<size_t>(e, 1))));
  return (lq * kGridErased + std::min(eq, kGridErased - 1)) * kGridData + std::min(dq, kGridData - 1);
}

void cell_features(const Codec &c, int op, int cell, float *f) {
  int lq = cell, eq = 0, dq = 0;
  if (op == RSGPU_OP_RECONSTRUCT) {
    dq = cell % kGridData;
    eq = (cell / kGridData) % kGridErased;
    lq = cell / (kGridData * kGridErased);
  }
  for (int i = 0; i < F; ++i) f[i] = 0.f;
  f[0] = c.family == RSGPU_FAMILY_CLASSIC ? 1.f : 0.f;
  f[1] = c.family == RSGPU_FAMILY_LEOPARD_GF8 ? 1.f : 0.f;
  f[2] = c.family == RSGPU_FAMILY_LEOPARD_GF16 ? 1.f : 0.f;
  f[3] = float(std::log2(double(c.k)) / 16.0);
  f[4] = float(std::log2(double(c.m)) / 16.0);
  f[5] = float((6.0 + lq / 4.0 - 12.0) / 10.0);
  f[6] = op == RSGPU_OP_ENCODE ? 1.f : 0.f;
  f[7] = op == RSGPU_OP_RECONSTRUCT ? 1.f : 0.f;
  f[8] = op == RSGPU_OP_VERIFY ? 1.f : 0.f;
  f[9] = float(eq / 64.0);
  f[10] = float(dq / 16.0);
}

// The grid for op's kind, built when missing or made by older weights.  The
// grids of every kind of the codec's shape (encode, verify, reconstruct with
// goal all and data) are built together, in one forward pass, so a serving
// stream meets at most one build per codec shape.
int grid_for(const rsgpu_mix_op &o, const Grid **out) {
  Codec &c = const_cast<rsgpu_codec *>(o.codec)->c;
  const GridKey key{c.family, int(c.k), int(c.m), o.op, o.op == RSGPU_OP_RECONSTRUCT ? o.goal : 0};
  const uint64_t version = model_version();
  std::lock_guard<std::mutex> g(grid_mu);
  Grid &gr = grids()[key];
  if (gr.best.empty() || gr.version != version) {
    struct Kind {
      int op, goal;
    };
    const Kind kinds[4] = {{RSGPU_OP_ENCODE, 0},
                           {RSGPU_OP_VERIFY, 0},
                           {RSGPU_OP_RECONSTRUCT, RSGPU_GOAL_ALL},
                           {RSGPU_OP_RECONSTRUCT, RSGPU_GOAL_DATA}};
    std::vector<float> feat;
    size_t rows = 0;
    for (const Kind &kd : kinds) rows += size_t(grid_cells(kd.op));
    feat.resize(rows * F);
    std::vector<float> pred(rows * P);
    size_t at = 0;
    for (const Kind &kd : kinds)
      for (int x = 0; x < grid_cells(kd.op); ++x, ++at) cell_features(c, kd.op, x, &feat[at * F]);
    uint64_t v = 0;
    int rc = model_predict(feat.data(), rows, pred.data(), false, &v);
    if (rc) return rc;
    at = 0;
    for (const Kind &kd : kinds) {
      Grid &kg = grids()[GridKey{c.family, int(c.k), int(c.m), kd.op, kd.goal}];
      const int cells = grid_cells(kd.op);
      kg.best.assign(cells, -1);
      for (int x = 0; x < cells; ++x, ++at) {
        int best = -1;
        for (int j = 0; j < P; ++j) {
          if (!mix_plan_valid(c, kd.op, plan_of_index(j))) continue;
          if (best < 0 || pred[at * P + j] > pred[at * P + best]) best = j;
        }
        kg.best[x] = int8_t(best);
      }
      kg.version = v;
    }
  }
  *out = &gr;  // std::map nodes are stable
  return RSGPU_OK;
}

}  // namespace

int mix_plan_batch(const rsgpu_mix_op *ops, size_t n, int planner, std::vector<rsgpu_plan> &plans) {
  if (planner == RSGPU_PLANNER_FIXED) return RSGPU_OK;
  std::vector<size_t> ask;
  for (size_t i = 0; i < n; ++i) {
    Codec &c = const_cast<rsgpu_codec *>(ops[i].codec)->c;
    rsgpu_plan p{};
    if (table_lookup(ops[i], &p) && mix_plan_valid(c, ops[i].op, p))
      plans[i] = p;
    else if (planner == RSGPU_PLANNER_MODEL)
      ask.push_back(i);
  }
  if (ask.empty() || !model_ready()) return RSGPU_OK;
  for (size_t i : ask) {
    const Grid *g = nullptr;
    int rc = grid_for(ops[i], &g);
    if (rc) return rc;
    const int best = g->best[grid_cell(ops[i])];
    if (best >= 0) plans[i] = plan_of_index(best);
  }
  return RSGPU_OK;
}

namespace {

// Device stripes for the sweep, grown on demand.
struct SweepBuffer {
  uint8_t *d = nullptr;
  size_t bytes = 0;
  ~SweepBuffer() {
    if (d) cudaFree(d);
  }
  int ensure(size_t n) {
    if (n <= bytes) return RSGPU_OK;
    if (d) {
      RS_CUDA(cudaDeviceSynchronize());
      cudaFree(d);
      d = nullptr;
      bytes = 0;
    }
    RS_CUDA(cudaMalloc(&d, n));
    RS_CUDA(cudaMemset(d, 0xA5, n));
    bytes = n;
    return RSGPU_OK;
  }
};

// Measure every candidate plan of the class of `rep` on n stripes of its
// shape; returns GB/s per plan index (0 where not measured).
int measure_class(const rsgpu_mix_op &rep, const rsgpu_tune_options &o, SweepBuffer &buf, cudaStream_t s,
                  float *gbps, uint8_t *measured) {
  Codec &c = const_cast<rsgpu_codec *>(rep.codec)->c;
  const size_t total = c.k + c.m, len = rep.shard_len;
  const size_t stripe = total * ((len + 255) & ~size_t(255));
  const size_t target = o.target_bytes ? o.target_bytes : (256u << 20);
  const size_t n = std::min<size_t>(std::max<size_t>(1, target / stripe), 8192);
  int rc = buf.ensure(n * stripe);
  if (rc) return rc;
  std::vector<uint8_t *> ptrs(n * total);
  for (size_t i = 0; i < n; ++i)
    for (size_t j = 0; j < total; ++j) ptrs[i * total + j] = buf.d + i * stripe + j * ((len + 255) & ~size_t(255));
  std::vector<rsgpu_mix_op> ops(n, rep);
  for (size_t i = 0; i < n; ++i) ops[i].shards = &ptrs[i * total];
  rsgpu_mix_options mo;
  rsgpu_mix_options_default(&mo);
  mo.planner = RSGPU_PLANNER_FIXED;
  cudaEvent_t e0, e1;
  RS_CUDA(cudaEventCreate(&e0));
  RS_CUDA(cudaEventCreate(&e1));
  const int reps = o.repeats > 0 ? o.repeats : 3;
  for (const rsgpu_plan &p : candidates(c, rep.op, len)) {
    std::vector<rsgpu_plan> plans(n, p);
    MixPtr b;
    rc = mix_build(ops.data(), n, plans.data(), mo, b);
    if (rc) break;
    const double bytes = double(mix_info(*b).algorithmic_bytes);
    rc = mix_launch(*b, s);
    if (rc) break;
    float best = 1e30f;
    for (int r = 0; r < reps && rc == RSGPU_OK; ++r) {
      cudaEventRecord(e0, s);
      rc = mix_launch(*b, s);
      cudaEventRecord(e1, s);
      if (cudaEventSynchronize(e1) != cudaSuccess) rc = RSGPU_ERR_CUDA;
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      best = std::min(best, ms);
    }
    if (rc) break;
    const int j = plan_index(p);
    gbps[j] = bytes > 0 ? float(bytes / (double(best) * 1e-3) / 1e9) : 0.f;
    measured[j] = 1;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return rc;
}

}  // namespace

int tune(const rsgpu_mix_op *ops, size_t n_ops, const rsgpu_tune_options &o, size_t *tuned) {
  // One representative per class: the first op of the class in `ops`.
  std::map<TuneKey, size_t> reps;
  for (size_t i = 0; i < n_ops; ++i) {
    if (!ops[i].codec || !ops[i].shards) return RSGPU_ERR_INVALID_ARGUMENT;
    reps.emplace(key_of(ops[i]), i);
  }
  SweepBuffer buf;
  cudaStream_t s = nullptr;
  RS_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  size_t done = 0;
  int rc = RSGPU_OK;
  for (auto &kv : reps) {
    const rsgpu_mix_op &rep = ops[kv.second];
    TuneEntry e;
    rc = measure_class(rep, o, buf, s, e.gbps, e.measured);
    if (rc) break;
    int best = -1;
    for (int j = 0; j < P; ++j)
      if (e.measured[j] && (best < 0 || e.gbps[j] > e.gbps[best])) best = j;
    if (best < 0) continue;
    e.best = plan_of_index(best);
    plan_features(rep, e.features);
    Tuner &t = tuner();
    std::lock_guard<std::mutex> g(t.mu);
    t.table[kv.first] = e;
    for (int j = 0; j < P; ++j)
      if (e.measured[j]) {
        rsgpu_tune_sample smp{};
        std::memcpy(smp.features, e.features, sizeof(smp.features));
        smp.plan = plan_of_index(j);
        smp.gbps = e.gbps[j];
        t.samples.push_back(smp);
      }
    ++done;
  }
  cudaStreamDestroy(s);
  if (tuned) *tuned = done;
  return rc;
}

size_t tuner_samples(rsgpu_tune_sample *out, size_t cap) {
  Tuner &t = tuner();
  std::lock_guard<std::mutex> g(t.mu);
  if (out)
    for (size_t i = 0; i < std::min(cap, t.samples.size()); ++i) out[i] = t.samples[i];
  return t.samples.size();
}

size_t tuner_table_size() {
  Tuner &t = tuner();
  std::lock_guard<std::mutex> g(t.mu);
  return t.table.size();
}

void tuner_clear() {
  Tuner &t = tuner();
  std::lock_guard<std::mutex> g(t.mu);
  t.table.clear();
  t.samples.clear();
}

// Text format, one record per line:
//   T family op goal ebucket lbucket k m best_algo best_tile f0..f10 (g measured) x P
//   S f0..f10 algo tile gbps
int tuner_save(const char *path) {
  Tuner &t = tuner();
  std::lock_guard<std::mutex> g(t.mu);
  FILE *fp = std::fopen(path, "w");
  if (!fp) return RSGPU_ERR_INVALID_ARGUMENT;
  for (auto &kv : t.table) {
    const TuneKey &k = kv.first;
    const TuneEntry &e = kv.second;
    std::fprintf(fp, "T %u %u %u %u %u %u %u %d %d", k.family, k.op, k.goal, k.ebucket, k.lbucket, k.k, k.m,
                 e.best.algo, e.best.tile);
    for (int i = 0; i < F; ++i) std::fprintf(fp, " %.9g", e.features[i]);
    for (int j = 0; j < P; ++j) std::fprintf(fp, " %.9g %u", e.gbps[j], e.measured[j]);
    std::fprintf(fp, "\n");
  }
  for (auto &smp : t.samples) {
    std::fprintf(fp, "S");
    for (int i = 0; i < F; ++i) std::fprintf(fp, " %.9g", smp.features[i]);
    std::fprintf(fp, " %d %d %.9g\n", smp.plan.algo, smp.plan.tile, smp.gbps);
  }
  std::fclose(fp);
  return RSGPU_OK;
}

int tuner_load(const char *path) {
  FILE *fp = std::fopen(path, "r");
  if (!fp) return RSGPU_ERR_INVALID_ARGUMENT;
  std::map<TuneKey, TuneEntry> table;
  std::vector<rsgpu_tune_sample> samples;
  char tag[4];
  int rc = RSGPU_OK;
  while (std::fscanf(fp, "%3s", tag) == 1) {
    if (tag[0] == 'T') {
      unsigned v[7];
      TuneEntry e;
      if (std::fscanf(fp, "%u %u %u %u %u %u %u %d %d", &v[0], &v[1], &v[2], &v[3], &v[4], &v[5], &v[6],
                      &e.best.algo, &e.best.tile) != 9) {
        rc = RSGPU_ERR_INVALID_ARGUMENT;
        break;
      }
      for (int i = 0; i < F && rc == RSGPU_OK; ++i)
        if (std::fscanf(fp, "%f", &e.features[i]) != 1) rc = RSGPU_ERR_INVALID_ARGUMENT;
      for (int j = 0; j < P && rc == RSGPU_OK; ++j) {
        unsigned mflag = 0;
        if (std::fscanf(fp, "%f %u", &e.gbps[j], &mflag) != 2) rc = RSGPU_ERR_INVALID_ARGUMENT;
        e.measured[j] = uint8_t(mflag);
      }
      if (rc) break;
      TuneKey k{uint8_t(v[0]), uint8_t(v[1]), uint8_t(v[2]), uint8_t(v[3]), uint8_t(v[4]), uint16_t(v[5]),
                uint16_t(v[6])};
      table[k] = e;
    } else if (tag[0] == 'S') {
      rsgpu_tune_sample smp{};
      for (int i = 0; i < F && rc == RSGPU_OK; ++i)
        if (std::fscanf(fp, "%f", &smp.features[i]) != 1) rc = RSGPU_ERR_INVALID_ARGUMENT;
      if (rc == RSGPU_OK && std::fscanf(fp, "%d %d %f", &smp.plan.algo, &smp.plan.tile, &smp.gbps) != 3)
        rc = RSGPU_ERR_INVALID_ARGUMENT;
      if (rc) break;
      samples.push_back(smp);
    } else {
      rc = RSGPU_ERR_INVALID_ARGUMENT;
      break;
    }
  }
  std::fclose(fp);
  if (rc) return rc;
  Tuner &t = tuner();
  std::lock_guard<std::mutex> g(t.mu);
  t.table = std::move(table);
  t.samples = std::move(samples);
  return RSGPU_OK;
}

// Training rows from the samples: one row per distinct feature vector, the
// best measurement of each plan as its target (log2 GB/s), mask = measured.
int tuner_training_rows(std::vector<float> &x, std::vector<float> &y, std::vector<uint8_t> &mask) {
  std::vector<rsgpu_tune_sample> samples;
  {
    Tuner &t = tuner();
    std::lock_guard<std::mutex> g(t.mu);
    samples = t.samples;
  }
  std::map<std::vector<float>, size_t> row_of;
  x.clear();
  y.clear();
  mask.clear();
  for (const auto &smp : samples) {
    const int j = plan_index(smp.plan);
    if (j < 0 || !(smp.gbps > 0)) continue;
    std::vector<float> key(smp.features, smp.features + F);
    auto it = row_of.find(key);
    size_t r;
    if (it == row_of.end()) {
      r = row_of.size();
      row_of.emplace(key, r);
      x.insert(x.end(), key.begin(), key.end());
      y.insert(y.end(), P, 0.f);
      mask.insert(mask.end(), P, 0);
    } else {
      r = it->second;
    }
    const float v = std::log2(smp.gbps);
    if (!mask[r * P + j] || v > y[r * P + j]) y[r * P + j] = v;
    mask[r * P + j] = 1;
  }
  return row_of.empty() ? RSGPU_ERR_INVALID_ARGUMENT : RSGPU_OK;
}

}  // namespace rsgpu

// ====================================================================== C ABI
extern "C" {

int32_t rsgpu_plan_features(const rsgpu_mix_op *op, float *out) {
  if (!op || !out) return RSGPU_ERR_INVALID_ARGUMENT;
  return rsgpu::plan_features(*op, out);
}

int32_t rsgpu_plan_index(rsgpu_plan plan) { return rsgpu::plan_index(plan); }

int32_t rsgpu_tune(const rsgpu_mix_op *ops, size_t n_ops, const rsgpu_tune_options *opts, size_t *classes_tuned) {
  if (!ops && n_ops) return RSGPU_ERR_INVALID_ARGUMENT;
  rsgpu_tune_options o{};
  if (opts) o = *opts;
  return rsgpu::tune(ops, n_ops, o, classes_tuned);
}

size_t rsgpu_tuner_samples(rsgpu_tune_sample *out, size_t cap) { return rsgpu::tuner_samples(out, cap); }
size_t rsgpu_tuner_table_size(void) { return rsgpu::tuner_table_size(); }

int32_t rsgpu_tuner_lookup(const rsgpu_mix_op *op, rsgpu_plan *out) {
  if (!op || !op->codec || !out) return RSGPU_ERR_INVALID_ARGUMENT;
  return rsgpu::table_lookup(*op, out) ? RSGPU_OK : RSGPU_ERR_INVALID_INDEX;
}

int32_t rsgpu_tuner_save(const char *path) { return path ? rsgpu::tuner_save(path) : RSGPU_ERR_INVALID_ARGUMENT; }
int32_t rsgpu_tuner_load(const char *path) { return path ? rsgpu::tuner_load(path) : RSGPU_ERR_INVALID_ARGUMENT; }
void rsgpu_tuner_clear(void) { rsgpu::tuner_clear(); }

size_t rsgpu_model_param_count(void) { return rsgpu::model_param_count(); }
int32_t rsgpu_model_get_params(float *out, size_t n) {
  return out ? rsgpu::model_get(out, n) : RSGPU_ERR_INVALID_ARGUMENT;
}
int32_t rsgpu_model_set_params(const float *in, size_t n) {
  return in ? rsgpu::model_set(in, n) : RSGPU_ERR_INVALID_ARGUMENT;
}

int32_t rsgpu_model_train(const float *features, const float *targets, const uint8_t *mask, size_t n,
                          const rsgpu_train_options *opts, float *final_loss) {
  if (!features || !targets || !mask) return RSGPU_ERR_INVALID_ARGUMENT;
  rsgpu_train_options o{};
  if (opts) o = *opts;
  return rsgpu::model_train(features, targets, mask, n, o, final_loss);
}

int32_t rsgpu_model_train_from_tuner(const rsgpu_train_options *opts, float *final_loss) {
  std::vector<float> x, y;
  std::vector<uint8_t> mask;
  int rc = rsgpu::tuner_training_rows(x, y, mask);
  if (rc) return rc;
  rsgpu_train_options o{};
  if (opts) o = *opts;
  return rsgpu::model_train(x.data(), y.data(), mask.data(), x.size() / RSGPU_MODEL_FEATURES, o, final_loss);
}

int32_t rsgpu_model_predict(const float *features, size_t n, float *out) {
  if ((!features || !out) && n) return RSGPU_ERR_INVALID_ARGUMENT;
  return rsgpu::model_predict(features, n, out);
}

int32_t rsgpu_model_gradients(const float *params, const float *features, const float *targets, const uint8_t *mask,
                              size_t n, float *loss, float *grads) {
  if (!params || !features || !targets || !mask || !loss || !grads) return RSGPU_ERR_INVALID_ARGUMENT;
  return rsgpu::model_gradients(params, features, targets, mask, n, loss, grads);
}

int32_t rsgpu_model_ready(void) { return rsgpu::model_ready() ? 1 : 0; }

}  // extern "C"
