// model.cu -- the learned cost model of the mixed-batch planner.
//
// A small MLP predicts, from the features of one operation (family, k, m,
// shard length, operation, erasure count and spread), the log2 throughput of
// every plan; the planner takes the best valid one.  Training data are the
// autotuner's own measurements.  Forward pass, backward pass and the Adam
// update are the kernels below; the host only sequences them.
//
//   x (F) -> W1, b1 -> ReLU (H) -> W2, b2 -> ReLU (H) -> W3, b3 -> y (P)
//   loss = mean over measured (mask) entries of (y - target)^2
//
// Gradients are accumulated in a fixed order (one thread per parameter,
// looping over the samples), so a training run is deterministic.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "batch.hpp"
#include "codec.hpp"
#include "model.hpp"

namespace rsgpu {

#define RS_CUDA(expr)                              \
  do {                                             \
    cudaError_t e_ = (expr);                       \
    if (e_ != cudaSuccess) return cuda_status(e_); \
  } while (0)

namespace {

constexpr int F = RSGPU_MODEL_FEATURES;
constexpr int H = RSGPU_MODEL_HIDDEN;
constexpr int P = RSGPU_MODEL_PLANS;
constexpr int oW1 = 0, oB1 = oW1 + F * H, oW2 = oB1 + H, oB2 = oW2 + H * H, oW3 = oB2 + H, oB3 = oW3 + H * P;
constexpr int kParams = oB3 + P;
static_assert(H == 32, "one warp per sample");

// Per-sample forward (and, with targets, backward to the pre-activations).
// One warp per sample; lane h owns hidden unit h.  Writes the activations
// a1, a2 and the error signals dz1, dz2, dy for the weight-gradient kernel,
// and the sample's summed squared error.
__global__ void __launch_bounds__(32) k_mlp_sample(const float *__restrict__ w, const float *__restrict__ x,
                                                   const float *__restrict__ t, const uint8_t *__restrict__ mask,
                                                   float inv_count, int n, float *__restrict__ y_out,
                                                   float *__restrict__ a1_out, float *__restrict__ a2_out,
                                                   float *__restrict__ dz1_out, float *__restrict__ dz2_out,
                                                   float *__restrict__ dy_out, float *__restrict__ sq_out) {
  const int s = blockIdx.x;
  const int h = threadIdx.x;
  if (s >= n) return;
  __shared__ float a1[H], a2[H], dy[P], dz2[H];
  const float *xs = x + size_t(s) * F;
  float z1 = w[oB1 + h];
  for (int f = 0; f < F; ++f) z1 += xs[f] * w[oW1 + f * H + h];
  a1[h] = z1 > 0.f ? z1 : 0.f;
  __syncwarp();
  float z2 = w[oB2 + h];
  for (int j = 0; j < H; ++j) z2 += a1[j] * w[oW2 + j * H + h];
  a2[h] = z2 > 0.f ? z2 : 0.f;
  __syncwarp();
  float sq = 0.f;
  if (h < P) {
    float y = w[oB3 + h];
    for (int j = 0; j < H; ++j) y += a2[j] * w[oW3 + j * P + h];
    if (y_out) y_out[size_t(s) * P + h] = y;
    float d = 0.f;
    if (t && mask[size_t(s) * P + h]) {
      const float e = y - t[size_t(s) * P + h];
      sq = e * e;
      d = 2.f * e * inv_count;
    }
    dy[h] = d;
  }
  __syncwarp();
  if (!t) return;
  // Sum of squared errors of this sample (lanes >= P contribute 0).
  for (int off = 16; off; off >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, off);
  if (h == 0) sq_out[s] = sq;
  float da2 = 0.f;
  for (int o = 0; o < P; ++o) da2 += w[oW3 + h * P + o] * dy[o];
  const float d2 = z2 > 0.f ? da2 : 0.f;
  dz2[h] = d2;
  __syncwarp();
  float da1 = 0.f;
  for (int j = 0; j < H; ++j) da1 += w[oW2 + h * H + j] * dz2[j];
  const float d1 = z1 > 0.f ? da1 : 0.f;
  a1_out[size_t(s) * H + h] = a1[h];
  a2_out[size_t(s) * H + h] = a2[h];
  dz1_out[size_t(s) * H + h] = d1;
  dz2_out[size_t(s) * H + h] = d2;
  if (h < P) dy_out[size_t(s) * P + h] = dy[h];
}

// Weight gradients: one thread per parameter, samples summed in order.
__global__ void k_mlp_wgrad(const float *__restrict__ x, const float *__restrict__ a1, const float *__restrict__ a2,
                            const float *__restrict__ dz1, const float *__restrict__ dz2,
                            const float *__restrict__ dy, int n, float *__restrict__ g) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kParams) return;
  float acc = 0.f;
  if (i < oB1) {
    const int f = i / H, hh = i % H;
    for (int s = 0; s < n; ++s) acc += x[size_t(s) * F + f] * dz1[size_t(s) * H + hh];
  } else if (i < oW2) {
    const int hh = i - oB1;
    for (int s = 0; s < n; ++s) acc += dz1[size_t(s) * H + hh];
  } else if (i < oB2) {
    const int j = (i - oW2) / H, hh = (i - oW2) % H;
    for (int s = 0; s < n; ++s) acc += a1[size_t(s) * H + j] * dz2[size_t(s) * H + hh];
  } else if (i < oW3) {
    const int hh = i - oB2;
    for (int s = 0; s < n; ++s) acc += dz2[size_t(s) * H + hh];
  } else if (i < oB3) {
    const int j = (i - oW3) / P, o = (i - oW3) % P;
    for (int s = 0; s < n; ++s) acc += a2[size_t(s) * H + j] * dy[size_t(s) * P + o];
  } else {
    const int o = i - oB3;
    for (int s = 0; s < n; ++s) acc += dy[size_t(s) * P + o];
  }
  g[i] = acc;
}

// Loss = sum of the per-sample squared errors * inv_count, summed in order
// by one warp.
__global__ void k_mlp_loss(const float *__restrict__ sq, int n, float inv_count, float *__restrict__ loss) {
  float acc = 0.f;
  for (int s = threadIdx.x; s < n; s += 32) acc += sq[s];
  for (int off = 16; off; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
  if (threadIdx.x == 0) *loss = acc * inv_count;
}

// Adam (Kingma & Ba, 2015), bias-corrected.
__global__ void k_adam(float *__restrict__ w, const float *__restrict__ g, float *__restrict__ m,
                       float *__restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kParams) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// Device buffers of one training / evaluation run.
struct Run {
  float *w = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
  float *x = nullptr, *t = nullptr, *y = nullptr;
  uint8_t *mask = nullptr;
  float *a1 = nullptr, *a2 = nullptr, *dz1 = nullptr, *dz2 = nullptr, *dy = nullptr, *sq = nullptr, *loss = nullptr;
  ~Run() {
    for (void *p : {(void *)w, (void *)g, (void *)m, (void *)v, (void *)x, (void *)t, (void *)y, (void *)mask,
                    (void *)a1, (void *)a2, (void *)dz1, (void *)dz2, (void *)dy, (void *)sq, (void *)loss})
      if (p) cudaFree(p);
  }
  int alloc(size_t n, bool train) {
    const size_t rows = n ? n : 1;
    RS_CUDA(cudaMalloc(&w, kParams * 4));
    RS_CUDA(cudaMalloc(&x, rows * F * 4));
    RS_CUDA(cudaMalloc(&y, rows * P * 4));
    if (train) {
      RS_CUDA(cudaMalloc(&g, kParams * 4));
      RS_CUDA(cudaMalloc(&m, kParams * 4));
      RS_CUDA(cudaMalloc(&v, kParams * 4));
      RS_CUDA(cudaMemset(m, 0, kParams * 4));
      RS_CUDA(cudaMemset(v, 0, kParams * 4));
      RS_CUDA(cudaMalloc(&t, rows * P * 4));
      RS_CUDA(cudaMalloc(&mask, rows * P));
      RS_CUDA(cudaMalloc(&a1, rows * H * 4));
      RS_CUDA(cudaMalloc(&a2, rows * H * 4));
      RS_CUDA(cudaMalloc(&dz1, rows * H * 4));
      RS_CUDA(cudaMalloc(&dz2, rows * H * 4));
      RS_CUDA(cudaMalloc(&dy, rows * P * 4));
      RS_CUDA(cudaMalloc(&sq, rows * 4));
      RS_CUDA(cudaMalloc(&loss, 4));
    }
    return RSGPU_OK;
  }
  // Forward + backward + weight gradients + loss, queued on the legacy stream.
  void grad_step(int n, float inv_count) {
    k_mlp_sample<<<n, 32>>>(w, x, t, mask, inv_count, n, y, a1, a2, dz1, dz2, dy, sq);
    k_mlp_wgrad<<<(kParams + 127) / 128, 128>>>(x, a1, a2, dz1, dz2, dy, n, g);
    k_mlp_loss<<<1, 32>>>(sq, n, inv_count, loss);
    launch_counter_add(3);
  }
};

struct ModelState {
  std::mutex mu;
  bool ready = false;
  std::vector<float> params;
  // Inference context: the weights stay on the device and inputs / outputs
  // go through pinned buffers on a private stream, so a planner call costs
  // one small kernel and waits only for that stream.
  int device = -1;
  cudaStream_t stream = nullptr;
  float *d_w = nullptr, *d_x = nullptr, *d_y = nullptr;
  float *h_x = nullptr, *h_y = nullptr;
  size_t cap = 0;
  bool w_dirty = true;
  // Predictions of this weight set by feature vector: a request stream
  // repeats a few operation shapes, and a planner call whose shapes were all
  // seen before launches nothing (its wait would queue behind whatever else
  // occupies the device).  Cleared when the weights change.
  std::unordered_map<std::string, std::vector<float>> memo;
  uint64_t version = 0;  // counts weight changes
};
ModelState &state() {
  static ModelState s;
  return s;
}

// Seeded uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)) weights, zero biases
// (splitmix64 stream).
std::vector<float> init_params(uint64_t seed) {
  std::vector<float> p(kParams, 0.f);
  uint64_t st = seed ? seed : 0x9E3779B97F4A7C15ull;
  auto next = [&]() {
    uint64_t z = (st += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return double(z >> 11) / double(1ull << 53);
  };
  auto fill = [&](int off, int count, int fan_in) {
    const double r = 1.0 / std::sqrt(double(fan_in));
    for (int i = 0; i < count; ++i) p[off + i] = float((2.0 * next() - 1.0) * r);
  };
  fill(oW1, F * H, F);
  fill(oW2, H * H, H);
  fill(oW3, H * P, H);
  return p;
}

}  // namespace

size_t model_param_count() { return kParams; }

bool model_ready() {
  std::lock_guard<std::mutex> g(state().mu);
  return state().ready;
}

int model_get(float *out, size_t n) {
  std::lock_guard<std::mutex> g(state().mu);
  if (!state().ready || n < size_t(kParams)) return RSGPU_ERR_INVALID_ARGUMENT;
  std::memcpy(out, state().params.data(), kParams * 4);
  return RSGPU_OK;
}

int model_set(const float *in, size_t n) {
  if (n != size_t(kParams)) return RSGPU_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> g(state().mu);
  state().params.assign(in, in + kParams);
  state().ready = true;
  state().w_dirty = true;
  state().memo.clear();
  ++state().version;
  return RSGPU_OK;
}

uint64_t model_version() {
  std::lock_guard<std::mutex> g(state().mu);
  return state().version;
}

int model_predict(const float *features, size_t n, float *out, bool memoize, uint64_t *version) {
  ModelState &m = state();
  std::lock_guard<std::mutex> g(m.mu);
  if (!m.ready) return RSGPU_ERR_INVALID_ARGUMENT;
  if (version) *version = m.version;
  if (n == 0) return RSGPU_OK;
  // Rows seen before come from the memo; the rest go to the device.
  std::vector<size_t> miss;
  for (size_t i = 0; i < n; ++i) {
    if (!memoize) {
      miss.push_back(i);
      continue;
    }
    auto it = m.memo.find(std::string(reinterpret_cast<const char *>(features + i * F), F * 4));
    if (it == m.memo.end())
      miss.push_back(i);
    else
      std::memcpy(out + i * P, it->second.data(), P * 4);
  }
  if (miss.empty()) return RSGPU_OK;
  const float *all = features;
  float *all_out = out;
  n = miss.size();
  int dev = 0;
  RS_CUDA(cudaGetDevice(&dev));
  if (m.device != dev) {  // first use (or a new device): fresh context
    m.device = dev;
    m.cap = 0;
    m.w_dirty = true;
    RS_CUDA(cudaStreamCreateWithFlags(&m.stream, cudaStreamNonBlocking));
    RS_CUDA(cudaMalloc(&m.d_w, kParams * 4));
  }
  if (n > m.cap) {
    const size_t cap = std::max<size_t>(n, 1024);
    if (m.d_x) cudaFree(m.d_x);
    if (m.d_y) cudaFree(m.d_y);
    if (m.h_x) cudaFreeHost(m.h_x);
    if (m.h_y) cudaFreeHost(m.h_y);
    RS_CUDA(cudaMalloc(&m.d_x, cap * F * 4));
    RS_CUDA(cudaMalloc(&m.d_y, cap * P * 4));
    RS_CUDA(cudaMallocHost(&m.h_x, cap * F * 4));
    RS_CUDA(cudaMallocHost(&m.h_y, cap * P * 4));
    m.cap = cap;
  }
  if (m.w_dirty) {
    RS_CUDA(cudaMemcpyAsync(m.d_w, m.params.data(), kParams * 4, cudaMemcpyHostToDevice, m.stream));
    RS_CUDA(cudaStreamSynchronize(m.stream));
    m.w_dirty = false;
  }
  for (size_t x = 0; x < n; ++x) std::memcpy(m.h_x + x * F, all + miss[x] * F, F * 4);
  RS_CUDA(cudaMemcpyAsync(m.d_x, m.h_x, n * F * 4, cudaMemcpyHostToDevice, m.stream));
  k_mlp_sample<<<int(n), 32, 0, m.stream>>>(m.d_w, m.d_x, nullptr, nullptr, 0.f, int(n), m.d_y, nullptr, nullptr,
                                            nullptr, nullptr, nullptr, nullptr);
  launch_counter_add(1);
  RS_CUDA(cudaGetLastError());
  RS_CUDA(cudaMemcpyAsync(m.h_y, m.d_y, n * P * 4, cudaMemcpyDeviceToHost, m.stream));
  RS_CUDA(cudaStreamSynchronize(m.stream));
  if (memoize && m.memo.size() + n > 65536) m.memo.clear();
  for (size_t x = 0; x < n; ++x) {
    std::memcpy(all_out + miss[x] * P, m.h_y + x * P, P * 4);
    if (memoize)
      m.memo.emplace(std::string(reinterpret_cast<const char *>(all + miss[x] * F), F * 4),
                     std::vector<float>(m.h_y + x * P, m.h_y + (x + 1) * P));
  }
  return RSGPU_OK;
}

namespace {
int upload_data(Run &r, const float *features, const float *targets, const uint8_t *mask, size_t n,
                float *inv_count) {
  size_t cnt = 0;
  for (size_t i = 0; i < n * P; ++i) cnt += mask[i] ? 1 : 0;
  if (cnt == 0) return RSGPU_ERR_INVALID_ARGUMENT;
  *inv_count = float(1.0 / double(cnt));
  RS_CUDA(cudaMemcpy(r.x, features, n * F * 4, cudaMemcpyHostToDevice));
  RS_CUDA(cudaMemcpy(r.t, targets, n * P * 4, cudaMemcpyHostToDevice));
  RS_CUDA(cudaMemcpy(r.mask, mask, n * P, cudaMemcpyHostToDevice));
  return RSGPU_OK;
}
}  // namespace

int model_gradients(const float *params, const float *features, const float *targets, const uint8_t *mask, size_t n,
                    float *loss, float *grads) {
  if (n == 0 || n > (1u << 30)) return RSGPU_ERR_INVALID_ARGUMENT;
  Run r;
  int rc = r.alloc(n, true);
  if (rc) return rc;
  float inv = 0.f;
  rc = upload_data(r, features, targets, mask, n, &inv);
  if (rc) return rc;
  RS_CUDA(cudaMemcpy(r.w, params, kParams * 4, cudaMemcpyHostToDevice));
  r.grad_step(int(n), inv);
  RS_CUDA(cudaGetLastError());
  RS_CUDA(cudaMemcpy(grads, r.g, kParams * 4, cudaMemcpyDeviceToHost));
  RS_CUDA(cudaMemcpy(loss, r.loss, 4, cudaMemcpyDeviceToHost));
  return RSGPU_OK;
}

int model_train(const float *features, const float *targets, const uint8_t *mask, size_t n,
                const rsgpu_train_options &o, float *final_loss) {
  if (n == 0 || n > (1u << 30)) return RSGPU_ERR_INVALID_ARGUMENT;
  const int epochs = o.epochs > 0 ? o.epochs : 2000;
  const float lr = o.lr > 0 ? o.lr : 3e-3f;
  Run r;
  int rc = r.alloc(n, true);
  if (rc) return rc;
  float inv = 0.f;
  rc = upload_data(r, features, targets, mask, n, &inv);
  if (rc) return rc;
  std::vector<float> w = init_params(o.seed);
  RS_CUDA(cudaMemcpy(r.w, w.data(), kParams * 4, cudaMemcpyHostToDevice));
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  double c1 = 1.0, c2 = 1.0;
  for (int e = 0; e < epochs; ++e) {
    r.grad_step(int(n), inv);
    c1 *= b1;
    c2 *= b2;
    k_adam<<<(kParams + 127) / 128, 128>>>(r.w, r.g, r.m, r.v, lr, b1, b2, eps, float(1.0 - c1), float(1.0 - c2));
    launch_counter_add(1);
  }
  // Loss of the final weights.
  r.grad_step(int(n), inv);
  RS_CUDA(cudaGetLastError());
  RS_CUDA(cudaMemcpy(w.data(), r.w, kParams * 4, cudaMemcpyDeviceToHost));
  float loss = 0.f;
  RS_CUDA(cudaMemcpy(&loss, r.loss, 4, cudaMemcpyDeviceToHost));
  if (final_loss) *final_loss = loss;
  return model_set(w.data(), w.size());
}

}  // namespace rsgpu
