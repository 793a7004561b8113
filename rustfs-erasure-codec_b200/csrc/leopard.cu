// leopard.cu -- Leopard FFT codecs over GF(2^8) and GF(2^16) on sm_100a.
//
// Every column of a shard is independent, so a CTA owns a tile of columns of
// one stripe and holds *all* transform lanes of that tile in shared memory:
// shards cross HBM exactly once (data in, parity or recovered shards out) and
// every IFFT / formal-derivative / FFT layer runs on chip.  A lane row is one
// 64-byte block (64 GF(2^8) columns, or 32 GF(2^16) columns in the
// reference's split byte layout, src/core/leopard_gf16/ops.rs:513-807) and is
// owned by one half-warp: 16 lanes x one 32-bit word.  Multiplication by a
// butterfly constant g^log_m uses nibble tables held one entry per lane and
// read with width-16 warp shuffles, so the two halves of a warp can work on
// different butterflies with different constants.
//
// Kernels:
//  K4/K6 k_leo_encode  grouped IFFT -> XOR-accumulate -> FFT
//                      (src/core/leopard_gf8/encode.rs:194-372,
//                       src/core/leopard_gf16/encode.rs:109-252)
//  K5/K7 k_leo_decode  err-locator scaling -> IFFT -> formal derivative ->
//                      FFT -> inverse scaling
//                      (src/core/leopard_gf8/decode.rs:291-420,
//                       src/core/leopard_gf16/decode.rs:704-910)
//  K7a   k_leo_locator FWHT error locator, one CTA per erasure pattern
//                      (src/core/leopard_gf16/decode.rs:177-216,
//                       src/core/leopard_gf8/decode.rs:58-113)
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <list>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "codec.hpp"
#include "leo_fft.cuh"
#include "leo_tile.cuh"
#include "launch_cfg.hpp"
#include "leopard.hpp"

namespace rsgpu {

#define RS_CUDA(expr)                              \
  do {                                             \
    cudaError_t e_ = (expr);                       \
    if (e_ != cudaSuccess) return cuda_status(e_); \
  } while (0)

// ====================================================================== tables
namespace {

size_t pow2_at_least(size_t n) {
  size_t p = 1;
  while (p < n) p <<= 1;
  return p;
}

// Leopard field tables (src/core/leopard_gf8/tables.rs:8-145,
// src/core/leopard_gf16/tables.rs:8-116): exp by LFSR over the field
// polynomial, log through the Cantor basis, the FFT skew factors and the
// Walsh transform of the log table.
struct LeoTables {
  int bits = 0;
  uint32_t order = 0, mod = 0;
  std::vector<uint16_t> log, exp, skew, walsh;

  uint16_t add_mod(uint32_t a, uint32_t b) const {
    const uint32_t s = a + b;
    return uint16_t((s + (s >> bits)) & (order - 1));
  }
  uint16_t sub_mod(uint32_t a, uint32_t b) const {
    const uint64_t d = uint64_t(a) - uint64_t(b);
    return uint16_t((d + (d >> bits)) & (order - 1));
  }
  uint16_t mul_log(uint16_t a, uint16_t log_b) const {
    return a == 0 ? 0 : exp[add_mod(log[a], log_b)];
  }

  void fwht(std::vector<uint16_t> &d, size_t mtrunc) const {
    for (size_t dist = 1, dist4 = 4; dist4 <= order; dist = dist4, dist4 <<= 2)
      for (size_t r = 0; r < mtrunc; r += dist4)
        for (size_t off = r; off < r + dist; ++off) {
          uint16_t *p = d.data();
          uint16_t t0 = add_mod(p[off], p[off + dist]), t1 = sub_mod(p[off], p[off + dist]);
          uint16_t t2 = add_mod(p[off + 2 * dist], p[off + 3 * dist]);
          uint16_t t3 = sub_mod(p[off + 2 * dist], p[off + 3 * dist]);
          p[off] = add_mod(t0, t2);
          p[off + 2 * dist] = sub_mod(t0, t2);
          p[off + dist] = add_mod(t1, t3);
          p[off + 3 * dist] = sub_mod(t1, t3);
        }
  }

  explicit LeoTables(int b) : bits(b), order(1u << b), mod((1u << b) - 1) {
    static const uint16_t cantor8[8] = {1, 214, 152, 146, 86, 200, 88, 230};
    static const uint16_t cantor16[16] = {0x0001, 0xACCA, 0x3C0E, 0x163E, 0xC582, 0xED2E, 0x914C, 0x4012,
                                          0x6C98, 0x10D8, 0x6A72, 0xB900, 0xFDB8, 0xFB34, 0xFF38, 0x991E};
    const uint16_t *cantor = b == 8 ? cantor8 : cantor16;
    const uint32_t poly = b == 8 ? 0x11D : 0x1002D;
    log.assign(order, 0);
    exp.assign(b == 8 ? order : 2 * order, 0);
    uint32_t state = 1;
    for (uint32_t i = 0; i < mod; ++i) {
      exp[state] = uint16_t(i);
      state <<= 1;
      if (state >= order) state ^= poly;
    }
    exp[0] = uint16_t(mod);
    log[0] = 0;
    for (int i = 0; i < b; ++i) {
      const uint32_t width = 1u << i;
      for (uint32_t j = 0; j < width; ++j) log[j + width] = log[j] ^ cantor[i];
    }
    for (uint32_t i = 0; i < order; ++i) log[i] = exp[log[i]];
    for (uint32_t i = 0; i < order; ++i) exp[log[i]] = uint16_t(i);
    exp[mod] = exp[0];

    skew.assign(mod, 0);
    std::vector<uint16_t> temp(b - 1);
    for (int i = 1; i < b; ++i) temp[i - 1] = uint16_t(1u << i);
    for (int mm = 0; mm < b - 1; ++mm) {
      const size_t step = size_t(1) << (mm + 1);
      skew[(size_t(1) << mm) - 1] = 0;
      for (int i = mm; i < b - 1; ++i) {
        const size_t s = size_t(1) << (i + 1);
        for (size_t j = (size_t(1) << mm) - 1; j < s; j += step) skew[j + s] = skew[j] ^ temp[i];
      }
      const uint16_t prod = mul_log(temp[mm], log[temp[mm] ^ 1]);
      temp[mm] = uint16_t(mod - log[prod]);
      for (int i = mm + 1; i < b - 1; ++i) temp[i] = mul_log(temp[i], add_mod(log[temp[i] ^ 1], temp[mm]));
    }
    for (uint32_t i = 0; i < mod; ++i) skew[i] = log[skew[i]];
    walsh.assign(order, 0);
    for (uint32_t i = 0; i < order; ++i) walsh[i] = log[i];
    walsh[0] = 0;
    fwht(walsh, order);
  }
};

}  // namespace

// Device-resident constants of one Leopard field, shared by every codec.
struct LeoField {
  int bits;
  LeoTables host;
  uint16_t *d_skew = nullptr;
  uint16_t *d_walsh = nullptr;
  uint32_t *d_bank = nullptr;   // multiplier tables indexed by log value (half-warp layer kernels)
  uint32_t *d_kbank = nullptr;  // tables of the register-stage kernels (GF(2^8): 5+3 split; GF(2^16): 5+5+5+1)
  uint32_t *d_sktab = nullptr;  // d_kbank's entry of each skew entry: entry i holds the tables of log skew[i]
  uint8_t *d_mul8 = nullptr;    // GF(2^8): products mul[a][b], 256 x 256 (device packing of dense maps)
  explicit LeoField(int b) : bits(b), host(b) {}
};

static int leo_field(int bits, LeoField **out) {
  static std::mutex mu;
  static LeoField *fields[2] = {nullptr, nullptr};
  std::lock_guard<std::mutex> g(mu);
  const int slot = bits == 8 ? 0 : 1;
  if (!fields[slot]) {
    LeoField *f = new LeoField(bits);
    const LeoTables &t = f->host;
    // The transforms test for a skipped multiply (a skew entry whose log is
    // the modulus) only in groups that can meet one, on the property that
    // those entries are exactly 2^i - 1.
    for (uint32_t i = 0; i < t.mod; ++i)
      if ((t.skew[i] == t.mod) != (((i + 1) & i) == 0)) {
        delete f;
        return RSGPU_ERR_CUDA;
      }
    RS_CUDA(cudaMalloc(&f->d_skew, t.skew.size() * 2));
    RS_CUDA(cudaMemcpy(f->d_skew, t.skew.data(), t.skew.size() * 2, cudaMemcpyHostToDevice));
    RS_CUDA(cudaMalloc(&f->d_walsh, t.walsh.size() * 2));
    RS_CUDA(cudaMemcpy(f->d_walsh, t.walsh.data(), t.walsh.size() * 2, cudaMemcpyHostToDevice));
    // Bank: for each log value, 16 lanes x (GF8: 2 words, GF16: 4 words).
    // GF8 word pair: c*n and c*(n<<4) replicated into all four bytes.
    // GF16 words k=0..3: c*(n << 4k) replicated into both 16-bit halves.
    const uint32_t words = bits == 8 ? 2 : 4;
    std::vector<uint32_t> bank(size_t(t.order) * 16 * words);
    for (uint32_t lm = 0; lm < t.order; ++lm)
      for (uint32_t n = 0; n < 16; ++n) {
        uint32_t *e = &bank[(size_t(lm) * 16 + n) * words];
        if (bits == 8) {
          e[0] = uint32_t(t.mul_log(uint16_t(n), uint16_t(lm))) * 0x01010101u;
          e[1] = uint32_t(t.mul_log(uint16_t(n << 4), uint16_t(lm))) * 0x01010101u;
        } else {
          for (uint32_t k = 0; k < 4; ++k) e[k] = uint32_t(t.mul_log(uint16_t(n << (4 * k)), uint16_t(lm))) * 0x10001u;
        }
      }
    RS_CUDA(cudaMalloc(&f->d_bank, bank.size() * 4));
    RS_CUDA(cudaMemcpy(f->d_bank, bank.data(), bank.size() * 4, cudaMemcpyHostToDevice));
    if (bits == 8) {
      // Per log value: c * i (i < 32) replicated into four bytes, then the
      // eight bytes c * (h << 5) packed into two words (layout of leo_fft.cuh).
      std::vector<uint32_t> kb(size_t(t.order) * kWBank8, 0);
      for (uint32_t lm = 0; lm < t.order; ++lm) {
        uint32_t *e = &kb[size_t(lm) * kWBank8];
        for (uint32_t i = 0; i < 32; ++i) e[i] = uint32_t(t.mul_log(uint16_t(i), uint16_t(lm))) * 0x01010101u;
        for (uint32_t h = 0; h < 8; ++h) e[32 + (h >> 2)] |= uint32_t(t.mul_log(uint16_t(h << 5), uint16_t(lm))) << (8 * (h & 3));
      }
      RS_CUDA(cudaMalloc(&f->d_kbank, kb.size() * 4));
      RS_CUDA(cudaMemcpy(f->d_kbank, kb.data(), kb.size() * 4, cudaMemcpyHostToDevice));
      std::vector<uint32_t> sk(size_t(t.mod) * kWBank8);
      for (uint32_t i = 0; i < t.mod; ++i)
        std::memcpy(&sk[size_t(i) * kWBank8], &kb[size_t(t.skew[i]) * kWBank8], kWBank8 * 4);
      RS_CUDA(cudaMalloc(&f->d_sktab, sk.size() * 4));
      RS_CUDA(cudaMemcpy(f->d_sktab, sk.data(), sk.size() * 4, cudaMemcpyHostToDevice));
      std::vector<uint8_t> mul(256 * 256, 0);
      for (uint32_t a = 1; a < 256; ++a)
        for (uint32_t b = 1; b < 256; ++b) mul[a * 256 + b] = uint8_t(t.exp[t.add_mod(t.log[a], t.log[b])]);
      RS_CUDA(cudaMalloc(&f->d_mul8, mul.size()));
      RS_CUDA(cudaMemcpy(f->d_mul8, mul.data(), mul.size(), cudaMemcpyHostToDevice));
    } else {
      // Per log value, 32 lanes x 4 words (layout of leo_fft.cuh): c * i,
      // c * (i << 5), c * (i << 10) for i = lane, and c * 2^15, each
      // replicated into both 16-bit halves.
      const size_t w = 32 * 4;
      std::vector<uint32_t> kb(size_t(t.order) * w);
      for (uint32_t lm = 0; lm < t.order; ++lm)
        for (uint32_t i = 0; i < 32; ++i) {
          uint32_t *e = &kb[size_t(lm) * w + i * 4];
          for (uint32_t q = 0; q < 3; ++q) e[q] = uint32_t(t.mul_log(uint16_t(i << (5 * q)), uint16_t(lm))) * 0x10001u;
          e[3] = uint32_t(t.mul_log(uint16_t(0x8000), uint16_t(lm))) * 0x10001u;
        }
      RS_CUDA(cudaMalloc(&f->d_kbank, kb.size() * 4));
      RS_CUDA(cudaMemcpy(f->d_kbank, kb.data(), kb.size() * 4, cudaMemcpyHostToDevice));
      std::vector<uint32_t> sk(size_t(t.mod) * w);
      for (uint32_t i = 0; i < t.mod; ++i) std::memcpy(&sk[size_t(i) * w], &kb[size_t(t.skew[i]) * w], w * 4);
      RS_CUDA(cudaMalloc(&f->d_sktab, sk.size() * 4));
      RS_CUDA(cudaMemcpy(f->d_sktab, sk.data(), sk.size() * 4, cudaMemcpyHostToDevice));
    }
    fields[slot] = f;
  }
  *out = fields[slot];
  return RSGPU_OK;
}

// ====================================================================== device
namespace {

constexpr int kLeoThreads = 512;

template <int BITS, bool VERIFY, bool GLOBAL_WORK>
__global__ void __launch_bounds__(kLeoThreads) k_leo_encode(LeoArgs a) {
  extern __shared__ uint32_t smem[];
  uint32_t *W = GLOBAL_WORK ? a.scratch + size_t(blockIdx.x) * a.lanes * a.nb * kRowWords : smem;
  const uint64_t tile_bytes = uint64_t(a.nb) * 64;
  const uint32_t tiles_per_job = uint32_t((a.len + tile_bytes - 1) / tile_bytes);
  const uint32_t total = tiles_per_job * a.n_jobs;
  __shared__ uint32_t bad;
  for (uint32_t t = blockIdx.x; t < total; t += gridDim.x) {
    const uint32_t job = t / tiles_per_job;
    const uint64_t col0 = uint64_t(t - job * tiles_per_job) * tile_bytes;
    const LeoJob jd = a.jobs[job];
    leo_encode_tile<BITS, VERIFY, kLeoThreads>(W, a, jd, col0, a.len, &bad);
  }
}

constexpr int kFftThreads = 256;
// Tiles whose shared memory allows one CTA per SM run one "wide" CTA of
// kWideThreads threads per SM; transforms whose work rows live in global
// memory run kGlobalBlocks CTAs of kWideThreads per SM.  Registers per thread:
// 65536 / (threads per SM).  The transforms are latency-bound (long-scoreboard
// waits on the constant tables and work rows dominate their stalls), so warps
// count for more than registers: at 1024 threads (64 registers, a few hundred
// bytes of spills) the config-3 GF(2^16) 1024+512 encode runs in 3.26 ms and
// the decode in 12.16 ms, against 4.48 and 16.83 ms at 512 threads (128
// registers); 2048+1024 at 8 KiB: 3.96 / 14.16 against 5.17 / 19.85 ms.  Two
// 512-thread CTAs per SM for global work rows gave 12.76 ms (decode), and
// 1024-thread CTAs two per SM (32 registers) spill kilobytes.
constexpr int kWideThreads = 1024;
// Other tiles run kNarrowBlocks CTAs of kFftThreads per SM, each within
// kFftSmemBudget bytes of shared memory: four (64 registers, narrower column
// tiles) rather than two (128 registers) made every such transform faster,
// e.g. GF(2^16) 300+100 at 64 KiB 4.19 / 15.66 -> 3.17 / 11.62 ms (encode /
// decode, 64 stripes), GF(2^8) 32+16 at 1 MiB decode 18.46 -> 13.00 ms.
constexpr int kNarrowBlocks = 4;
constexpr int kGlobalBlocks = 1;

// Register-stage kernels (leo_fft.cuh).  Tile: 4 * kFftThreads bytes when the
// transform fits in registers (m or n <= 16), else 64 * nb bytes with the
// work rows in shared memory (or a per-CTA slab of global memory).
__host__ __device__ inline uint64_t fft_tile_bytes(uint32_t lanes_one_thread, uint32_t nb) {
  return lanes_one_thread <= 16 ? uint64_t(4 * kFftThreads) : uint64_t(64) * nb;
}

// NT = kWideThreads is used when a tile's shared memory leaves room for one
// CTA per SM, and for work rows in global memory.
template <int BITS, bool VERIFY, bool GLOBAL_WORK, int NT = kFftThreads>
__global__ void __launch_bounds__(NT, NT == kFftThreads ? kNarrowBlocks : (GLOBAL_WORK ? kGlobalBlocks : 1)) k_fft_encode(LeoArgs a) {
  extern __shared__ __align__(16) uint32_t smem[];
  __shared__ uint32_t bad;
  uint32_t *W = GLOBAL_WORK ? a.scratch + size_t(blockIdx.x) * a.lanes * a.nb * kRowWords : smem;
  const uint64_t tile_bytes = fft_tile_bytes(a.m, a.nb);
  const uint32_t tiles_per_job = uint32_t((a.len + tile_bytes - 1) / tile_bytes);
  const uint32_t total = tiles_per_job * a.n_jobs;
  for (uint32_t t = blockIdx.x; t < total; t += gridDim.x) {
    const uint32_t job = t / tiles_per_job;
    const uint64_t col0 = uint64_t(t - job * tiles_per_job) * tile_bytes;
    const LeoJob jd = a.jobs[job];
    fft_encode_tile<BITS, VERIFY, NT>(W, a, jd, col0, a.len, &bad);
  }
}

template <int BITS, bool GLOBAL_WORK, int NT = kFftThreads>
__global__ void __launch_bounds__(NT, NT == kFftThreads ? kNarrowBlocks : (GLOBAL_WORK ? kGlobalBlocks : 1)) k_fft_decode(LeoArgs a) {
  extern __shared__ __align__(16) uint32_t smem[];
  uint32_t *W = GLOBAL_WORK ? a.scratch + size_t(blockIdx.x) * a.lanes * a.nb * kRowWords : smem;
  const uint64_t tile_bytes = fft_tile_bytes(a.n, a.nb);
  const uint32_t tiles_per_job = uint32_t((a.len + tile_bytes - 1) / tile_bytes);
  const uint32_t total = tiles_per_job * a.n_jobs;
  for (uint32_t t = blockIdx.x; t < total; t += gridDim.x) {
    const uint32_t job = t / tiles_per_job;
    const uint64_t col0 = uint64_t(t - job * tiles_per_job) * tile_bytes;
    const LeoJob jd = a.jobs[job];
    fft_decode_tile<BITS, NT>(W, a, jd, col0, a.len);
  }
}

template <int BITS, bool GLOBAL_WORK>
__global__ void __launch_bounds__(kLeoThreads) k_leo_decode(LeoArgs a) {
  extern __shared__ uint32_t smem[];
  uint32_t *W = GLOBAL_WORK ? a.scratch + size_t(blockIdx.x) * a.lanes * a.nb * kRowWords : smem;
  const uint64_t tile_bytes = uint64_t(a.nb) * 64;
  const uint32_t tiles_per_job = uint32_t((a.len + tile_bytes - 1) / tile_bytes);
  const uint32_t total = tiles_per_job * a.n_jobs;
  for (uint32_t t = blockIdx.x; t < total; t += gridDim.x) {
    const uint32_t job = t / tiles_per_job;
    const uint64_t col0 = uint64_t(t - job * tiles_per_job) * tile_bytes;
    const LeoJob jd = a.jobs[job];
    leo_decode_tile<BITS, kLeoThreads>(W, a, jd, col0, a.len);
  }
}

// K7a: one CTA per erasure pattern.  data[] = indicator of erased positions
// (parity i at i, padding p..m, data j at m + j), FWHT limited to blocks below
// work_size, times log_walsh mod (2^bits - 1), full FWHT; err = first n values.
template <int BITS>
__global__ void __launch_bounds__(1024) k_leo_locator(const uint8_t *const *presents, uint16_t *const *outs,
                                                      const uint16_t *walsh, uint32_t k, uint32_t p, uint32_t m,
                                                      uint32_t n) {
  extern __shared__ uint16_t d[];
  constexpr uint32_t order = 1u << BITS, mod = order - 1;
  const uint8_t *present = presents[blockIdx.x];
  for (uint32_t i = threadIdx.x; i < order; i += blockDim.x) {
    uint16_t v = 0;
    if (i < p)
      v = present[k + i] ? 0 : 1;
    else if (i < m)
      v = 1;
    else if (i < m + k)
      v = present[i - m] ? 0 : 1;
    d[i] = v;
  }
  __syncthreads();
  auto add = [](uint32_t x, uint32_t y) -> uint32_t {
    const uint32_t s = x + y;
    return (s + (s >> BITS)) & mod;
  };
  auto sub = [](uint32_t x, uint32_t y) -> uint32_t {
    const uint32_t df = x - y;
    return (df + (df >> BITS)) & mod;
  };
  for (int pass = 0; pass < 2; ++pass) {
    const uint32_t mtrunc = pass == 0 ? m + k : order;
    for (uint32_t dist = 1, dist4 = 4; dist4 <= order; dist = dist4, dist4 <<= 2) {
      const uint32_t nblk = (mtrunc + dist4 - 1) / dist4;
      for (uint32_t q = threadIdx.x; q < nblk * dist; q += blockDim.x) {
        const uint32_t off = (q / dist) * dist4 + q % dist;
        const uint32_t a0 = d[off], a1 = d[off + dist], a2 = d[off + 2 * dist], a3 = d[off + 3 * dist];
        const uint32_t t0 = add(a0, a1), t1 = sub(a0, a1), t2 = add(a2, a3), t3 = sub(a2, a3);
        d[off] = uint16_t(add(t0, t2));
        d[off + 2 * dist] = uint16_t(sub(t0, t2));
        d[off + dist] = uint16_t(add(t1, t3));
        d[off + 3 * dist] = uint16_t(sub(t1, t3));
      }
      __syncthreads();
    }
    if (pass == 0) {
      for (uint32_t i = threadIdx.x; i < order; i += blockDim.x)
        if (d[i]) d[i] = uint16_t((uint64_t(d[i]) * walsh[i]) % mod);
      __syncthreads();
    }
  }
  uint16_t *out = outs[blockIdx.x];
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) out[i] = d[i];
}

}  // namespace

// ====================================================================== host
using EventPtr = std::shared_ptr<CUevent_st>;

// A cached error-locator array.  Launches never read it in place: every
// build copies the locators it needs into memory the launch owns, in stream
// order, under the cache lock (copy_locators), and records an event after the
// copies.  A plan evicted from the cache gives its block back only behind
// those events, so a copy still queued on some stream always reads the
// pattern it was queued for.
struct LeoPlan {
  uint16_t *err = nullptr;  // device, n entries (one block of the locator pool)
  uint32_t input_count = 0;
  // Completion of the launch that builds err (null once seen complete):
  // a copy that uses the plan waits on it in stream order instead of the
  // builder waiting on the host.
  EventPtr ready;
  // Copies from err that may still be queued (pruned as they complete).
  std::vector<EventPtr> readers;
  std::list<std::string>::iterator lru;
  uint64_t pinned_by = 0;  // the build that last used it cannot evict it
};

// A block of an evicted plan, reusable once its readers (and its own
// locator launch) have finished in stream order.
struct RetiredBlock {
  uint16_t *err;
  EventPtr ready;
  std::vector<EventPtr> readers;
};

// Locator arrays cached per codec: least recently used patterns beyond this
// many bytes are evicted (the reference bounds its GF(2^16) decode-plan cache
// the same way, src/core/leopard_gf16/decode.rs:268-305, 405-445).  At least
// 64 patterns are kept whatever the code's width.
constexpr size_t kLocatorCacheBytes = size_t(32) << 20;
constexpr size_t kLocatorCacheMinPlans = 64;

struct LeopardState {
  LeoField *field = nullptr;
  uint32_t m = 0, n = 0, mtrunc = 0, last = 0;
  std::mutex mu;
  std::unordered_map<std::string, LeoPlan> plans;
  std::list<std::string> plan_lru;  // least recently used first
  size_t plan_block = 0;            // bytes of one locator block (2n, 256-aligned)
  size_t plan_budget = 0;           // bytes the cached plans may hold
  rsgpu_cache_stats plan_stats{};   // requests, hits, misses, inserts, evictions
  uint64_t build_seq = 0;           // id of the build in progress (under mu)
  std::vector<void *> owned;    // retired scratch slabs, freed with the codec
  // Locator blocks are carved from these slabs, so a new pattern costs no
  // cudaMalloc once the pool has grown to the cache's budget.
  std::vector<void *> plan_slabs;
  std::vector<uint16_t *> free_blocks;
  std::vector<RetiredBlock> retired_blocks;
  uint32_t *scratch = nullptr;  // global work rows for the decode of very wide codes
  size_t scratch_bytes = 0;
  // Launches that use `scratch` are ordered across streams by this event:
  // each waits for the previous user's record, then records its own.
  cudaEvent_t scratch_done = nullptr;
  std::mutex scratch_mu;
  std::vector<uint8_t> dense_enc;  // GF(2^8): the encode map as an m x k matrix
  uint32_t *d_dense_enc = nullptr;  // ... packed for K1, device-resident (filled with dense_enc)
  // GF(2^8) decode maps by (presence pattern, goal), with their K1 tables,
  // least recently used first out beyond kDenseCacheBytes (under mu).
  struct DenseEntry {
    std::string key;
    std::shared_ptr<const LeoDenseMap> map;
    size_t bytes;
  };
  std::list<DenseEntry> dense_lru;
  std::unordered_map<std::string, std::list<DenseEntry>::iterator> dense_index;
  size_t dense_bytes = 0;
  // Bytes reconstructed so far under patterns whose map is not derived yet
  // (bounded: cleared when it holds kDenseSeenMax patterns).
  std::unordered_map<std::string, size_t> dense_seen;
  ~LeopardState() {
    cudaDeviceSynchronize();
    for (void *p : plan_slabs) cudaFree(p);
    if (scratch) cudaFree(scratch);
    for (void *p : owned) cudaFree(p);
    if (d_dense_enc) cudaFree(d_dense_enc);
    if (scratch_done) cudaEventDestroy(scratch_done);
  }
};

struct LeoLaunch {
  Codec *codec = nullptr;
  bool decode = false, verify = false;
  int engine = 1;  // 1: register-stage kernels, 0: half-warp layer kernels
  LeoArgs args{};
  void *d_blob = nullptr;  // jobs | pointers | roles
  // One-shot launches allocate the blob on their stream and free it there
  // after the kernel; prepared launches own it until destroyed.
  bool blob_ordered = false;
  cudaStream_t blob_stream = nullptr;
  int threads = 256;  // register-stage kernels: 256, or kWideThreads for one CTA per SM
  int grid = 0;
  size_t smem = 0;
  bool global_work = false;
  // Work rows in a caller-owned buffer private to the launch's stream
  // (instead of the codec's shared slab, which launches on different streams
  // take in turn).
  void *own_scratch = nullptr;
  ~LeoLaunch() {
    if (!d_blob) return;
    if (blob_ordered)
      cudaFreeAsync(d_blob, blob_stream);
    else
      cudaFree(d_blob);
  }
};

// Grow the codec's scratch slab to `need` bytes.  A slab another thread may
// still have in a built launch is retired (kept until the codec is
// destroyed), never freed under it.
int grow_scratch(LeopardState &st, size_t need) {
  std::lock_guard<std::mutex> g(st.scratch_mu);
  if (st.scratch_bytes >= need) return RSGPU_OK;
  if (st.scratch) st.owned.push_back(st.scratch);
  st.scratch = nullptr;
  st.scratch_bytes = 0;
  RS_CUDA(cudaMalloc(&st.scratch, need));
  st.scratch_bytes = need;
  return RSGPU_OK;
}

int Codec::init_leopard() {
  RS_CUDA(cudaGetDevice(&device));
  auto st = std::make_shared<LeopardState>();
  int rc = leo_field(family == RSGPU_FAMILY_LEOPARD_GF8 ? 8 : 16, &st->field);
  if (rc) return rc;
  st->m = uint32_t(pow2_at_least(m));
  st->n = uint32_t(pow2_at_least(st->m + k));
  st->mtrunc = uint32_t(std::min<size_t>(k, st->m));
  st->last = uint32_t(k % st->m);
  st->plan_block = (size_t(st->n) * 2 + 255) & ~size_t(255);
  st->plan_budget = std::max(kLocatorCacheBytes, kLocatorCacheMinPlans * st->plan_block);
  const uint32_t mod = st->field->host.mod;
  if (st->m > mod) return RSGPU_ERR_TOO_MANY_SHARDS;
  leo = st;
  return RSGPU_OK;
}

namespace {

constexpr size_t kSmemBudget = 200 * 1024;

// Column blocks per tile: enough rows of work per CTA without exceeding the
// shared-memory budget.
uint32_t pick_nb(uint32_t lanes, size_t len) {
  const size_t row = 64;
  uint32_t nb = 1;
  while (nb < 16 && size_t(lanes) * (nb * 2) * row <= 96 * 1024 && size_t(nb * 2) * 64 <= len) nb *= 2;
  return nb;
}

int sm_count() {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  }
  return sms;
}

int ilog2(uint32_t v) {
  int b = 0;
  while ((1u << b) < v) ++b;
  return b;
}

uint8_t stage_byte(int lg, int lgdm) { return uint8_t(lg | (lgdm << 3)); }

// At most four stages: 16 bits of lanes (GF(2^16)) in four-bit stages.
constexpr int kMaxStages = 4;

// Stage plans of the register-stage kernels (leo_fft.cuh).  IFFT: radix-4
// layers from distance 1 up, then a radix-2 layer when log2 L is odd; two
// radix-4 layers per 16-lane stage.  FFT: radix-4 layers from the top down,
// then the distance-1 radix-2 layer when log2 L is odd.
int ifft_stages(uint32_t L, uint8_t *out) {
  const int b = ilog2(L);
  int used = 0, n = 0;
  while (b - used >= 4 && n < kMaxStages) {
    out[n++] = stage_byte(4, used);
    used += 4;
  }
  if (b - used > 0 && n < kMaxStages) out[n++] = stage_byte(b - used, used);
  return n;
}

int fft_stages(uint32_t L, uint8_t *out) {
  const int b = ilog2(L);
  int n = 0;
  if (b == 0) return 0;
  const bool odd = b & 1;
  int cur = b;
  const int floor_bits = odd ? 3 : 0;
  if (b == 1) {
    out[n++] = stage_byte(1, 0);
    return n;
  }
  if (((cur - floor_bits) % 4) == 2) {
    out[n++] = stage_byte(2, cur - 2);
    cur -= 2;
  }
  while (cur - floor_bits >= 4 && n < kMaxStages) {
    out[n++] = stage_byte(4, cur - 4);
    cur -= 4;
  }
  if (odd && n < kMaxStages) out[n++] = stage_byte(3, 0);
  return n;
}

uint32_t pack_stages(const uint8_t *st) {
  return uint32_t(st[0]) | uint32_t(st[1]) << 8 | uint32_t(st[2]) << 16 | uint32_t(st[3]) << 24;
}

void fill_stages(LeoArgs &a) {
  uint8_t st[kMaxStages] = {0, 0, 0, 0};
  a.n_ienc = uint32_t(ifft_stages(a.m, st));
  a.st_ienc = pack_stages(st);
  std::memset(st, 0, sizeof(st));
  a.n_fenc = uint32_t(fft_stages(a.m, st));
  a.st_fenc = pack_stages(st);
  std::memset(st, 0, sizeof(st));
  a.n_idec = uint32_t(ifft_stages(a.n, st));
  a.st_idec = pack_stages(st);
  std::memset(st, 0, sizeof(st));
  a.n_fdec = uint32_t(fft_stages(a.n, st));
  a.st_fdec = pack_stages(st);
}

}  // namespace

// Which Leopard kernels run: 1 = register-stage kernels (leo_fft.cuh, the
// default), 0 = the half-warp layer kernels (leo_tile.cuh).  Both write the
// same bytes; RSGPU_LEO_ENGINE overrides, and the mixed-batch planner may
// pick either per operation.
int &leo_engine() {
  static int v = [] {
    const char *e = getenv("RSGPU_LEO_ENGINE");
    return e ? atoi(e) : 1;
  }();
  return v;
}

namespace {

constexpr size_t kFftSmemBudget = (192 * 1024) / kNarrowBlocks;  // kNarrowBlocks resident CTAs per SM

// Work rows and tile width of a register-stage launch: `rows` rows of work
// (encoder 2m, decoder n) when the transform needs shared memory, i.e. when
// `reg_lanes` (m or n) exceeds 16.
template <class K, class K2>
int configure_fft(const K kernel, const K2 kernel_wide, LeoLaunch &L, uint32_t rows, uint32_t reg_lanes, size_t len,
                  size_t n_jobs) {
  LeopardState &st = *L.codec->leo;
  L.args.lanes = rows;
  size_t smem = 0;
  uint32_t nb = 2;
  if (reg_lanes > 16) {
    while (nb < 8 && size_t(rows) * (nb * 2) * 64 <= kFftSmemBudget && size_t(nb * 2) * 64 <= len) nb *= 2;
    smem = size_t(rows) * nb * 64;
  }
  L.args.nb = nb;
  L.global_work = smem > 200 * 1024;
  const uint64_t tile = fft_tile_bytes(reg_lanes, nb);
  const uint64_t tiles = ((len + tile - 1) / tile) * std::max<size_t>(n_jobs, 1);
  L.threads = kFftThreads;
  if (!L.global_work) {
    L.smem = smem;
    const void *fn = reinterpret_cast<const void *>(kernel);
    if (smem > kFftSmemBudget) {  // one CTA per SM: give it more warps
      L.threads = kWideThreads;
      fn = reinterpret_cast<const void *>(kernel_wide);
    }
    RS_CUDA(ensure_smem_limit(fn, smem));
    int per_sm = 0;
    RS_CUDA(blocks_per_sm(fn, L.threads, smem, &per_sm));
    L.grid = int(std::min<uint64_t>(tiles, uint64_t(std::max(per_sm, 1)) * sm_count()));
  } else {
    // Work rows in a global slab (L2-resident): one wide CTA per SM keeps the
    // slab smaller than several narrower CTAs would.
    L.smem = 0;
    L.threads = kWideThreads;
    L.grid = int(std::min<uint64_t>(tiles, uint64_t(kGlobalBlocks) * sm_count()));
    const size_t need = size_t(L.grid) * rows * nb * 64;
    if (L.own_scratch) {  // sized by the caller for a full grid
      L.args.scratch = static_cast<uint32_t *>(L.own_scratch);
      return RSGPU_OK;
    }
    int rc = grow_scratch(st, need);
    if (rc) return rc;
    {
      std::lock_guard<std::mutex> g(st.scratch_mu);
      L.args.scratch = st.scratch;
    }
  }
  return RSGPU_OK;
}

template <class K>
int configure(const K kernel, LeoLaunch &L, uint32_t lanes, size_t len, uint64_t tiles) {
  LeopardState &st = *L.codec->leo;
  uint32_t nb = pick_nb(lanes, len);
  size_t smem = size_t(lanes) * nb * 64;
  L.global_work = smem > kSmemBudget;
  L.args.nb = nb;
  L.args.lanes = lanes;
  if (!L.global_work) {
    L.smem = smem;
    RS_CUDA(ensure_smem_limit(reinterpret_cast<const void *>(kernel), smem));
    int per_sm = 0;
    RS_CUDA(blocks_per_sm(reinterpret_cast<const void *>(kernel), kLeoThreads, smem, &per_sm));
    L.grid = int(std::min<uint64_t>(tiles, uint64_t(std::max(per_sm, 1)) * sm_count()));
  } else {
    // Work rows in a device slab: one region per resident CTA.
    L.smem = 0;
    L.grid = int(std::min<uint64_t>(tiles, uint64_t(2 * sm_count())));
    const size_t need = size_t(L.grid) * lanes * nb * 64;
    int rc = grow_scratch(st, need);
    if (rc) return rc;
    {
      std::lock_guard<std::mutex> g(st.scratch_mu);
      L.args.scratch = st.scratch;
    }
  }
  return RSGPU_OK;
}

// Makes stream s wait for the events that are still pending (a null or
// completed event needs no wait).
int wait_events(const std::vector<EventPtr> &evs, cudaStream_t s) {
  for (const EventPtr &e : evs)
    if (e && cudaEventQuery(e.get()) != cudaSuccess) RS_CUDA(cudaStreamWaitEvent(s, e.get(), 0));
  return RSGPU_OK;
}

// A locator block for a new plan, its previous users ordered before stream
// s: a free block, else a retired one (s waits for the copies that read it
// and for the launch that wrote it), else a new slab's worth.
int take_block(LeopardState &st, cudaStream_t s, uint16_t **out) {
  if (st.free_blocks.empty() && !st.retired_blocks.empty()) {
    RetiredBlock r = std::move(st.retired_blocks.back());
    st.retired_blocks.pop_back();
    r.readers.push_back(r.ready);
    const int rc = wait_events(r.readers, s);
    if (rc) return rc;
    *out = r.err;
    return RSGPU_OK;
  }
  if (st.free_blocks.empty()) {
    const size_t per = std::max<size_t>(1, (size_t(1) << 20) / st.plan_block);
    void *p = nullptr;
    RS_CUDA(cudaMalloc(&p, per * st.plan_block));
    st.plan_slabs.push_back(p);
    for (size_t i = 0; i < per; ++i)
      st.free_blocks.push_back(reinterpret_cast<uint16_t *>(static_cast<uint8_t *>(p) + i * st.plan_block));
  }
  *out = st.free_blocks.back();
  st.free_blocks.pop_back();
  return RSGPU_OK;
}

// Evicts least recently used plans until one more block fits the budget;
// plans the current build uses stay (the cache may then run over its budget
// until a later build).
void evict_for_one(LeopardState &st) {
  while ((st.plans.size() + 1) * st.plan_block > st.plan_budget && !st.plan_lru.empty()) {
    auto it = st.plans.find(st.plan_lru.front());
    if (it->second.pinned_by == st.build_seq) break;  // every older plan is gone already
    st.retired_blocks.push_back(RetiredBlock{it->second.err, it->second.ready, std::move(it->second.readers)});
    st.plan_lru.pop_front();
    st.plans.erase(it);
    ++st.plan_stats.evictions;
  }
}

// Error locators for a presence pattern, built on the GPU (K7a) and cached
// (least recently used out beyond the budget); returns the plan, pinned for
// the current build.  Caller holds st.mu and has started a build
// (st.build_seq).
int decode_plan(Codec &c, const uint8_t *present, LeoPlan **out, cudaStream_t s,
                std::vector<std::pair<std::string, const uint8_t *>> &pending) {
  LeopardState &st = *c.leo;
  std::string key(reinterpret_cast<const char *>(present), c.k + c.m);
  ++st.plan_stats.requests;
  auto it = st.plans.find(key);
  if (it != st.plans.end()) {
    ++st.plan_stats.hits;
    st.plan_lru.splice(st.plan_lru.end(), st.plan_lru, it->second.lru);
    it->second.pinned_by = st.build_seq;
    *out = &it->second;
    return RSGPU_OK;
  }
  ++st.plan_stats.misses;
  evict_for_one(st);
  LeoPlan plan;
  int rc = take_block(st, s, &plan.err);
  if (rc) return rc;
  plan.input_count = st.m;
  for (size_t i = 0; i < c.k; ++i)
    if (present[i]) plan.input_count = uint32_t(st.m + i + 1);
  plan.pinned_by = st.build_seq;
  auto ins = st.plans.emplace(key, std::move(plan));
  st.plan_lru.push_back(key);
  ins.first->second.lru = std::prev(st.plan_lru.end());
  ++st.plan_stats.inserts;
  pending.emplace_back(key, present);
  *out = &ins.first->second;
  return RSGPU_OK;
}

int build_locators(Codec &c, std::vector<std::pair<std::string, const uint8_t *>> &pending, cudaStream_t s) {
  if (pending.empty()) return RSGPU_OK;
  LeopardState &st = *c.leo;
  const size_t total = c.k + c.m;
  std::vector<uint8_t> pres(pending.size() * total);
  for (size_t i = 0; i < pending.size(); ++i) std::memcpy(&pres[i * total], pending[i].first.data(), total);
  // Stream-ordered scratch: nothing here waits for other streams' work.
  uint8_t *d_pres = nullptr;
  RS_CUDA(cudaError_t(lib_malloc_async(reinterpret_cast<void **>(&d_pres), pres.size(), s)));
  int rc = upload_to(d_pres, pres.data(), pres.size(), s);
  if (rc) return rc;
  std::vector<const uint8_t *> pp(pending.size());
  std::vector<uint16_t *> oo(pending.size());
  for (size_t i = 0; i < pending.size(); ++i) {
    pp[i] = d_pres + i * total;
    oo[i] = st.plans[pending[i].first].err;
  }
  void *d_pp = nullptr, *d_oo = nullptr;
  RS_CUDA(cudaError_t(lib_malloc_async(&d_pp, pp.size() * sizeof(void *), s)));
  RS_CUDA(cudaError_t(lib_malloc_async(&d_oo, oo.size() * sizeof(void *), s)));
  if ((rc = upload_to(d_pp, pp.data(), pp.size() * sizeof(void *), s))) return rc;
  if ((rc = upload_to(d_oo, oo.data(), oo.size() * sizeof(void *), s))) return rc;
  const int bits = st.field->bits;
  const size_t smem = size_t(1u << bits) * 2;
  if (bits == 16) {
    RS_CUDA(ensure_smem_limit(reinterpret_cast<const void *>(k_leo_locator<16>), smem));
    k_leo_locator<16><<<int(pending.size()), 1024, smem, s>>>(
        static_cast<const uint8_t *const *>(d_pp), static_cast<uint16_t *const *>(d_oo), st.field->d_walsh,
        uint32_t(c.k), uint32_t(c.m), st.m, st.n);
  } else {
    k_leo_locator<8><<<int(pending.size()), 256, smem, s>>>(
        static_cast<const uint8_t *const *>(d_pp), static_cast<uint16_t *const *>(d_oo), st.field->d_walsh,
        uint32_t(c.k), uint32_t(c.m), st.m, st.n);
  }
  launch_counter_add(1);
  RS_CUDA(cudaGetLastError());
  cudaFreeAsync(d_pres, s);
  cudaFreeAsync(d_pp, s);
  cudaFreeAsync(d_oo, s);
  // The new plans are visible to other streams once the lock is released:
  // their users wait for this event (wait_plans) rather than this thread
  // waiting here, where the locator launch may queue behind other streams'
  // long-running kernels.
  cudaEvent_t ev = nullptr;
  RS_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  std::shared_ptr<CUevent_st> ready(ev, [](cudaEvent_t e) { cudaEventDestroy(e); });
  RS_CUDA(cudaEventRecord(ev, s));
  for (auto &p : pending) st.plans[p.first].ready = ready;
  pending.clear();
  return RSGPU_OK;
}

// Makes stream s wait for the locator launches of these plans that may still
// be running, and forgets the ones that have finished.  Caller holds st.mu.
int wait_plans(const std::vector<LeoPlan *> &plans, cudaStream_t s) {
  const CUevent_st *last = nullptr;
  for (LeoPlan *p : plans) {
    if (!p || !p->ready) continue;
    if (cudaEventQuery(p->ready.get()) == cudaSuccess) {
      p->ready.reset();
      continue;
    }
    if (p->ready.get() == last) continue;
    last = p->ready.get();
    RS_CUDA(cudaStreamWaitEvent(s, p->ready.get(), 0));
  }
  return RSGPU_OK;
}

// Copies the locators of `plans` (distinct) to dst + i * n on stream s, after
// their locator launches.  With `ordered` the copies stay queued on s and an
// event recorded behind them joins each plan's readers (an evicted block is
// reused only after it); otherwise the call waits for s.  Caller holds st.mu.
int copy_locators(LeopardState &st, const std::vector<LeoPlan *> &plans, uint16_t *dst, cudaStream_t s,
                  bool ordered) {
  if (plans.empty()) return RSGPU_OK;
  int rc = wait_plans(plans, s);
  if (rc) return rc;
  for (size_t i = 0; i < plans.size(); ++i)
    RS_CUDA(cudaMemcpyAsync(dst + i * st.n, plans[i]->err, size_t(st.n) * 2, cudaMemcpyDeviceToDevice, s));
  if (!ordered) return cuda_status(cudaStreamSynchronize(s));
  cudaEvent_t ev = nullptr;
  RS_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  EventPtr read(ev, [](cudaEvent_t e) { cudaEventDestroy(e); });
  RS_CUDA(cudaEventRecord(ev, s));
  for (LeoPlan *p : plans) {
    auto &r = p->readers;
    r.erase(std::remove_if(r.begin(), r.end(), [](const EventPtr &e) { return cudaEventQuery(e.get()) == cudaSuccess; }),
            r.end());
    r.push_back(read);
  }
  return RSGPU_OK;
}

int build_leo(Codec &c, int op, size_t n_stripes, uint8_t *const *shards, const uint8_t *present, size_t len,
              int goal, const uint8_t *required, size_t n_required, uint32_t *flags, LeoLaunch &L,
              cudaStream_t s, bool one_shot) {
  LeopardState &st = *c.leo;
  const size_t total = c.k + c.m;
  L.codec = &c;
  L.decode = op == RSGPU_OP_RECONSTRUCT;
  L.verify = op == RSGPU_OP_VERIFY;
  std::vector<LeoJob> jobs;
  std::vector<uint8_t> roles;
  std::vector<size_t> role_off;
  {
    // The lock covers the plans, their locator launches and the copies of the
    // locators into this launch's blob.
    std::lock_guard<std::mutex> g(st.mu);
    ++st.build_seq;
    std::vector<std::pair<std::string, const uint8_t *>> pending;
    std::vector<LeoPlan *> used;       // distinct plans, in first-use order
    std::vector<uint32_t> slot_of_job;  // index into `used` per decode job
    std::unordered_map<LeoPlan *, uint32_t> slot;
    int bad = RSGPU_OK;  // an unrecoverable stripe: plans already cached still get their locators
    for (size_t i = 0; i < n_stripes && bad == RSGPU_OK; ++i) {
      LeoJob j{};
      j.ptr_off = uint32_t(i * total);
      j.flag_idx = uint32_t(i);
      if (L.decode) {
        const uint8_t *pr = present + i * total;
        size_t np = 0;
        bool any_target = false;
        const size_t base = roles.size();
        for (size_t x = 0; x < total; ++x) {
          np += pr[x] ? 1 : 0;
          bool want = goal == RSGPU_GOAL_ALL || (goal == RSGPU_GOAL_DATA && x < c.k) ||
                      (goal == RSGPU_GOAL_REQUIRED && x < n_required && required[x]);
          uint8_t role = pr[x] ? 1 : (want ? 2 : 0);
          any_target |= role == 2;
          roles.push_back(role);
        }
        // Missing beyond the parity count cannot be recovered
        // (src/core/leopard_gf16/decode.rs:744-748).
        if (total - np > c.m) {
          bad = RSGPU_ERR_TOO_FEW_SHARDS_PRESENT;
          break;
        }
        if (np == total || !any_target) {
          roles.resize(base);
          continue;
        }
        LeoPlan *plan = nullptr;
        if ((bad = decode_plan(c, pr, &plan, s, pending))) break;
        auto sl = slot.emplace(plan, uint32_t(used.size()));
        if (sl.second) used.push_back(plan);
        slot_of_job.push_back(sl.first->second);
        j.input_count = plan->input_count;
        role_off.push_back(base);
      }
      jobs.push_back(j);
    }
    int rc = build_locators(c, pending, s);  // plans already cached get their locators even on an error
    if (rc) return rc;
    if (bad) return bad;
    // Blob: jobs | pointers | roles | locators (one array per distinct pattern).
    const size_t jb = jobs.size() * sizeof(LeoJob);
    const size_t pb = n_stripes * total * sizeof(void *);
    const size_t lo = (jb + pb + roles.size() + 255) & ~size_t(255);
    const size_t lb = used.size() * size_t(st.n) * 2;
    std::vector<uint8_t> blob(lo);
    std::memcpy(blob.data() + jb, shards, pb);
    std::memcpy(blob.data() + jb + pb, roles.data(), roles.size());
    if (one_shot) {
      RS_CUDA(cudaError_t(lib_malloc_async(&L.d_blob, lo + lb + 16, s)));
      L.blob_ordered = true;
      L.blob_stream = s;
    } else {
      RS_CUDA(cudaMalloc(&L.d_blob, lo + lb + 16));
    }
    uint8_t *dbase = static_cast<uint8_t *>(L.d_blob);
    uint16_t *locs = reinterpret_cast<uint16_t *>(dbase + lo);
    for (size_t i = 0; i < jobs.size() && L.decode; ++i) {
      jobs[i].role = dbase + jb + pb + role_off[i];
      jobs[i].err = locs + size_t(slot_of_job[i]) * st.n;
    }
    std::memcpy(blob.data(), jobs.data(), jb);
    if (one_shot) {
      if ((rc = upload_to(L.d_blob, blob.data(), blob.size(), s))) return rc;
    } else {
      RS_CUDA(cudaMemcpy(L.d_blob, blob.data(), blob.size(), cudaMemcpyHostToDevice));
    }
    if ((rc = copy_locators(st, used, locs, s, one_shot))) return rc;
  }
  const size_t jb = jobs.size() * sizeof(LeoJob);
  uint8_t *dbase = static_cast<uint8_t *>(L.d_blob);
  LeoArgs &a = L.args;
  a.jobs = reinterpret_cast<const LeoJob *>(dbase);
  a.ptrs = reinterpret_cast<const uint8_t *const *>(dbase + jb);
  a.skew = st.field->d_skew;
  a.bank = st.field->d_bank;
  a.flags = flags;
  a.len = len;
  a.n_jobs = uint32_t(jobs.size());
  a.k = uint32_t(c.k);
  a.p = uint32_t(c.m);
  a.m = st.m;
  a.n = st.n;
  a.mtrunc = st.mtrunc;
  a.last = st.last;
  a.mod = st.field->host.mod;
  a.kbank = st.field->d_kbank;
  a.sktab = st.field->d_sktab;
  fill_stages(a);
  L.engine = leo_engine();
  if (L.engine == 1) {
    const bool b16f = st.field->bits == 16;
    const size_t nj = jobs.size();
    if (L.decode)
      return b16f ? configure_fft(k_fft_decode<16, false>, k_fft_decode<16, false, kWideThreads>, L, st.n, st.n, len, nj)
                  : configure_fft(k_fft_decode<8, false>, k_fft_decode<8, false, kWideThreads>, L, st.n, st.n, len, nj);
    if (L.verify)
      return b16f ? configure_fft(k_fft_encode<16, true, false>, k_fft_encode<16, true, false, kWideThreads>, L, 2 * st.m,
                                  st.m, len, nj)
                  : configure_fft(k_fft_encode<8, true, false>, k_fft_encode<8, true, false, kWideThreads>, L, 2 * st.m, st.m,
                                  len, nj);
    return b16f ? configure_fft(k_fft_encode<16, false, false>, k_fft_encode<16, false, false, kWideThreads>, L, 2 * st.m,
                                st.m, len, nj)
                : configure_fft(k_fft_encode<8, false, false>, k_fft_encode<8, false, false, kWideThreads>, L, 2 * st.m, st.m,
                                len, nj);
  }
  const uint32_t lanes = L.decode ? st.n : 2 * st.m;
  const uint32_t nb_guess = pick_nb(lanes, len);
  const uint64_t tiles = ((len + nb_guess * 64 - 1) / (nb_guess * 64)) * std::max<size_t>(jobs.size(), 1);
  const bool b16 = st.field->bits == 16;
  int rc;
  if (L.decode)
    rc = b16 ? configure(k_leo_decode<16, false>, L, lanes, len, tiles)
             : configure(k_leo_decode<8, false>, L, lanes, len, tiles);
  else if (L.verify)
    rc = b16 ? configure(k_leo_encode<16, true, false>, L, lanes, len, tiles)
             : configure(k_leo_encode<8, true, false>, L, lanes, len, tiles);
  else
    rc = b16 ? configure(k_leo_encode<16, false, false>, L, lanes, len, tiles)
             : configure(k_leo_encode<8, false, false>, L, lanes, len, tiles);
  if (rc) return rc;
  return RSGPU_OK;
}

}  // namespace

namespace {
int leo_launch_kernel(const LeoLaunch &L, cudaStream_t s);
}

// Launches that use the codec's shared scratch slab (global work rows) wait
// for the previous such launch on any stream.  Under stream capture the
// graph's own dependencies order them instead (an event recorded outside a
// capture cannot be waited on inside it).
int leo_launch(const LeoLaunch &L, cudaStream_t s) {
  if (L.args.n_jobs == 0) return RSGPU_OK;
  if (!L.global_work || L.own_scratch) return leo_launch_kernel(L, s);
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  RS_CUDA(cudaStreamIsCapturing(s, &cap));
  if (cap != cudaStreamCaptureStatusNone) return leo_launch_kernel(L, s);
  LeopardState &st = *L.codec->leo;
  std::lock_guard<std::mutex> g(st.scratch_mu);
  if (!st.scratch_done) RS_CUDA(cudaEventCreateWithFlags(&st.scratch_done, cudaEventDisableTiming));
  RS_CUDA(cudaStreamWaitEvent(s, st.scratch_done, 0));
  int rc = leo_launch_kernel(L, s);
  if (rc) return rc;
  return cuda_status(cudaEventRecord(st.scratch_done, s));
}

namespace {
int leo_launch_kernel(const LeoLaunch &L, cudaStream_t s) {
  const bool b16 = L.codec->leo->field->bits == 16;
  const LeoArgs &a = L.args;
  if (L.engine == 1) {
    const dim3 grid(L.grid), block(L.threads);
    const bool wide = L.threads != kFftThreads;
#define FFT_GO(KERNEL) KERNEL<<<grid, block, L.smem, s>>>(a)
    if (L.decode) {
      if (L.global_work) {
        if (b16) FFT_GO((k_fft_decode<16, true, kWideThreads>)); else FFT_GO((k_fft_decode<8, true, kWideThreads>));
      } else if (wide) {
        if (b16) FFT_GO((k_fft_decode<16, false, kWideThreads>)); else FFT_GO((k_fft_decode<8, false, kWideThreads>));
      } else {
        if (b16) FFT_GO((k_fft_decode<16, false>)); else FFT_GO((k_fft_decode<8, false>));
      }
    } else if (L.verify) {
      if (L.global_work) {
        if (b16) FFT_GO((k_fft_encode<16, true, true, kWideThreads>)); else FFT_GO((k_fft_encode<8, true, true, kWideThreads>));
      } else if (wide) {
        if (b16) FFT_GO((k_fft_encode<16, true, false, kWideThreads>)); else FFT_GO((k_fft_encode<8, true, false, kWideThreads>));
      } else {
        if (b16) FFT_GO((k_fft_encode<16, true, false>)); else FFT_GO((k_fft_encode<8, true, false>));
      }
    } else {
      if (L.global_work) {
        if (b16) FFT_GO((k_fft_encode<16, false, true, kWideThreads>)); else FFT_GO((k_fft_encode<8, false, true, kWideThreads>));
      } else if (wide) {
        if (b16) FFT_GO((k_fft_encode<16, false, false, kWideThreads>)); else FFT_GO((k_fft_encode<8, false, false, kWideThreads>));
      } else {
        if (b16) FFT_GO((k_fft_encode<16, false, false>)); else FFT_GO((k_fft_encode<8, false, false>));
      }
    }
#undef FFT_GO
    launch_counter_add(1);
    return cuda_status(cudaGetLastError());
  }
  const dim3 grid(L.grid), block(kLeoThreads);
#define LEO_GO(KERNEL) KERNEL<<<grid, block, L.smem, s>>>(a)
  if (L.decode) {
    if (L.global_work) {
      if (b16) LEO_GO((k_leo_decode<16, true>)); else LEO_GO((k_leo_decode<8, true>));
    } else {
      if (b16) LEO_GO((k_leo_decode<16, false>)); else LEO_GO((k_leo_decode<8, false>));
    }
  } else if (L.verify) {
    if (L.global_work) {
      if (b16) LEO_GO((k_leo_encode<16, true, true>)); else LEO_GO((k_leo_encode<8, true, true>));
    } else {
      if (b16) LEO_GO((k_leo_encode<16, true, false>)); else LEO_GO((k_leo_encode<8, true, false>));
    }
  } else {
    if (L.global_work) {
      if (b16) LEO_GO((k_leo_encode<16, false, true>)); else LEO_GO((k_leo_encode<8, false, true>));
    } else {
      if (b16) LEO_GO((k_leo_encode<16, false, false>)); else LEO_GO((k_leo_encode<8, false, false>));
    }
  }
#undef LEO_GO
  launch_counter_add(1);
  return cuda_status(cudaGetLastError());
}
}  // namespace

uint32_t leo_kernel_count(const LeoLaunch &L) { return L.args.n_jobs ? 1 : 0; }

int prepare_other(Codec &c, int op, size_t n_stripes, uint8_t *const *shards, const uint8_t *present, size_t len,
                  int goal, uint32_t *flags, std::shared_ptr<LeoLaunch> &out) {
  if (c.family == RSGPU_FAMILY_CLASSIC) return prepare_tower(c, op, n_stripes, shards, present, len, goal, flags, out);
  auto L = std::make_shared<LeoLaunch>();
  int rc = build_leo(c, op, n_stripes, shards, present, len, goal, nullptr, 0, flags, *L, nullptr, false);
  if (rc) return rc;
  out = L;
  return RSGPU_OK;
}

// Work rows of a full grid of the decode kernel when they live in global
// memory (configure_fft: n rows of two 64-byte blocks per CTA, beyond
// 200 KiB of shared memory); 0 when they fit shared memory.
size_t leo_reconstruct_scratch_bytes(Codec &c) {
  const size_t rows = c.leo->n, per_cta = rows * 2 * 64;
  return per_cta > 200 * 1024 ? size_t(kGlobalBlocks) * sm_count() * per_cta : 0;
}

void leo_set_scratch(LeoLaunch &L, void *scratch) {
  if (!L.own_scratch) return;
  L.own_scratch = scratch;
  L.args.scratch = static_cast<uint32_t *>(scratch);
}

int prepare_leo_reconstruct_once(Codec &c, size_t n, uint8_t *const *shards, const uint8_t *present, size_t len,
                                 int goal, cudaStream_t s, void *scratch, std::shared_ptr<LeoLaunch> &out) {
  auto L = std::make_shared<LeoLaunch>();
  L->own_scratch = leo_reconstruct_scratch_bytes(c) ? scratch : nullptr;
  int rc = build_leo(c, RSGPU_OP_RECONSTRUCT, n, shards, present, len, goal, nullptr, 0, nullptr, *L, s, true);
  if (rc) return rc;
  out = L;
  return RSGPU_OK;
}

static int run_once(Codec &c, int op, size_t n, uint8_t *const *shards, const uint8_t *present, size_t len, int goal,
                    const uint8_t *required, size_t n_required, uint32_t *flags, cudaStream_t s) {
  // Stream-ordered: the launch's job blob is freed on `s` behind the kernel
  // when L goes out of scope, so the call returns without waiting.
  LeoLaunch L;
  int rc = build_leo(c, op, n, shards, present, len, goal, required, n_required, flags, L, s, true);
  if (rc) return rc;
  return leo_launch(L, s);
}

// GF(2^8) codes with at most 4 parity shards encode shards of 128 KiB and
// more through K1 with the codec's dense encode map (the FFT encode's own
// linear map, so the same bytes; its packed tables stay on the device):
// per call, 10+4 at 1 MiB 1.3x and at 4 MiB 1.6x faster than the FFT encode
// (the kernels alone: 3.1 against 0.54 TB/s).  Below 128 KiB the FFT call's
// smaller host cost wins; with more parity the transform is as fast (32+16)
// or much faster (128+64), so it stays.
constexpr size_t kDenseEncMinLen = size_t(128) << 10;

int leopard_encode(Codec &c, size_t n, uint8_t *const *shards, size_t len, cudaStream_t s) {
  if (c.leo->field->bits == 8 && c.m <= 4 && len >= kDenseEncMinLen && n > 0) {
    std::vector<uint8_t> rows;
    int rc = leopard_dense_encode(c, rows);
    if (rc) return rc;
    const uint32_t *tbl = nullptr;
    {
      std::lock_guard<std::mutex> g(c.leo->mu);
      tbl = c.leo->d_dense_enc;
    }
    const size_t total = c.k + c.m;
    std::vector<JobDesc> jobs(n);
    std::vector<const uint8_t *> ptrs(shards, shards + n * total);
    for (size_t i = 0; i < n; ++i) {
      jobs[i].ptr_off = uint32_t(i * total);
      jobs[i].n_in = uint16_t(c.k);
      jobs[i].n_out = uint16_t(c.m);
      jobs[i].tbl = tbl;
    }
    return c.apply_jobs(jobs, ptrs, len, s);
  }
  return run_once(c, RSGPU_OP_ENCODE, n, shards, nullptr, len, 0, nullptr, 0, nullptr, s);
}

int leopard_verify(Codec &c, size_t n, const uint8_t *const *shards, size_t len, uint8_t *ok, cudaStream_t s) {
  // The same rule as encode: small-parity GF(2^8) codes on shards of 128 KiB
  // and more compare against the dense encode map through K1.
  if (c.leo->field->bits == 8 && c.m <= 4 && len >= kDenseEncMinLen && n > 0) {
    std::vector<uint8_t> rows;
    int rc = leopard_dense_encode(c, rows);
    if (rc) return rc;
    const uint32_t *tbl = nullptr;
    {
      std::lock_guard<std::mutex> g(c.leo->mu);
      tbl = c.leo->d_dense_enc;
    }
    return c.verify_dev(n, shards, len, ok, s, tbl);
  }
  uint32_t *flags = nullptr;
  RS_CUDA(cudaError_t(lib_malloc_async(reinterpret_cast<void **>(&flags), std::max<size_t>(n, 1) * 4, s)));
  RS_CUDA(cudaMemsetAsync(flags, 0, std::max<size_t>(n, 1) * 4, s));
  int rc = run_once(c, RSGPU_OP_VERIFY, n, const_cast<uint8_t *const *>(shards), nullptr, len, 0, nullptr, 0, flags, s);
  std::vector<uint32_t> f(n);
  if (rc == RSGPU_OK) rc = cuda_status(cudaMemcpyAsync(f.data(), flags, n * 4, cudaMemcpyDeviceToHost, s));
  cudaFreeAsync(flags, s);
  if (rc == RSGPU_OK) rc = cuda_status(cudaStreamSynchronize(s));
  if (rc == RSGPU_OK)
    for (size_t i = 0; i < n; ++i) ok[i] = f[i] ? 0 : 1;
  return rc;
}

namespace {

constexpr size_t kDenseCacheBytes = size_t(64) << 20;
// A pattern's map is derived once the calls of this codec have moved this
// many bytes under it (this call included): deriving costs a small FFT
// launch, a wait and host packing (about a millisecond), which the FFT decode
// (~150 GB/s) of fewer bytes finishes sooner, while a pattern that keeps
// coming back (a failed disk seen by every stripe) soon pays for it.
constexpr size_t kDenseDeriveBytes = size_t(64) << 20;
constexpr size_t kDenseSeenMax = 4096;
constexpr size_t kDenseWideLen = size_t(1) << 20;  // maps of > 4 output groups: dense from here
constexpr int kDenseNotTaken = -1;

// Whether a pattern (key = presence flags + goal) with `targets` outputs runs
// through its dense map now, counting `bytes` more moved under it.  Caller
// holds st.mu.
bool dense_due_locked(LeopardState &st, const std::string &key, size_t targets, size_t bytes, size_t len) {
  if (targets > 16 && len < kDenseWideLen) return false;
  if (st.dense_index.count(key)) return true;
  if (st.dense_seen.size() >= kDenseSeenMax) st.dense_seen.clear();
  size_t &seen = st.dense_seen[key];
  seen += bytes;
  if (seen < kDenseDeriveBytes) return false;
  st.dense_seen.erase(key);
  return true;
}

// GF(2^8) reconstruct as a dense K1 launch: each stripe's map (its present
// shards -> its targets) comes from the per-codec map cache, derived with
// the FFT decode where missing (leopard_dense_decode).  The map is the FFT
// pipeline's own linear map, so the bytes are the FFT decode's on any
// inputs; measured 2.8-6x faster than the per-call FFT decode on 32+16
// codes (1-4 MiB shards) and on 128+64 with up to 16 erasures.
// A pattern stays on the FFT decode while its map is not cached and fewer
// than kDenseDeriveBytes have been moved under it, and when its map has more
// than 16 targets and the shards are under 1 MiB (its K1 tables and extra
// passes over the inputs then cost more than the transform: 128+64 with 64
// erasures at 256 KiB took 7.2 ms dense against 3.9 ms FFT); those stripes
// run in one FFT launch beside the dense one.  kDenseNotTaken when no
// pattern goes dense.
int reconstruct_dense8(Codec &c, size_t n, uint8_t *const *shards, const uint8_t *present, size_t len, int goal,
                       cudaStream_t s) {
  LeopardState &st = *c.leo;
  const size_t k = c.k, total = k + c.m;
  // Distinct patterns of the stripes that have something to rebuild.
  std::unordered_map<std::string, size_t> uniq;
  std::vector<size_t> which(n, SIZE_MAX), stripes_of, targets_of;
  std::vector<std::string> keys;
  for (size_t i = 0; i < n; ++i) {
    const uint8_t *pr = present + i * total;
    size_t targets = 0;
    for (size_t x = 0; x < total; ++x) targets += !pr[x] && (goal == RSGPU_GOAL_ALL || x < k);
    if (!targets) continue;
    std::string key(reinterpret_cast<const char *>(pr), total);
    auto it = uniq.find(key);
    if (it == uniq.end()) {
      it = uniq.emplace(key, keys.size()).first;
      keys.push_back(key);
      stripes_of.push_back(0);
      targets_of.push_back(targets);
    }
    which[i] = it->second;
    ++stripes_of[it->second];
  }
  if (keys.empty()) return RSGPU_OK;
  // Which patterns run dense.
  std::vector<char> dense(keys.size(), 1);
  size_t n_dense = 0;
  {
    std::lock_guard<std::mutex> g(st.mu);
    for (size_t u = 0; u < keys.size(); ++u) {
      dense[u] = dense_due_locked(st, keys[u] + char(goal), targets_of[u], stripes_of[u] * total * len, len);
      n_dense += dense[u];
    }
  }
  if (n_dense == 0) return kDenseNotTaken;
  // The other patterns' stripes: one FFT decode launch on the same stream.
  if (n_dense < keys.size()) {
    std::vector<uint8_t *> fsh;
    std::vector<uint8_t> fpr;
    for (size_t i = 0; i < n; ++i) {
      if (which[i] == SIZE_MAX || dense[which[i]]) continue;
      fsh.insert(fsh.end(), shards + i * total, shards + (i + 1) * total);
      fpr.insert(fpr.end(), present + i * total, present + (i + 1) * total);
    }
    const int rc = run_once(c, RSGPU_OP_RECONSTRUCT, fsh.size() / total, fsh.data(), fpr.data(), len, goal, nullptr,
                            0, nullptr, s);
    if (rc) return rc;
  }
  // Dense patterns: maps (cached or derived), then one K1 launch.
  std::vector<size_t> slot(keys.size(), SIZE_MAX);
  std::vector<uint8_t> pres;
  for (size_t u = 0; u < keys.size(); ++u)
    if (dense[u]) {
      slot[u] = pres.size() / total;
      pres.insert(pres.end(), keys[u].begin(), keys[u].end());
    }
  std::vector<LeoDenseMap> maps;
  int rc = leopard_dense_decode(c, n_dense, pres.data(), goal, maps, s);
  if (rc) return rc;
  std::vector<uint32_t> tables;
  std::vector<size_t> map_off(maps.size());
  for (size_t d = 0; d < maps.size(); ++d) {
    map_off[d] = tables.size();
    tables.insert(tables.end(), maps[d].packed->begin(), maps[d].packed->end());
  }
  std::vector<JobDesc> jobs;
  std::vector<size_t> tbl_off;
  std::vector<const uint8_t *> ptrs;
  for (size_t i = 0; i < n; ++i) {
    if (which[i] == SIZE_MAX || !dense[which[i]]) continue;
    const size_t d = slot[which[i]];
    const LeoDenseMap &mp = maps[d];
    JobDesc j{};
    j.ptr_off = uint32_t(ptrs.size());
    j.n_in = uint16_t(mp.inputs.size());
    j.n_out = uint16_t(mp.targets.size());
    for (uint16_t x : mp.inputs) ptrs.push_back(shards[i * total + x]);
    for (uint16_t t : mp.targets) ptrs.push_back(shards[i * total + t]);
    jobs.push_back(j);
    tbl_off.push_back(map_off[d]);
  }
  return c.apply_with_tables(jobs, tbl_off, ptrs, tables, len, s);
}

}  // namespace

bool leopard_dense_due(Codec &c, const uint8_t *present, int goal, size_t len) {
  if (c.leo->field->bits != 8) return false;
  const size_t k = c.k, total = k + c.m;
  size_t targets = 0;
  for (size_t x = 0; x < total; ++x) targets += !present[x] && (goal == RSGPU_GOAL_ALL || x < k);
  if (!targets) return false;
  const std::string key = std::string(reinterpret_cast<const char *>(present), total) + char(goal);
  LeopardState &st = *c.leo;
  std::lock_guard<std::mutex> g(st.mu);
  return dense_due_locked(st, key, targets, total * len, len);
}

int leopard_reconstruct(Codec &c, size_t n, uint8_t *const *shards, const uint8_t *present, size_t len, int goal,
                        const uint8_t *required, size_t n_required, cudaStream_t s) {
  if (c.leo->field->bits == 8 && goal != RSGPU_GOAL_REQUIRED) {
    const int rc = reconstruct_dense8(c, n, shards, present, len, goal, s);
    if (rc != kDenseNotTaken) return rc;
  }
  return run_once(c, RSGPU_OP_RECONSTRUCT, n, shards, present, len, goal, required, n_required, nullptr, s);
}

// ====================================================================== mixed batches
int leopard_geometry(Codec &c, LeoGeometry *g) {
  if (!c.leo) return RSGPU_ERR_INVALID_ARGUMENT;
  const LeopardState &st = *c.leo;
  g->bits = st.field->bits;
  g->k = uint32_t(c.k);
  g->p = uint32_t(c.m);
  g->m = st.m;
  g->n = st.n;
  g->mtrunc = st.mtrunc;
  g->last = st.last;
  g->mod = st.field->host.mod;
  g->skew = st.field->d_skew;
  g->bank = st.field->d_bank;
  g->kbank = st.field->d_kbank;
  g->sktab = st.field->d_sktab;
  LeoArgs a{};
  a.m = st.m;
  a.n = st.n;
  fill_stages(a);
  g->st_ienc = a.st_ienc;
  g->st_fenc = a.st_fenc;
  g->st_idec = a.st_idec;
  g->st_fdec = a.st_fdec;
  g->n_ienc = a.n_ienc;
  g->n_fenc = a.n_fenc;
  g->n_idec = a.n_idec;
  g->n_fdec = a.n_fdec;
  return RSGPU_OK;
}

int leopard_locators(Codec &c, size_t n, const uint8_t *present, uint16_t *dst, const uint16_t **err,
                     uint32_t *input_count, cudaStream_t s, bool ordered) {
  LeopardState &st = *c.leo;
  const size_t total = c.k + c.m;
  std::lock_guard<std::mutex> g(st.mu);
  ++st.build_seq;
  std::vector<std::pair<std::string, const uint8_t *>> pending;
  std::vector<LeoPlan *> used;
  std::unordered_map<LeoPlan *, uint32_t> slot;
  std::vector<uint32_t> slot_of(n, 0);
  int bad = RSGPU_OK;
  for (size_t i = 0; i < n && bad == RSGPU_OK; ++i) {
    LeoPlan *p = nullptr;
    bad = decode_plan(c, present + i * total, &p, s, pending);
    if (bad) break;
    auto sl = slot.emplace(p, uint32_t(used.size()));
    if (sl.second) used.push_back(p);
    slot_of[i] = sl.first->second;
    input_count[i] = p->input_count;
  }
  int rc = build_locators(c, pending, s);  // plans already cached get their locators even on an error
  if (!rc) rc = bad;
  if (!rc) rc = copy_locators(st, used, dst, s, ordered);
  if (rc) return rc;
  for (size_t i = 0; i < n; ++i) err[i] = dst + size_t(slot_of[i]) * st.n;
  return RSGPU_OK;
}

void leopard_cache_stats(Codec &c, rsgpu_cache_stats *out) {
  LeopardState &st = *c.leo;
  std::lock_guard<std::mutex> g(st.mu);
  *out = st.plan_stats;
  out->entries = st.plans.size();
  out->retained_bytes = st.plans.size() * st.plan_block;
}

const uint8_t (*leopard_mul8())[256] {
  static uint8_t mul[256][256];
  static std::once_flag once;
  std::call_once(once, [] {
    LeoField *f = nullptr;
    if (leo_field(8, &f) != RSGPU_OK) return;
    const LeoTables &t = f->host;
    for (uint32_t a = 0; a < 256; ++a)
      for (uint32_t b = 0; b < 256; ++b)
        mul[a][b] = (a && b) ? uint8_t(t.exp[t.add_mod(t.log[a], t.log[b])]) : 0;
  });
  return mul;
}

namespace {

// The element whose log is 0 (the multiplicative identity of the Leopard
// field's representation).
uint8_t leo8_one() {
  LeoField *f = nullptr;
  leo_field(8, &f);
  return uint8_t(f->host.exp[0]);
}

}  // namespace

int leopard_dense_encode(Codec &c, std::vector<uint8_t> &rows) {
  LeopardState &st = *c.leo;
  if (st.field->bits != 8) return RSGPU_ERR_INVALID_ARGUMENT;
  {
    std::lock_guard<std::mutex> g(st.mu);
    if (!st.dense_enc.empty()) {
      rows = st.dense_enc;
      return RSGPU_OK;
    }
  }
  // Encode the unit vectors: data shard j holds the identity element at
  // column j, so parity shard r column j is coefficient (r, j) of the map.
  const size_t k = c.k, m = c.m, total = k + m;
  const size_t L = (k + 63) / 64 * 64;
  std::vector<uint8_t> host(total * L, 0);
  const uint8_t one = leo8_one();
  for (size_t j = 0; j < k; ++j) host[j * L + j] = one;
  cudaStream_t s = nullptr;
  RS_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  uint8_t *d = nullptr;
  int rc = cuda_status(cudaError_t(lib_malloc_async(reinterpret_cast<void **>(&d), host.size(), s)));
  if (rc == RSGPU_OK) rc = cuda_status(cudaMemcpyAsync(d, host.data(), host.size(), cudaMemcpyHostToDevice, s));
  std::vector<uint8_t *> ptrs(total);
  for (size_t i = 0; i < total; ++i) ptrs[i] = d + i * L;
  if (rc == RSGPU_OK) rc = run_once(c, RSGPU_OP_ENCODE, 1, ptrs.data(), nullptr, L, 0, nullptr, 0, nullptr, s);
  if (rc == RSGPU_OK) rc = cuda_status(cudaMemcpyAsync(host.data(), d, host.size(), cudaMemcpyDeviceToHost, s));
  if (d) cudaFreeAsync(d, s);
  if (cudaStreamSynchronize(s) != cudaSuccess && rc == RSGPU_OK) rc = RSGPU_ERR_CUDA;
  cudaStreamDestroy(s);
  if (rc) return rc;
  rows.assign(m * k, 0);
  for (size_t r = 0; r < m; ++r)
    for (size_t j = 0; j < k; ++j) rows[r * k + j] = host[(k + r) * L + j];
  std::vector<uint32_t> packed(packed_table_words(m, k));
  pack_tables_with(leopard_mul8(), rows.data(), m, k, packed.data());
  uint32_t *d_tbl = nullptr;
  RS_CUDA(cudaMalloc(&d_tbl, packed.size() * 4));
  RS_CUDA(cudaMemcpy(d_tbl, packed.data(), packed.size() * 4, cudaMemcpyHostToDevice));
  std::lock_guard<std::mutex> g(st.mu);
  if (!st.dense_enc.empty()) {  // another thread finished first
    cudaFree(d_tbl);
    return RSGPU_OK;
  }
  st.dense_enc = rows;
  st.d_dense_enc = d_tbl;
  return RSGPU_OK;
}

namespace {

// Maps are derived with one FFT decode over unit-vector stripes: the q-th
// present shard of pattern i holds the identity element at column q, so
// target t column q of the decoded stripes is coefficient (t, q) of that
// pattern's map.  dense_layout fills every map's inputs and targets and
// returns the column count L (the widest map's inputs, in 64-byte blocks);
// dense_units writes the unit vectors into a host image of n stripes;
// dense_extract reads the coefficients back out and packs the K1 tables.
size_t dense_layout(const Codec &c, size_t n, const uint8_t *present, int goal, std::vector<LeoDenseMap> &maps) {
  const size_t k = c.k, total = k + c.m;
  maps.assign(n, LeoDenseMap{});
  size_t max_in = 1;
  for (size_t i = 0; i < n; ++i) {
    const uint8_t *pr = present + i * total;
    LeoDenseMap &mp = maps[i];
    for (size_t x = 0; x < total; ++x) {
      if (pr[x])
        mp.inputs.push_back(uint16_t(x));
      else if (goal == RSGPU_GOAL_ALL || x < k)
        mp.targets.push_back(uint16_t(x));
    }
    max_in = std::max(max_in, mp.inputs.size());
  }
  return (max_in + 63) / 64 * 64;
}

void dense_units(const Codec &c, const std::vector<LeoDenseMap> &maps, size_t L, uint8_t *host) {
  const size_t total = c.k + c.m;
  std::memset(host, 0, maps.size() * total * L);
  const uint8_t one = leo8_one();
  for (size_t i = 0; i < maps.size(); ++i)
    for (size_t q = 0; q < maps[i].inputs.size(); ++q) host[(i * total + maps[i].inputs[q]) * L + q] = one;
}

void dense_extract(const Codec &c, std::vector<LeoDenseMap> &maps, size_t L, const uint8_t *host) {
  const size_t total = c.k + c.m;
  for (size_t i = 0; i < maps.size(); ++i) {
    LeoDenseMap &mp = maps[i];
    const size_t ni = mp.inputs.size(), nt = mp.targets.size();
    mp.rows.assign(nt * ni, 0);
    for (size_t t = 0; t < nt; ++t)
      for (size_t q = 0; q < ni; ++q) mp.rows[t * ni + q] = host[(i * total + mp.targets[t]) * L + q];
    auto packed = std::make_shared<std::vector<uint32_t>>(packed_table_words(nt, ni));
    pack_tables_with(leopard_mul8(), mp.rows.data(), nt, ni, packed->data());
    mp.packed = std::move(packed);
  }
}

// Derives the maps of n patterns (one FFT decode, stream-ordered on s; the
// host waits for s only, to read the maps back).
int derive_dense8(Codec &c, size_t n, const uint8_t *present, int goal, std::vector<LeoDenseMap> &maps,
                  cudaStream_t s) {
  const size_t total = c.k + c.m;
  const size_t L = dense_layout(c, n, present, goal, maps);
  std::vector<uint8_t> host(n * total * L, 0);
  dense_units(c, maps, L, host.data());
  uint8_t *d = nullptr;
  RS_CUDA(cudaError_t(lib_malloc_async(reinterpret_cast<void **>(&d), host.size(), s)));
  int rc = cuda_status(cudaMemcpyAsync(d, host.data(), host.size(), cudaMemcpyHostToDevice, s));
  std::vector<uint8_t *> ptrs(n * total);
  for (size_t i = 0; i < n * total; ++i) ptrs[i] = d + i * L;
  if (rc == RSGPU_OK) rc = run_once(c, RSGPU_OP_RECONSTRUCT, n, ptrs.data(), present, L, goal, nullptr, 0, nullptr, s);
  if (rc == RSGPU_OK) rc = cuda_status(cudaMemcpyAsync(host.data(), d, host.size(), cudaMemcpyDeviceToHost, s));
  cudaFreeAsync(d, s);
  if (cudaStreamSynchronize(s) != cudaSuccess && rc == RSGPU_OK) rc = RSGPU_ERR_CUDA;
  if (rc) return rc;
  dense_extract(c, maps, L, host.data());
  return RSGPU_OK;
}

// Adds derived maps to the codec's map cache (least recently used out
// beyond kDenseCacheBytes).  Caller holds st.mu.
void dense_insert_locked(LeopardState &st, const std::string &key, LeoDenseMap &&map) {
  if (st.dense_index.count(key)) return;
  const size_t bytes = key.size() + map.rows.size() + map.packed->size() * 4 +
                       (map.inputs.size() + map.targets.size()) * 2;
  st.dense_lru.push_front({key, std::make_shared<const LeoDenseMap>(std::move(map)), bytes});
  st.dense_index.emplace(key, st.dense_lru.begin());
  st.dense_bytes += bytes;
  while (st.dense_bytes > kDenseCacheBytes && st.dense_lru.size() > 1) {
    auto &old = st.dense_lru.back();
    st.dense_bytes -= old.bytes;
    st.dense_index.erase(old.key);
    st.dense_lru.pop_back();
  }
}

std::string dense_key(const Codec &c, const uint8_t *present, int goal) {
  return std::string(reinterpret_cast<const char *>(present), c.k + c.m) + char(goal);
}

}  // namespace

int leopard_dense_decode(Codec &c, size_t n, const uint8_t *present, int goal, std::vector<LeoDenseMap> &maps,
                         cudaStream_t s) {
  LeopardState &st = *c.leo;
  if (st.field->bits != 8) return RSGPU_ERR_INVALID_ARGUMENT;
  const size_t total = c.k + c.m;
  maps.assign(n, LeoDenseMap{});
  std::vector<size_t> miss;
  {
    std::lock_guard<std::mutex> g(st.mu);
    for (size_t i = 0; i < n; ++i) {
      auto it = st.dense_index.find(dense_key(c, present + i * total, goal));
      if (it == st.dense_index.end()) {
        miss.push_back(i);
        continue;
      }
      st.dense_lru.splice(st.dense_lru.begin(), st.dense_lru, it->second);
      maps[i] = *it->second->map;
    }
  }
  if (miss.empty()) return RSGPU_OK;
  std::vector<uint8_t> pres(miss.size() * total);
  for (size_t x = 0; x < miss.size(); ++x) std::memcpy(&pres[x * total], present + miss[x] * total, total);
  std::vector<LeoDenseMap> got;
  const int rc = derive_dense8(c, miss.size(), pres.data(), goal, got, s);
  if (rc) return rc;
  std::lock_guard<std::mutex> g(st.mu);
  for (size_t x = 0; x < miss.size(); ++x) {
    maps[miss[x]] = got[x];
    dense_insert_locked(st, dense_key(c, &pres[x * total], goal), std::move(got[x]));
  }
  return RSGPU_OK;
}

bool leopard_dense_cached(Codec &c, const uint8_t *present, int goal) {
  LeopardState &st = *c.leo;
  std::lock_guard<std::mutex> g(st.mu);
  return st.dense_index.count(dense_key(c, present, goal)) != 0;
}

size_t leopard_dense_derive_bytes(Codec &c, const uint8_t *present, int goal) {
  std::vector<LeoDenseMap> maps;
  return dense_layout(c, 1, present, goal, maps) * (c.k + c.m);
}

int leopard_dense_derive_start(Codec &c, const uint8_t *present, int goal, uint8_t *pinned, cudaStream_t s,
                               DenseDerivation &d) {
  if (c.leo->field->bits != 8) return RSGPU_ERR_INVALID_ARGUMENT;
  const size_t total = c.k + c.m;
  std::vector<LeoDenseMap> maps;
  d.codec = &c;
  d.goal = goal;
  d.pattern.assign(reinterpret_cast<const char *>(present), total);
  d.L = dense_layout(c, 1, present, goal, maps);
  d.bytes = total * d.L;
  d.pinned = pinned;
  dense_units(c, maps, d.L, pinned);
  RS_CUDA(cudaError_t(lib_malloc_async(reinterpret_cast<void **>(&d.dev), d.bytes, s)));
  RS_CUDA(cudaMemcpyAsync(d.dev, pinned, d.bytes, cudaMemcpyHostToDevice, s));
  std::vector<uint8_t *> ptrs(total);
  for (size_t i = 0; i < total; ++i) ptrs[i] = d.dev + i * d.L;
  int rc = run_once(c, RSGPU_OP_RECONSTRUCT, 1, ptrs.data(), present, d.L, goal, nullptr, 0, nullptr, s);
  if (rc) {
    cudaFreeAsync(d.dev, s);
    d.dev = nullptr;
    return rc;
  }
  RS_CUDA(cudaMemcpyAsync(pinned, d.dev, d.bytes, cudaMemcpyDeviceToHost, s));
  RS_CUDA(cudaFreeAsync(d.dev, s));
  d.dev = nullptr;
  RS_CUDA(cudaEventCreateWithFlags(&d.done, cudaEventDisableTiming));
  return cuda_status(cudaEventRecord(d.done, s));
}

int leopard_dense_derive_finish(DenseDerivation &d) {
  const cudaError_t e = cudaEventQuery(d.done);
  if (e == cudaErrorNotReady) return RSGPU_ERR_INVALID_ARGUMENT;
  cudaEventDestroy(d.done);
  d.done = nullptr;
  if (e != cudaSuccess) return cuda_status(e);
  Codec &c = *d.codec;
  std::vector<LeoDenseMap> maps;
  dense_layout(c, 1, reinterpret_cast<const uint8_t *>(d.pattern.data()), d.goal, maps);
  dense_extract(c, maps, d.L, d.pinned);
  LeopardState &st = *c.leo;
  std::lock_guard<std::mutex> g(st.mu);
  dense_insert_locked(st, d.pattern + char(d.goal), std::move(maps[0]));
  return RSGPU_OK;
}

// ---------------------------------------------------------------- dense maps derived in stream order
namespace {

// Packs the K1 tables of one dense map on the device, in the layout of
// pack_tables_with (common.hpp: kTableWords words per group of four targets
// and input), from the decoded unit-vector stripe: coefficient (t, q) is
// byte q of shard targets[t].  One thread per table word.
__global__ void __launch_bounds__(256) k_pack_dense8(const uint8_t *units, uint32_t L, const uint16_t *targets,
                                                     uint32_t nt, uint32_t ni, const uint8_t *mul, uint32_t *out) {
  const uint32_t groups = (nt + 3) / 4;
  const uint64_t total = uint64_t(groups) * ni * kTableWords;
  for (uint64_t x = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; x < total; x += uint64_t(gridDim.x) * blockDim.x) {
    const uint32_t w = uint32_t(x % kTableWords);
    const uint64_t gj = x / kTableWords;
    const uint32_t j = uint32_t(gj % ni), g = uint32_t(gj / ni);
    uint32_t word = 0;
    for (uint32_t r = 0; r < 4; ++r) {
      const uint32_t o = g * 4 + r;
      if (o >= nt) break;
      const uint8_t *row = mul + uint32_t(units[size_t(targets[o]) * L + j]) * 256;
      if (w < 16)
        word |= uint32_t(row[w]) << (8 * r);
      else if (w < 32)
        word |= uint32_t(row[(w - 16) << 4]) << (8 * r);
      else if (w < 64)
        word |= uint32_t(row[w - 32]) << (8 * r);
      else if (((w - 64) >> 1) == r) {
        const uint32_t h0 = 4 * ((w - 64) & 1);
        for (uint32_t b = 0; b < 4; ++b) word |= uint32_t(row[(h0 + b) << 5]) << (8 * b);
      }
    }
    out[x] = word;
  }
}

}  // namespace

// Bytes of the device image leopard_dense_inline works in: the unit-vector
// stripe (k + m shards of L = the inputs rounded up to 64 bytes) and the
// target list.
size_t leopard_dense_inline_bytes(Codec &c, const uint8_t *present, int goal) {
  std::vector<LeoDenseMap> maps;
  const size_t L = dense_layout(c, 1, present, goal, maps);
  return (c.k + c.m) * L + ((maps[0].targets.size() * 2 + 15) & ~size_t(15)) + 16;
}

int leopard_dense_inline(Codec &c, const uint8_t *present, int goal, uint8_t *d_img, uint32_t *d_tbl,
                         std::vector<uint16_t> &inputs, std::vector<uint16_t> &targets, cudaStream_t s) {
  LeopardState &st = *c.leo;
  if (st.field->bits != 8) return RSGPU_ERR_INVALID_ARGUMENT;
  const size_t total = c.k + c.m;
  std::vector<LeoDenseMap> maps;
  const size_t L = dense_layout(c, 1, present, goal, maps);
  inputs = maps[0].inputs;
  targets = maps[0].targets;
  if (targets.empty()) return RSGPU_OK;
  const size_t units = total * L;
  std::vector<uint8_t> host(leopard_dense_inline_bytes(c, present, goal), 0);
  dense_units(c, maps, L, host.data());
  std::memcpy(host.data() + units, targets.data(), targets.size() * 2);
  int rc = upload_to(d_img, host.data(), host.size(), s);
  if (rc) return rc;
  std::vector<uint8_t *> ptrs(total);
  for (size_t i = 0; i < total; ++i) ptrs[i] = d_img + i * L;
  // The FFT decode of the unit vectors (the pattern's own transform), then
  // the packing, both queued on s ahead of the batch that applies the map.
  rc = run_once(c, RSGPU_OP_RECONSTRUCT, 1, ptrs.data(), present, L, goal, nullptr, 0, nullptr, s);
  if (rc) return rc;
  const uint64_t words = packed_table_words(targets.size(), inputs.size());
  const int grid = int(std::min<uint64_t>((words + 255) / 256, uint64_t(sm_count()) * 8));
  k_pack_dense8<<<grid, 256, 0, s>>>(d_img, uint32_t(L), reinterpret_cast<const uint16_t *>(d_img + units),
                                     uint32_t(targets.size()), uint32_t(inputs.size()), st.field->d_mul8, d_tbl);
  launch_counter_add(1);
  return cuda_status(cudaGetLastError());
}

// ====================================================================== no allocation
// Reconstruction for callers that cannot allocate device memory: the work
// rows, the pointer table, the presence/role flags, the error locators and the
// job descriptor live in file-scope static device arrays instead of
// allocations.  Host code never hands these names to a kernel (in host code
// they are stand-ins, not device addresses): set-up resolves each one with
// cudaGetSymbolAddress once per device, with that device current, and the
// kernels receive the resolved pointers.
namespace {

constexpr size_t kNaLanes = RSGPU_NOALLOC_MAX_LANES;
constexpr size_t kNaScratchWords = RSGPU_NOALLOC_SCRATCH_BYTES / 4;
static_assert(RSGPU_NOALLOC_SCRATCH_BYTES >= kNaLanes * 64, "one CTA at the lane limit must fit");

static __device__ __align__(256) uint32_t na_scratch[kNaScratchWords];  // work rows, one region per CTA
static __device__ __align__(256) const uint8_t *na_ptrs[kNaLanes];      // shard pointers (k + p <= lanes)
static __device__ __align__(256) uint8_t na_present[kNaLanes];
static __device__ __align__(256) uint8_t na_role[kNaLanes];
static __device__ __align__(256) uint16_t na_err[kNaLanes];
static __device__ __align__(256) LeoJob na_job;
static __device__ __align__(256) const uint8_t *na_present_ref[1];
static __device__ __align__(256) uint16_t *na_err_ref[1];

struct NaDevice {
  bool ready = false;
  uint32_t *scratch = nullptr;
  const uint8_t **ptrs = nullptr;
  uint8_t *present = nullptr, *role = nullptr;
  uint16_t *err = nullptr;
  LeoJob *job = nullptr;
  const uint8_t *const *present_ref = nullptr;
  uint16_t *const *err_ref = nullptr;
};

constexpr int kNaMaxDevices = 64;
NaDevice na_dev[kNaMaxDevices];
std::mutex na_mu;
// Host-side staging: static arrays, so a call allocates no host memory either.
// Copies from them are issued from pageable memory, which the driver consumes
// before cudaMemcpyAsync returns, so the next call may overwrite them at once.
const uint8_t *na_h_ptrs[kNaLanes];
uint8_t na_h_present[kNaLanes];
uint8_t na_h_role[kNaLanes];
LeoJob na_h_job;

int na_setup(int dev, NaDevice &d) {
  void *p = nullptr;
  RS_CUDA(cudaGetSymbolAddress(&p, na_scratch));
  d.scratch = static_cast<uint32_t *>(p);
  RS_CUDA(cudaGetSymbolAddress(&p, na_ptrs));
  d.ptrs = static_cast<const uint8_t **>(p);
  RS_CUDA(cudaGetSymbolAddress(&p, na_present));
  d.present = static_cast<uint8_t *>(p);
  RS_CUDA(cudaGetSymbolAddress(&p, na_role));
  d.role = static_cast<uint8_t *>(p);
  RS_CUDA(cudaGetSymbolAddress(&p, na_err));
  d.err = static_cast<uint16_t *>(p);
  RS_CUDA(cudaGetSymbolAddress(&p, na_job));
  d.job = static_cast<LeoJob *>(p);
  RS_CUDA(cudaGetSymbolAddress(&p, na_present_ref));
  d.present_ref = static_cast<const uint8_t *const *>(p);
  RS_CUDA(cudaGetSymbolAddress(&p, na_err_ref));
  d.err_ref = static_cast<uint16_t *const *>(p);
  // The locator kernel reads its pattern and output through one-entry
  // pointer arrays; point them at the static presence and locator arrays.
  const uint8_t *pres = d.present;
  uint16_t *err = d.err;
  RS_CUDA(cudaMemcpy(const_cast<const uint8_t **>(d.present_ref), &pres, sizeof(pres), cudaMemcpyHostToDevice));
  RS_CUDA(cudaMemcpy(const_cast<uint16_t **>(d.err_ref), &err, sizeof(err), cudaMemcpyHostToDevice));
  // The GF(2^16) locator needs 128 KiB of dynamic shared memory (raised once
  // per device here, not at every call).
  RS_CUDA(ensure_smem_limit(reinterpret_cast<const void *>(k_leo_locator<16>), size_t(1u << 16) * 2));
  (void)dev;
  d.ready = true;
  return RSGPU_OK;
}

}  // namespace

int leopard_reconstruct_noalloc(Codec &c, uint8_t *const *shards, const uint8_t *present, size_t len,
                                cudaStream_t s) {
  LeopardState &st = *c.leo;
  const size_t total = c.k + c.m;
  if (st.n > kNaLanes || total > kNaLanes) return RSGPU_ERR_SCRATCH_LIMIT;
  size_t np = 0;
  for (size_t i = 0; i < total; ++i) np += present[i] ? 1 : 0;
  if (np == total) return RSGPU_OK;
  if (total - np > c.m) return RSGPU_ERR_TOO_FEW_SHARDS_PRESENT;
  if (c.device < 0 || c.device >= kNaMaxDevices) return RSGPU_ERR_INVALID_ARGUMENT;
  int prev = 0;
  RS_CUDA(cudaGetDevice(&prev));
  if (prev != c.device) RS_CUDA(cudaSetDevice(c.device));
  std::lock_guard<std::mutex> g(na_mu);
  NaDevice &d = na_dev[c.device];
  int rc = d.ready ? RSGPU_OK : na_setup(c.device, d);
  if (rc == RSGPU_OK) {
    uint32_t input_count = st.m;
    for (size_t i = 0; i < total; ++i) {
      na_h_ptrs[i] = shards[i];
      na_h_present[i] = present[i] ? 1 : 0;
      na_h_role[i] = present[i] ? 1 : 2;
      if (i < c.k && present[i]) input_count = uint32_t(st.m + i + 1);
    }
    na_h_job = LeoJob{};
    na_h_job.err = d.err;
    na_h_job.role = d.role;
    na_h_job.input_count = input_count;
    cudaError_t e = cudaMemcpyAsync(d.ptrs, na_h_ptrs, total * sizeof(void *), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d.present, na_h_present, total, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d.role, na_h_role, total, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d.job, &na_h_job, sizeof(LeoJob), cudaMemcpyHostToDevice, s);
    rc = cuda_status(e);
  }
  if (rc == RSGPU_OK) {
    // Error locators for this pattern (K7a) into the static locator array;
    // every entry the decode reads (indices < n) is rewritten.
    const int bits = st.field->bits;
    const size_t lsmem = size_t(1u << bits) * 2;
    if (bits == 16) {
      k_leo_locator<16><<<1, 1024, lsmem, s>>>(d.present_ref, d.err_ref, st.field->d_walsh, uint32_t(c.k),
                                               uint32_t(c.m), st.m, st.n);
    } else {
      k_leo_locator<8><<<1, 256, lsmem, s>>>(d.present_ref, d.err_ref, st.field->d_walsh, uint32_t(c.k),
                                             uint32_t(c.m), st.m, st.n);
    }
    LeoArgs a{};
    a.jobs = d.job;
    a.ptrs = d.ptrs;
    a.skew = st.field->d_skew;
    a.bank = st.field->d_bank;
    a.scratch = d.scratch;
    a.len = len;
    a.n_jobs = 1;
    a.k = uint32_t(c.k);
    a.p = uint32_t(c.m);
    a.m = st.m;
    a.n = st.n;
    a.mtrunc = st.mtrunc;
    a.last = st.last;
    a.nb = 1;
    a.lanes = st.n;
    a.mod = st.field->host.mod;
    // Every row a CTA reads is written first (step 1 loads or zeroes all n
    // rows of its region), so the scratch needs no clearing between calls.
    const uint64_t tiles = len / 64;
    const uint64_t slots = kNaScratchWords / (uint64_t(st.n) * kRowWords);
    const int grid = int(std::min<uint64_t>(tiles, std::min<uint64_t>(slots, 4 * uint64_t(sm_count()))));
    if (bits == 16)
      k_leo_decode<16, true><<<grid, kLeoThreads, 0, s>>>(a);
    else
      k_leo_decode<8, true><<<grid, kLeoThreads, 0, s>>>(a);
    launch_counter_add(2);
    rc = cuda_status(cudaGetLastError());
  }
  if (prev != c.device) cudaSetDevice(prev);
  return rc;
}

}  // namespace rsgpu
