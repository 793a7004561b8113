// tower.cu -- classic Reed-Solomon over the GF((2^8)^2) tower field
// (galois_16::ReedSolomon, src/galois_16.rs) on sm_100a.
//
// An element x*X + c is stored as the byte pair [x, c].  Multiplying by a
// constant [cx, cc] is linear over the two byte planes:
//   out_x = (cc + 2cx) x + cx c,   out_c = 128cx x + cc c   (X^2 = 2X + 128),
// so a coefficient becomes four GF(2^8) constants.  The kernel packs, for two
// outputs r0 and r1, the x-byte contributions (out_x r0, out_c r0, out_x r1,
// out_c r1) into one table word and the c-byte contributions into another;
// four nibble lookups per element (warp shuffles, as in the GF(2^8) matrix
// apply) then produce both outputs of that element at once.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "codec.hpp"
#include "launch_cfg.hpp"
#include "leopard.hpp"

namespace rsgpu {

#define RS_CUDA(expr)                              \
  do {                                             \
    cudaError_t e_ = (expr);                       \
    if (e_ != cudaSuccess) return cuda_status(e_); \
  } while (0)

namespace {

constexpr int kTowerWords = 64;  // per (output pair, input): x lo, x hi, c lo, c hi

__device__ __forceinline__ uint32_t tshfl(uint32_t table, uint32_t idx) {
  uint32_t r;
  asm("shfl.sync.idx.b32 %0, %1, %2, 31, -1;" : "=r"(r) : "r"(table), "r"(idx));
  return r;
}

// Tables of one (pair, input): lanes hold entry (lane & 15) of each.
struct TT {
  uint32_t xl, xh, cl, ch;
};

// Word w holds elements e0 = bytes 0,1 and e1 = bytes 2,3 ([x, c] each).
__device__ __forceinline__ void mac_tower(uint32_t w, const TT &t, uint32_t &a0, uint32_t &a1) {
  a0 ^= tshfl(t.xl, w) ^ tshfl(t.xh, w >> 4) ^ tshfl(t.cl, w >> 8) ^ tshfl(t.ch, w >> 12);
  a1 ^= tshfl(t.xl, w >> 16) ^ tshfl(t.xh, w >> 20) ^ tshfl(t.cl, w >> 24) ^ tshfl(t.ch, w >> 28);
}

template <bool VERIFY>
__global__ void __launch_bounds__(256) k_apply_tower(ApplyArgs a) {
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t tile = 256 * 16;
  const uint32_t tiles_per_job = uint32_t((a.len + tile - 1) / tile);
  const uint32_t total = tiles_per_job * a.n_jobs;
  for (uint32_t t = blockIdx.x; t < total; t += gridDim.x) {
    const uint32_t job = t / tiles_per_job;
    const JobDesc d = a.jobs[job];
    const uint64_t col = uint64_t(t - job * tiles_per_job) * tile + threadIdx.x * 16ull;
    const bool vec = col + 16 <= d.vec_len;
    const uint8_t *const *ptr = a.ptrs + d.ptr_off;
    for (uint32_t g = 0; g * 2 < d.n_out; ++g) {
      uint32_t acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      for (uint32_t j = 0; j < d.n_in; ++j) {
        uint4 x = make_uint4(0, 0, 0, 0);
        if (vec) {
          x = __ldg(reinterpret_cast<const uint4 *>(ptr[j] + col));
        } else if (col < a.len) {
          // Tail: assemble the vector bytewise (shard lengths are even).
          uint8_t b[16];
          for (int i = 0; i < 16; ++i) b[i] = col + i < a.len ? ptr[j][col + i] : 0;
          std::memcpy(&x, b, 16);
        }
        const uint32_t *tb = d.tbl + (g * d.n_in + j) * kTowerWords;
        const TT tt{__ldg(tb + (lane & 15)), __ldg(tb + 16 + (lane & 15)), __ldg(tb + 32 + (lane & 15)),
                    __ldg(tb + 48 + (lane & 15))};
        mac_tower(x.x, tt, acc[0], acc[1]);
        mac_tower(x.y, tt, acc[2], acc[3]);
        mac_tower(x.z, tt, acc[4], acc[5]);
        mac_tower(x.w, tt, acc[6], acc[7]);
      }
      bool bad = false;
      for (uint32_t r = 0; r < 2 && g * 2 + r < d.n_out; ++r) {
        const uint32_t sel = r == 0 ? 0x5410 : 0x7632;
        uint4 o = make_uint4(__byte_perm(acc[0], acc[1], sel), __byte_perm(acc[2], acc[3], sel),
                             __byte_perm(acc[4], acc[5], sel), __byte_perm(acc[6], acc[7], sel));
        uint8_t *dst = const_cast<uint8_t *>(ptr[d.n_in + g * 2 + r]) + col;
        if (vec) {
          if (VERIFY) {
            uint4 e = *reinterpret_cast<const uint4 *>(dst);
            bad |= (e.x != o.x) | (e.y != o.y) | (e.z != o.z) | (e.w != o.w);
          } else if (a.accumulate) {  // incremental parity update
            const uint4 e = *reinterpret_cast<const uint4 *>(dst);
            *reinterpret_cast<uint4 *>(dst) = make_uint4(o.x ^ e.x, o.y ^ e.y, o.z ^ e.z, o.w ^ e.w);
          } else {
            *reinterpret_cast<uint4 *>(dst) = o;
          }
        } else if (col < a.len) {
          uint8_t b[16];
          std::memcpy(b, &o, 16);
          for (int i = 0; i < 16 && col + i < a.len; ++i) {
            if (VERIFY)
              bad |= dst[i] != b[i];
            else if (a.accumulate)
              dst[i] ^= b[i];
            else
              dst[i] = b[i];
          }
        }
      }
      if (VERIFY && bad) atomicOr(a.flags + d.flag_idx, 1u);
    }
  }
}

// Host packing: rows is n_out x n_in tower coefficients.
void pack_tower(const T16 *rows, size_t n_out, size_t n_in, uint32_t *out) {
  const Gf8 &f = gf8();
  const size_t pairs = (n_out + 1) / 2;
  for (size_t g = 0; g < pairs; ++g)
    for (size_t j = 0; j < n_in; ++j) {
      uint32_t *t = out + (g * n_in + j) * kTowerWords;
      std::memset(t, 0, kTowerWords * 4);
      for (size_t r = 0; r < 2 && g * 2 + r < n_out; ++r) {
        const T16 co = rows[(g * 2 + r) * n_in + j];
        const uint8_t A = co.c ^ f.mul[2][co.x], B = co.x, C = f.mul[128][co.x], D = co.c;
        for (unsigned n = 0; n < 16; ++n) {
          const unsigned sh = 16 * unsigned(r);
          t[n] |= (uint32_t(f.mul[A][n]) | uint32_t(f.mul[C][n]) << 8) << sh;
          t[16 + n] |= (uint32_t(f.mul[A][n << 4]) | uint32_t(f.mul[C][n << 4]) << 8) << sh;
          t[32 + n] |= (uint32_t(f.mul[B][n]) | uint32_t(f.mul[D][n]) << 8) << sh;
          t[48 + n] |= (uint32_t(f.mul[B][n << 4]) | uint32_t(f.mul[D][n << 4]) << 8) << sh;
        }
      }
    }
}

size_t tower_words(size_t n_out, size_t n_in) { return ((n_out + 1) / 2) * n_in * kTowerWords; }

}  // namespace

struct TowerState {
  uint32_t *enc = nullptr;
  std::mutex mu;
  std::unordered_map<std::string, uint32_t *> decode;  // pattern -> device tables
  ~TowerState() {
    cudaDeviceSynchronize();
    if (enc) cudaFree(enc);
    for (auto &kv : decode) cudaFree(kv.second);
  }
};

static TowerState *tower_state(const Codec &c) { return c.tower.get(); }

int Codec::init_tower(const uint8_t *custom_rows) {
  RS_CUDA(cudaGetDevice(&device));
  if (custom_rows) {
    // src/core/codec.rs:546-615 (with_custom_matrix): identity on top, the
    // caller's m x k rows ([X coefficient, constant] per element) below.
    tmatrix.assign((k + m) * k, T16{0, 0});
    for (size_t i = 0; i < k; ++i) tmatrix[i * k + i] = T16{0, 1};
    for (size_t r = 0; r < m; ++r)
      for (size_t j = 0; j < k; ++j)
        tmatrix[(k + r) * k + j] = T16{custom_rows[2 * (r * k + j)], custom_rows[2 * (r * k + j) + 1]};
  } else {
    int rc = build_tower_matrix(k, m, tmatrix);
    if (rc) return rc;
  }
  auto st = std::make_shared<TowerState>();
  std::vector<uint32_t> packed(tower_words(m, k));
  pack_tower(&tmatrix[k * k], m, k, packed.data());
  RS_CUDA(cudaMalloc(&st->enc, packed.size() * 4));
  RS_CUDA(cudaMemcpy(st->enc, packed.data(), packed.size() * 4, cudaMemcpyHostToDevice));
  tower = st;
  return RSGPU_OK;
}

static int launch_tower(const std::vector<JobDesc> &jobs, const std::vector<const uint8_t *> &ptrs, size_t len,
                        bool verify, uint32_t *flags, cudaStream_t s, bool accumulate = false) {
  if (jobs.empty()) return RSGPU_OK;
  std::vector<JobDesc> js = jobs;
  for (auto &j : js) {
    bool aligned = true;
    for (uint32_t i = 0; i < uint32_t(j.n_in) + j.n_out; ++i)
      aligned &= (reinterpret_cast<uintptr_t>(ptrs[j.ptr_off + i]) & 15) == 0;
    j.vec_len = aligned ? (len & ~uint64_t(15)) : 0;
  }
  const size_t jb = js.size() * sizeof(JobDesc);
  std::vector<uint8_t> blob(jb + ptrs.size() * sizeof(void *));
  std::memcpy(blob.data(), js.data(), jb);
  std::memcpy(blob.data() + jb, ptrs.data(), ptrs.size() * sizeof(void *));
  void *d = nullptr;
  RS_CUDA(cudaMalloc(&d, blob.size()));
  RS_CUDA(cudaMemcpy(d, blob.data(), blob.size(), cudaMemcpyHostToDevice));
  ApplyArgs a{};
  a.jobs = static_cast<const JobDesc *>(d);
  a.ptrs = reinterpret_cast<const uint8_t *const *>(static_cast<char *>(d) + jb);
  a.flags = flags;
  a.len = len;
  a.n_jobs = uint32_t(js.size());
  a.accumulate = accumulate ? 1 : 0;
  const uint64_t tiles = ((len + 4095) / 4096) * js.size();
  const int grid = int(std::min<uint64_t>(tiles, uint64_t(device_sm_count()) * 8));
  if (verify)
    k_apply_tower<true><<<grid, 256, 0, s>>>(a);
  else
    k_apply_tower<false><<<grid, 256, 0, s>>>(a);
  launch_counter_add(1);
  RS_CUDA(cudaGetLastError());
  RS_CUDA(cudaStreamSynchronize(s));
  cudaFree(d);
  return RSGPU_OK;
}

int tower_apply_columns(Codec &c, const std::vector<const uint8_t *> &inputs, const std::vector<size_t> &cols,
                        uint8_t *const *parity, size_t len, bool accumulate, cudaStream_t s) {
  if (inputs.empty()) return RSGPU_OK;
  const size_t k = c.k, m = c.m, n_in = inputs.size();
  std::vector<T16> rows(m * n_in);
  for (size_t r = 0; r < m; ++r)
    for (size_t j = 0; j < n_in; ++j) rows[r * n_in + j] = c.tmatrix[(k + r) * k + cols[j]];
  std::vector<uint32_t> packed(tower_words(m, n_in));
  pack_tower(rows.data(), m, n_in, packed.data());
  uint32_t *d_tbl = nullptr;
  RS_CUDA(cudaMalloc(&d_tbl, packed.size() * 4));
  RS_CUDA(cudaMemcpy(d_tbl, packed.data(), packed.size() * 4, cudaMemcpyHostToDevice));
  std::vector<JobDesc> jobs(1);
  jobs[0].n_in = uint16_t(n_in);
  jobs[0].n_out = uint16_t(m);
  jobs[0].tbl = d_tbl;
  std::vector<const uint8_t *> ptrs(inputs);
  for (size_t r = 0; r < m; ++r) ptrs.push_back(parity[r]);
  int rc = launch_tower(jobs, ptrs, len, false, nullptr, s, accumulate);
  cudaFree(d_tbl);
  return rc;
}

int tower_encode(Codec &c, size_t n, uint8_t *const *shards, size_t len, cudaStream_t s) {
  TowerState *st = tower_state(c);
  std::vector<JobDesc> jobs(n);
  std::vector<const uint8_t *> ptrs(shards, shards + n * (c.k + c.m));
  for (size_t i = 0; i < n; ++i) {
    jobs[i] = JobDesc{};
    jobs[i].ptr_off = uint32_t(i * (c.k + c.m));
    jobs[i].n_in = uint16_t(c.k);
    jobs[i].n_out = uint16_t(c.m);
    jobs[i].tbl = st->enc;
  }
  return launch_tower(jobs, ptrs, len, false, nullptr, s);
}

int tower_verify(Codec &c, size_t n, const uint8_t *const *shards, size_t len, uint8_t *ok, cudaStream_t s) {
  TowerState *st = tower_state(c);
  std::vector<JobDesc> jobs(n);
  std::vector<const uint8_t *> ptrs(shards, shards + n * (c.k + c.m));
  for (size_t i = 0; i < n; ++i) {
    jobs[i] = JobDesc{};
    jobs[i].ptr_off = uint32_t(i * (c.k + c.m));
    jobs[i].n_in = uint16_t(c.k);
    jobs[i].n_out = uint16_t(c.m);
    jobs[i].flag_idx = uint32_t(i);
    jobs[i].tbl = st->enc;
  }
  uint32_t *flags = nullptr;
  RS_CUDA(cudaMalloc(&flags, std::max<size_t>(n, 1) * 4));
  RS_CUDA(cudaMemset(flags, 0, std::max<size_t>(n, 1) * 4));
  int rc = launch_tower(jobs, ptrs, len, true, flags, s);
  std::vector<uint32_t> f(n);
  if (rc == RSGPU_OK) {
    RS_CUDA(cudaMemcpy(f.data(), flags, n * 4, cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < n; ++i) ok[i] = f[i] ? 0 : 1;
  }
  cudaFree(flags);
  return rc;
}

// Composed recovery rows over the first k present shards (the classic plan of
// src/core/recovery_plan.rs:262-517 in the tower field); tables cached per
// (pattern, targets).
int tower_reconstruct(Codec &c, size_t n, uint8_t *const *shards, const uint8_t *present, size_t len, int goal,
                      const uint8_t *required, size_t n_required, cudaStream_t s) {
  TowerState *st = tower_state(c);
  const size_t total = c.k + c.m;
  std::vector<JobDesc> jobs;
  std::vector<const uint8_t *> ptrs;
  std::lock_guard<std::mutex> g(st->mu);
  for (size_t i = 0; i < n; ++i) {
    ClassicPlan p;
    int rc = c.plan_classic(present + i * total, goal, required, n_required, p);
    if (rc) return rc;
    if (p.all_present || p.targets.empty()) continue;
    std::string key(reinterpret_cast<const char *>(p.survivors.data()), p.survivors.size() * 2);
    key.push_back('|');
    key.append(reinterpret_cast<const char *>(p.targets.data()), p.targets.size() * 2);
    uint32_t *tbl = nullptr;
    auto it = st->decode.find(key);
    if (it != st->decode.end()) {
      tbl = it->second;
    } else {
      const size_t k = c.k;
      std::vector<T16> dec(k * k);
      if (p.needs_inverse) {
        std::vector<T16> sel(k * k);
        for (size_t r = 0; r < k; ++r)
          for (size_t col = 0; col < k; ++col) sel[r * k + col] = c.tmatrix[p.survivors[r] * k + col];
        if (!t16_invert(k, sel.data(), dec.data())) return RSGPU_ERR_INVALID_CUSTOM_MATRIX;
      } else {
        for (size_t r = 0; r < k; ++r)
          for (size_t col = 0; col < k; ++col) dec[r * k + col] = T16{0, uint8_t(p.survivors[col] == r)};
      }
      std::vector<T16> rows(p.targets.size() * k);
      for (size_t t = 0; t < p.targets.size(); ++t) {
        const size_t idx = p.targets[t];
        for (size_t col = 0; col < k; ++col) {
          T16 acc{0, 0};
          if (idx < k) {
            acc = dec[idx * k + col];
          } else {
            for (size_t j = 0; j < k; ++j) {
              T16 pr = t16_mul(c.tmatrix[idx * k + j], dec[j * k + col]);
              acc.x ^= pr.x;
              acc.c ^= pr.c;
            }
          }
          rows[t * k + col] = acc;
        }
      }
      std::vector<uint32_t> packed(tower_words(p.targets.size(), k));
      pack_tower(rows.data(), p.targets.size(), k, packed.data());
      RS_CUDA(cudaMalloc(&tbl, packed.size() * 4));
      RS_CUDA(cudaMemcpy(tbl, packed.data(), packed.size() * 4, cudaMemcpyHostToDevice));
      st->decode.emplace(key, tbl);
    }
    JobDesc j{};
    j.ptr_off = uint32_t(ptrs.size());
    j.n_in = uint16_t(c.k);
    j.n_out = uint16_t(p.targets.size());
    j.tbl = tbl;
    for (uint16_t sv : p.survivors) ptrs.push_back(shards[i * total + sv]);
    for (uint16_t tg : p.targets) ptrs.push_back(shards[i * total + tg]);
    jobs.push_back(j);
  }
  return launch_tower(jobs, ptrs, len, false, nullptr, s);
}

// Prepared tower batches run through the per-call path (no graph capture).
int prepare_tower(Codec &, int, size_t, uint8_t *const *, const uint8_t *, size_t, int, uint32_t *,
                  std::shared_ptr<LeoLaunch> &) {
  return RSGPU_ERR_UNSUPPORTED_CODEC_FAMILY;
}

}  // namespace rsgpu
