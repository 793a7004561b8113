// k_classic.cu -- sm_100a kernels of the classic Reed-Solomon path.
//
// K1 (matrix apply): out[r] = sum_j c[r][j] * in[j] over GF(2^8), bytewise,
//   for encode, reconstruct (composed recovery rows) and verify (compare
//   instead of store).  It replaces the reference's row dot-product loops
//   (src/core/encode.rs:532-602, src/galois_8/x86/gfni_rows.rs:15-288).
//   Design: each thread owns 16 (or 32) byte columns of one stripe and reads
//   every input shard exactly once with coalesced 128-bit loads.  Products
//   are table lookups split over the bits of the data byte, and the tables of
//   four outputs are packed into one 32-bit word per entry, so one lookup
//   serves four parity rows.  Two formulations share the work so that
//   neither the shuffle (LSU) pipe nor the integer (ALU) pipe saturates:
//     4+4 split: two warp-shuffle lookups into 16-entry tables held one entry
//       per lane (mirrored into lanes 16..31, so the raw shifted data word is
//       a valid index: the shuffle only reads bits 0..4);
//     5+3 split: one shuffle into a 32-entry table for the low five bits and
//       one byte-permute (PRMT) per output for the high three bits, whose
//       eight-entry byte table fits the two PRMT source registers and whose
//       result lands directly in per-output column order.
//   All m outputs of a column are accumulated in registers and written once.
//
// K3 (decode tables): Gauss-Jordan inversion of the selected survivor rows,
//   composition of the requested parity rows and packing of the nibble
//   tables, one CTA per erasure pattern (src/core/reconstruct.rs:1068-1174,
//   src/core/recovery_plan.rs:425-517).
#include <cuda_runtime.h>

#include <cstdlib>

#include "common.hpp"
#include "kernels.hpp"

namespace rsgpu {

namespace {

__device__ __forceinline__ uint32_t tshfl(uint32_t table, uint32_t idx) {
  uint32_t r;
  asm("shfl.sync.idx.b32 %0, %1, %2, 31, -1;" : "=r"(r) : "r"(table), "r"(idx));
  return r;
}

// Accumulate the four columns of data word w into a[0..3] (four packed outputs each).
__device__ __forceinline__ void mac4(uint32_t w, uint32_t lo, uint32_t hi, uint32_t *a) {
  a[0] ^= tshfl(lo, w) ^ tshfl(hi, w >> 4);
  a[1] ^= tshfl(lo, w >> 8) ^ tshfl(hi, w >> 12);
  a[2] ^= tshfl(lo, w >> 16) ^ tshfl(hi, w >> 20);
  a[3] ^= tshfl(lo, w >> 24) ^ tshfl(hi, w >> 28);
}

// Transpose 4 columns x 4 packed outputs into 4 output words.
__device__ __forceinline__ void transpose4(const uint32_t *a, uint32_t *o) {
  uint32_t t0 = __byte_perm(a[0], a[1], 0x5140);
  uint32_t t1 = __byte_perm(a[2], a[3], 0x5140);
  uint32_t t2 = __byte_perm(a[0], a[1], 0x7362);
  uint32_t t3 = __byte_perm(a[2], a[3], 0x7362);
  o[0] = __byte_perm(t0, t1, 0x5410);
  o[1] = __byte_perm(t0, t1, 0x7632);
  o[2] = __byte_perm(t2, t3, 0x5410);
  o[3] = __byte_perm(t2, t3, 0x7632);
}

// 5+3 split, shuffle half: low five bits of each byte of w index t5.
__device__ __forceinline__ void mac4_lo5(uint32_t w, uint32_t t5, uint32_t *a) {
  a[0] ^= tshfl(t5, w);
  a[1] ^= tshfl(t5, w >> 8);
  a[2] ^= tshfl(t5, w >> 16);
  a[3] ^= tshfl(t5, w >> 24);
}

// 5+3 split, PRMT half: selector nibble c = high three bits of byte c of w.
__device__ __forceinline__ uint32_t hi3_selector(uint32_t w) {
  const uint32_t x = (w >> 5) & 0x07070707u;
  const uint32_t y = x | ((w >> 9) & 0x00707070u);
  return __byte_perm(y, 0, 0x3320);
}

__device__ __forceinline__ uint4 ld_stream(const uint8_t *p) {
  uint4 v;
  asm volatile("ld.global.nc.L1::no_allocate.v4.u32 {%0,%1,%2,%3}, [%4];"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "l"(p));
  return v;
}

__device__ __forceinline__ void st_stream(uint8_t *p, uint4 v) {
  asm volatile("st.global.L1::no_allocate.v4.u32 [%0], {%1,%2,%3,%4};" ::"l"(p), "r"(v.x), "r"(v.y),
               "r"(v.z), "r"(v.w)
               : "memory");
}


// One tile = kApplyThreads threads x V 128-bit vectors of columns of one job.
// NG = number of 4-output groups per pass (outputs g*4 .. g*4+3).
// MIX: 0 = every input uses the 4+4 split, 1 = odd inputs use 5+3, 2 = all 5+3.
template <int NG, int V, int kBatch, int MIX, bool VERIFY>
__global__ void __launch_bounds__(kApplyThreads) k_apply_vec(ApplyArgs a) {
  constexpr uint32_t kTile = kApplyThreads * kApplyVec * V;
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t tiles_per_job = uint32_t((a.len + kTile - 1) / kTile);
  const uint32_t total = tiles_per_job * a.n_jobs;
  for (uint32_t t = blockIdx.x; t < total; t += gridDim.x) {
    const uint32_t job = t / tiles_per_job;
    const uint64_t tile_base = uint64_t(t - job * tiles_per_job) * kTile;
    const JobDesc d = a.jobs[job];
    if (tile_base >= d.vec_len) continue;  // CTA-uniform
    // Thread column of vector v: tile_base + (v * kApplyThreads + tid) * 16, so a
    // warp's 32 loads of one vector cover 512 contiguous bytes.
    uint64_t col[V];
    bool active[V];
#pragma unroll
    for (int v = 0; v < V; ++v) {
      col[v] = tile_base + (uint64_t(v) * kApplyThreads + threadIdx.x) * kApplyVec;
      active[v] = col[v] < d.vec_len;
    }
    const uint8_t *const *ptr = a.ptrs + d.ptr_off;
    const uint32_t n_in = d.n_in;
    for (uint32_t g0 = 0; g0 * 4 < d.n_out; g0 += NG) {
      uint32_t acc[NG][V][16];   // per column: 4 packed outputs
      uint32_t oacc[NG][V][16];  // per output r, word w (index r*4+w): 4 columns
#pragma unroll
      for (int g = 0; g < NG; ++g)
#pragma unroll
        for (int v = 0; v < V; ++v)
#pragma unroll
          for (int i = 0; i < 16; ++i) acc[g][v][i] = oacc[g][v][i] = 0;
      for (uint32_t j0 = 0; j0 < n_in; j0 += kBatch) {
        uint4 x[kBatch][V];
#pragma unroll
        for (int b = 0; b < kBatch; ++b) {
          const uint8_t *src = (j0 + b < n_in) ? ptr[j0 + b] : nullptr;
#pragma unroll
          for (int v = 0; v < V; ++v) {
            x[b][v] = make_uint4(0, 0, 0, 0);
            if (src && active[v]) x[b][v] = ld_stream(src + col[v]);
          }
        }
#pragma unroll
        for (int b = 0; b < kBatch; ++b) {
          if (j0 + b >= n_in) break;  // warp-uniform
          const bool split53 = MIX == 2 || (MIX == 1 && (b & 1));  // compile-time
#pragma unroll
          for (int g = 0; g < NG; ++g) {
            const uint32_t *tb = d.tbl + ((g0 + g) * n_in + (j0 + b)) * kTableWords;
            if (!split53) {
              const uint32_t lo = __ldg(tb + (lane & 15));
              const uint32_t hi = __ldg(tb + 16 + (lane & 15));
#pragma unroll
              for (int v = 0; v < V; ++v) {
                mac4(x[b][v].x, lo, hi, &acc[g][v][0]);
                mac4(x[b][v].y, lo, hi, &acc[g][v][4]);
                mac4(x[b][v].z, lo, hi, &acc[g][v][8]);
                mac4(x[b][v].w, lo, hi, &acc[g][v][12]);
              }
            } else {
              const uint32_t t5 = __ldg(tb + 32 + lane);
              const uint4 h01 = __ldg(reinterpret_cast<const uint4 *>(tb + 64));
              const uint4 h23 = __ldg(reinterpret_cast<const uint4 *>(tb + 68));
              const uint32_t h3[8] = {h01.x, h01.y, h01.z, h01.w, h23.x, h23.y, h23.z, h23.w};
#pragma unroll
              for (int v = 0; v < V; ++v) {
                const uint32_t wv[4] = {x[b][v].x, x[b][v].y, x[b][v].z, x[b][v].w};
#pragma unroll
                for (int w = 0; w < 4; ++w) {
                  mac4_lo5(wv[w], t5, &acc[g][v][w * 4]);
                  const uint32_t sel = hi3_selector(wv[w]);
#pragma unroll
                  for (int r = 0; r < 4; ++r) oacc[g][v][r * 4 + w] ^= __byte_perm(h3[2 * r], h3[2 * r + 1], sel);
                }
              }
            }
          }
        }
      }
      bool bad = false;
#pragma unroll
      for (int g = 0; g < NG; ++g) {
#pragma unroll
        for (int v = 0; v < V; ++v) {
          uint32_t o[4][4];  // [output r][word w]
#pragma unroll
          for (int w = 0; w < 4; ++w) {
            uint32_t tmp[4];
            transpose4(&acc[g][v][w * 4], tmp);
#pragma unroll
            for (int r = 0; r < 4; ++r) o[r][w] = tmp[r] ^ (MIX ? oacc[g][v][r * 4 + w] : 0u);
          }
#pragma unroll
          for (int r = 0; r < 4; ++r) {
            const uint32_t out = (g0 + g) * 4 + r;
            if (out < d.n_out && active[v]) {
              uint8_t *dst = const_cast<uint8_t *>(ptr[n_in + out]) + col[v];
              if (VERIFY) {
                uint4 e = ld_stream(dst);
                bad |= (e.x != o[r][0]) | (e.y != o[r][1]) | (e.z != o[r][2]) | (e.w != o[r][3]);
              } else {
                st_stream(dst, make_uint4(o[r][0], o[r][1], o[r][2], o[r][3]));
              }
            }
          }
        }
      }
      if (VERIFY) {
        if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(a.flags + d.flag_idx, 1u);
      }
    }
  }
}

// Byte-granular path for the columns past each job's vec_len (shard tails
// that are not a multiple of 16 bytes, or jobs whose pointers are not 16-byte
// aligned).  One thread per byte column.
template <bool VERIFY>
__global__ void k_apply_tail(ApplyArgs a, uint64_t max_tail) {
  const uint64_t n = max_tail * a.n_jobs;
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n;
       i += uint64_t(gridDim.x) * blockDim.x) {
    const uint32_t job = uint32_t(i / max_tail);
    const JobDesc d = a.jobs[job];
    const uint64_t col = d.vec_len + (i - uint64_t(job) * max_tail);
    if (col >= a.len) continue;
    const uint8_t *const *ptr = a.ptrs + d.ptr_off;
    bool bad = false;
    for (uint32_t g = 0; g * 4 < d.n_out; ++g) {
      uint32_t acc = 0;
      for (uint32_t j = 0; j < d.n_in; ++j) {
        const uint32_t x = ptr[j][col];
        const uint32_t *tb = d.tbl + (g * d.n_in + j) * kTableWords;
        acc ^= __ldg(tb + (x & 15)) ^ __ldg(tb + 16 + (x >> 4));
      }
      for (uint32_t r = 0; r < 4 && g * 4 + r < d.n_out; ++r) {
        uint8_t *dst = const_cast<uint8_t *>(ptr[d.n_in + g * 4 + r]) + col;
        const uint8_t b = uint8_t(acc >> (8 * r));
        if (VERIFY)
          bad |= (*dst != b);
        else
          *dst = b;
      }
    }
    if (VERIFY && bad) atomicOr(a.flags + d.flag_idx, 1u);
  }
}

// ------------------------------------------------------------------ K3
// GF(2^8) arithmetic from log/exp tables staged in shared memory.
struct SmemGf {
  uint8_t log[256];
  uint8_t exp[512];
  __device__ uint8_t mul(uint8_t a, uint8_t b) const {
    return (a && b) ? exp[log[a] + log[b]] : 0;
  }
  __device__ uint8_t inv(uint8_t a) const { return a ? exp[255 - log[a]] : 0; }
};

__global__ void __launch_bounds__(256) k_decode_tables(DecodeTableArgs a) {
  extern __shared__ uint8_t smem[];
  __shared__ SmemGf gf;
  __shared__ uint8_t factor[256];
  __shared__ int pivot_row;
  __shared__ int singular;
  const DecodeTask task = a.tasks[blockIdx.x];
  const int k = a.k;
  const int w = 2 * k;
  uint8_t *aug = smem;              // k x 2k  [S | I]
  uint8_t *rows = smem + k * w;     // n_out x k composed rows
  for (int i = threadIdx.x; i < 256; i += blockDim.x) gf.log[i] = a.gf_log[i];
  for (int i = threadIdx.x; i < 512; i += blockDim.x) gf.exp[i] = a.gf_exp[i % 255];
  for (int i = threadIdx.x; i < k * w; i += blockDim.x) {
    const int r = i / w, c = i % w;
    uint8_t v;
    if (c < k)
      v = a.matrix[task.survivors[r] * k + c];
    else
      v = (c - k == r) ? 1 : 0;
    aug[i] = v;
  }
  if (threadIdx.x == 0) singular = 0;
  __syncthreads();
  if (task.needs_inverse) {
    for (int col = 0; col < k; ++col) {
      if (threadIdx.x == 0) {
        int p = col;
        while (p < k && aug[p * w + col] == 0) ++p;
        pivot_row = p;
        if (p == k) singular = 1;
      }
      __syncthreads();
      if (singular) break;
      const int p = pivot_row;
      if (p != col)
        for (int c = threadIdx.x; c < w; c += blockDim.x) {
          uint8_t t = aug[p * w + c];
          aug[p * w + c] = aug[col * w + c];
          aug[col * w + c] = t;
        }
      __syncthreads();
      const uint8_t s = gf.inv(aug[col * w + col]);
      __syncthreads();
      for (int c = threadIdx.x; c < w; c += blockDim.x) aug[col * w + c] = gf.mul(s, aug[col * w + c]);
      __syncthreads();
      for (int r = threadIdx.x; r < k; r += blockDim.x) factor[r] = (r == col) ? 0 : aug[r * w + col];
      __syncthreads();
      for (int i = threadIdx.x; i < k * w; i += blockDim.x) {
        const int r = i / w, c = i % w;
        const uint8_t f = factor[r];
        if (f) aug[i] ^= gf.mul(f, aug[col * w + c]);
      }
      __syncthreads();
    }
  }
  if (singular) {
    if (threadIdx.x == 0) a.status[blockIdx.x] = 1;
    return;
  }
  // Compose the requested rows over the survivor columns.  Without missing
  // data the survivors are the data shards in order and the inverse is the
  // identity.
  const int n_out = task.n_out;
  for (int i = threadIdx.x; i < n_out * k; i += blockDim.x) {
    const int t = i / k, c = i % k;
    const int idx = task.targets[t];
    uint8_t v = 0;
    if (idx < k) {
      v = task.needs_inverse ? aug[idx * w + k + c] : uint8_t(task.survivors[c] == idx);
    } else {
      const uint8_t *erow = a.matrix + idx * k;
      if (task.needs_inverse) {
        for (int j = 0; j < k; ++j) v ^= gf.mul(erow[j], aug[j * w + k + c]);
      } else {
        v = erow[task.survivors[c]];
      }
    }
    rows[i] = v;
  }
  __syncthreads();
  // Pack the lookup tables (layout of common.hpp).
  uint32_t *out = task.tbl_out;
  const int groups = (n_out + 3) / 4;
  for (int i = threadIdx.x; i < groups * k * kTableWords; i += blockDim.x) {
    const int e = i % kTableWords, j = (i / kTableWords) % k, g = (i / kTableWords) / k;
    uint32_t word = 0;
    if (e < 64) {
      const uint8_t x = e < 16 ? uint8_t(e) : e < 32 ? uint8_t((e - 16) << 4) : uint8_t(e - 32);
      for (int r = 0; r < 4; ++r) {
        const int o = g * 4 + r;
        if (o < n_out) word |= uint32_t(gf.mul(rows[o * k + j], x)) << (8 * r);
      }
    } else {
      const int r = (e - 64) >> 1, h0 = ((e - 64) & 1) * 4, o = g * 4 + r;
      if (o < n_out)
        for (int h = 0; h < 4; ++h) word |= uint32_t(gf.mul(rows[o * k + j], uint8_t((h0 + h) << 5))) << (8 * h);
    }
    out[i] = word;
  }
  if (threadIdx.x == 0) a.status[blockIdx.x] = 0;
}

int grid_for(const void *fn, int threads, size_t smem) {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  }
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem);
  if (per_sm < 1) per_sm = 1;
  return sms * per_sm;
}

template <int NG, int V, int B, int MIX, bool VERIFY>
void launch_vec(const ApplyArgs &a, cudaStream_t s) {
  static int grid_max = 0;
  if (!grid_max) grid_max = grid_for((const void *)k_apply_vec<NG, V, B, MIX, VERIFY>, kApplyThreads, 0);
  const uint64_t tile = uint64_t(kApplyThreads) * kApplyVec * V;
  const uint64_t tiles = ((a.len + tile - 1) / tile) * a.n_jobs;
  const int grid = int(tiles < uint64_t(grid_max) ? tiles : grid_max);
  k_apply_vec<NG, V, B, MIX, VERIFY><<<grid, kApplyThreads, 0, s>>>(a);
}

// Tile variants the autotuner chooses from: (vectors per thread, inputs in
// flight, lookup mix).
template <bool VERIFY>
void launch_variant(const ApplyArgs &a, int variant, cudaStream_t s) {
  if (a.max_out > 4) {
    launch_vec<2, 1, 4, 1, VERIFY>(a, s);
    return;
  }
  switch (variant) {
    case 0: launch_vec<1, 2, 4, 0, VERIFY>(a, s); break;
    case 2: launch_vec<1, 2, 4, 2, VERIFY>(a, s); break;
    case 3: launch_vec<1, 1, 8, 1, VERIFY>(a, s); break;
    case 4: launch_vec<1, 1, 4, 1, VERIFY>(a, s); break;
    case 1: launch_vec<1, 2, 4, 1, VERIFY>(a, s); break;
    default: launch_vec<1, 2, 4, 0, VERIFY>(a, s); break;
  }
}

}  // namespace

int &apply_variant() {
  static int v = [] {
    const char *e = getenv("RSGPU_APPLY_VARIANT");
    return e ? atoi(e) : 0;
  }();
  return v;
}

cudaError_t launch_apply(const ApplyArgs &a, bool verify, uint64_t max_tail, cudaStream_t s) {
  if (a.n_jobs == 0) return cudaSuccess;
  uint64_t launches = 0;
  if (a.any_vec && a.len >= 16) {
    if (verify)
      launch_variant<true>(a, apply_variant(), s);
    else
      launch_variant<false>(a, apply_variant(), s);
    ++launches;
  }
  if (max_tail) {
    const uint64_t n = max_tail * a.n_jobs;
    const int threads = 256;
    const uint64_t want = (n + threads - 1) / threads;
    const int grid = int(want < 148 * 16 ? want : 148 * 16);
    if (verify)
      k_apply_tail<true><<<grid, threads, 0, s>>>(a, max_tail);
    else
      k_apply_tail<false><<<grid, threads, 0, s>>>(a, max_tail);
    ++launches;
  }
  launch_counter_add(launches);
  return cudaGetLastError();
}

cudaError_t launch_decode_tables(const DecodeTableArgs &a, int n_tasks, int max_out, cudaStream_t s) {
  if (n_tasks == 0) return cudaSuccess;
  const size_t smem = size_t(a.k) * 2 * a.k + size_t(max_out) * a.k;
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(k_decode_tables, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         int(smem));
    if (e != cudaSuccess) return e;
  }
  k_decode_tables<<<n_tasks, 256, smem, s>>>(a);
  launch_counter_add(1);
  return cudaGetLastError();
}

}  // namespace rsgpu
