// k_classic.cu -- sm_100a kernels of the classic Reed-Solomon path.
//
// K1 (matrix apply): out[r] = sum_j c[r][j] * in[j] over GF(2^8), bytewise,
//   for encode, reconstruct (composed recovery rows) and verify (compare
//   instead of store).  It replaces the reference's row dot-product loops
//   (src/core/encode.rs:532-602, src/galois_8/x86/gfni_rows.rs:15-288).
//   Design: each thread owns 16 byte columns of one stripe and reads every
//   input shard exactly once with a coalesced 128-bit load.  A product
//   c * x is the XOR of two 16-entry nibble-table lookups; the tables of four
//   outputs are packed into one 32-bit word per entry, so one lookup serves
//   four parity rows at once.  The lookups are warp shuffles: lane l holds
//   table entry (l & 15), so a shuffle indexed by the raw shifted data word
//   (only bits 0..3 matter once the 16-entry table is mirrored into lanes
//   16..31) performs 32 independent table lookups without touching shared
//   memory and without bank conflicts.  All m outputs of a column are
//   accumulated in registers and written once.
//
// K3 (decode tables): Gauss-Jordan inversion of the selected survivor rows,
//   composition of the requested parity rows and packing of the nibble
//   tables, one CTA per erasure pattern (src/core/reconstruct.rs:1068-1174,
//   src/core/recovery_plan.rs:425-517).
#include <cuda_runtime.h>

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

constexpr int kBatch = 8;  // input vectors kept in flight per thread

// NG = number of 4-output groups handled in one pass (outputs g*4 .. g*4+3).
template <int NG, bool VERIFY>
__global__ void __launch_bounds__(kApplyThreads) k_apply_vec(ApplyArgs a) {
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t tiles_per_job = (a.len + kApplyTile - 1) / kApplyTile;
  const uint64_t total = tiles_per_job * a.n_jobs;
  for (uint64_t t = blockIdx.x; t < total; t += gridDim.x) {
    const uint32_t job = uint32_t(t / tiles_per_job);
    const uint64_t col = (t - uint64_t(job) * tiles_per_job) * kApplyTile + uint64_t(threadIdx.x) * kApplyVec;
    const JobDesc d = a.jobs[job];
    if ((t - uint64_t(job) * tiles_per_job) * kApplyTile >= d.vec_len) continue;  // CTA-uniform
    const bool active = col < d.vec_len;
    const uint8_t *const *ptr = a.ptrs + d.ptr_off;
    const uint32_t n_in = d.n_in;
    for (uint32_t g0 = 0; g0 * 4 < d.n_out; g0 += NG) {
      uint32_t acc[NG][16];
#pragma unroll
      for (int g = 0; g < NG; ++g)
#pragma unroll
        for (int i = 0; i < 16; ++i) acc[g][i] = 0;
      for (uint32_t j0 = 0; j0 < n_in; j0 += kBatch) {
        uint4 v[kBatch];
#pragma unroll
        for (int b = 0; b < kBatch; ++b) {
          v[b] = make_uint4(0, 0, 0, 0);
          if (active && j0 + b < n_in) v[b] = ld_stream(ptr[j0 + b] + col);
        }
#pragma unroll
        for (int b = 0; b < kBatch; ++b) {
          if (j0 + b >= n_in) break;  // warp-uniform
#pragma unroll
          for (int g = 0; g < NG; ++g) {
            const uint32_t *tb = d.tbl + ((g0 + g) * n_in + (j0 + b)) * 32;
            const uint32_t lo = __ldg(tb + (lane & 15));
            const uint32_t hi = __ldg(tb + 16 + (lane & 15));
            mac4(v[b].x, lo, hi, &acc[g][0]);
            mac4(v[b].y, lo, hi, &acc[g][4]);
            mac4(v[b].z, lo, hi, &acc[g][8]);
            mac4(v[b].w, lo, hi, &acc[g][12]);
          }
        }
      }
      bool bad = false;
#pragma unroll
      for (int g = 0; g < NG; ++g) {
        uint32_t o[4][4];  // [output r][word w]
#pragma unroll
        for (int w = 0; w < 4; ++w) {
          uint32_t tmp[4];
          transpose4(&acc[g][w * 4], tmp);
#pragma unroll
          for (int r = 0; r < 4; ++r) o[r][w] = tmp[r];
        }
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          const uint32_t out = (g0 + g) * 4 + r;
          if (out < d.n_out && active) {
            uint8_t *dst = const_cast<uint8_t *>(ptr[n_in + out]) + col;
            if (VERIFY) {
              uint4 e = ld_stream(dst);
              bad |= (e.x != o[r][0]) | (e.y != o[r][1]) | (e.z != o[r][2]) | (e.w != o[r][3]);
            } else {
              st_stream(dst, make_uint4(o[r][0], o[r][1], o[r][2], o[r][3]));
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
        const uint32_t *tb = d.tbl + (g * d.n_in + j) * 32;
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
  // Pack nibble tables (layout of common.hpp).
  uint32_t *out = task.tbl_out;
  const int groups = (n_out + 3) / 4;
  for (int i = threadIdx.x; i < groups * k * 32; i += blockDim.x) {
    const int e = i & 31, j = (i >> 5) % k, g = (i >> 5) / k;
    const uint8_t x = (e < 16) ? uint8_t(e) : uint8_t((e - 16) << 4);
    uint32_t word = 0;
    for (int r = 0; r < 4; ++r) {
      const int o = g * 4 + r;
      if (o < n_out) word |= uint32_t(gf.mul(rows[o * k + j], x)) << (8 * r);
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

}  // namespace

cudaError_t launch_apply(const ApplyArgs &a, bool verify, uint64_t max_tail, cudaStream_t s) {
  if (a.n_jobs == 0) return cudaSuccess;
  const uint64_t tiles = ((a.len + kApplyTile - 1) / kApplyTile) * a.n_jobs;
  uint64_t launches = 0;
  if (tiles && a.any_vec) {
    const void *fn;
    if (a.max_out > 4)
      fn = verify ? (const void *)k_apply_vec<2, true> : (const void *)k_apply_vec<2, false>;
    else
      fn = verify ? (const void *)k_apply_vec<1, true> : (const void *)k_apply_vec<1, false>;
    static int grid_cache[4] = {0, 0, 0, 0};
    const int slot = (a.max_out > 4 ? 2 : 0) + (verify ? 1 : 0);
    if (!grid_cache[slot]) grid_cache[slot] = grid_for(fn, kApplyThreads, 0);
    const int grid = int(tiles < uint64_t(grid_cache[slot]) ? tiles : grid_cache[slot]);
    if (a.max_out > 4) {
      if (verify)
        k_apply_vec<2, true><<<grid, kApplyThreads, 0, s>>>(a);
      else
        k_apply_vec<2, false><<<grid, kApplyThreads, 0, s>>>(a);
    } else {
      if (verify)
        k_apply_vec<1, true><<<grid, kApplyThreads, 0, s>>>(a);
      else
        k_apply_vec<1, false><<<grid, kApplyThreads, 0, s>>>(a);
    }
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
