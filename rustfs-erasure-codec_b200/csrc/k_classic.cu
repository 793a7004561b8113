// k_classic.cu -- sm_100a kernels of the classic Reed-Solomon path.
//
// K1 (matrix apply): out[r] = sum_j c[r][j] * in[j] over GF(2^8), bytewise,
//   for encode, reconstruct (composed recovery rows) and verify (compare
//   instead of store).  It replaces the reference's row dot-product loops
//   (src/core/encode.rs:532-602, src/galois_8/x86/gfni_rows.rs:15-288).  The
//   per-tile device code and its design notes are in apply_tile.cuh; this file
//   holds the grid-stride launches over one batch.
//
// K3 (decode tables): Gauss-Jordan inversion of the selected survivor rows,
//   composition of the requested parity rows and packing of the nibble
//   tables, one CTA per erasure pattern (src/core/reconstruct.rs:1068-1174,
//   src/core/recovery_plan.rs:425-517).
#include <cuda_runtime.h>

#include <cstdlib>

#include "apply_tile.cuh"
#include "common.hpp"
#include "kernels.hpp"

namespace rsgpu {

namespace {

// L2 prefetch of `bytes` (a multiple of 16) at a 16-byte-aligned address.
__device__ __forceinline__ void prefetch_l2(const void *p, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// Grid-stride loop of apply_tile over every (job, tile) of a launch.  With
// PF, the CTA first asks L2 for the input columns of the tile it will take
// next (one bulk prefetch per input shard), so those loads are L2 hits.
template <int NG, int V, int kBatch, int MIX, bool VERIFY, bool PF = false, int MINB = 0, bool ACC = false>
__global__ void __launch_bounds__(kApplyThreads, MINB ? MINB : ((NG == 1 && V <= 2) ? 4 : 1)) k_apply_vec(ApplyArgs a) {
  constexpr uint32_t kTile = kApplyThreads * kApplyVec * V;
  const uint32_t tiles_per_job = uint32_t((a.len + kTile - 1) / kTile);
  const uint32_t total = tiles_per_job * a.n_jobs;
  for (uint32_t t = blockIdx.x; t < total; t += gridDim.x) {
    const uint32_t job = t / tiles_per_job;
    const uint64_t tile_base = uint64_t(t - job * tiles_per_job) * kTile;
    const JobDesc d = a.jobs[job];
    if (PF) {
      const uint32_t t2 = t + gridDim.x;
      if (t2 < total) {
        const uint32_t job2 = t2 / tiles_per_job;
        const uint64_t base2 = uint64_t(t2 - job2 * tiles_per_job) * kTile;
        const JobDesc d2 = a.jobs[job2];
        if (threadIdx.x < d2.n_in && base2 < d2.vec_len) {
          const uint64_t left = d2.vec_len - base2;
          prefetch_l2(a.ptrs[d2.ptr_off + threadIdx.x] + base2, uint32_t(left < kTile ? left : kTile));
        }
      }
    }
    if (tile_base >= d.vec_len) continue;  // CTA-uniform
    apply_tile<NG, V, kBatch, MIX, VERIFY, ACC>(a.ptrs, a.flags, d, tile_base);
  }
}

// Byte-granular path for the columns past each job's vec_len.  One thread per
// byte column.
template <bool VERIFY, bool ACC = false>
__global__ void k_apply_tail(ApplyArgs a, uint64_t max_tail) {
  const uint64_t n = max_tail * a.n_jobs;
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n;
       i += uint64_t(gridDim.x) * blockDim.x) {
    const uint32_t job = uint32_t(i / max_tail);
    const JobDesc d = a.jobs[job];
    const uint64_t col = d.vec_len + (i - uint64_t(job) * max_tail);
    if (col >= a.len) continue;
    if (apply_column<VERIFY, ACC>(a.ptrs, d, col) && VERIFY) atomicOr(a.flags + d.flag_idx, 1u);
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

template <int NG, int V, int B, int MIX, bool VERIFY, bool PF = false, int MINB = 0, bool ACC = false>
void launch_vec(const ApplyArgs &a, cudaStream_t s) {
  static int grid_max = 0;
  if (!grid_max)
    grid_max = grid_for((const void *)k_apply_vec<NG, V, B, MIX, VERIFY, PF, MINB, ACC>, kApplyThreads, 0);
  const uint64_t tile = uint64_t(kApplyThreads) * kApplyVec * V;
  const uint64_t tiles = ((a.len + tile - 1) / tile) * a.n_jobs;
  const int grid = int(tiles < uint64_t(grid_max) ? tiles : grid_max);
  k_apply_vec<NG, V, B, MIX, VERIFY, PF, MINB, ACC><<<grid, kApplyThreads, 0, s>>>(a);
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
    case 5: launch_vec<1, 2, 4, 0, VERIFY, true>(a, s); break;
    case 6: launch_vec<1, 1, 8, 0, VERIFY>(a, s); break;
    case 7: launch_vec<1, 1, 8, 0, VERIFY, true>(a, s); break;
    case 8: launch_vec<1, 4, 2, 0, VERIFY>(a, s); break;
    case 9: launch_vec<1, 2, 2, 0, VERIFY, true>(a, s); break;
    case 10: launch_vec<1, 1, 4, 0, VERIFY, false, 6>(a, s); break;
    case 11: launch_vec<1, 1, 2, 0, VERIFY, false, 8>(a, s); break;
    case 12: launch_vec<1, 2, 2, 0, VERIFY, false, 6>(a, s); break;
    case 13: launch_vec<1, 1, 4, 0, VERIFY, false, 4>(a, s); break;
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
    if (a.accumulate)
      launch_vec<1, 2, 4, 0, false, false, 0, true>(a, s);
    else if (verify)
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
    if (a.accumulate)
      k_apply_tail<false, true><<<grid, threads, 0, s>>>(a, max_tail);
    else if (verify)
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
