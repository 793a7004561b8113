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
#include "launch_cfg.hpp"

namespace rsgpu {

namespace {

// Grid-stride loop of apply_tile over every (job, tile) of a launch, inputs
// loaded straight into registers: the tile for more than 4 outputs and for
// accumulating (incremental parity) launches.
template <int NG, int V, int kBatch, int MIX, bool VERIFY, bool ACC = false>
__global__ void __launch_bounds__(kApplyThreads, (NG == 1 && V <= 2) ? 4 : 1) k_apply_vec(ApplyArgs a) {
  constexpr uint32_t kTile = kApplyThreads * kApplyVec * V;
  const uint32_t tiles_per_job = uint32_t((a.len + kTile - 1) / kTile);
  const uint32_t total = tiles_per_job * a.n_jobs;
  for (uint32_t t = blockIdx.x; t < total; t += gridDim.x) {
    const uint32_t job = t / tiles_per_job;
    const uint64_t tile_base = uint64_t(t - job * tiles_per_job) * kTile;
    const JobDesc d = a.jobs[job];
    if (tile_base >= d.vec_len) continue;  // CTA-uniform
    apply_tile<NG, V, kBatch, MIX, VERIFY, ACC>(a.ptrs, a.flags, d, tile_base);
  }
}

// ------------------------------------------------------------------ K1, TMA-staged
// The same product as k_apply_vec<1, V, 4, 0> with the input tiles staged in
// shared memory by the bulk-copy (TMA) unit: one producer warp streams each
// step's tile slices (one contiguous 256 * 16 * V-byte slice per input shard,
// cp.async.bulk with completion on the stage's mbarrier) into a ring of S
// stages of 4 slots; kApplyThreads consumer threads wait for a stage, run the
// table arithmetic from shared memory and release it.  A step is up to 4
// input shards of one tile, or for verify the tile's <= 4 parity shards.
// n_out <= 4 only.  Every wait is bounded (about 2 s of SM clock); a wait
// that runs out sets *a.stall (the codec's status word, read back by the
// next synchronous call as RSGPU_ERR_DEVICE_TIMEOUT), and the producer then
// waits, bounded again, for the copies it has in flight before it exits.
// Measured against the register-path tile (k_apply_vec<1, 2, 4, 0>) on
// 1024 x 1 MiB stripes: 10+4 encode 4650 vs 4268 GB/s; global-load stalls per
// issued instruction fall from 4.1 to 1.7, and the bulk copies do not compete
// with the table shuffles for the L1 data pipe (cp.async staging, which
// does, was 7-14% slower than the register path).
constexpr long long kStallCycles = 4000000000ll;

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
// Wait for the completion of the barrier phase with this parity; false when
// the wait ran out.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  const long long t0 = clock64();
  for (;;) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
    if (clock64() - t0 > kStallCycles) return false;
  }
}
__device__ __forceinline__ void bulk_load(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}
__device__ __forceinline__ uint32_t lds32(uint32_t addr) {
  uint32_t v;
  asm volatile("ld.shared.u32 %0, [%1];" : "=r"(v) : "r"(addr) : "memory");
  return v;
}
__device__ __forceinline__ uint4 lds128(uint32_t addr) {
  uint4 v;
  asm volatile("ld.shared.v4.u32 {%0,%1,%2,%3}, [%4];" : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "r"(addr)
               : "memory");
  return v;
}

template <int V, int S, bool VERIFY>
__global__ void __launch_bounds__(kApplyThreads + 32, 2) k_apply_tma(ApplyArgs a) {
  constexpr uint32_t kSlot = kApplyThreads * kApplyVec * V;  // one input's slice of a tile
  extern __shared__ __align__(128) uint8_t tma_smem[];
  __shared__ __align__(8) uint64_t full[S], empty[S];
  // The 4+4 nibble tables (words 0..31 of each input's packed table) of each
  // stage's inputs, copied with the data when the launch's jobs carry
  // different tables (a batch of stripes with different erasure patterns):
  // read from L2 after the stage's wait, they put an L2 round trip on every
  // step (10+4 rebuild 3.2 -> 4.2 TB/s).  A table that every job shares stays
  // L1-resident and is read with plain loads.
  __shared__ __align__(16) uint32_t tma_tbl[S][4][32];
  const uint32_t tid = threadIdx.x, lane = tid & 31;
  const uint32_t sbase = uint32_t(__cvta_generic_to_shared(tma_smem));
  const uint32_t tbase = uint32_t(__cvta_generic_to_shared(&tma_tbl[0][0][0]));
  const uint32_t fbar = uint32_t(__cvta_generic_to_shared(full));
  const uint32_t ebar = uint32_t(__cvta_generic_to_shared(empty));
  if (tid == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(fbar + 8 * s, 1);
      mbar_init(ebar + 8 * s, kApplyThreads / 32);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  const uint32_t tiles_per_job = uint32_t((a.len + kSlot - 1) / kSlot);
  const uint32_t total = tiles_per_job * a.n_jobs;

  if (tid >= kApplyThreads) {  // producer warp: one lane issues every copy
    if (tid != kApplyThreads) return;
    uint32_t it = 0;
    bool ok = true;
    for (uint32_t t = blockIdx.x; t < total && ok; t += gridDim.x) {
      const uint32_t job = t / tiles_per_job;
      const uint64_t base = uint64_t(t - job * tiles_per_job) * kSlot;
      const JobDesc d = a.jobs[job];
      if (base >= d.vec_len) continue;
      const uint32_t valid = uint32_t(d.vec_len - base < kSlot ? d.vec_len - base : kSlot);
      const uint8_t *const *ptr = a.ptrs + d.ptr_off;
      const bool tbl_copy = a.tbl_stage && d.tbl && (reinterpret_cast<uintptr_t>(d.tbl) & 15) == 0;
      const uint32_t steps = (d.n_in + 3) / 4 + (VERIFY ? 1 : 0);
      for (uint32_t step = 0; step < steps; ++step, ++it) {
        const uint32_t s = it % S, ph = (it / S) & 1;
        if (!mbar_wait(ebar + 8 * s, ph ^ 1)) {
          ok = false;
          break;
        }
        const bool par = VERIFY && step * 4 >= d.n_in;
        const uint32_t j0 = par ? d.n_in : step * 4;
        const uint32_t rows = par ? d.n_out : min(4u, d.n_in - j0);
        const bool tbl_here = tbl_copy && !par;
        mbar_expect_tx(fbar + 8 * s, rows * valid + (tbl_here ? rows * 128 : 0));
        for (uint32_t b = 0; b < rows; ++b)
          bulk_load(sbase + (s * 4 + b) * kSlot, ptr[j0 + b] + base, valid, fbar + 8 * s);
        if (tbl_here)
          for (uint32_t b = 0; b < rows; ++b)
            bulk_load(tbase + (s * 4 + b) * 128, d.tbl + (j0 + b) * kTableWords, 128, fbar + 8 * s);
      }
    }
    if (!ok) {
      if (a.stall) atomicOr(a.stall, 1u);
      // Copies already issued land in stages the consumers stopped reading:
      // wait (bounded) for them before the CTA's shared memory goes away.
      for (uint32_t k = 0; k < S && k < it; ++k) {
        const uint32_t i = it - 1 - k;
        mbar_wait(fbar + 8 * (i % S), (i / S) & 1);
      }
    }
    return;
  }

  // Consumers: the same (tile, step) sequence as the producer.
  uint32_t it = 0;
  for (uint32_t t = blockIdx.x; t < total; t += gridDim.x) {
    const uint32_t job = t / tiles_per_job;
    const uint64_t base = uint64_t(t - job * tiles_per_job) * kSlot;
    const JobDesc d = a.jobs[job];
    if (base >= d.vec_len) continue;
    const uint32_t n_in = d.n_in;
    const bool tbl_copy = a.tbl_stage && d.tbl && (reinterpret_cast<uintptr_t>(d.tbl) & 15) == 0;  // as the producer decides
    const uint32_t steps = (n_in + 3) / 4 + (VERIFY ? 1 : 0);
    uint64_t col[V];
    bool active[V];
#pragma unroll
    for (int v = 0; v < V; ++v) {
      col[v] = base + (uint64_t(v) * kApplyThreads + tid) * kApplyVec;
      active[v] = col[v] < d.vec_len;
    }
    uint32_t acc[V][16];
#pragma unroll
    for (int v = 0; v < V; ++v)
#pragma unroll
      for (int i = 0; i < 16; ++i) acc[v][i] = 0;
    bool bad = false;
    for (uint32_t step = 0; step < steps; ++step, ++it) {
      const uint32_t s = it % S, ph = (it / S) & 1;
      if (!mbar_wait(fbar + 8 * s, ph)) {
        if (a.stall) atomicOr(a.stall, 1u);
        return;
      }
      const uint32_t slot0 = sbase + s * 4 * kSlot + tid * kApplyVec;
      const bool par = VERIFY && step * 4 >= n_in;
      if (!par) {
        const uint32_t j0 = step * 4;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          if (j0 + b >= n_in) break;  // warp-uniform
          uint32_t lo, hi;
          if (tbl_copy) {
            const uint32_t ta = tbase + (s * 4 + b) * 128 + (lane & 15) * 4;
            lo = lds32(ta);
            hi = lds32(ta + 64);
          } else {
            const uint32_t *tb = d.tbl + (j0 + b) * kTableWords;
            lo = __ldg(tb + (lane & 15));
            hi = __ldg(tb + 16 + (lane & 15));
          }
#pragma unroll
          for (int v = 0; v < V; ++v) {
            const uint4 x = lds128(slot0 + b * kSlot + v * kApplyThreads * kApplyVec);
            mac4(x.x, lo, hi, &acc[v][0]);
            mac4(x.y, lo, hi, &acc[v][4]);
            mac4(x.z, lo, hi, &acc[v][8]);
            mac4(x.w, lo, hi, &acc[v][12]);
          }
        }
      }
      if (step + 1 == steps) {  // outputs of this tile (parity rows are in this stage when VERIFY)
#pragma unroll
        for (int v = 0; v < V; ++v) {
          uint32_t o[4][4];
#pragma unroll
          for (int w = 0; w < 4; ++w) {
            uint32_t tmp[4];
            transpose4(&acc[v][w * 4], tmp);
#pragma unroll
            for (int r = 0; r < 4; ++r) o[r][w] = tmp[r];
          }
#pragma unroll
          for (int r = 0; r < 4; ++r) {
            if (uint32_t(r) < d.n_out && active[v]) {
              if (VERIFY) {
                const uint4 e = lds128(slot0 + r * kSlot + v * kApplyThreads * kApplyVec);
                bad |= (e.x != o[r][0]) | (e.y != o[r][1]) | (e.z != o[r][2]) | (e.w != o[r][3]);
                if (d.verify_store)
                  st_stream(const_cast<uint8_t *>(a.ptrs[d.ptr_off + n_in + d.n_out + r]) + col[v],
                            make_uint4(o[r][0], o[r][1], o[r][2], o[r][3]));
              } else {
                uint8_t *dst = const_cast<uint8_t *>(a.ptrs[d.ptr_off + n_in + r]) + col[v];
                st_stream(dst, make_uint4(o[r][0], o[r][1], o[r][2], o[r][3]));
              }
            }
          }
        }
        if (VERIFY && __any_sync(0xffffffffu, bad) && lane == 0) atomicOr(a.flags + d.flag_idx, 1u);
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(ebar + 8 * s);
    }
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

// Pair kernel: blockIdx.y selects the pair, the x dimension strides over
// its 16-byte chunks; pairs whose pointers are not both 16-byte aligned, and
// the bytes past the last full chunk, go byte by byte.
template <int MODE>
__global__ void __launch_bounds__(256) k_pairs(const PairOp *pairs, uint32_t *flag) {
  const PairOp p = pairs[blockIdx.y];
  const bool aligned = ((reinterpret_cast<uintptr_t>(p.a) | reinterpret_cast<uintptr_t>(p.b)) & 15) == 0;
  const uint64_t vec = aligned ? p.len / 16 : 0;
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  bool bad = false;
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < vec; i += stride) {
    const uint4 x = ld_stream(p.a + 16 * i);
    if (MODE == PAIR_COMPARE) {
      const uint4 y = ld_stream(p.b + 16 * i);
      bad |= (x.x != y.x) | (x.y != y.y) | (x.z != y.z) | (x.w != y.w);
    } else {
      uint4 *dst = reinterpret_cast<uint4 *>(p.b + 16 * i);
      const uint4 y = *dst;
      st_stream(p.b + 16 * i, make_uint4(x.x ^ y.x, x.y ^ y.y, x.z ^ y.z, x.w ^ y.w));
    }
  }
  for (uint64_t i = 16 * vec + blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < p.len; i += stride) {
    if (MODE == PAIR_COMPARE)
      bad |= p.a[i] != p.b[i];
    else
      p.b[i] ^= p.a[i];
  }
  if (MODE == PAIR_COMPARE && __any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(flag, 1u);
}

__global__ void __launch_bounds__(256) k_gather_tables(const uint32_t *full, uint32_t *out, GatherCols cols,
                                                       uint32_t groups, uint32_t k_full, uint32_t n_sel) {
  const uint32_t n = groups * n_sel * kTableWords;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t e = i % kTableWords, j = (i / kTableWords) % n_sel, g = i / (kTableWords * n_sel);
    out[i] = full[(g * k_full + cols.cols[j]) * kTableWords + e];
  }
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

template <int NG, int V, int B, int MIX, bool VERIFY, bool ACC = false>
void launch_vec(const ApplyArgs &a, cudaStream_t s) {
  static int grid_max = 0;
  if (!grid_max) grid_max = grid_for((const void *)k_apply_vec<NG, V, B, MIX, VERIFY, ACC>, kApplyThreads, 0);
  const uint64_t tile = uint64_t(kApplyThreads) * kApplyVec * V;
  const uint64_t tiles = ((a.len + tile - 1) / tile) * a.n_jobs;
  const int grid = int(tiles < uint64_t(grid_max) ? tiles : grid_max);
  k_apply_vec<NG, V, B, MIX, VERIFY, ACC><<<grid, kApplyThreads, 0, s>>>(a);
}

template <int V, int S, bool VERIFY>
void launch_tma(const ApplyArgs &a, cudaStream_t s) {
  constexpr size_t smem = size_t(S) * 4 * kApplyThreads * kApplyVec * V;
  static int grid_max = 0;
  const void *fn = (const void *)k_apply_tma<V, S, VERIFY>;
  ensure_smem_limit(fn, smem);  // per device, set once
  if (!grid_max) grid_max = grid_for(fn, kApplyThreads + 32, smem);
  const uint64_t tile = uint64_t(kApplyThreads) * kApplyVec * V;
  const uint64_t tiles = ((a.len + tile - 1) / tile) * a.n_jobs;
  const int grid = int(tiles < uint64_t(grid_max) ? tiles : grid_max);
  k_apply_tma<V, S, VERIFY><<<grid, kApplyThreads + 32, smem, s>>>(a);
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
    case 1: launch_vec<1, 2, 4, 0, VERIFY>(a, s); break;  // register path
    case 2: launch_tma<2, 2, VERIFY>(a, s); break;
    case 3: launch_tma<1, 4, VERIFY>(a, s); break;
    default: launch_tma<2, 3, VERIFY>(a, s); break;  // 0: TMA-staged, 2 x 16 B per thread, 3 stages
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
      launch_vec<1, 2, 4, 0, false, true>(a, s);
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
    const uint64_t cap = uint64_t(device_sm_count()) * 16;
    const int grid = int(want < cap ? want : cap);
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

cudaError_t launch_pairs(const PairOp *pairs, uint32_t n, uint64_t max_len, int mode, uint32_t *flag,
                         cudaStream_t s) {
  if (n == 0 || max_len == 0) return cudaSuccess;
  if (n > 65535) return cudaErrorInvalidValue;  // one grid row per pair
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  }
  // About 8 CTAs per SM in total, at least one per 64 KiB of the longest pair.
  const uint64_t per_pair = (max_len + 65535) / 65536;
  uint64_t want = (uint64_t(sms) * 8 + n - 1) / n;
  if (want > per_pair) want = per_pair;
  if (want < 1) want = 1;
  const dim3 grid(uint32_t(want), n);
  if (mode == PAIR_COMPARE)
    k_pairs<PAIR_COMPARE><<<grid, 256, 0, s>>>(pairs, flag);
  else
    k_pairs<PAIR_XOR><<<grid, 256, 0, s>>>(pairs, flag);
  launch_counter_add(1);
  return cudaGetLastError();
}

cudaError_t launch_gather_tables(const uint32_t *full, uint32_t *out, const GatherCols &cols, uint32_t groups,
                                 uint32_t k_full, uint32_t n_sel, cudaStream_t s) {
  const uint32_t n = groups * n_sel * kTableWords;
  if (n == 0) return cudaSuccess;
  const uint32_t grid = (n + 255) / 256 < 1184 ? (n + 255) / 256 : 1184;
  k_gather_tables<<<grid, 256, 0, s>>>(full, out, cols, groups, k_full, n_sel);
  launch_counter_add(1);
  return cudaGetLastError();
}

cudaError_t launch_decode_tables(const DecodeTableArgs &a, int n_tasks, int max_out, cudaStream_t s) {
  if (n_tasks == 0) return cudaSuccess;
  const size_t smem = size_t(a.k) * 2 * a.k + size_t(max_out) * a.k;
  cudaError_t e = ensure_smem_limit(reinterpret_cast<const void *>(k_decode_tables), smem);
  if (e != cudaSuccess) return e;
  k_decode_tables<<<n_tasks, 256, smem, s>>>(a);
  launch_counter_add(1);
  return cudaGetLastError();
}

}  // namespace rsgpu
