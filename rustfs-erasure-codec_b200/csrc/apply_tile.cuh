// apply_tile.cuh -- device code of the classic matrix-apply kernel (K1), one
// column tile at a time, shared by k_apply_vec (k_classic.cu) and the
// mixed-batch persistent kernel (batch.cu).
//
// out[r] = sum_j c[r][j] * in[j] over GF(2^8), bytewise.  Each thread owns 16
// (or 32) byte columns of one stripe and reads every input shard exactly once
// with coalesced 128-bit loads.  Products are table lookups split over the
// bits of the data byte, and the tables of four outputs are packed into one
// 32-bit word per entry, so one lookup serves four output rows.  Two
// formulations can share the work so that neither the shuffle (LSU) pipe nor
// the integer (ALU) pipe saturates:
//   4+4 split: two warp-shuffle lookups into 16-entry tables held one entry
//     per lane (mirrored into lanes 16..31, so the raw shifted data word is a
//     valid index: the shuffle only reads bits 0..4);
//   5+3 split: one shuffle into a 32-entry table for the low five bits and one
//     byte-permute (PRMT) per output for the high three bits, whose eight-entry
//     byte table fits the two PRMT source registers and whose result lands
//     directly in per-output column order.
// All outputs of a column are accumulated in registers and written once.
// The tables need not come from the classic field: any GF(2)-linear byte map
// (multiplication by a constant in the Leopard GF(2^8) field, for one) packs
// the same way.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "common.hpp"

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
// y = x | (x >> 4) puts byte i + 1's field in the high nibble of byte i; the
// fields do not overlap, so it equals x + (x >> 4), which one multiply-high
// and add computes on the FMA pipe (the GF(2^8) transforms are bound by the
// integer pipe).
__device__ __forceinline__ uint32_t hi3_selector(uint32_t w) {
  const uint32_t x = (w >> 5) & 0x07070707u;
  const uint32_t y = __umulhi(x, 1u << 28) + x;
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

// One tile = kApplyThreads threads x V 128-bit vectors of columns of job d,
// starting at byte tile_base (< d.vec_len).  NG = number of 4-output groups
// per pass over the inputs (outputs g*4 .. g*4+3).  MIX: 0 = every input uses
// the 4+4 split, 1 = odd inputs use 5+3, 2 = all 5+3.  Must be called by all
// kApplyThreads threads of the CTA (warp shuffles need full warps).
// ACC: outputs accumulate (dst ^= product) instead of being overwritten,
// for incremental parity updates (encode_single with i > 0, update).
template <int NG, int V, int kBatch, int MIX, bool VERIFY, bool ACC = false>
__device__ __forceinline__ void apply_tile(const uint8_t *const *ptrs, uint32_t *flags, const JobDesc &d,
                                           uint64_t tile_base) {
  const uint32_t lane = threadIdx.x & 31;
  // Thread column of vector v: tile_base + (v * kApplyThreads + tid) * 16, so a
  // warp's 32 loads of one vector cover 512 contiguous bytes.
  uint64_t col[V];
  bool active[V];
#pragma unroll
  for (int v = 0; v < V; ++v) {
    col[v] = tile_base + (uint64_t(v) * kApplyThreads + threadIdx.x) * kApplyVec;
    active[v] = col[v] < d.vec_len;
  }
  const uint8_t *const *ptr = ptrs + d.ptr_off;
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
              if (d.verify_store)
                st_stream(const_cast<uint8_t *>(ptr[n_in + d.n_out + out]) + col[v],
                          make_uint4(o[r][0], o[r][1], o[r][2], o[r][3]));
            } else if (ACC) {
              const uint4 e = *reinterpret_cast<const uint4 *>(dst);
              st_stream(dst, make_uint4(o[r][0] ^ e.x, o[r][1] ^ e.y, o[r][2] ^ e.z, o[r][3] ^ e.w));
            } else {
              st_stream(dst, make_uint4(o[r][0], o[r][1], o[r][2], o[r][3]));
            }
          }
        }
      }
    }
    if (VERIFY) {
      if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(flags + d.flag_idx, 1u);
    }
  }
}

// Byte-granular product of one column col (>= d.vec_len, < the shard length)
// of job d: the path for shard tails that are not a multiple of 16 bytes, or
// jobs whose pointers are not 16-byte aligned.  Returns true on a verify
// mismatch.
template <bool VERIFY, bool ACC = false>
__device__ __forceinline__ bool apply_column(const uint8_t *const *ptrs, const JobDesc &d, uint64_t col) {
  const uint8_t *const *ptr = ptrs + d.ptr_off;
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
      if (VERIFY) {
        bad |= (*dst != b);
        if (d.verify_store) const_cast<uint8_t *>(ptr[d.n_in + d.n_out + g * 4 + r])[col] = b;
      } else if (ACC)
        *dst ^= b;
      else
        *dst = b;
    }
  }
  return bad;
}

}  // namespace
}  // namespace rsgpu
