// leo_fft.cuh -- Leopard FFT encode / decode, register-resident stages.
//
// The Leopard transforms (src/core/leopard_gf16/ops.rs:375-511 and the plan
// builders of src/core/leopard_gf16/mod.rs, src/core/leopard_gf8/mod.rs) are
// layers of radix-4 butterflies with distances 1, 4, 16, ... (IFFT) or ...,
// 16, 4, 1 (FFT), plus one radix-2 layer when log2 of the size is odd.  Two
// consecutive radix-4 layers only mix the 16 lanes {R + a + d*j : j < 16}, so
// a thread loads those 16 lanes of one 32-bit column word into registers,
// runs both layers there, and stores them back: one shared-memory round trip
// and one barrier per two layers, instead of per layer.  A transform of L
// lanes is a list of such stages (16, 8, 4 or 2 lanes per thread); codes with
// at most 16 lanes run entirely in registers, straight from and to HBM.
//
// All 32 threads of a warp work on the same lanes of 32 adjacent column
// words, so every butterfly constant is warp-uniform: its table is loaded
// once per warp (one entry per thread) and read with full-warp shuffles, and
// a constant whose log is the field modulus (the reference skips the
// multiply, ops.rs:375-465) is a uniform branch around the multiply.
//
// Multiplication by a constant c:
//   GF(2^8): 5+3 split.  Each byte's low five bits index a 32-entry table of
//     c*i held one entry per lane (one shuffle per byte); the high three bits
//     select, with one byte-permute for all four bytes of a word, from an
//     8-entry byte table of c*(h << 5) held in two registers.
//   GF(2^16): 5+5+5+1 split.  Bits 0-4, 5-9 and 10-14 of each element index
//     three 32-entry tables (c * (i << 5q)) held one entry per lane (one
//     shuffle each, so six per word of two elements, against eight for
//     nibble tables); bit 15 of both elements becomes a mask with one
//     sign-replicating byte-permute, applied to c * 2^15 (the split byte
//     layout is converted to 16-bit elements on load and back on store).
//
// Which lanes a stage may skip: the reference only runs the butterflies of
// blocks that start below `mtrunc`.  Lanes of skipped IFFT blocks are zero
// (absent inputs and padding), and butterflies on zeros leave zeros; lanes of
// skipped FFT blocks never reach an output lane.  So a stage group whose base
// lane is >= mtrunc is skipped, and every other group runs all of its
// butterflies: the outputs are bit-identical to the reference.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "apply_tile.cuh"
#include "leo_types.hpp"

namespace rsgpu {
namespace {

// ------------------------------------------------------------------ constants
template <int BITS>
struct KTab;
template <>
struct KTab<8> {
  uint32_t lo5, h0, h1;
};
template <>
struct KTab<16> {
  uint32_t t0, t1, t2, c15;  // c * (lane << 0 / 5 / 10) and c * 2^15, each in both halves
};

// GF(2^8) table bank, one record of kWBank8 words per log value:
// [0, 32): c * i (i < 32) replicated into all four bytes; [32, 34): byte h of
// the pair = c * (h << 5).
constexpr int kWBank8 = 36;

template <int BITS>
__device__ __forceinline__ KTab<BITS> kload(const uint32_t *bank, uint32_t lm, uint32_t lane);
template <>
__device__ __forceinline__ KTab<8> kload<8>(const uint32_t *bank, uint32_t lm, uint32_t lane) {
  const uint32_t *r = bank + lm * kWBank8;
  const uint2 h = __ldg(reinterpret_cast<const uint2 *>(r + 32));
  return KTab<8>{__ldg(r + lane), h.x, h.y};
}
// GF(2^16) table bank, one record of 32 lanes x 4 words per log value.
template <>
__device__ __forceinline__ KTab<16> kload<16>(const uint32_t *bank, uint32_t lm, uint32_t lane) {
  const uint4 v = __ldg(reinterpret_cast<const uint4 *>(bank) + lm * 32 + lane);
  return KTab<16>{v.x, v.y, v.z, v.w};
}

__device__ __forceinline__ uint32_t kmul(uint32_t w, const KTab<8> &t) {
  const uint32_t s0 = tshfl(t.lo5, w);
  const uint32_t s1 = tshfl(t.lo5, w >> 8);
  const uint32_t s2 = tshfl(t.lo5, w >> 16);
  const uint32_t s3 = tshfl(t.lo5, w >> 24);
  const uint32_t lo = __byte_perm(__byte_perm(s0, s1, 0x0040), __byte_perm(s2, s3, 0x4000), 0x7610);
  return lo ^ __byte_perm(t.h0, t.h1, hi3_selector(w));
}
// Byte permute with sign replication: selector nibble 9 (B) fills a byte
// with the top bit of source byte 1 (3).  __byte_perm reads only three
// bits of each selector nibble, so this is written in PTX.
__device__ __forceinline__ uint32_t top_bit_masks(uint32_t w) {
  uint32_t r;
  asm("prmt.b32 %0, %1, 0, 0xBB99;" : "=r"(r) : "r"(w));
  return r;  // low half: bit 15 of w replicated, high half: bit 31
}
__device__ __forceinline__ uint32_t kmul(uint32_t w, const KTab<16> &t) {
  const uint32_t a = tshfl(t.t0, w) ^ tshfl(t.t1, w >> 5) ^ tshfl(t.t2, w >> 10);
  const uint32_t b = tshfl(t.t0, w >> 16) ^ tshfl(t.t1, w >> 21) ^ tshfl(t.t2, w >> 26);
  return __byte_perm(a, b, 0x7610) ^ (top_bit_masks(w) & t.c15);
}

// Warp-uniform butterfly constant: its log value and this thread's tables.
template <int BITS>
struct Kc {
  uint32_t lm;
  KTab<BITS> t;
};

// skew: the field's FFT skew logs; sktab: the multiplier tables of each skew
// entry (entry i = the bank's tables of log skew[i]).  A transform's skew
// base is an offset into both.
struct FftCtx {
  const uint32_t *bank;
  uint32_t mod;
  uint32_t lane;
  const uint16_t *skew;
  const uint32_t *sktab;
};

// The butterfly constant at skew entry skb + idx.  Its log (for the
// reference's skip of a multiply by a log-modulus constant) and its tables
// are independent loads, so their latencies overlap; with the tables looked
// up by log value instead, the table load had to wait for the log.
// SK = false: the caller knows that no constant of its group has that log,
// so the log is not loaded and every butterfly multiplies.
template <int BITS, bool SK>
__device__ __forceinline__ Kc<BITS> kc(const FftCtx &x, int32_t skb, uint32_t idx) {
  const uint32_t i = uint32_t(skb + int32_t(idx));
  return Kc<BITS>{SK ? uint32_t(__ldg(x.skew + i)) : 0u, kload<BITS>(x.sktab, i, x.lane)};
}

// Inverse butterfly (IFFT): y ^= x; x ^= y * c.  Forward (FFT): x ^= y * c; y ^= x.
template <int BITS, bool SK>
__device__ __forceinline__ void ibf(uint32_t &x, uint32_t &y, const Kc<BITS> &c, uint32_t mod) {
  y ^= x;
  if (!SK || c.lm != mod) x ^= kmul(y, c.t);
}
template <int BITS, bool SK>
__device__ __forceinline__ void fbf(uint32_t &x, uint32_t &y, const Kc<BITS> &c, uint32_t mod) {
  if (!SK || c.lm != mod) x ^= kmul(y, c.t);
  y ^= x;
}

// Radix-4 on (a, b, c, d) = lanes i, i+d, i+2d, i+3d of one block.
// Inverse order: (a,b) m01, (c,d) m23, (a,c) m02, (b,d) m02.
// Forward order: (a,c) m02, (b,d) m02, (a,b) m01, (c,d) m23.
template <int BITS, bool SK>
__device__ __forceinline__ void iq(uint32_t &a, uint32_t &b, uint32_t &c, uint32_t &d, const Kc<BITS> &m01,
                                   const Kc<BITS> &m02, const Kc<BITS> &m23, uint32_t mod) {
  ibf<BITS, SK>(a, b, m01, mod);
  ibf<BITS, SK>(c, d, m23, mod);
  ibf<BITS, SK>(a, c, m02, mod);
  ibf<BITS, SK>(b, d, m02, mod);
}
template <int BITS, bool SK>
__device__ __forceinline__ void fq(uint32_t &a, uint32_t &b, uint32_t &c, uint32_t &d, const Kc<BITS> &m01,
                                   const Kc<BITS> &m02, const Kc<BITS> &m23, uint32_t mod) {
  fbf<BITS, SK>(a, c, m02, mod);
  fbf<BITS, SK>(b, d, m02, mod);
  fbf<BITS, SK>(a, b, m01, mod);
  fbf<BITS, SK>(c, d, m23, mod);
}

// One stage on the registers v[0..G) holding lanes R + a + dm * j.  skb is
// the transform's skew base (an offset into the field's skew entries): a
// radix-4 block starting at lane r with distance d uses entries skb + r + d,
// skb + r + 2d, skb + r + 3d (m01, m02, m23); a radix-2 block uses skb + r + d.  LG = log2 G; FWD selects FFT (true) or IFFT.
//   IFFT: G=16: radix-4 (d = dm) then radix-4 (4dm); G=8: radix-4 (dm) then
//         radix-2 (4dm); G=4: radix-4 (dm); G=2: radix-2 (dm).
//   FFT:  G=16: radix-4 (4dm) then radix-4 (dm); G=8: radix-4 (2dm) then
//         radix-2 (dm); G=4: radix-4 (dm); G=2: radix-2 (dm).
template <int BITS, int LG, bool FWD, bool SK>
__device__ __forceinline__ void stage_regs_k(uint32_t *v, const FftCtx &x, int32_t skb, uint32_t R,
                                             uint32_t dm) {
  const uint32_t mod = x.mod;
  if (LG == 4) {
    if (!FWD) {
#pragma unroll
      for (int s = 0; s < 4; ++s) {
        const uint32_t r = R + 4 * s * dm;
        const Kc<BITS> m01 = kc<BITS, SK>(x, skb, r + dm), m02 = kc<BITS, SK>(x, skb, r + 2 * dm),
                       m23 = kc<BITS, SK>(x, skb, r + 3 * dm);
        iq<BITS, SK>(v[4 * s], v[4 * s + 1], v[4 * s + 2], v[4 * s + 3], m01, m02, m23, mod);
      }
      const Kc<BITS> m01 = kc<BITS, SK>(x, skb, R + 4 * dm), m02 = kc<BITS, SK>(x, skb, R + 8 * dm),
                     m23 = kc<BITS, SK>(x, skb, R + 12 * dm);
#pragma unroll
      for (int t = 0; t < 4; ++t) iq<BITS, SK>(v[t], v[t + 4], v[t + 8], v[t + 12], m01, m02, m23, mod);
    } else {
      const Kc<BITS> m01 = kc<BITS, SK>(x, skb, R + 4 * dm), m02 = kc<BITS, SK>(x, skb, R + 8 * dm),
                     m23 = kc<BITS, SK>(x, skb, R + 12 * dm);
#pragma unroll
      for (int t = 0; t < 4; ++t) fq<BITS, SK>(v[t], v[t + 4], v[t + 8], v[t + 12], m01, m02, m23, mod);
#pragma unroll
      for (int s = 0; s < 4; ++s) {
        const uint32_t r = R + 4 * s * dm;
        const Kc<BITS> n01 = kc<BITS, SK>(x, skb, r + dm), n02 = kc<BITS, SK>(x, skb, r + 2 * dm),
                       n23 = kc<BITS, SK>(x, skb, r + 3 * dm);
        fq<BITS, SK>(v[4 * s], v[4 * s + 1], v[4 * s + 2], v[4 * s + 3], n01, n02, n23, mod);
      }
    }
  } else if (LG == 3) {
    if (!FWD) {
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        const uint32_t r = R + 4 * s * dm;
        const Kc<BITS> m01 = kc<BITS, SK>(x, skb, r + dm), m02 = kc<BITS, SK>(x, skb, r + 2 * dm),
                       m23 = kc<BITS, SK>(x, skb, r + 3 * dm);
        iq<BITS, SK>(v[4 * s], v[4 * s + 1], v[4 * s + 2], v[4 * s + 3], m01, m02, m23, mod);
      }
      const Kc<BITS> c = kc<BITS, SK>(x, skb, R + 4 * dm);
#pragma unroll
      for (int t = 0; t < 4; ++t) ibf<BITS, SK>(v[t], v[t + 4], c, mod);
    } else {
      const Kc<BITS> m01 = kc<BITS, SK>(x, skb, R + 2 * dm), m02 = kc<BITS, SK>(x, skb, R + 4 * dm),
                     m23 = kc<BITS, SK>(x, skb, R + 6 * dm);
#pragma unroll
      for (int t = 0; t < 2; ++t) fq<BITS, SK>(v[t], v[t + 2], v[t + 4], v[t + 6], m01, m02, m23, mod);
#pragma unroll
      for (int s = 0; s < 4; ++s) {
        const Kc<BITS> c = kc<BITS, SK>(x, skb, R + 2 * s * dm + dm);
        fbf<BITS, SK>(v[2 * s], v[2 * s + 1], c, mod);
      }
    }
  } else if (LG == 2) {
    const Kc<BITS> m01 = kc<BITS, SK>(x, skb, R + dm), m02 = kc<BITS, SK>(x, skb, R + 2 * dm),
                   m23 = kc<BITS, SK>(x, skb, R + 3 * dm);
    if (!FWD)
      iq<BITS, SK>(v[0], v[1], v[2], v[3], m01, m02, m23, mod);
    else
      fq<BITS, SK>(v[0], v[1], v[2], v[3], m01, m02, m23, mod);
  } else if (LG == 1) {
    const Kc<BITS> c = kc<BITS, SK>(x, skb, R + dm);
    if (!FWD)
      ibf<BITS, SK>(v[0], v[1], c, mod);
    else
      fbf<BITS, SK>(v[0], v[1], c, mod);
  }
}

// True when a constant of the group of lanes R + a + dm * j (j < G) may be a
// skew entry whose log is the field modulus.  Those entries are exactly
// 2^i - 1 in both fields' skew tables (checked when the tables are built),
// and the group's constants are entries skb + R + dm * t, 0 < t < G, so the
// question is whether base + dm * t, base = skb + 1 + R, is a power of two
// for such a t.  A power of two of at least dm is a multiple of dm, so base
// must be one, and then base / dm + t must be a power of two.
__device__ __forceinline__ bool group_may_skip(int32_t skb, uint32_t R, uint32_t dm, uint32_t G) {
  const uint32_t base = uint32_t(skb + 1) + R;
  if (base & (dm - 1)) return false;
  const uint32_t q = base / dm + 1;  // smallest candidate
  const uint32_t p2 = q <= 1 ? 1u : 1u << (32 - __clz(q - 1));
  return p2 <= q + G - 2;
}

// One register stage (see stage_regs_k).  GF(2^16): groups that cannot meet
// a skipped multiply run without the per-butterfly test (the choice is
// warp-uniform).  GF(2^8) keeps the test everywhere: the second copy of every
// stage body made its decodes 5-8% slower (config-4 shapes, B200), the
// encodes 3-6% faster.
template <int BITS, int LG, bool FWD>
__device__ __forceinline__ void stage_regs(uint32_t *v, const FftCtx &x, int32_t skb, uint32_t R, uint32_t dm) {
  if (BITS == 8 || group_may_skip(skb, R, dm, 1u << LG))
    stage_regs_k<BITS, LG, FWD, true>(v, x, skb, R, dm);
  else
    stage_regs_k<BITS, LG, FWD, false>(v, x, skb, R, dm);
}

template <int BITS, bool FWD>
__device__ __forceinline__ void stage_regs_rt(uint32_t *v, int lg, const FftCtx &x, int32_t skb, uint32_t R,
                                              uint32_t dm) {
  switch (lg) {
    case 4: stage_regs<BITS, 4, FWD>(v, x, skb, R, dm); break;
    case 3: stage_regs<BITS, 3, FWD>(v, x, skb, R, dm); break;
    case 2: stage_regs<BITS, 2, FWD>(v, x, skb, R, dm); break;
    case 1: stage_regs<BITS, 1, FWD>(v, x, skb, R, dm); break;
    default: break;
  }
}

// Formal derivative of n <= 16 lanes held in registers (all lanes of one
// column word): lane l gains the XOR of lanes l | 2^t over the zero bits t of
// l (src/core/leopard_gf16/decode.rs:1100-1116, restated without the
// in-place sequencing).
__device__ __forceinline__ void derivative_regs(uint32_t *v, uint32_t n) {
  uint32_t o[16];
#pragma unroll
  for (int l = 0; l < 16; ++l) o[l] = v[l];
#pragma unroll
  for (int l = 0; l < 16; ++l)
#pragma unroll
    for (int t = 1; t < 16; t <<= 1)
      if (!(l & t) && uint32_t(l | t) < n) v[l] ^= o[l | t];
}

// ------------------------------------------------------------------ layout
// Split-layout conversion of GF(2^16) words: word w of a 64-byte block holds
// bytes 4w..4w+3; element i of the block is byte i | byte (i + 32) << 8.  The
// partner of word w (< 8) is word w + 8, held by thread lane ^ 8.
template <int BITS>
__device__ __forceinline__ uint32_t fft_to_work(uint32_t w, uint32_t lane) {
  if (BITS == 8) return w;
  const uint32_t other = __shfl_xor_sync(0xffffffffu, w, 8);
  return (lane & 8) ? __byte_perm(other, w, 0x7362) : __byte_perm(w, other, 0x5140);
}
template <int BITS>
__device__ __forceinline__ uint32_t fft_to_user(uint32_t w, uint32_t lane) {
  if (BITS == 8) return w;
  const uint32_t other = __shfl_xor_sync(0xffffffffu, w, 8);
  return (lane & 8) ? __byte_perm(other, w, 0x7531) : __byte_perm(w, other, 0x6420);
}

__device__ __forceinline__ uint32_t ldg_u32(const uint8_t *p) { return __ldg(reinterpret_cast<const uint32_t *>(p)); }

// ------------------------------------------------------------------ stage plans
// A stage is one byte: log2(lanes per thread) in bits 0..2, log2(dm) above.
__device__ __forceinline__ int st_lg(uint8_t s) { return s & 7; }
__device__ __forceinline__ uint8_t st_at(uint32_t plan, uint32_t s) { return uint8_t(plan >> (8 * s)); }

// One shared-memory stage over L lanes held as rows of C words in S (in
// place).  Groups whose base lane is >= mtrunc are skipped.  Every warp takes
// (group, 32-word slice) items; all threads of the CTA call it.  The stage
// shape is a template parameter so that each loop body is straight-line code.
template <int BITS, bool FWD, int LG, int NT>
__device__ __forceinline__ void smem_stage_lg(uint32_t *S, uint32_t C, uint32_t lgC32, uint32_t L, uint32_t lgdm,
                                              const FftCtx &x, int32_t skb, uint32_t mtrunc) {
  constexpr uint32_t G = 1u << LG;
  const uint32_t dm = 1u << lgdm;
  const uint32_t warp = threadIdx.x >> 5;
  const uint32_t items = (L >> LG) << lgC32;
  for (uint32_t it = warp; it < items; it += NT / 32) {
    const uint32_t grp = it >> lgC32, slice = it & ((1u << lgC32) - 1);
    const uint32_t a = grp & (dm - 1), R = (grp >> lgdm) << (LG + lgdm);
    if (R >= mtrunc) continue;  // warp-uniform
    uint32_t *base = S + size_t(R + a) * C + slice * 32 + x.lane;
    const size_t step = size_t(dm) * C;
    uint32_t v[G];
#pragma unroll
    for (uint32_t j = 0; j < G; ++j) v[j] = base[j * step];
    stage_regs<BITS, LG, FWD>(v, x, skb, R, dm);
#pragma unroll
    for (uint32_t j = 0; j < G; ++j) base[j * step] = v[j];
  }
}

template <int BITS, bool FWD, int NT>
__device__ __forceinline__ void smem_stage(uint32_t *S, uint32_t C, uint32_t lgC32, uint32_t L, uint8_t st,
                                        const FftCtx &x, int32_t skb, uint32_t mtrunc) {
  const uint32_t lgdm = st >> 3;
  switch (st_lg(st)) {
    case 4: smem_stage_lg<BITS, FWD, 4, NT>(S, C, lgC32, L, lgdm, x, skb, mtrunc); break;
    case 3: smem_stage_lg<BITS, FWD, 3, NT>(S, C, lgC32, L, lgdm, x, skb, mtrunc); break;
    case 2: smem_stage_lg<BITS, FWD, 2, NT>(S, C, lgC32, L, lgdm, x, skb, mtrunc); break;
    default: smem_stage_lg<BITS, FWD, 1, NT>(S, C, lgC32, L, lgdm, x, skb, mtrunc); break;
  }
}

// Formal derivative over n >= 32 lanes held as rows of C >= 32 words (shared
// memory, or the global work rows), in place: lane l gains the XOR of the old
// lanes l | 2^t over the zero bits t of l (src/core/leopard_gf16/decode.rs:
// 1100-1116, restated without the in-place sequencing).  A warp takes one
// group of 16 consecutive lanes of a 32-word slice per round, as the stages
// do: bits 0-3 come from its own 16 registers (lane j's sources are lanes
// above j, so an ascending in-place pass reads only old values), and each
// zero bit t >= 4 of the group's base adds the 16 lanes 2^t above it, 16
// independent loads.  New lane l depends only on old lanes above it, and the
// groups are taken in ascending order, so each round reads everything it
// needs, waits for the whole CTA, then writes.
template <int NT>
__device__ void smem_derivative(uint32_t *S, uint32_t C, uint32_t lgC, uint32_t n) {
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t lgC32 = lgC - 5, lgn = 31 - __clz(n);
  const uint32_t items = (n >> 4) << lgC32;
  for (uint32_t r0 = 0; r0 < items; r0 += NT / 32) {
    const uint32_t it = r0 + warp;
    const bool have = it < items;  // warp-uniform
    uint32_t v[16];
    uint32_t *base = S;
    if (have) {
      const uint32_t R = (it >> lgC32) << 4;
      base = S + size_t(R) * C + ((it & ((1u << lgC32) - 1)) << 5) + lane;
#pragma unroll
      for (int j = 0; j < 16; ++j) v[j] = base[size_t(j) * C];
#pragma unroll
      for (int j = 0; j < 16; ++j)
#pragma unroll
        for (int t = 1; t < 16; t <<= 1)
          if (!(j & t)) v[j] ^= v[j | t];
      for (uint32_t t = 4; t < lgn; ++t) {
        if (R & (1u << t)) continue;  // warp-uniform
        const uint32_t *src = base + (size_t(1) << t) * C;
#pragma unroll
        for (int h = 0; h < 16; h += 8) {  // eight loads in flight at a time (register cap)
          uint32_t u[8];
#pragma unroll
          for (int j = 0; j < 8; ++j) u[j] = src[size_t(h + j) * C];
#pragma unroll
          for (int j = 0; j < 8; ++j) v[h + j] ^= u[j];
        }
      }
    }
    __syncthreads();
    if (have) {
#pragma unroll
      for (int j = 0; j < 16; ++j) base[size_t(j) * C] = v[j];
    }
    __syncthreads();
  }
}

// The same derivative one word per thread, up to kHold words per round: the
// form the mixed kernel keeps (its K1 tiles share the kernel's 80 registers,
// and the grouped form's 16-lane registers made the whole kernel spill more:
// the mixed workload 2.7% slower).
template <int NT>
__device__ void flat_derivative(uint32_t *S, uint32_t C, uint32_t lgC, uint32_t n) {
  constexpr int kHold = 8;
  const uint32_t total = n << lgC;
  for (uint32_t base = 0; base < total; base += NT * kHold) {
    uint32_t nv[kHold];
#pragma unroll
    for (int h = 0; h < kHold; ++h) {
      const uint32_t q = base + h * NT + threadIdx.x;
      nv[h] = 0;
      if (q < total) {
        const uint32_t l = q >> lgC, w = q & (C - 1);
        uint32_t v = S[q];
        for (uint32_t t = 1; (l | t) < n; t <<= 1)
          if (!(l & t)) v ^= S[size_t(l | t) * C + w];
        nv[h] = v;
      }
    }
    __syncthreads();
#pragma unroll
    for (int h = 0; h < kHold; ++h) {
      const uint32_t q = base + h * NT + threadIdx.x;
      if (q < total) S[q] = nv[h];
    }
    __syncthreads();
  }
}

}  // namespace
}  // namespace rsgpu

namespace rsgpu {
namespace {

// ------------------------------------------------------------------ encode
// Encoder IFFT stage 0 of group g (16 consecutive lanes per thread), straight
// from the data shards (zero past cnt); writes T, or the accumulator A when
// it is the only stage (assign for the first group, XOR after).
template <int BITS, int NT>
__device__ __forceinline__ void enc_stage0(uint32_t *dst, bool accumulate, const LeoArgs &a, const uint8_t *const *ptr,
                                        uint32_t g, uint32_t cnt, uint32_t C, uint32_t lgC32, uint64_t col0,
                                        uint64_t len, const FftCtx &x, int32_t skb) {
  const uint32_t warp = threadIdx.x >> 5, m = a.m;
  const uint32_t items = (m >> 4) << lgC32;
  for (uint32_t it = warp; it < items; it += NT / 32) {
    const uint32_t R = (it >> lgC32) << 4, slice = it & ((1u << lgC32) - 1);
    const uint32_t wi = slice * 32 + x.lane;
    const uint64_t col = col0 + 4ull * wi;
    uint32_t v[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      uint32_t w = 0;
      if (R + j < cnt && col < len) w = ldg_u32(ptr[g * m + R + j] + col);
      v[j] = fft_to_work<BITS>(w, x.lane);
    }
    if (R < cnt) stage_regs<BITS, 4, false>(v, x, skb, R, 1);
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      uint32_t *d = dst + size_t(R + j) * C + wi;
      *d = accumulate ? (*d ^ v[j]) : v[j];
    }
  }
}

// Last encoder IFFT stage: T -> registers -> accumulator (assign for the
// first group, XOR for the rest).  No group is skipped here.
template <int BITS, int LG, int NT>
__device__ __forceinline__ void enc_last_ifft_lg(const uint32_t *T, uint32_t *A, bool accumulate, uint32_t C,
                                                 uint32_t lgC32, uint32_t m, uint32_t lgdm, const FftCtx &x,
                                                 int32_t skb) {
  constexpr uint32_t G = 1u << LG;
  const uint32_t dm = 1u << lgdm, warp = threadIdx.x >> 5;
  const uint32_t items = (m >> LG) << lgC32;
  const size_t step = size_t(dm) * C;
  for (uint32_t it = warp; it < items; it += NT / 32) {
    const uint32_t grp = it >> lgC32, slice = it & ((1u << lgC32) - 1);
    const uint32_t aa = grp & (dm - 1), R = (grp >> lgdm) << (LG + lgdm);
    const size_t off = size_t(R + aa) * C + slice * 32 + x.lane;
    uint32_t v[G];
#pragma unroll
    for (uint32_t j = 0; j < G; ++j) v[j] = T[off + j * step];
    stage_regs<BITS, LG, false>(v, x, skb, R, dm);
#pragma unroll
    for (uint32_t j = 0; j < G; ++j) {
      uint32_t *d = A + off + j * step;
      *d = accumulate ? (*d ^ v[j]) : v[j];
    }
  }
}

template <int BITS, int NT>
__device__ __forceinline__ void enc_last_ifft(const uint32_t *T, uint32_t *A, bool accumulate, uint32_t C,
                                           uint32_t lgC32, uint32_t m, uint8_t st, const FftCtx &x,
                                           int32_t skb) {
  const uint32_t lgdm = st >> 3;
  switch (st_lg(st)) {
    case 4: enc_last_ifft_lg<BITS, 4, NT>(T, A, accumulate, C, lgC32, m, lgdm, x, skb); break;
    case 3: enc_last_ifft_lg<BITS, 3, NT>(T, A, accumulate, C, lgC32, m, lgdm, x, skb); break;
    case 2: enc_last_ifft_lg<BITS, 2, NT>(T, A, accumulate, C, lgC32, m, lgdm, x, skb); break;
    default: enc_last_ifft_lg<BITS, 1, NT>(T, A, accumulate, C, lgC32, m, lgdm, x, skb); break;
  }
}

// Last encoder FFT stage (consecutive lanes): accumulator -> registers ->
// parity shards 0..p (or compared with them).  Returns this thread's mismatch.
template <int BITS, bool VERIFY, int LG, int NT>
__device__ __forceinline__ uint32_t enc_out_lg(const uint32_t *A, const LeoArgs &a, const uint8_t *const *ptr,
                                               uint32_t C, uint32_t lgC32, uint64_t col0, uint64_t len,
                                               const FftCtx &x, int32_t skf) {
  constexpr uint32_t G = 1u << LG;
  const uint32_t warp = threadIdx.x >> 5, m = a.m, p = a.p, k = a.k;
  const uint32_t items = (m >> LG) << lgC32;
  uint32_t mismatch = 0;
  for (uint32_t it = warp; it < items; it += NT / 32) {
    const uint32_t R = (it >> lgC32) << LG, slice = it & ((1u << lgC32) - 1);
    if (R >= p) continue;  // warp-uniform
    const uint32_t wi = slice * 32 + x.lane;
    const uint64_t col = col0 + 4ull * wi;
    uint32_t v[G];
#pragma unroll
    for (uint32_t j = 0; j < G; ++j) v[j] = A[size_t(R + j) * C + wi];
    stage_regs<BITS, LG, true>(v, x, skf, R, 1);
#pragma unroll
    for (uint32_t j = 0; j < G; ++j) {
      if (R + j >= p) break;  // warp-uniform
      const uint32_t u = fft_to_user<BITS>(v[j], x.lane);
      if (col < len) {
        uint32_t *out = reinterpret_cast<uint32_t *>(const_cast<uint8_t *>(ptr[k + R + j]) + col);
        if (VERIFY)
          mismatch |= (__ldg(out) != u);
        else
          *out = u;
      }
    }
  }
  return mismatch;
}

template <int BITS, bool VERIFY, int NT>
__device__ __forceinline__ uint32_t enc_out(const uint32_t *A, const LeoArgs &a, const uint8_t *const *ptr, uint32_t C,
                                         uint32_t lgC32, uint8_t st, uint64_t col0, uint64_t len, const FftCtx &x,
                                         int32_t skf) {
  switch (st_lg(st)) {
    case 4: return enc_out_lg<BITS, VERIFY, 4, NT>(A, a, ptr, C, lgC32, col0, len, x, skf);
    case 3: return enc_out_lg<BITS, VERIFY, 3, NT>(A, a, ptr, C, lgC32, col0, len, x, skf);
    case 2: return enc_out_lg<BITS, VERIFY, 2, NT>(A, a, ptr, C, lgC32, col0, len, x, skf);
    default: return enc_out_lg<BITS, VERIFY, 1, NT>(A, a, ptr, C, lgC32, col0, len, x, skf);
  }
}

// Registers-only encode (m <= 16): one word per thread, all m lanes in
// registers.  Returns this thread's mismatch.
template <int BITS, bool VERIFY, int LG>
__device__ __forceinline__ uint32_t enc_regs_lg(const LeoArgs &a, const uint8_t *const *ptr, uint64_t col0,
                                                uint64_t len, const FftCtx &x) {
  constexpr uint32_t M = 1u << LG;
  const uint32_t k = a.k, p = a.p;
  const uint64_t col = col0 + 4ull * threadIdx.x;
  const bool act = col < len;  // whole 64-byte blocks, so uniform per half-warp
  uint32_t acc[M];
#pragma unroll
  for (uint32_t j = 0; j < M; ++j) acc[j] = 0;
  for (uint32_t g = 0; g * M < k; ++g) {
    const uint32_t cnt = min(M, k - g * M);
    uint32_t v[M];
#pragma unroll
    for (uint32_t j = 0; j < M; ++j) {
      uint32_t w = 0;
      if (j < cnt && act) w = ldg_u32(ptr[g * M + j] + col);
      v[j] = fft_to_work<BITS>(w, x.lane);
    }
    stage_regs<BITS, LG, false>(v, x, int32_t(M - 1 + g * M), 0, 1);
#pragma unroll
    for (uint32_t j = 0; j < M; ++j) acc[j] ^= v[j];
  }
  stage_regs<BITS, LG, true>(acc, x, -1, 0, 1);
  uint32_t mismatch = 0;
#pragma unroll
  for (uint32_t j = 0; j < M; ++j) {
    if (j >= p) break;
    const uint32_t u = fft_to_user<BITS>(acc[j], x.lane);
    if (act) {
      uint32_t *out = reinterpret_cast<uint32_t *>(const_cast<uint8_t *>(ptr[k + j]) + col);
      if (VERIFY)
        mismatch |= (__ldg(out) != u);
      else
        *out = u;
    }
  }
  return mismatch;
}

template <int BITS, bool VERIFY>
__device__ __forceinline__ uint32_t enc_regs(const LeoArgs &a, const uint8_t *const *ptr, uint64_t col0, uint64_t len,
                                          const FftCtx &x) {
  switch (a.m) {
    case 16: return enc_regs_lg<BITS, VERIFY, 4>(a, ptr, col0, len, x);
    case 8: return enc_regs_lg<BITS, VERIFY, 3>(a, ptr, col0, len, x);
    case 4: return enc_regs_lg<BITS, VERIFY, 2>(a, ptr, col0, len, x);
    case 2: return enc_regs_lg<BITS, VERIFY, 1>(a, ptr, col0, len, x);
    default: return enc_regs_lg<BITS, VERIFY, 0>(a, ptr, col0, len, x);
  }
}

// Encode (or, with VERIFY, recompute and compare) one column tile of job jd.
// src/core/leopard_gf8/encode.rs:194-372, src/core/leopard_gf16/encode.rs:109-252:
// each group of m data shards (zero past k) goes through the encoder IFFT
// (skew base fft_skew + m - 1 + g*m) and is XORed into an accumulator, which
// then goes through the FFT (skew base fft_skew - 1); lanes 0..p are parity.
//
// m <= 16: registers only; the tile is NT words (4 NT bytes) of every shard,
//   one word per thread, and W is unused.
// m >= 32: W holds 2m rows of C = 16 * a.nb words (IFFT scratch, then the
//   accumulator); the tile is 4C bytes of every shard.
template <int BITS, bool VERIFY, int NT>
__device__ void fft_encode_tile(uint32_t *W, const LeoArgs &a, const LeoJob &jd, uint64_t col0, uint64_t len,
                                uint32_t *bad) {
  const uint32_t lane = threadIdx.x & 31;
  const FftCtx x{a.kbank, a.mod, lane, a.skew, a.sktab};
  const uint32_t m = a.m, k = a.k;
  const uint8_t *const *ptr = a.ptrs + jd.ptr_off;
  uint32_t mismatch = 0;
  if (VERIFY) {
    if (threadIdx.x == 0) *bad = 0;
    __syncthreads();  // the reset lands before any warp can report
  }
  if (m <= 16) {
    mismatch = enc_regs<BITS, VERIFY>(a, ptr, col0, len, x);
  } else {
    const uint32_t C = a.nb * 16, lgC32 = 31 - __clz(C >> 5);
    uint32_t *T = W, *A = W + size_t(m) * C;
    for (uint32_t g = 0; g * m < k; ++g) {
      const uint32_t cnt = min(m, k - g * m);
      const int32_t skb = int32_t(m - 1 + g * m);
      enc_stage0<BITS, NT>(T, false, a, ptr, g, cnt, C, lgC32, col0, len, x, skb);
      __syncthreads();
      for (uint32_t s = 1; s + 1 < a.n_ienc; ++s) {
        smem_stage<BITS, false, NT>(T, C, lgC32, m, st_at(a.st_ienc, s), x, skb, cnt);
        __syncthreads();
      }
      enc_last_ifft<BITS, NT>(T, A, g != 0, C, lgC32, m, st_at(a.st_ienc, a.n_ienc - 1), x, skb);
      __syncthreads();
    }
    // FFT over the accumulator; the last stage (consecutive lanes) writes parity.
    const int32_t skf = -1;
    for (uint32_t s = 0; s + 1 < a.n_fenc; ++s) {
      smem_stage<BITS, true, NT>(A, C, lgC32, m, st_at(a.st_fenc, s), x, skf, a.p);
      __syncthreads();
    }
    mismatch = enc_out<BITS, VERIFY, NT>(A, a, ptr, C, lgC32, st_at(a.st_fenc, a.n_fenc - 1), col0, len, x, skf);
  }
  if (VERIFY) {
    if (__any_sync(0xffffffffu, mismatch) && lane == 0) atomicOr(bad, 1u);
    __syncthreads();
    if (threadIdx.x == 0 && *bad) atomicOr(a.flags + jd.flag_idx, 1u);
  }
  __syncthreads();
}

// ------------------------------------------------------------------ decode
// Shard behind decode lane l: parity i at lane i, data j at lane m + j.
__device__ __forceinline__ int lane_shard(uint32_t l, uint32_t k, uint32_t p, uint32_t m) {
  if (l < p) return int(k + l);
  if (l >= m && l < m + k) return int(l - m);
  return -1;
}

// Load decode lane l of the thread's word: present shards scaled by their
// error locator, everything else zero.
template <int BITS>
__device__ __forceinline__ uint32_t dec_load(const LeoArgs &a, const LeoJob &jd, const uint8_t *const *ptr,
                                             uint32_t l, uint64_t col, bool act, const FftCtx &x) {
  const int sh = lane_shard(l, a.k, a.p, a.m);
  const bool present = sh >= 0 && jd.role[sh] == 1;  // warp-uniform
  uint32_t w = 0;
  if (present && act) w = ldg_u32(ptr[sh] + col);
  w = fft_to_work<BITS>(w, x.lane);
  if (present) w = kmul(w, kload<BITS>(x.bank, jd.err[l], x.lane));
  return w;
}

// Store decode lane l if its shard is a target: scaled by mod - err[l].
template <int BITS>
__device__ __forceinline__ void dec_store(const LeoArgs &a, const LeoJob &jd, const uint8_t *const *ptr, uint32_t l,
                                          uint64_t col, bool act, uint32_t v, const FftCtx &x) {
  const int sh = lane_shard(l, a.k, a.p, a.m);
  if (sh < 0 || jd.role[sh] != 2) return;  // warp-uniform
  v = kmul(v, kload<BITS>(x.bank, a.mod - jd.err[l], x.lane));
  v = fft_to_user<BITS>(v, x.lane);
  if (act) *reinterpret_cast<uint32_t *>(const_cast<uint8_t *>(ptr[sh]) + col) = v;
}

// Decoder IFFT stage 0 (16 consecutive lanes per thread), straight from HBM.
template <int BITS, int NT>
__device__ __forceinline__ void dec_stage0(uint32_t *S, const LeoArgs &a, const LeoJob &jd, const uint8_t *const *ptr,
                                        uint32_t C, uint32_t lgC32, uint64_t col0, uint64_t len, const FftCtx &x,
                                        int32_t skd) {
  const uint32_t warp = threadIdx.x >> 5, in_cnt = jd.input_count;
  const uint32_t items = (a.n >> 4) << lgC32;
  for (uint32_t it = warp; it < items; it += NT / 32) {
    const uint32_t R = (it >> lgC32) << 4, slice = it & ((1u << lgC32) - 1);
    const uint32_t wi = slice * 32 + x.lane;
    const uint64_t col = col0 + 4ull * wi;
    uint32_t v[16];
    if (R < in_cnt) {
#pragma unroll
      for (int j = 0; j < 16; ++j) v[j] = dec_load<BITS>(a, jd, ptr, R + j, col, col < len, x);
      stage_regs<BITS, 4, false>(v, x, skd, R, 1);
    } else {
#pragma unroll
      for (int j = 0; j < 16; ++j) v[j] = 0;
    }
#pragma unroll
    for (int j = 0; j < 16; ++j) S[size_t(R + j) * C + wi] = v[j];
  }
}

// Last decoder FFT stage (consecutive lanes): S -> registers -> targets.
template <int BITS, int LG, int NT>
__device__ __forceinline__ void dec_out_lg(const uint32_t *S, const LeoArgs &a, const LeoJob &jd,
                                           const uint8_t *const *ptr, uint32_t C, uint32_t lgC32, uint64_t col0,
                                           uint64_t len, const FftCtx &x, int32_t skd) {
  constexpr uint32_t G = 1u << LG;
  const uint32_t warp = threadIdx.x >> 5, out_cnt = a.m + a.k;
  const uint32_t items = (a.n >> LG) << lgC32;
  for (uint32_t it = warp; it < items; it += NT / 32) {
    const uint32_t R = (it >> lgC32) << LG, slice = it & ((1u << lgC32) - 1);
    if (R >= out_cnt) continue;  // warp-uniform
    const uint32_t wi = slice * 32 + x.lane;
    const uint64_t col = col0 + 4ull * wi;
    uint32_t v[G];
#pragma unroll
    for (uint32_t j = 0; j < G; ++j) v[j] = S[size_t(R + j) * C + wi];
    stage_regs<BITS, LG, true>(v, x, skd, R, 1);
#pragma unroll
    for (uint32_t j = 0; j < G; ++j) dec_store<BITS>(a, jd, ptr, R + j, col, col < len, v[j], x);
  }
}

template <int BITS, int NT>
__device__ __forceinline__ void dec_out(const uint32_t *S, const LeoArgs &a, const LeoJob &jd, const uint8_t *const *ptr,
                                     uint32_t C, uint32_t lgC32, uint8_t st, uint64_t col0, uint64_t len,
                                     const FftCtx &x, int32_t skd) {
  switch (st_lg(st)) {
    case 4: dec_out_lg<BITS, 4, NT>(S, a, jd, ptr, C, lgC32, col0, len, x, skd); break;
    case 3: dec_out_lg<BITS, 3, NT>(S, a, jd, ptr, C, lgC32, col0, len, x, skd); break;
    case 2: dec_out_lg<BITS, 2, NT>(S, a, jd, ptr, C, lgC32, col0, len, x, skd); break;
    default: dec_out_lg<BITS, 1, NT>(S, a, jd, ptr, C, lgC32, col0, len, x, skd); break;
  }
}

// Registers-only decode (n <= 16): one word per thread, all n lanes in registers.
template <int BITS, int LG>
__device__ __forceinline__ void dec_regs_lg(const LeoArgs &a, const LeoJob &jd, const uint8_t *const *ptr,
                                            uint64_t col0, uint64_t len, const FftCtx &x) {
  constexpr uint32_t N = 1u << LG;
  const uint64_t col = col0 + 4ull * threadIdx.x;
  const bool act = col < len;
  const int32_t skd = -1;
  uint32_t v[16];
#pragma unroll
  for (uint32_t j = 0; j < 16; ++j) v[j] = j < N ? dec_load<BITS>(a, jd, ptr, j, col, act, x) : 0u;
  stage_regs<BITS, LG, false>(v, x, skd, 0, 1);
  derivative_regs(v, N);
  stage_regs<BITS, LG, true>(v, x, skd, 0, 1);
#pragma unroll
  for (uint32_t j = 0; j < N; ++j) dec_store<BITS>(a, jd, ptr, j, col, act, v[j], x);
}

template <int BITS>
__device__ __forceinline__ void dec_regs(const LeoArgs &a, const LeoJob &jd, const uint8_t *const *ptr, uint64_t col0,
                                      uint64_t len, const FftCtx &x) {
  switch (a.n) {
    case 16: dec_regs_lg<BITS, 4>(a, jd, ptr, col0, len, x); break;
    case 8: dec_regs_lg<BITS, 3>(a, jd, ptr, col0, len, x); break;
    case 4: dec_regs_lg<BITS, 2>(a, jd, ptr, col0, len, x); break;
    default: dec_regs_lg<BITS, 1>(a, jd, ptr, col0, len, x); break;
  }
}

// Reconstruct one column tile of job jd (src/core/leopard_gf8/decode.rs:291-420,
// src/core/leopard_gf16/decode.rs:704-910): scale present lanes by their error
// locators, IFFT (blocks below input_count), formal derivative, FFT (blocks
// below m + k), scale targets by mod - locator.
// n <= 16: registers only, tile = 4 NT bytes.  n >= 32: W holds n rows of
// C = 16 * a.nb words, tile = 4C bytes.
// GROUPED: the formal derivative by 16-lane groups (smem_derivative) or one
// word per thread (flat_derivative; the mixed kernel's choice).
template <int BITS, int NT, bool GROUPED = true>
__device__ void fft_decode_tile(uint32_t *W, const LeoArgs &a, const LeoJob &jd, uint64_t col0, uint64_t len) {
  const uint32_t lane = threadIdx.x & 31;
  const FftCtx x{a.kbank, a.mod, lane, a.skew, a.sktab};
  const uint32_t n = a.n;
  const uint8_t *const *ptr = a.ptrs + jd.ptr_off;
  const int32_t skd = -1;
  if (n <= 16) {
    dec_regs<BITS>(a, jd, ptr, col0, len, x);
    __syncthreads();
    return;
  }
  const uint32_t C = a.nb * 16, lgC32 = 31 - __clz(C >> 5), lgC = lgC32 + 5;
  uint32_t *S = W;
  dec_stage0<BITS, NT>(S, a, jd, ptr, C, lgC32, col0, len, x, skd);
  __syncthreads();
  for (uint32_t s = 1; s < a.n_idec; ++s) {
    smem_stage<BITS, false, NT>(S, C, lgC32, n, st_at(a.st_idec, s), x, skd, jd.input_count);
    __syncthreads();
  }
  if (GROUPED)
    smem_derivative<NT>(S, C, lgC, n);
  else
    flat_derivative<NT>(S, C, lgC, n);
  for (uint32_t s = 0; s + 1 < a.n_fdec; ++s) {
    smem_stage<BITS, true, NT>(S, C, lgC32, n, st_at(a.st_fdec, s), x, skd, a.m + a.k);
    __syncthreads();
  }
  dec_out<BITS, NT>(S, a, jd, ptr, C, lgC32, st_at(a.st_fdec, a.n_fdec - 1), col0, len, x, skd);
  __syncthreads();
}

}  // namespace
}  // namespace rsgpu
