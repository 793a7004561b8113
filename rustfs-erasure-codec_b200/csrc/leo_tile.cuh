// leo_tile.cuh -- device code of the Leopard FFT codecs, one column tile at a
// time, shared by the per-codec kernels (leopard.cu) and the mixed-batch
// persistent kernel (batch.cu).
//
// Every column of a shard is independent, so a CTA owns a tile of columns of
// one stripe and holds *all* transform lanes of that tile in a work area
// (shared memory, or a per-CTA slab of global memory for very wide codes):
// shards cross HBM exactly once (data in, parity or recovered shards out) and
// every IFFT / formal-derivative / FFT layer runs on chip.  A lane row is one
// 64-byte block (64 GF(2^8) columns, or 32 GF(2^16) columns in the
// reference's split byte layout, src/core/leopard_gf16/ops.rs:513-807) and is
// owned by one half-warp: 16 lanes x one 32-bit word.  Multiplication by a
// butterfly constant g^log_m uses nibble tables held one entry per lane and
// read with width-16 warp shuffles, so the two halves of a warp can work on
// different butterflies with different constants.
//
// NT is the CTA size (a multiple of 32); every function below is called by
// all NT threads of the CTA together.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "leo_types.hpp"

namespace rsgpu {
namespace {

template <int BITS>
struct Tab;
template <>
struct Tab<8> {
  uint32_t lo, hi;
};
template <>
struct Tab<16> {
  uint32_t t0, t1, t2, t3;
};

__device__ __forceinline__ uint32_t shfl16(uint32_t v, uint32_t idx) {
  uint32_t r;
  asm("shfl.sync.idx.b32 %0, %1, %2, 0x101f, -1;" : "=r"(r) : "r"(v), "r"(idx));
  return r;
}

template <int BITS>
__device__ __forceinline__ Tab<BITS> load_tab(const uint32_t *bank, uint32_t lm, uint32_t hl);
template <>
__device__ __forceinline__ Tab<8> load_tab<8>(const uint32_t *bank, uint32_t lm, uint32_t hl) {
  const uint2 v = __ldg(reinterpret_cast<const uint2 *>(bank) + lm * 16 + hl);
  return Tab<8>{v.x, v.y};
}
template <>
__device__ __forceinline__ Tab<16> load_tab<16>(const uint32_t *bank, uint32_t lm, uint32_t hl) {
  const uint4 v = __ldg(reinterpret_cast<const uint4 *>(bank) + lm * 16 + hl);
  return Tab<16>{v.x, v.y, v.z, v.w};
}

// Products of the elements of word w with the half-warp's constant.
__device__ __forceinline__ uint32_t mulw(uint32_t w, const Tab<8> &t) {
  const uint32_t s0 = shfl16(t.lo, w) ^ shfl16(t.hi, w >> 4);
  const uint32_t s1 = shfl16(t.lo, w >> 8) ^ shfl16(t.hi, w >> 12);
  const uint32_t s2 = shfl16(t.lo, w >> 16) ^ shfl16(t.hi, w >> 20);
  const uint32_t s3 = shfl16(t.lo, w >> 24) ^ shfl16(t.hi, w >> 28);
  return __byte_perm(__byte_perm(s0, s1, 0x0040), __byte_perm(s2, s3, 0x4000), 0x7610);
}
__device__ __forceinline__ uint32_t mulw(uint32_t w, const Tab<16> &t) {
  const uint32_t a = shfl16(t.t0, w) ^ shfl16(t.t1, w >> 4) ^ shfl16(t.t2, w >> 8) ^ shfl16(t.t3, w >> 12);
  const uint32_t b = shfl16(t.t0, w >> 16) ^ shfl16(t.t1, w >> 20) ^ shfl16(t.t2, w >> 24) ^ shfl16(t.t3, w >> 28);
  return __byte_perm(a, b, 0x7610);
}

// Split-layout conversion of a 64-byte GF(2^16) block held as 16 words by a
// half-warp (word t = bytes 4t..4t+3 of the block).
__device__ __forceinline__ uint32_t user_to_work16(uint32_t w, uint32_t hl) {
  const uint32_t other = __shfl_xor_sync(0xffffffffu, w, 8, 16);
  return hl < 8 ? __byte_perm(w, other, 0x5140) : __byte_perm(other, w, 0x7362);
}
__device__ __forceinline__ uint32_t work_to_user16(uint32_t w, uint32_t hl) {
  const uint32_t other = __shfl_xor_sync(0xffffffffu, w, 8, 16);
  return hl < 8 ? __byte_perm(w, other, 0x6420) : __byte_perm(other, w, 0x7531);
}

template <int BITS>
__device__ __forceinline__ uint32_t from_user(uint32_t w, uint32_t hl) {
  return BITS == 16 ? user_to_work16(w, hl) : w;
}
template <int BITS>
__device__ __forceinline__ uint32_t to_user(uint32_t w, uint32_t hl) {
  return BITS == 16 ? work_to_user16(w, hl) : w;
}

// Row r, column block cb: 16 words.
__device__ __forceinline__ uint32_t *row_ptr(uint32_t *W, uint32_t nb, uint32_t r, uint32_t cb) {
  return W + (size_t(r) * nb + cb) * kRowWords;
}

// dit2 on rows x, y of column block cb (forward: x ^= y*c, y ^= x;
// inverse: y ^= x, x ^= y*c; log_m == mod means only y ^= x).  Both
// half-warps always execute the shuffles; `valid` gates the stores.
template <int BITS, bool FWD>
__device__ __forceinline__ void dit2(uint32_t *W, uint32_t nb, uint32_t cb, uint32_t x, uint32_t y, uint32_t lm,
                                     const Tab<BITS> &t, uint32_t mod, bool valid, uint32_t hl) {
  uint32_t *px = row_ptr(W, nb, valid ? x : 0, cb) + hl;
  uint32_t *py = row_ptr(W, nb, valid ? y : 0, cb) + hl;
  uint32_t xv = *px, yv = *py;
  const bool skip = lm == mod;
  if (FWD) {
    const uint32_t prod = mulw(yv, t);
    if (!skip) xv ^= prod;
    yv ^= xv;
  } else {
    yv ^= xv;
    const uint32_t prod = mulw(yv, t);
    if (!skip) xv ^= prod;
  }
  if (valid) {
    *px = xv;
    *py = yv;
  }
}

// One radix-4 layer over lanes [0, nl): blocks r < mtrunc step 4*dist, each
// spanning lanes i, i+dist, i+2dist, i+3dist for i in [r, r+dist).
// Skew factors: sk[iend + adj], sk[iend + dist + adj], sk[iend + 2dist + adj].
template <int BITS, bool FWD, int NT>
__device__ void layer4(uint32_t *W, const LeoArgs &a, const uint16_t *sk, int adj, uint32_t nl, uint32_t mtrunc,
                       uint32_t dist) {
  constexpr uint32_t kHalfWarps = NT / 16;
  const uint32_t hw = threadIdx.x >> 4, hl = threadIdx.x & 15;
  const uint32_t dist4 = dist * 4;
  const uint32_t nblk = (mtrunc + dist4 - 1) / dist4;
  const uint32_t items = nblk * dist * a.nb;
  const uint32_t rounds = (items + kHalfWarps - 1) / kHalfWarps;
  for (uint32_t rd = 0; rd < rounds; ++rd) {
    const uint32_t q = rd * kHalfWarps + hw;
    const bool valid = q < items;
    const uint32_t qq = valid ? q : 0;
    const uint32_t cb = qq % a.nb, bq = qq / a.nb;
    const uint32_t r = (bq / dist) * dist4, i = r + bq % dist;
    const uint32_t iend = r + dist;
    const uint32_t m01 = sk[int(iend) + adj], m02 = sk[int(iend + dist) + adj], m23 = sk[int(iend + 2 * dist) + adj];
    const Tab<BITS> t01 = load_tab<BITS>(a.bank, m01, hl);
    const Tab<BITS> t23 = load_tab<BITS>(a.bank, m23, hl);
    const Tab<BITS> t02 = load_tab<BITS>(a.bank, m02, hl);
    const uint32_t ia = i, ib = i + dist, ic = i + 2 * dist, id = i + 3 * dist;
    const bool ha = ia < nl, hb = ib < nl, hc = ic < nl, hd = id < nl;
    if (FWD) {
      dit2<BITS, true>(W, a.nb, cb, ia, ic, m02, t02, a.mod, valid && ha && hc, hl);
      dit2<BITS, true>(W, a.nb, cb, ib, id, m02, t02, a.mod, valid && hb && hd, hl);
      dit2<BITS, true>(W, a.nb, cb, ia, ib, m01, t01, a.mod, valid && ha && hb, hl);
      dit2<BITS, true>(W, a.nb, cb, ic, id, m23, t23, a.mod, valid && hc && hd, hl);
    } else {
      dit2<BITS, false>(W, a.nb, cb, ia, ib, m01, t01, a.mod, valid && ha && hb, hl);
      dit2<BITS, false>(W, a.nb, cb, ic, id, m23, t23, a.mod, valid && hc && hd, hl);
      dit2<BITS, false>(W, a.nb, cb, ia, ic, m02, t02, a.mod, valid && ha && hc, hl);
      dit2<BITS, false>(W, a.nb, cb, ib, id, m02, t02, a.mod, valid && hb && hd, hl);
    }
  }
}

// Final radix-2 layer: pairs (i, i + dist) for i in [0, count), constant per pair.
template <int BITS, bool FWD, int NT>
__device__ void layer2(uint32_t *W, const LeoArgs &a, uint32_t nl, uint32_t count, uint32_t dist, uint32_t stride,
                       const uint16_t *lm_of, int lm_fixed) {
  constexpr uint32_t kHalfWarps = NT / 16;
  const uint32_t hw = threadIdx.x >> 4, hl = threadIdx.x & 15;
  const uint32_t items = count * a.nb;
  const uint32_t rounds = (items + kHalfWarps - 1) / kHalfWarps;
  for (uint32_t rd = 0; rd < rounds; ++rd) {
    const uint32_t q = rd * kHalfWarps + hw;
    const bool valid = q < items;
    const uint32_t qq = valid ? q : 0;
    const uint32_t cb = qq % a.nb, i = (qq / a.nb) * stride;
    const uint32_t lm = lm_fixed >= 0 ? uint32_t(lm_fixed) : lm_of[i];
    const Tab<BITS> t = load_tab<BITS>(a.bank, lm, hl);
    dit2<BITS, FWD>(W, a.nb, cb, i, i + dist, lm, t, a.mod, valid && i + dist < nl, hl);
  }
}

// Encoder IFFT (src/core/leopard_gf16/mod.rs build_ifft_dit16_plan): lanes >=
// mtrunc hold zeros, skew base = fft_skew + (m - 1) + group offset.
template <int BITS, int NT>
__device__ void ifft_encoder(uint32_t *W, const LeoArgs &a, const uint16_t *sk, uint32_t mtrunc) {
  const uint32_t m = a.m;
  uint32_t dist = 1, dist4 = 4;
  while (dist4 <= m) {
    layer4<BITS, false, NT>(W, a, sk, 0, m, mtrunc, dist);
    __syncthreads();
    dist = dist4;
    dist4 <<= 2;
  }
  if (dist < m) {
    layer2<BITS, false, NT>(W, a, m, dist, dist, 1, nullptr, sk[dist]);
    __syncthreads();
  }
}

// FFT (build_fft_dit16_plan): skew = fft_skew, i_end - 1 indexing.
template <int BITS, int NT>
__device__ void fft(uint32_t *W, const LeoArgs &a, uint32_t nl, uint32_t mtrunc, uint32_t msize) {
  uint32_t dist4 = msize, dist = msize >> 2;
  while (dist != 0) {
    layer4<BITS, true, NT>(W, a, a.skew, -1, nl, mtrunc, dist);
    __syncthreads();
    dist4 = dist;
    dist >>= 2;
  }
  if (dist4 == 2) {
    layer2<BITS, true, NT>(W, a, nl, (mtrunc + 1) / 2, 1, 2, a.skew, -1);
    __syncthreads();
  }
}

// Decoder IFFT (build_ifft_decode_dit16_plan): blocks r < input_count.
template <int BITS, int NT>
__device__ void ifft_decoder(uint32_t *W, const LeoArgs &a, uint32_t mtrunc) {
  const uint32_t n = a.n;
  uint32_t dist = 1, dist4 = 4;
  while (dist4 <= n) {
    layer4<BITS, false, NT>(W, a, a.skew, -1, n, mtrunc, dist);
    __syncthreads();
    dist = dist4;
    dist4 <<= 2;
  }
  if (dist < n) {
    layer2<BITS, false, NT>(W, a, n, dist, dist, 1, nullptr, a.skew[dist - 1]);
    __syncthreads();
  }
}

// Formal derivative (decode.rs compute_formal_derivative16): lane l gains the
// XOR of lanes l + 2^t for every zero bit t of l with l + 2^t < n.  Lanes
// are rewritten in increasing order in rounds, so every read sees the value
// from before the pass.
template <int NT>
__device__ void derivative(uint32_t *W, const LeoArgs &a) {
  constexpr uint32_t kHalfWarps = NT / 16;
  const uint32_t hw = threadIdx.x >> 4, hl = threadIdx.x & 15;
  const uint32_t items = a.n * a.nb;
  for (uint32_t base = 0; base < items; base += kHalfWarps) {
    const uint32_t q = base + hw;
    uint32_t v = 0;
    const bool valid = q < items;
    uint32_t l = 0, cb = 0;
    if (valid) {
      l = q / a.nb;
      cb = q % a.nb;
      v = row_ptr(W, a.nb, l, cb)[hl];
      for (uint32_t w = 1; l + w < a.n; w <<= 1)
        if (!(l & w)) v ^= row_ptr(W, a.nb, l + w, cb)[hl];
    }
    __syncthreads();
    if (valid) row_ptr(W, a.nb, l, cb)[hl] = v;
    __syncthreads();
  }
}

__device__ __forceinline__ uint32_t ld_u32(const uint8_t *p) {
  return __ldg(reinterpret_cast<const uint32_t *>(p));
}

// Encode (or, with VERIFY, recompute and compare) the column tile starting at
// byte col0 of job jd, whose shards are len bytes long.  W holds 2m rows of
// a.nb blocks.  `bad` is a shared-memory word of the CTA (verify only).
// src/core/leopard_gf8/encode.rs:194-372, src/core/leopard_gf16/encode.rs:109-252.
template <int BITS, bool VERIFY, int NT>
__device__ void leo_encode_tile(uint32_t *W, const LeoArgs &a, const LeoJob &jd, uint64_t col0, uint64_t len,
                                uint32_t *bad) {
  constexpr uint32_t kHalfWarps = NT / 16;
  const uint32_t hw = threadIdx.x >> 4, hl = threadIdx.x & 15;
  const uint32_t m = a.m;
  uint32_t *acc = W, *tmp = W + size_t(m) * a.nb * kRowWords;
  const uint8_t *const *ptr = a.ptrs + jd.ptr_off;
  if (VERIFY && threadIdx.x == 0) *bad = 0;
  // Each group of m data shards passes through an IFFT and is XORed into acc.
  for (uint32_t g = 0; g * m < a.k; ++g) {
    uint32_t *dst = g == 0 ? acc : tmp;
    const uint32_t cnt = g == 0 ? a.mtrunc : (a.k - g * m < m ? a.k - g * m : m);
    // Rounds keep both halves of every warp in step (the layout shuffle
    // needs all 32 lanes).
    for (uint32_t base = 0; base < m * a.nb; base += kHalfWarps) {
      const uint32_t q = base + hw;
      const bool valid = q < m * a.nb;
      const uint32_t l = valid ? q / a.nb : 0, cb = valid ? q % a.nb : 0;
      const uint64_t col = col0 + uint64_t(cb) * 64;
      uint32_t v = 0;
      if (valid && l < cnt && col < len) v = ld_u32(ptr[g * m + l] + col + hl * 4);
      v = from_user<BITS>(v, hl);
      if (valid) row_ptr(dst, a.nb, l, cb)[hl] = v;
    }
    __syncthreads();
    const uint16_t *sk = a.skew + (m - 1) + g * m;
    ifft_encoder<BITS, NT>(dst, a, sk, cnt);
    if (g > 0) {
      for (uint32_t i = threadIdx.x; i < m * a.nb * kRowWords; i += NT) acc[i] ^= tmp[i];
      __syncthreads();
    }
  }
  fft<BITS, NT>(acc, a, m, a.p, m);
  // Parity lanes 0..p back to user layout (or compared against the stored parity).
  uint32_t mismatch = 0;
  for (uint32_t base = 0; base < a.p * a.nb; base += kHalfWarps) {
    const uint32_t q = base + hw;
    const bool valid = q < a.p * a.nb;
    const uint32_t l = valid ? q / a.nb : 0, cb = valid ? q % a.nb : 0;
    const uint64_t col = col0 + uint64_t(cb) * 64;
    const uint32_t v = to_user<BITS>(row_ptr(acc, a.nb, l, cb)[hl], hl);
    if (valid && col < len) {
      uint32_t *out = reinterpret_cast<uint32_t *>(const_cast<uint8_t *>(ptr[a.k + l]) + col) + hl;
      if (VERIFY)
        mismatch |= (*out != v);
      else
        *out = v;
    }
  }
  if (VERIFY) {
    if (mismatch) atomicOr(bad, 1u);
    __syncthreads();
    if (threadIdx.x == 0 && *bad) atomicOr(a.flags + jd.flag_idx, 1u);
  }
  __syncthreads();
}

// Reconstruct the column tile starting at byte col0 of job jd.  W holds n
// rows of a.nb blocks.  src/core/leopard_gf8/decode.rs:291-420,
// src/core/leopard_gf16/decode.rs:704-910.
template <int BITS, int NT>
__device__ void leo_decode_tile(uint32_t *W, const LeoArgs &a, const LeoJob &jd, uint64_t col0, uint64_t len) {
  constexpr uint32_t kHalfWarps = NT / 16;
  const uint32_t hw = threadIdx.x >> 4, hl = threadIdx.x & 15;
  const uint32_t m = a.m, n = a.n, k = a.k, p = a.p;
  const uint8_t *const *ptr = a.ptrs + jd.ptr_off;
  // Step 1: lanes 0..p parity, m..m+k data; present lanes scaled by their
  // error locator, everything else zero.
  for (uint32_t base = 0; base < n * a.nb; base += kHalfWarps) {
    const uint32_t q = base + hw;
    const bool valid = q < n * a.nb;
    const uint32_t l = valid ? q / a.nb : 0, cb = valid ? q % a.nb : 0;
    const uint64_t col = col0 + uint64_t(cb) * 64;
    int shard = -1;
    if (l < p)
      shard = int(k + l);
    else if (l >= m && l < m + k)
      shard = int(l - m);
    const bool load = valid && shard >= 0 && jd.role[shard] == 1 && col < len;
    uint32_t v = 0;
    if (load) v = ld_u32(ptr[shard] + col + hl * 4);
    // Every half-warp converts and multiplies (shuffles must stay
    // converged); unused rows multiply zero by the identity.
    v = from_user<BITS>(v, hl);
    const uint32_t lm = load ? jd.err[l] : a.mod;
    const Tab<BITS> tb = load_tab<BITS>(a.bank, lm, hl);
    v = mulw(v, tb);
    if (valid) row_ptr(W, a.nb, l, cb)[hl] = v;
  }
  __syncthreads();
  ifft_decoder<BITS, NT>(W, a, jd.input_count);
  derivative<NT>(W, a);
  fft<BITS, NT>(W, a, n, m + k, n);
  // Step 5: each target scaled by mod - err and written in user layout.
  for (uint32_t base = 0; base < (k + p) * a.nb; base += kHalfWarps) {
    const uint32_t q = base + hw;
    const bool valid = q < (k + p) * a.nb;
    const uint32_t i = valid ? q / a.nb : 0, cb = valid ? q % a.nb : 0;
    const uint64_t col = col0 + uint64_t(cb) * 64;
    const bool target = valid && jd.role[i] == 2;
    const uint32_t lane = i >= k ? i - k : m + i;
    const uint32_t lm = target ? (a.mod - jd.err[lane]) : a.mod;
    const Tab<BITS> tb = load_tab<BITS>(a.bank, lm, hl);
    const uint32_t v = to_user<BITS>(mulw(row_ptr(W, a.nb, lane, cb)[hl], tb), hl);
    if (target && col < len) reinterpret_cast<uint32_t *>(const_cast<uint8_t *>(ptr[i]) + col)[hl] = v;
  }
  __syncthreads();
}

}  // namespace
}  // namespace rsgpu
