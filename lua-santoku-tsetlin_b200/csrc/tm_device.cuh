// Device helpers shared by the train kernels (tm_kernels.cu,
// tm_train_wpt.cu): the Philox draws of the draw contract, mbarrier waits and
// TMA bulk row copies, and the bit-sliced automaton updates.
#pragma once

#include "tm_internal.h"

namespace tmb {

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11).  Counter words are
// (sample, epoch, unit, stream); the key is the machine's seed.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                       uint64_t key, uint32_t *o) {
  uint32_t k0 = (uint32_t)key, k1 = (uint32_t)(key >> 32);
#pragma unroll
  for (int r = 0; r < 10; r++) {
    const uint32_t hi0 = __umulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
    const uint32_t hi1 = __umulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
    const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
    c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  o[0] = c0; o[1] = c1; o[2] = c2; o[3] = c3;
}

// draw < a with p = a / range  <=>  floor(u * range / 2^32) < a
__device__ __forceinline__ uint64_t bounded64(uint32_t u, uint64_t range) {
  return ((uint64_t)u * range) >> 32;
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// ---------------------------------------------------------------------------
// mbarrier + TMA bulk copy helpers (sm_90+ PTX; no cluster multicast)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// Sample rows are streamed once per unit; they are loaded with an L2
// evict-first policy so that they do not displace the automata of units
// whose state lives in global memory.
__device__ __forceinline__ void tma_row(uint64_t *bar, void *dst, const void *src,
                                        uint32_t bytes) {
  uint64_t pol;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], "
      "[%1], %2, [%3], %4;" ::"r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar)), "l"(pol)
      : "memory");
}
// Bounded wait for the phase with the given parity; false on time-out.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity,
                                          uint32_t limit = TM_WAIT_LIMIT) {
  const uint32_t a = smem_u32(bar);
  for (uint32_t it = 0; it < limit; it++) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// ---------------------------------------------------------------------------
// Bit-sliced automaton updates on one 32-bit word of one clause.
//   act_j   : action row of the clause
//   cnt_j   : its m = B-1 count planes, stride Wp
// ---------------------------------------------------------------------------

// Saturating +1 on bits I and -1 on bits D (I & D == 0).  A decrement is an
// increment in complemented space: flip the D bits of every plane, ripple a
// carry of (I|D) through the count planes and (masked by am) the action
// plane, saturate overflowing bits at all ones, flip back.  Equivalent to
// tk_automata_inc on I followed by tk_automata_dec on D (automata.h:88-318).
__device__ __forceinline__ void w_add(uint32_t *__restrict__ act_j, uint32_t *__restrict__ cnt_j,
                                      uint32_t Wp, uint32_t m, uint32_t w, uint32_t I, uint32_t D,
                                      uint32_t am) {
  uint32_t c = I | D;
  if (!c) return;
  for (uint32_t b = 0; b < m && c; b++) {
    const uint32_t p = cnt_j[b * Wp + w] ^ D;
    cnt_j[b * Wp + w] = (p ^ c) ^ D;
    c &= p;
  }
  if (!c) return;
  const uint32_t a = act_j[w] ^ D;
  const uint32_t ca = c & am;
  uint32_t na = a ^ ca;
  c = a & ca;
  if (c) {
    for (uint32_t b = 0; b < m; b++) cnt_j[b * Wp + w] = ((cnt_j[b * Wp + w] ^ D) | c) ^ D;
    na |= c;
  }
  act_j[w] = na ^ D;
}

// Saturating subtraction of 2^l on bits M (Type Ib picks, counted in binary).
__device__ __forceinline__ void w_sub_pow2(uint32_t *__restrict__ act_j,
                                           uint32_t *__restrict__ cnt_j, uint32_t Wp, uint32_t m,
                                           uint32_t w, uint32_t l, uint32_t M, uint32_t am) {
  if (!M) return;
  if (l > m) {  // 2^l exceeds every value
    for (uint32_t b = 0; b < m; b++) cnt_j[b * Wp + w] &= ~M;
    act_j[w] &= ~M;
    return;
  }
  uint32_t bw = M;
  for (uint32_t b = l; b < m && bw; b++) {
    const uint32_t p = cnt_j[b * Wp + w];
    cnt_j[b * Wp + w] = p ^ bw;
    bw &= ~p;
  }
  if (!bw) return;
  const uint32_t a = act_j[w];
  const uint32_t ba = bw & am;
  uint32_t na = a ^ ba;
  bw = ~a & ba;
  if (bw) {
    for (uint32_t b = 0; b < m; b++) cnt_j[b * Wp + w] &= ~bw;
    na &= ~bw;
  }
  act_j[w] = na;
}

// automata.h:499-512
__device__ __forceinline__ uint32_t w_included(const uint32_t *act_j, const uint32_t *cnt_j,
                                               uint32_t Wp, uint32_t m, uint32_t ib, uint32_t w) {
  uint32_t inc = act_j[w];
  for (uint32_t i = 1; i < ib && i <= m; i++) inc &= cnt_j[(m - i) * Wp + w];
  return inc;
}

// Register-resident forms of the same updates.  The B-1 count planes and
// the action of one word are loaded together (all loads in flight at once),
// updated in registers and stored together; BM bounds B-1 at compile time
// so every plane index is static.
template <int BM>
__device__ __forceinline__ void ld_word(const uint32_t *__restrict__ act_j,
                                        const uint32_t *__restrict__ cnt_j, uint32_t Wp,
                                        uint32_t m, uint32_t w, uint32_t (&p)[BM], uint32_t &a) {
#pragma unroll
  for (int b = 0; b < BM; b++)
    if (b < (int)m) p[b] = cnt_j[b * Wp + w];
  a = act_j[w];
}

template <int BM>
__device__ __forceinline__ void st_word(uint32_t *__restrict__ act_j, uint32_t *__restrict__ cnt_j,
                                        uint32_t Wp, uint32_t m, uint32_t w,
                                        const uint32_t (&p)[BM], uint32_t a) {
#pragma unroll
  for (int b = 0; b < BM; b++)
    if (b < (int)m) cnt_j[b * Wp + w] = p[b];
  act_j[w] = a;
}

// automata.h:499-512: action AND the top include_bits-1 count planes
template <int BM>
__device__ __forceinline__ uint32_t rg_included(const uint32_t (&p)[BM], uint32_t a, uint32_t m,
                                                uint32_t ib) {
  uint32_t inc = a;
#pragma unroll
  for (int b = 0; b < BM; b++)
    if (b < (int)m && b + (int)ib > (int)m) inc &= p[b];
  return inc;
}

// w_add on registers
template <int BM>
__device__ __forceinline__ void rg_add(uint32_t (&p)[BM], uint32_t &a, uint32_t m, uint32_t I,
                                       uint32_t D, uint32_t am) {
  uint32_t c = I | D;
#pragma unroll
  for (int b = 0; b < BM; b++)
    if (b < (int)m) {
      const uint32_t q = p[b] ^ D;
      p[b] = (q ^ c) ^ D;
      c &= q;
    }
  const uint32_t af = a ^ D, ca = c & am;
  uint32_t na = af ^ ca;
  c = af & ca;
  if (c) {
#pragma unroll
    for (int b = 0; b < BM; b++)
      if (b < (int)m) p[b] = ((p[b] ^ D) | c) ^ D;
    na |= c;
  }
  a = na ^ D;
}

// w_sub_pow2 on registers
template <int BM>
__device__ __forceinline__ void rg_sub_pow2(uint32_t (&p)[BM], uint32_t &a, uint32_t m,
                                            uint32_t l, uint32_t M, uint32_t am) {
  if (!M) return;
  if (l > m) {
#pragma unroll
    for (int b = 0; b < BM; b++)
      if (b < (int)m) p[b] &= ~M;
    a &= ~M;
    return;
  }
  uint32_t bw = M;
#pragma unroll
  for (int b = 0; b < BM; b++)
    if (b >= (int)l && b < (int)m) {
      const uint32_t q = p[b];
      p[b] = q ^ bw;
      bw &= ~q;
    }
  const uint32_t ba = bw & am;
  uint32_t na = a ^ ba;
  bw = ~a & ba;
  if (bw) {
#pragma unroll
    for (int b = 0; b < BM; b++)
      if (b < (int)m) p[b] &= ~bw;
    na &= ~bw;
  }
  a = na;
}

// Two consecutive words at once: the B-1 planes and the action of words
// w0, w0+1 (w0 even) are moved with 64-bit accesses and updated word by word
// in registers (two words keep the live state within 128 registers).
template <int BM>
__device__ __forceinline__ void ld_pair(const uint32_t *__restrict__ act_c,
                                        const uint32_t *__restrict__ cnt_c, uint32_t Wp,
                                        uint32_t m, uint32_t w0, uint32_t (&p)[2][BM],
                                        uint32_t (&a)[2]) {
#pragma unroll
  for (int b = 0; b < BM; b++)
    if (b < (int)m) {
      const uint2 t = *(const uint2 *)(cnt_c + b * Wp + w0);
      p[0][b] = t.x;
      p[1][b] = t.y;
    }
  const uint2 t = *(const uint2 *)(act_c + w0);
  a[0] = t.x;
  a[1] = t.y;
}

template <int BM>
__device__ __forceinline__ void st_pair(uint32_t *__restrict__ act_c, uint32_t *__restrict__ cnt_c,
                                        uint32_t Wp, uint32_t m, uint32_t w0,
                                        const uint32_t (&p)[2][BM], const uint32_t (&a)[2]) {
#pragma unroll
  for (int b = 0; b < BM; b++)
    if (b < (int)m) *(uint2 *)(cnt_c + b * Wp + w0) = make_uint2(p[0][b], p[1][b]);
  *(uint2 *)(act_c + w0) = make_uint2(a[0], a[1]);
}

// rg_add with no decrements (Type II): plain carry ripple.
template <int BM>
__device__ __forceinline__ void rg_inc(uint32_t (&p)[BM], uint32_t &a, uint32_t m, uint32_t I,
                                       uint32_t am) {
  uint32_t c = I;
#pragma unroll
  for (int b = 0; b < BM; b++)
    if (b < (int)m) {
      const uint32_t q = p[b];
      p[b] = q ^ c;
      c &= q;
    }
  const uint32_t ca = c & am;
  uint32_t na = a ^ ca;
  c = a & ca;
  if (c) {
#pragma unroll
    for (int b = 0; b < BM; b++)
      if (b < (int)m) p[b] |= c;
    na |= c;
  }
  a = na;
}

// rg_add with no increments (Type Ia when L > clause_maximum): plain borrow
// ripple, saturating at zero.
template <int BM>
__device__ __forceinline__ void rg_dec(uint32_t (&p)[BM], uint32_t &a, uint32_t m, uint32_t D,
                                       uint32_t am) {
  uint32_t bw = D;
#pragma unroll
  for (int b = 0; b < BM; b++)
    if (b < (int)m) {
      const uint32_t q = p[b];
      p[b] = q ^ bw;
      bw &= ~q;
    }
  const uint32_t ba = bw & am;
  uint32_t na = a ^ ba;
  bw = ~a & ba;
  if (bw) {
#pragma unroll
    for (int b = 0; b < BM; b++)
      if (b < (int)m) p[b] &= ~bw;
    na &= ~bw;
  }
  a = na;
}

// Mask of word w0 + k given the last-word mask `last` and W words.
__device__ __forceinline__ uint32_t word_mask(uint32_t w, uint32_t W, uint32_t last) {
  return w + 1 < W ? 0xFFFFFFFFu : (w + 1 == W ? last : 0u);
}

}  // namespace tmb
