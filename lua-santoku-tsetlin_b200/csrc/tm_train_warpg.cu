// k_train_warpg: one warp per unit for rows of at most 32 x WPL words
// (WPL = 4 or 8: up to 128 or 256 words) with 8-bit automata -- the encoder
// and mid-width classifier rows.  As in k_train_warp (tm_kernels.cu) a warp
// trains its unit alone, warp-synchronously: no CTA barrier, no sample ring,
// the chance draws of 32 epoch positions made at once (one position per
// lane) and broadcast by shuffles.  Lane l owns words l + 32 h (h < WPL)
// of all eight clauses.  Only the action plane (read by every evaluation)
// lives in the warp's shared memory (8 KB for 256-word rows, so up to 16
// units per SM); the seven count planes stay in global memory, where the
// owning lane reads and writes a word's planes only when feedback reaches
// that word (coalesced: the lanes' words are consecutive).  The feedback of
// one clause loads the planes of two of the lane's words before updating
// either, to keep loads in flight.  Same rules and draws as k_train
// (capi.c:163-243): bit-identical results.
#include <cuda_runtime.h>

#include "tm_device.cuh"
#include "tm_internal.h"

namespace tmb {

namespace {

constexpr uint32_t kM = 7;  // count planes of 8-bit automata

// One word's seven count planes (global memory, read through L2 only: the
// lanes of the warp write them between reads) and its action (shared
// memory).
__device__ __forceinline__ void ldg_word(const uint32_t *act_c, const uint32_t *cnt_c,
                                         uint32_t Wp, uint32_t w, uint32_t (&p)[kM],
                                         uint32_t &a) {
#pragma unroll
  for (uint32_t b = 0; b < kM; b++) p[b] = __ldcg(cnt_c + b * Wp + w);
  a = act_c[w];
}

__device__ __forceinline__ void stg_word(uint32_t *act_c, uint32_t *cnt_c, uint32_t Wp,
                                         uint32_t w, const uint32_t (&p)[kM], uint32_t a) {
#pragma unroll
  for (uint32_t b = 0; b < kM; b++) __stcg(cnt_c + b * Wp + w, p[b]);
  act_c[w] = a;
}

template <int WPL>
__global__ void __launch_bounds__(32, 16)
    k_train_warpg(const TrainDev *__restrict__ machines, const WorkItem *__restrict__ work,
                  uint32_t nwork, uint32_t *__restrict__ counter, uint32_t e_begin,
                  uint32_t e_end, uint32_t act_words, uint32_t ib_words, uint32_t ovf_cap,
                  unsigned long long *__restrict__ pairs) {
  extern __shared__ __align__(128) uint8_t smem[];
  const uint32_t lane = threadIdx.x & 31;
  uint32_t *act = (uint32_t *)smem;  // 8 x Wp words of the current unit
  uint32_t *lev0 = act + act_words, *lev1 = lev0 + ib_words, *ovf = lev1 + ib_words;
  uint32_t *cnt_ovf = ovf + ovf_cap;  // [0]: overflow entries
  for (uint32_t i = lane; i < 2 * ib_words; i += 32) lev0[i] = 0;
  if (lane == 0) cnt_ovf[0] = 0;
  __syncwarp();
  while (true) {
    uint32_t u = 0;
    if (lane == 0) {
      // the next unit, passing over those of machines whose gate is closed
      u = atomicAdd(counter, 1u);
      while (u < nwork) {
        const uint32_t *gt = machines[work[u].m].gate;
        if (!gt || *gt) break;
        u = atomicAdd(counter, 1u);
      }
    }
    u = __shfl_sync(0xFFFFFFFFu, u, 0);
    if (u >= nwork) break;
    const WorkItem wi = work[u];
    const TrainDev &M = machines[wi.m];
    const ClassDev C = M.cls[wi.h];
    const uint32_t Wp = C.Wp, W = C.W;
    const uint32_t g = wi.h * M.clause_chunks + wi.k;
    uint32_t *gact = M.act + C.act_off + (uint64_t)wi.k * 8 * Wp;
    uint32_t *gcnt = M.cnt + C.cnt_off + (uint64_t)wi.k * 8 * kM * Wp;
    for (uint32_t i = lane; i < 2 * Wp; i += 32) ((uint4 *)act)[i] = ((const uint4 *)gact)[i];
    __syncwarp();
    const uint32_t T = M.T;
    const uint64_t T2 = 2ull * T;
    const uint32_t ep_end = e_end < M.epochs ? e_end : M.epochs;
    const uint32_t *xbase = M.x + C.x_off;
    uint32_t lits = 0;  // lane q < 8: literal count of clause q (valid when !dirty)
    uint32_t dirty = 0xFFu;

    for (uint32_t e = e_begin; e < ep_end; e++) {
      const uint32_t ee = M.epoch_base + e;
      const uint32_t *perm = M.perm + (uint64_t)(e - e_begin) * M.n;
      for (uint32_t base = 0; base < M.n; base += 32) {
        const uint32_t i = base + lane;
        bool live = false;
        uint32_t s = 0, pos = 0;
        uint32_t d[8];
        if (i < M.n) {
          s = perm[i];
          if (M.type == 0) {
            pos = (uint32_t)M.labels[s] == wi.h;
            live = pos;
            if (!pos) {
              uint32_t o[4];
              philox(s, ee, g, ST_NEG, M.seed, o);
              live = (uint64_t)o[0] >= M.thr_neg;
            }
          } else {
            pos = (M.codes[(uint64_t)s * M.code_bytes + (wi.h >> 3)] >> (wi.h & 7)) & 1u;
            live = true;
          }
          if (live) {
            philox(s, ee, g, ST_CH0, M.seed, d);
            philox(s, ee, g, ST_CH1, M.seed, d + 4);
          }
        }
        uint32_t bal = __ballot_sync(0xFFFFFFFFu, live);
        if (lane == 0 && pairs && bal) atomicAdd(pairs, (unsigned long long)__popc(bal));
        if (!bal) continue;
        while (bal) {
          const uint32_t src = __ffs(bal) - 1;
          bal &= bal - 1;
          const uint32_t sp = __shfl_sync(0xFFFFFFFFu, s, src);
          const uint32_t pa = __shfl_sync(0xFFFFFFFFu, pos, src);
          uint32_t dd[8];
#pragma unroll
          for (int k = 0; k < 8; k++) dd[k] = __shfl_sync(0xFFFFFFFFu, d[k], src);
          // the sample's row: word lane + 32 h (the loads of all the lane's
          // words in flight at once; other warps cover their latency)
          uint32_t xa[WPL];
#pragma unroll
          for (int h = 0; h < WPL; h++) {
            const uint32_t w = lane + 32 * h;
            xa[h] = w < W ? xbase[(uint64_t)sp * Wp + w] : 0u;
          }
          // evaluation of the 8 clauses (capi.c:97-122)
          uint32_t Lq = 0, Fq = 0;
#pragma unroll 2
          for (uint32_t c = 0; c < 8; c++) {
            const bool dl = (dirty >> c) & 1u;
            uint32_t fc = 0, lc = 0;
#pragma unroll
            for (int h = 0; h < WPL; h++) {
              const uint32_t w = lane + 32 * h;
              const uint32_t a = (w < W ? act[c * Wp + w] : 0u) & word_mask(w, W, C.emask);
              fc += __popc(a & ~xa[h]);
              if (dl) lc += __popc(a);
            }
            fc = __reduce_add_sync(0xFFFFFFFFu, fc);
            if (lane == c) Fq = fc;
            if (dl) {
              lc = __reduce_add_sync(0xFFFFFFFFu, lc);
              if (lane == c) Lq = lc;
            } else if (lane == c) {
              Lq = lits;
            }
          }
          lits = Lq;
          dirty = 0;
          int32_t vq = 0;
          if (lane < 8) {
            if (Lq == 0)
              vq = (int32_t)M.tol;
            else {
              vq = (int32_t)(Lq < M.tol ? Lq : M.tol) - (int32_t)Fq;
              vq = vq < 0 ? 0 : vq;
            }
          }
          int32_t v = __reduce_add_sync(0xFFFFFFFFu, (lane & 1) ? -vq : vq);
          v = v > (int32_t)T ? (int32_t)T : v;
          v = v < -(int32_t)T ? -(int32_t)T : v;
          const uint64_t av = (uint64_t)(pa ? (int64_t)T - v : (int64_t)T + v);
          // lane c < 8 decides clause c (capi.c:226-242)
          const uint32_t odd = lane & 1u;
          const bool type1 = pa ? !odd : odd;
          uint32_t dsel = 0;
#pragma unroll
          for (int k = 0; k < 8; k++)
            if ((uint32_t)k == ((lane & 7) & ~1u) + (type1 ? 0u : 1u)) dsel = dd[k];
          const bool fire = lane < 8 && bounded64(dsel, T2) < av;
          const uint32_t ibm = __ballot_sync(0xFFFFFFFFu, fire && type1 && vq == 0);
          const uint32_t fbm = __ballot_sync(0xFFFFFFFFu, fire && vq > 0);
          const uint32_t t1m = __ballot_sync(0xFFFFFFFFu, fire && type1 && vq > 0);
          const uint32_t incm =
              __ballot_sync(0xFFFFFFFFu, fire && type1 && vq > 0 && Lq <= M.maxlit);
          dirty = fbm | ibm;
          // Type Ia / II (capi.c:177-180, 192-196) on the lane's words, two
          // at a time: their planes are loaded before either is updated
          for (uint32_t cm = fbm; cm; cm &= cm - 1) {
            const uint32_t c = __ffs(cm) - 1;
            uint32_t *act_c = act + c * Wp, *cnt_c = gcnt + (size_t)c * kM * Wp;
            const bool t1 = (t1m >> c) & 1u, incx = (incm >> c) & 1u;
#pragma unroll
            for (int h0 = 0; h0 < WPL; h0 += 2) {
              uint32_t pp[2][kM], aq[2];
              bool on[2];
#pragma unroll
              for (int j = 0; j < 2; j++) {
                const uint32_t w = lane + 32 * (h0 + j);
                const uint32_t x = xa[h0 + j], vm = word_mask(w, W, C.vmask);
                // only Type Ia with increments changes a word whose literals are all 1
                on[j] = w < W && ((t1 && incx) || (~x & vm) != 0);
                if (on[j]) ldg_word(act_c, cnt_c, Wp, w, pp[j], aq[j]);
              }
#pragma unroll
              for (int j = 0; j < 2; j++) {
                if (!on[j]) continue;
                const uint32_t w = lane + 32 * (h0 + j);
                const uint32_t x = xa[h0 + j], vm = word_mask(w, W, C.vmask);
                const uint32_t am = word_mask(w, W, C.amask);
                const uint32_t nx = ~x & ~rg_included<kM>(pp[j], aq[j], kM, M.ib) & vm;
                if (t1 && incx)
                  rg_add<kM>(pp[j], aq[j], kM, x & vm, nx, am);
                else if (t1)
                  rg_dec<kM>(pp[j], aq[j], kM, nx, am);
                else
                  rg_inc<kM>(pp[j], aq[j], kM, nx, am);
                stg_word(act_c, cnt_c, Wp, w, pp[j], aq[j]);
              }
            }
          }
          // Type Ib (capi.c:181-190): picks counted per bit in two levels
          // (plus overflow entries worth 4), then applied word by word
          for (uint32_t cm = ibm; cm; cm &= cm - 1) {
            const uint32_t c = __ffs(cm) - 1;
            uint32_t *act_c = act + c * Wp, *cnt_c = gcnt + (size_t)c * kM * Wp;
            const uint32_t npk = C.s_picks, nq = (npk + 3) >> 2;
            for (uint32_t q = lane; q < nq; q += 32) {
              uint32_t o[4];
              philox(sp, ee, g, ST_IB | (c << 20) | q, M.seed, o);
#pragma unroll
              for (uint32_t r = 0; r < 4; r++) {
                if (4 * q + r < npk) {
                  const uint32_t bit = __umulhi(o[r], C.input_bits);
                  const uint32_t w = bit >> 5, mk = 1u << (bit & 31);
                  if (atomicXor(&lev0[w], mk) & mk) {
                    if (atomicXor(&lev1[w], mk) & mk) {
                      const uint32_t at = atomicAdd(&cnt_ovf[0], 1u);
                      if (at < ovf_cap) ovf[at] = bit;
                    }
                  }
                }
              }
            }
            __syncwarp();
#pragma unroll
            for (int h0 = 0; h0 < WPL; h0 += 2) {
              uint32_t pp[2][kM], aq[2], m0[2], m1[2];
              bool on[2];
#pragma unroll
              for (int j = 0; j < 2; j++) {
                const uint32_t w = lane + 32 * (h0 + j);
                m0[j] = w < W ? lev0[w] : 0u;
                m1[j] = w < W ? lev1[w] : 0u;
                on[j] = (m0[j] | m1[j]) != 0;
                if (on[j]) {
                  lev0[w] = 0;
                  lev1[w] = 0;
                  ldg_word(act_c, cnt_c, Wp, w, pp[j], aq[j]);
                }
              }
#pragma unroll
              for (int j = 0; j < 2; j++) {
                if (!on[j]) continue;
                const uint32_t w = lane + 32 * (h0 + j);
                const uint32_t am = word_mask(w, W, C.amask);
                rg_sub_pow2<kM>(pp[j], aq[j], kM, 0, m0[j], am);
                rg_sub_pow2<kM>(pp[j], aq[j], kM, 1, m1[j], am);
                stg_word(act_c, cnt_c, Wp, w, pp[j], aq[j]);
              }
            }
            // the overflow entries' words may belong to any lane: their
            // planes were written by those lanes above
            __syncwarp();
            const uint32_t no = cnt_ovf[0];
            if (no) {
              if (lane == 0) {
                for (uint32_t t = 0; t < no && t < ovf_cap; t++) {
                  const uint32_t bit = ovf[t], w = bit >> 5;
                  const uint32_t am = word_mask(w, W, C.amask);
                  uint32_t pp[kM], aq;
                  ldg_word(act_c, cnt_c, Wp, w, pp, aq);
                  rg_sub_pow2<kM>(pp, aq, kM, 2, 1u << (bit & 31), am);
                  stg_word(act_c, cnt_c, Wp, w, pp, aq);
                }
                cnt_ovf[0] = 0;
              }
              __syncwarp();
            }
          }
          __syncwarp();
        }
      }
    }
    __syncwarp();
    for (uint32_t i = lane; i < 2 * Wp; i += 32) ((uint4 *)gact)[i] = ((const uint4 *)act)[i];
    __syncwarp();
  }
}

// shared memory of one unit, in words: the action plane, two Type Ib
// levels of ib_words, the overflow entries and their count (a multiple of
// 32 words: every slice starts 16-byte aligned)
uint32_t warpg_words(uint32_t Wpmax, uint32_t ovf_cap) {
  return (8 * Wpmax + 2 * Wpmax + ovf_cap + 32 + 31) / 32 * 32;
}

template <int WPL>
int warpg_occ(size_t bytes) {
  cudaFuncSetAttribute(k_train_warpg<WPL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)bytes);
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_train_warpg<WPL>, 32, bytes) !=
      cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return nb;
}

}  // namespace

int train_warpg_wpl(uint32_t Wpmax) { return Wpmax <= 128 ? 4 : (Wpmax <= 256 ? 8 : 0); }

int train_warpg_occupancy(uint32_t Wpmax, uint32_t smax, size_t *smem_bytes) {
  const int wpl = train_warpg_wpl(Wpmax);
  if (!wpl) return 0;
  const uint32_t ovf_cap = smax / 4 > 0 ? smax / 4 : 1;
  const size_t bytes = (size_t)warpg_words(Wpmax, ovf_cap) * 4;
  *smem_bytes = bytes;
  return wpl == 4 ? warpg_occ<4>(bytes) : warpg_occ<8>(bytes);
}

cudaError_t launch_train_warpg(const TrainDev *machines, const WorkItem *work, uint32_t nwork,
                               uint32_t *counter, uint32_t e_begin, uint32_t e_end,
                               uint32_t Wpmax, uint32_t smax, int grid, cudaStream_t st,
                               unsigned long long *pairs) {
  const int wpl = train_warpg_wpl(Wpmax);
  if (!wpl || grid <= 0) return cudaErrorInvalidValue;
  const uint32_t ovf_cap = smax / 4 > 0 ? smax / 4 : 1;
  const size_t bytes = (size_t)warpg_words(Wpmax, ovf_cap) * 4;
  if (wpl == 4)
    k_train_warpg<4><<<grid, 32, bytes, st>>>(machines, work, nwork, counter, e_begin, e_end,
                                              8 * Wpmax, Wpmax, ovf_cap, pairs);
  else
    k_train_warpg<8><<<grid, 32, bytes, st>>>(machines, work, nwork, counter, e_begin, e_end,
                                              8 * Wpmax, Wpmax, ovf_cap, pairs);
  return cudaGetLastError();
}

}  // namespace tmb
