// sm_100a kernels of the Tsetlin-machine hot path.
//
//   k_repack    reference byte rows -> padded 32-bit word rows
//   k_setup     automata initial state (automata.h:72-86)
//   k_perm_keys + CUB radix sort: the epoch's sample order
//   k_train     fused clause evaluation + Type I/II feedback, one CTA per
//               unit of 8 clauses (capi.c:85-243, automata.h:88-742)
//   k_lits      literal count of every clause (capi.c:103-108)
//   k_predict   tiled clause evaluation + per-class vote sums
//               (capi.c:903-1086)
//   k_finalize  argmax (ties to the lowest class) / code bits / scores
#include <cooperative_groups.h>
#include <cub/cub.cuh>

#include "tm_device.cuh"

namespace tmb {

// ---------------------------------------------------------------------------
// Layout kernels
// ---------------------------------------------------------------------------
__global__ void k_repack(const uint8_t *__restrict__ src, uint64_t n, uint64_t row_bytes,
                         uint64_t src_stride, uint32_t *__restrict__ dst, uint32_t dst_words,
                         uint32_t *__restrict__ zero, uint64_t zero_words) {
  // the vote sums of the predict that reads these rows start at zero
  for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < zero_words;
       t += (uint64_t)gridDim.x * blockDim.x)
    zero[t] = 0;
  const uint64_t total = n * dst_words;
  for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t r = t / dst_words;
    const uint64_t b0 = (t - r * dst_words) * 4;
    const uint8_t *row = src + r * src_stride;
    uint32_t v = 0;
#pragma unroll
    for (int b = 0; b < 4; b++)
      if (b0 + b < row_bytes) v |= (uint32_t)row[b0 + b] << (8 * b);
    dst[t] = v;
  }
}

cudaError_t launch_repack(const uint8_t *src, uint64_t n, uint64_t row_bytes, uint64_t src_stride,
                          uint32_t *dst, uint32_t dst_words, cudaStream_t st, uint32_t *zero,
                          uint64_t zero_words) {
  const uint64_t total = std::max<uint64_t>(n * dst_words, zero_words);
  if (!total) return cudaSuccess;
  const int blocks = (int)std::min<uint64_t>((total + 255) / 256, 148ull * 32);
  k_repack<<<blocks, 256, 0, st>>>(src, n, row_bytes, src_stride, dst, dst_words, zero,
                                   zero_words);
  return cudaGetLastError();
}

__global__ void k_labels(const int64_t *__restrict__ src, int32_t *__restrict__ dst, uint64_t n) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    dst[i] = (int32_t)(uint32_t)src[i];  // capi.c:1161: (unsigned int) lbls[sample]
}

cudaError_t launch_labels(const int64_t *src, int32_t *dst, uint64_t n, cudaStream_t st) {
  if (!n) return cudaSuccess;
  const int blocks = (int)std::min<uint64_t>((n + 255) / 256, 148ull * 16);
  k_labels<<<blocks, 256, 0, st>>>(src, dst, n);
  return cudaGetLastError();
}

// automata.h:72-86: count planes all ones, actions zero (padding words zero).
__global__ void k_setup(uint32_t *__restrict__ act, uint32_t *__restrict__ cnt,
                        const ClassDev *__restrict__ cls, uint32_t clauses, uint32_t B) {
  const ClassDev C = cls[blockIdx.y];
  const uint32_t m = B - 1;
  const uint64_t rows = (uint64_t)clauses;
  const uint64_t aw = rows * C.Wp;
  for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < aw;
       t += (uint64_t)gridDim.x * blockDim.x)
    act[C.act_off + t] = 0;
  const uint64_t cw = rows * m * C.Wp;
  for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < cw;
       t += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t w = (uint32_t)(t % C.Wp);
    cnt[C.cnt_off + t] = w + 1 < C.W ? 0xFFFFFFFFu : (w + 1 == C.W ? C.vmask : 0u);
  }
}

cudaError_t launch_setup(uint32_t *act, uint32_t *cnt, const ClassDev *cls, uint32_t classes,
                         uint32_t clauses, uint32_t B, uint64_t act_words, cudaStream_t st) {
  (void)act_words;
  dim3 grid(64, classes);
  k_setup<<<grid, 256, 0, st>>>(act, cnt, cls, clauses, B);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Epoch order: sort samples by a 64-bit Philox key (stable, ties by index).
// ---------------------------------------------------------------------------
__global__ void k_perm_keys(uint64_t seed, uint32_t epoch, uint32_t n, uint64_t *keys,
                            uint32_t *idx, const uint32_t *epoch_dev) {
  // epoch_dev (optional): the epoch is read from device memory, so that a
  // captured graph builds the order of whatever epoch it is replayed for
  if (epoch_dev) epoch += *epoch_dev;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    uint32_t o[4];
    philox(i, epoch, 0u, ST_PERM, seed, o);
    keys[i] = ((uint64_t)o[0] << 32) | o[1];
    idx[i] = i;
  }
}

static size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

size_t perm_scratch_bytes(uint32_t n) {
  size_t temp = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, temp, (uint64_t *)nullptr, (uint64_t *)nullptr,
                                  (uint32_t *)nullptr, (uint32_t *)nullptr, (int)n, 0, 64);
  return align256(temp) + 2 * align256((size_t)n * 8) + align256((size_t)n * 4);
}

cudaError_t launch_perm(uint64_t seed, uint32_t epoch, uint32_t n, uint32_t *out, void *scratch,
                        size_t scratch_bytes, cudaStream_t st, const uint32_t *epoch_dev) {
  if (!n) return cudaSuccess;
  size_t temp = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, temp, (uint64_t *)nullptr, (uint64_t *)nullptr,
                                  (uint32_t *)nullptr, (uint32_t *)nullptr, (int)n, 0, 64);
  uint8_t *p = (uint8_t *)scratch;
  uint64_t *k_in = (uint64_t *)p;
  p += align256((size_t)n * 8);
  uint64_t *k_out = (uint64_t *)p;
  p += align256((size_t)n * 8);
  uint32_t *v_in = (uint32_t *)p;
  p += align256((size_t)n * 4);
  void *tmp = p;
  if ((size_t)(p - (uint8_t *)scratch) + temp > scratch_bytes) return cudaErrorInvalidValue;
  const int blocks = (int)std::min<uint32_t>((n + 255) / 256, 148u * 8);
  k_perm_keys<<<blocks, 256, 0, st>>>(seed, epoch, n, k_in, v_in, epoch_dev);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return cub::DeviceRadixSort::SortPairs(tmp, temp, k_in, k_out, v_in, out, (int)n, 0, 64, st);
}

// ---------------------------------------------------------------------------
// k_train: trains units (8 clauses of one class of one machine), pulling
// them from a work list.
//
// Two shapes:
//   single  one CTA of 8 warps per unit; warp j owns clause j.  The unit's
//           automata live in shared memory (SMEM_STATE, copied in and out
//           once per unit) or stay in global memory.
//   PAIR    a cluster of 2 CTAs per unit, for units too large for one SM
//           (the large sparse classifier: 256 KB): CTA r holds clauses
//           4r..4r+3 with all their bit planes in shared memory; two warps
//           own each clause.  Clause partial sums are written to both CTAs'
//           shared memory (DSMEM) and one cluster barrier per sample makes
//           all eight visible to both.
//
// Per batch of TM_BATCH sample positions of the epoch order, every thread
// examines one position: negative-sampling skip (capi.c:215) and the eight
// chance draws (capi.c:232-239) are independent of the automata, so they
// are drawn up front and the surviving samples are compacted into a list
// (both CTAs of a pair compute the same list).  Per surviving sample:
//   1. its padded row arrives in a 4-slot shared-memory ring by TMA bulk
//      copy (issued 3 samples ahead, completion on an mbarrier; no
//      multicast -- each CTA of a pair fetches its own copy);
//   2. the warps of clause j reduce its literal and failed counts
//      (__reduce_add_sync) and publish them;
//   3. one barrier (CTA, or cluster for a pair); every warp forms all eight
//      votes and the clamped chunk vote and decides its clause's feedback
//      from the pre-drawn chance values;
//   4. the Type Ia / Ib / II feedback of all fed-back clauses is spread over
//      every thread of the CTA as (clause, word) items, so that no warp waits
//      for another's clause; a barrier ends the sample.
// ---------------------------------------------------------------------------
namespace cg = cooperative_groups;

template <bool PAIR>
__device__ __forceinline__ void unit_sync() {
  if constexpr (PAIR)
    cg::this_cluster().sync();
  else
    __syncthreads();
}

// EXACT: every machine of the launch has exactly BM count planes, so the
// plane loops have no run-time bound; those single-CTA variants (256
// threads) fit in 85 registers, three CTAs per SM, the others are capped at
// 128 registers, two CTAs per SM; a pair CTA (512 threads, its shared
// memory fills the SM) at 128.
// CPW: clauses evaluated by one warp (1, 2 or 4): a single CTA has 256 /
// CPW threads, so small units fit more CTAs per SM.
template <bool SMEM_STATE, bool PAIR, int BM, bool EXACT = false, int CPW = 1>
__global__ void __launch_bounds__(PAIR ? 2 * TM_TRAIN_THREADS : TM_TRAIN_THREADS / CPW,
                                  PAIR ? 1 : (EXACT ? 3 * CPW : 2))
    k_train(const TrainDev *__restrict__ machines, const WorkItem *__restrict__ work,
            uint32_t nwork, uint32_t *__restrict__ counter, uint32_t e_begin, uint32_t e_end,
            TrainSmem lay, uint32_t *__restrict__ err) {
  static_assert(CPW == 1 || !PAIR, "clause pairs evaluate one clause per warp group");
  constexpr uint32_t NW = PAIR ? 4 : 1;   // warps per clause
  constexpr uint32_t CPC = PAIR ? 4 : 8;  // clauses per CTA
  constexpr uint32_t GS = 32 * NW;        // lanes per clause group
  extern __shared__ __align__(128) uint8_t smem[];
  const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t rank = PAIR ? cg::this_cluster().block_rank() : 0;
  const uint32_t lc = warp / NW * CPW;      // first local clause of this warp
  const uint32_t gl = (warp % NW) * 32 + lane;  // lane within the clause group
  const uint32_t j = rank * CPC + lc;       // clause of the unit (0..7)
  uint32_t *ring = (uint32_t *)(smem + lay.ring_off);
  uint64_t *bars = (uint64_t *)(smem + lay.bar_off);
  uint32_t *list_s = (uint32_t *)(smem + lay.list_off);
  uint32_t *list_d = list_s + blockDim.x;
  // parts[buf][clause][warp of the clause][literal count, failed count]
  uint32_t *parts = (uint32_t *)(smem + lay.votes_off);
  uint32_t *misc = (uint32_t *)(smem + lay.misc_off);
  // misc: [0] unit, [1..16] warp active counts, [20] abort, [24..31] overflow counts
  uint32_t *peer_parts = parts, *peer_misc = misc;
  if constexpr (PAIR) {
    cg::cluster_group cl = cg::this_cluster();
    peer_parts = cl.map_shared_rank(parts, rank ^ 1u);
    peer_misc = cl.map_shared_rank(misc, rank ^ 1u);
  }

  if (tid == 0) {
    for (int r = 0; r < TM_RING; r++) mbar_init(&bars[r], 1);
    mbar_fence_init();
    misc[20] = 0;
  }
  // Type Ib level counters: TM_IB_SLOTS slots of two levels
  for (uint32_t i = tid; i < 2 * TM_IB_SLOTS * lay.ib_words; i += blockDim.x)
    ((uint32_t *)(smem + lay.ib_off))[i] = 0;
  if (tid < 8) misc[24 + tid] = 0;
  unit_sync<PAIR>();

  uint32_t gs = 0;  // rows issued to the ring so far (slot/phase of row k: k % R, k / R)
  uint32_t issued = 0;
  bool aborted = false;

  while (true) {
    if (tid == 0 && rank == 0) {
      // the next unit; units of a machine whose gate is closed (a search
      // trial that stopped) are passed over
      uint32_t u = atomicAdd(counter, 1u);
      while (u < nwork) {
        const uint32_t *gt = machines[work[u].m].gate;
        if (!gt || *gt) break;
        u = atomicAdd(counter, 1u);
      }
      misc[0] = u;
      if constexpr (PAIR) peer_misc[0] = u;
    }
    unit_sync<PAIR>();
    const uint32_t u = misc[0];
    if (u >= nwork) break;
    const WorkItem wi = work[u];
    const TrainDev &M = machines[wi.m];
    const ClassDev C = M.cls[wi.h];
    const uint32_t m = EXACT ? (uint32_t)BM : M.B - 1;
    const uint32_t Wp = C.Wp, W = C.W;
    const uint32_t g = wi.h * M.clause_chunks + wi.k;
    // this CTA's clauses: rows rank*CPC .. rank*CPC+CPC-1 of the unit
    uint32_t *gact = M.act + C.act_off + ((uint64_t)wi.k * 8 + rank * CPC) * Wp;
    uint32_t *gcnt = M.cnt + C.cnt_off + ((uint64_t)wi.k * 8 + rank * CPC) * m * Wp;
    uint32_t *act, *cnt;
    if (SMEM_STATE) {
      act = (uint32_t *)(smem + lay.state_off);
      cnt = act + CPC * Wp;
      const uint32_t na4 = CPC * Wp / 4, nc4 = CPC * m * Wp / 4;  // uint4 counts
      for (uint32_t i = tid; i < na4; i += blockDim.x)
        ((uint4 *)act)[i] = ((const uint4 *)gact)[i];
      for (uint32_t i = tid; i < nc4; i += blockDim.x)
        ((uint4 *)cnt)[i] = ((const uint4 *)gcnt)[i];
      __syncthreads();
    } else {
      // count planes stay in global memory (L2-resident working set); the
      // action plane, read by every evaluation, is held in shared memory
      act = (uint32_t *)(smem + lay.state_off);
      cnt = gcnt;
      const uint32_t na4 = CPC * Wp / 4;
      for (uint32_t i = tid; i < na4; i += blockDim.x) ((uint4 *)act)[i] = ((const uint4 *)gact)[i];
      __syncthreads();
    }
    uint32_t *act_j = act + lc * Wp;
    bool dirty[CPW];         // this warp's clauses changed since their literal counts were taken
    uint32_t lit_cache[CPW];  // their literal counts when clean
#pragma unroll
    for (int q = 0; q < CPW; q++) {
      dirty[q] = true;
      lit_cache[q] = 0;
    }
    const uint32_t T = M.T;
    const uint64_t T2 = 2ull * T;
    const uint32_t ep_end = e_end < M.epochs ? e_end : M.epochs;
    const uint32_t row_bytes = Wp * 4;
    const uint32_t *xbase = M.x + C.x_off;

    for (uint32_t e = e_begin; e < ep_end && !aborted; e++) {
      const uint32_t ee = M.epoch_base + e;
      const uint32_t *perm = M.perm + (uint64_t)(e - e_begin) * M.n;
      for (uint32_t base = 0; base < M.n && !aborted; base += blockDim.x) {
        // ---- batch phase: skip decisions and chance draws ----------------
        const uint32_t i = base + tid;
        bool live = false;
        uint32_t s = 0, pos = 0;
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
        }
        const uint32_t bal = __ballot_sync(0xFFFFFFFFu, live);
        if (lane == 0) misc[1 + warp] = __popc(bal);
        __syncthreads();
        uint32_t off = 0, nact = 0;
        for (uint32_t w = 0; w < (blockDim.x >> 5); w++) {
          const uint32_t c = misc[1 + w];
          off += w < warp ? c : 0;
          nact += c;
        }
        if (live) {
          const uint32_t slot = off + __popc(bal & ((1u << lane) - 1u));
          list_s[slot] = s | (pos << 31);
          uint32_t d[8];
          philox(s, ee, g, ST_CH0, M.seed, d);
          philox(s, ee, g, ST_CH1, M.seed, d + 4);
#pragma unroll
          for (int k = 0; k < 8; k++) list_d[slot * 8 + k] = d[k];
        }
        __syncthreads();
        if (tid == 0) {
          const uint32_t pre = nact < TM_RING - 1 ? nact : TM_RING - 1;
          for (uint32_t a = 0; a < pre; a++) {
            const uint32_t k = gs + a, sl = k % TM_RING;
            tma_row(&bars[sl], ring + sl * lay.ring_words,
                    xbase + (uint64_t)(list_s[a] & 0x7FFFFFFFu) * Wp, row_bytes);
          }
          issued = gs + pre;
        }

        // ---- sequential per-sample steps ---------------------------------
        for (uint32_t a = 0; a < nact; a++) {
          const uint32_t k = gs + a, sl = k % TM_RING;
          if (!mbar_wait(&bars[sl], (k / TM_RING) & 1u, lay.wait_limit)) {
            misc[20] = 1;
            if constexpr (PAIR) peer_misc[20] = 1;
            atomicOr(err, 1u);
          }
          const uint32_t *xr = ring + sl * lay.ring_words;
          const uint32_t ent = list_s[a];
          const uint32_t pa = ent >> 31;
          // lane c (< CPC) decides local clause c below; its chance draw and
          // the draw's scaled value do not depend on the automata, so they
          // are read before the evaluation, off the decision's critical path
          const uint32_t cl = lane % CPC, jj = rank * CPC + cl;
          const bool type1 = pa ? !(jj & 1u) : (jj & 1u);
          const uint64_t drv = bounded64(list_d[a * 8 + 2 * (jj >> 1) + (type1 ? 0 : 1)], T2);

          // clauses j .. j+CPW-1: literal count L and failed count F
          // (capi.c:97-122).  L only changes when the clause is updated, so
          // it is recounted only after feedback to the clause (`dirty`).
          uint32_t *slot_parts = parts + (a & 1) * 64;
          {
            // each word of the sample row is loaded once for all CPW clauses
            uint32_t l[CPW], f[CPW];
#pragma unroll
            for (int q = 0; q < CPW; q++) l[q] = f[q] = 0;
            const uint32_t Q = Wp >> 2, qlast = (W - 1) >> 2;
#pragma unroll 4
            for (uint32_t qi = gl; qi < Q; qi += GS) {
              const uint4 x4 = *(const uint4 *)(xr + 4 * qi);
#pragma unroll
              for (int q = 0; q < CPW; q++) {
                uint4 a4 = *(const uint4 *)(act_j + q * Wp + 4 * qi);
                if (qi == qlast) {  // evaluation mask on word W-1 (capi.c:104-106)
                  const uint32_t k = (W - 1) & 3;
                  if (k == 0) a4.x &= C.emask;
                  if (k == 1) a4.y &= C.emask;
                  if (k == 2) a4.z &= C.emask;
                  if (k == 3) a4.w &= C.emask;
                }
                f[q] += __popc(a4.x & ~x4.x) + __popc(a4.y & ~x4.y) + __popc(a4.z & ~x4.z) +
                        __popc(a4.w & ~x4.w);
                if (dirty[q]) l[q] += __popc(a4.x) + __popc(a4.y) + __popc(a4.z) + __popc(a4.w);
              }
            }
#pragma unroll
            for (int q = 0; q < CPW; q++) {
              uint32_t lq;
              if (dirty[q]) {
                lq = __reduce_add_sync(0xFFFFFFFFu, l[q]);
              } else {
                lq = (warp % NW == 0) ? lit_cache[q] : 0u;
              }
              const uint32_t fq = __reduce_add_sync(0xFFFFFFFFu, f[q]);
              if (lane == 0) {
                const uint32_t at = (j + q) * 8 + (warp % NW) * 2;
                slot_parts[at] = lq;
                slot_parts[at + 1] = fq;
                if constexpr (PAIR) {
                  peer_parts[(a & 1) * 64 + at] = lq;
                  peer_parts[(a & 1) * 64 + at + 1] = fq;
                }
              }
            }
          }
          unit_sync<PAIR>();
          if (misc[20]) {
            // rows gs + a .. issued - 1 are still to be drained: row gs + a
            // first (its phase may or may not have completed -- waiting on
            // a completed phase returns at once), then the ones issued
            // ahead of it, each in its own ring slot
            aborted = true;
            gs += a;
            break;
          }
          if (tid == 0 && a + TM_RING - 1 < nact) {
            const uint32_t k2 = gs + a + TM_RING - 1, sl2 = k2 % TM_RING;
            tma_row(&bars[sl2], ring + sl2 * lay.ring_words,
                    xbase + (uint64_t)(list_s[a + TM_RING - 1] & 0x7FFFFFFFu) * Wp, row_bytes);
            issued = k2 + 1;
          }
          // votes of all eight clauses (capi.c:110-118), lane q computing
          // clause q's; chunk vote, clamp, feedback probability
          // (capi.c:217-225) by warp reduction
          uint32_t Lq = 0;
          int32_t vq = 0;
          if (lane < 8) {
            Lq = 0;
            uint32_t Fq = 0;
#pragma unroll
            for (uint32_t h = 0; h < NW; h++) {
              Lq += slot_parts[lane * 8 + 2 * h];
              Fq += slot_parts[lane * 8 + 2 * h + 1];
            }
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
#pragma unroll
          for (int q = 0; q < CPW; q++) {
            lit_cache[q] = __shfl_sync(0xFFFFFFFFu, Lq, j + q);
            dirty[q] = false;
          }
          // feedback of this CTA's clauses (capi.c:226-242), lane c deciding
          // local clause c: draw 2p decides Type I of pair p, draw 2p+1 Type
          // II; the positive case gives Type I to the even clause.  Masks over
          // local clauses: Ia/II, Ib, Type I, Ia increments where x = 1.  In a
          // single CTA lane c already holds clause c's vote and literal count.
          int32_t vj = vq;
          uint32_t lj = Lq;
          if constexpr (PAIR) {
            vj = __shfl_sync(0xFFFFFFFFu, vq, jj);
            lj = __shfl_sync(0xFFFFFFFFu, Lq, jj);
          }
          const bool fire = lane < CPC && drv < av;
          const uint32_t ibm = __ballot_sync(0xFFFFFFFFu, fire && type1 && vj == 0);
          const uint32_t fbm = __ballot_sync(0xFFFFFFFFu, fire && vj > 0);
          const uint32_t t1m = __ballot_sync(0xFFFFFFFFu, fire && type1 && vj > 0);
          const uint32_t incm = __ballot_sync(0xFFFFFFFFu, fire && type1 && vj > 0 && lj <= M.maxlit);
          const uint32_t all = fbm | ibm;
          if (!all) continue;
          // Feedback work is shared by the whole CTA: Type Ib picks of every
          // Ib clause are drawn by all threads, then (clause, word) items of
          // every fed-back clause are spread over all threads.  Ib clauses
          // go in groups of TM_IB_SLOTS (one level-counter slot each); a
          // sample with more Ib clauses than slots takes further rounds.
          uint32_t *ibase = (uint32_t *)(smem + lay.ib_off);
          const uint32_t sp = ent & 0x7FFFFFFFu;
          uint32_t rest = ibm, pass = fbm;
          while (true) {
            uint32_t grp = 0;
            for (int q = 0; q < TM_IB_SLOTS && rest; q++) {
              grp |= rest & (0u - rest);
              rest &= rest - 1u;
            }
            pass |= grp;
            if (grp) {
              // Type Ib (capi.c:181-190): s single-automaton decrements with
              // replacement, counted per bit in binary (two levels in shared
              // memory, larger counts as overflow entries of 4 each), then
              // applied as saturating subtractions -- order-free, so equal to
              // the reference's sequential decrements.
              const uint32_t npk = C.s_picks;
              const uint32_t nq = (npk + 3) >> 2;
              uint32_t slot = 0;
              for (uint32_t cm = grp; cm; cm &= cm - 1, slot++) {
                const uint32_t c = __ffs(cm) - 1, jj = rank * CPC + c;
                uint32_t *l0 = ibase + (size_t)slot * 2 * lay.ib_words, *l1 = l0 + lay.ib_words;
                uint32_t *ov = (uint32_t *)(smem + lay.ovf_off) + (size_t)slot * lay.ovf_cap;
                for (uint32_t q = tid; q < nq; q += blockDim.x) {
                  uint32_t o[4];
                  philox(sp, ee, g, ST_IB | (jj << 20) | q, M.seed, o);
#pragma unroll
                  for (uint32_t r = 0; r < 4; r++) {
                    if (4 * q + r < npk) {
                      const uint32_t bit = __umulhi(o[r], C.input_bits);
                      const uint32_t w = bit >> 5, mk = 1u << (bit & 31);
                      if (atomicXor(&l0[w], mk) & mk) {
                        if (atomicXor(&l1[w], mk) & mk) {
                          const uint32_t at = atomicAdd(&misc[24 + slot], 1u);
                          if (at < lay.ovf_cap) ov[at] = bit;
                        }
                      }
                    }
                  }
                }
              }
              __syncthreads();
            }
            // (clause, pair) items: item i -> the (i / P)-th fed-back clause,
            // words 2(i % P) and 2(i % P) + 1
            {
              // fed-back clauses in ascending order, 4 bits each
              uint32_t clist = 0, nfed = 0;
              for (uint32_t cm = pass; cm; cm &= cm - 1, nfed++)
                clist |= (uint32_t)(__ffs(cm) - 1) << (4 * nfed);
              const uint32_t P2 = Wp >> 1;
              const uint32_t total = nfed * P2;
              const uint32_t NT = blockDim.x;
              uint32_t kk = tid / P2, qi = tid - kk * P2;
              for (uint32_t it = tid; it < total; it += NT) {
                const uint32_t c = (clist >> (4 * kk)) & 15u;
                const uint32_t w0 = 2 * qi;
                uint32_t *act_c = act + c * Wp, *cnt_c = cnt + (size_t)c * m * Wp;
                uint32_t pq[2][BM], aq[2];
                if ((grp >> c) & 1u) {
                  uint32_t *l0 = ibase + (size_t)__popc(grp & ((1u << c) - 1u)) * 2 * lay.ib_words;
                  const uint2 m0 = *(const uint2 *)(l0 + w0);
                  const uint2 m1 = *(const uint2 *)(l0 + lay.ib_words + w0);
                  if ((m0.x | m0.y | m1.x | m1.y) != 0) {
                    *(uint2 *)(l0 + w0) = make_uint2(0, 0);
                    *(uint2 *)(l0 + lay.ib_words + w0) = make_uint2(0, 0);
                    ld_pair<BM>(act_c, cnt_c, Wp, m, w0, pq, aq);
#pragma unroll
                    for (int k = 0; k < 2; k++) {
                      const uint32_t am = word_mask(w0 + k, W, C.amask);
                      rg_sub_pow2<BM>(pq[k], aq[k], m, 0, k ? m0.y : m0.x, am);
                      rg_sub_pow2<BM>(pq[k], aq[k], m, 1, k ? m1.y : m1.x, am);
                    }
                    st_pair<BM>(act_c, cnt_c, Wp, m, w0, pq, aq);
                  }
                } else {
                  const uint2 x2 = *(const uint2 *)(xr + w0);
                  const bool t1 = (t1m >> c) & 1u, incx = (incm >> c) & 1u;
                  const uint32_t vm0 = word_mask(w0, W, C.vmask), vm1 = word_mask(w0 + 1, W, C.vmask);
                  // only Type Ia with increments changes words whose literals
                  // are all 1: Type II and the Type Ia decrements act where x = 0
                  const bool need = (t1 && incx) || ((~x2.x & vm0) | (~x2.y & vm1)) != 0;
                  if (need) {
                    ld_pair<BM>(act_c, cnt_c, Wp, m, w0, pq, aq);
#pragma unroll
                    for (int k = 0; k < 2; k++) {
                      const uint32_t x = k ? x2.y : x2.x, vm = k ? vm1 : vm0;
                      const uint32_t am = word_mask(w0 + k, W, C.amask);
                      const uint32_t nx = ~x & ~rg_included<BM>(pq[k], aq[k], m, M.ib) & vm;
                      // Type Ia (capi.c:177-180): inc where x=1 (if L <= maximum),
                      // dec where x=0 and not included.  Type II (capi.c:192-196):
                      // inc where x=0 and not included.
                      if (t1 && incx)
                        rg_add<BM>(pq[k], aq[k], m, x & vm, nx, am);
                      else if (t1)
                        rg_dec<BM>(pq[k], aq[k], m, nx, am);
                      else
                        rg_inc<BM>(pq[k], aq[k], m, nx, am);
                    }
                    st_pair<BM>(act_c, cnt_c, Wp, m, w0, pq, aq);
                  }
                }
                qi += NT;
                while (qi >= P2) {
                  qi -= P2;
                  kk++;
                }
              }
            }
            if (grp) {
              uint32_t novf = 0;
              for (uint32_t q = 0; q < (uint32_t)__popc(grp); q++) novf += misc[24 + q];
              if (novf) {
                // bits picked 4 or more times: rare, applied by one thread
                __syncthreads();
                if (tid == 0) {
                  uint32_t slot = 0;
                  for (uint32_t cm = grp; cm; cm &= cm - 1, slot++) {
                    const uint32_t c = __ffs(cm) - 1;
                    const uint32_t *ov = (uint32_t *)(smem + lay.ovf_off) + (size_t)slot * lay.ovf_cap;
                    const uint32_t no = misc[24 + slot];
                    for (uint32_t t = 0; t < no && t < lay.ovf_cap; t++) {
                      const uint32_t bit = ov[t], w = bit >> 5;
                      const uint32_t am = w + 1 == W ? C.amask : 0xFFFFFFFFu;
                      uint32_t pp[BM], aq;
                      ld_word<BM>(act + c * Wp, cnt + (size_t)c * m * Wp, Wp, m, w, pp, aq);
                      rg_sub_pow2<BM>(pp, aq, m, 2, 1u << (bit & 31), am);
                      st_word<BM>(act + c * Wp, cnt + (size_t)c * m * Wp, Wp, m, w, pp, aq);
                    }
                    misc[24 + slot] = 0;
                  }
                }
              }
            }
            if (!rest) break;
            // the next group's picks reuse the level slots
            __syncthreads();
            pass = 0;
          }
#pragma unroll
          for (int q = 0; q < CPW; q++)
            if (all & (1u << (lc + q))) dirty[q] = true;
          // the next sample's evaluation reads clauses this step updated
          __syncthreads();
        }
        if (!aborted) gs += nact;
        // active steps of the batch (a fire-and-forget reduction)
        if (tid == 0 && rank == 0 && nact) atomicAdd((unsigned long long *)(err + 2), (unsigned long long)nact);
        unit_sync<PAIR>();
      }
    }
    if (aborted) break;
    __syncthreads();
    {
      const uint32_t na4 = CPC * Wp / 4;
      for (uint32_t i = tid; i < na4; i += blockDim.x)
        ((uint4 *)gact)[i] = ((const uint4 *)act)[i];
    }
    if (SMEM_STATE) {
      const uint32_t nc4 = CPC * m * Wp / 4;
      for (uint32_t i = tid; i < nc4; i += blockDim.x)
        ((uint4 *)gcnt)[i] = ((const uint4 *)cnt)[i];
    }
    unit_sync<PAIR>();
  }
  if (aborted && tid == 0) {
    // wait (bounded) for this CTA's copies still in flight before exiting
    for (uint32_t k = gs; k < issued; k++) mbar_wait(&bars[k % TM_RING], (k / TM_RING) & 1u);
  }
  // no CTA of a pair leaves while its peer may still write to its shared memory
  unit_sync<PAIR>();
}

// ---------------------------------------------------------------------------
// k_train_warp: short rows (Wp <= 64 words, B <= 8 state bits) -- one warp
// per unit, warp-synchronous, no CTA barriers.  Lane l owns words l and
// l + 32 of all 8 clauses; the unit's planes live in the warp's slice of
// shared memory.  Per 32 positions of the epoch order each lane draws one
// position's skip decision and chance draws into registers; surviving
// positions are visited in order through the ballot mask, their draws
// broadcast by shuffles.  The next surviving sample's row is loaded while
// the current one is processed.  Same rules and draws as k_train.  WPC
// warps (units) share a CTA: 4, or 1 so that the SM's shared memory is
// divided among units without rounding to CTAs of four.
// ---------------------------------------------------------------------------
template <int BM, bool EXACT, int WPC>
__global__ void __launch_bounds__(WPC * 32)
    k_train_warp(const TrainDev *__restrict__ machines, const WorkItem *__restrict__ work,
                 uint32_t nwork, uint32_t *__restrict__ counter, uint32_t e_begin, uint32_t e_end,
                 uint32_t slice_words, uint32_t ib_words, uint32_t ovf_cap, uint32_t stride,
                 unsigned long long *__restrict__ pairs) {
  extern __shared__ __align__(128) uint8_t smem[];
  const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  // stride: words per warp, a multiple of 32 (16-byte alignment of every slice)
  uint32_t *slice = (uint32_t *)smem + (size_t)wid * stride;
  uint32_t *lev0 = slice + slice_words, *lev1 = lev0 + ib_words, *ovf = lev1 + ib_words;
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
    const uint32_t m = EXACT ? (uint32_t)BM : M.B - 1;
    const uint32_t Wp = C.Wp, W = C.W;
    const uint32_t g = wi.h * M.clause_chunks + wi.k;
    uint32_t *gact = M.act + C.act_off + (uint64_t)wi.k * 8 * Wp;
    uint32_t *gcnt = M.cnt + C.cnt_off + (uint64_t)wi.k * 8 * m * Wp;
    uint32_t *act = slice, *cnt = slice + 8 * Wp;
    for (uint32_t i = lane; i < 2 * Wp; i += 32) ((uint4 *)act)[i] = ((const uint4 *)gact)[i];
    for (uint32_t i = lane; i < 2 * m * Wp; i += 32) ((uint4 *)cnt)[i] = ((const uint4 *)gcnt)[i];
    __syncwarp();
    const uint32_t T = M.T;
    const uint64_t T2 = 2ull * T;
    const uint32_t ep_end = e_end < M.epochs ? e_end : M.epochs;
    const uint32_t *xbase = M.x + C.x_off;
    const uint32_t w0 = lane, w1 = lane + 32;
    const uint32_t vm0 = word_mask(w0, W, C.vmask), vm1 = word_mask(w1, W, C.vmask);
    const uint32_t em0 = word_mask(w0, W, C.emask), em1 = word_mask(w1, W, C.emask);
    const uint32_t am0 = word_mask(w0, W, C.amask), am1 = word_mask(w1, W, C.amask);
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
        // row of the first surviving sample
        uint32_t src = __ffs(bal) - 1;
        uint32_t sc = __shfl_sync(0xFFFFFFFFu, s, src);
        uint32_t x0 = xbase[(uint64_t)sc * Wp + (w0 < Wp ? w0 : 0)];
        uint32_t x1 = w1 < Wp ? xbase[(uint64_t)sc * Wp + w1] : 0u;
        while (bal) {
          src = __ffs(bal) - 1;
          bal &= bal - 1;
          const uint32_t sp = __shfl_sync(0xFFFFFFFFu, s, src);
          const uint32_t pa = __shfl_sync(0xFFFFFFFFu, pos, src);
          uint32_t dd[8];
#pragma unroll
          for (int k = 0; k < 8; k++) dd[k] = __shfl_sync(0xFFFFFFFFu, d[k], src);
          const uint32_t xa = w0 < W ? x0 : 0u, xb = w1 < W ? x1 : 0u;
          // prefetch the next surviving sample's row
          if (bal) {
            const uint32_t sn = __shfl_sync(0xFFFFFFFFu, s, __ffs(bal) - 1);
            x0 = xbase[(uint64_t)sn * Wp + (w0 < Wp ? w0 : 0)];
            x1 = w1 < Wp ? xbase[(uint64_t)sn * Wp + w1] : 0u;
          }
          // evaluation of the 8 clauses (capi.c:97-122)
          uint32_t Lq = 0, Fq = 0;
#pragma unroll
          for (uint32_t c = 0; c < 8; c++) {
            const uint32_t a0 = (w0 < Wp ? act[c * Wp + w0] : 0u) & em0;
            const uint32_t a1 = (w1 < Wp ? act[c * Wp + w1] : 0u) & em1;
            const uint32_t fc = __reduce_add_sync(0xFFFFFFFFu, __popc(a0 & ~xa) + __popc(a1 & ~xb));
            if (lane == c) Fq = fc;
            if ((dirty >> c) & 1u) {
              const uint32_t lc = __reduce_add_sync(0xFFFFFFFFu, __popc(a0) + __popc(a1));
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
          // Type Ia / II (capi.c:177-180, 192-196) on the lane's two words
          for (uint32_t cm = fbm; cm; cm &= cm - 1) {
            const uint32_t c = __ffs(cm) - 1;
            uint32_t *act_c = act + c * Wp, *cnt_c = cnt + (size_t)c * m * Wp;
            const bool t1 = (t1m >> c) & 1u, incx = (incm >> c) & 1u;
#pragma unroll
            for (int h = 0; h < 2; h++) {
              const uint32_t w = h ? w1 : w0, x = h ? xb : xa, vm = h ? vm1 : vm0;
              const uint32_t am = h ? am1 : am0;
              if (w >= W) continue;
              // only Type Ia with increments changes a word whose literals are all 1
              if (!(t1 && incx) && (~x & vm) == 0) continue;
              uint32_t pp[BM], aq;
              ld_word<BM>(act_c, cnt_c, Wp, m, w, pp, aq);
              const uint32_t nx = ~x & ~rg_included<BM>(pp, aq, m, M.ib) & vm;
              if (t1 && incx)
                rg_add<BM>(pp, aq, m, x & vm, nx, am);
              else if (t1)
                rg_dec<BM>(pp, aq, m, nx, am);
              else
                rg_inc<BM>(pp, aq, m, nx, am);
              st_word<BM>(act_c, cnt_c, Wp, m, w, pp, aq);
            }
          }
          // Type Ib (capi.c:181-190), counted per bit then applied
          for (uint32_t cm = ibm; cm; cm &= cm - 1) {
            const uint32_t c = __ffs(cm) - 1;
            uint32_t *act_c = act + c * Wp, *cnt_c = cnt + (size_t)c * m * Wp;
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
            for (int h = 0; h < 2; h++) {
              const uint32_t w = h ? w1 : w0, am = h ? am1 : am0;
              if (w >= W) continue;
              const uint32_t m0 = lev0[w], m1 = lev1[w];
              if (!(m0 | m1)) continue;
              lev0[w] = 0;
              lev1[w] = 0;
              uint32_t pp[BM], aq;
              ld_word<BM>(act_c, cnt_c, Wp, m, w, pp, aq);
              rg_sub_pow2<BM>(pp, aq, m, 0, m0, am);
              rg_sub_pow2<BM>(pp, aq, m, 1, m1, am);
              st_word<BM>(act_c, cnt_c, Wp, m, w, pp, aq);
            }
            __syncwarp();
            const uint32_t no = cnt_ovf[0];
            if (no) {
              if (lane == 0) {
                for (uint32_t t = 0; t < no && t < ovf_cap; t++) {
                  const uint32_t bit = ovf[t], w = bit >> 5;
                  const uint32_t am = word_mask(w, W, C.amask);
                  uint32_t pp[BM], aq;
                  ld_word<BM>(act_c, cnt_c, Wp, m, w, pp, aq);
                  rg_sub_pow2<BM>(pp, aq, m, 2, 1u << (bit & 31), am);
                  st_word<BM>(act_c, cnt_c, Wp, m, w, pp, aq);
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
    for (uint32_t i = lane; i < 2 * m * Wp; i += 32) ((uint4 *)gcnt)[i] = ((const uint4 *)cnt)[i];
    __syncwarp();
  }
}

// shared memory per warp of k_train_warp, in words (a multiple of 32)
static uint32_t warp_slice_words(uint32_t Wpmax, uint32_t Bmax, uint32_t ib_words,
                                 uint32_t ovf_cap) {
  return (8 * Bmax * Wpmax + 2 * ib_words + ovf_cap + 32 + 31) / 32 * 32;
}

template <int WPC>
static int warp_occ(bool exact, size_t bytes) {
  cudaFuncSetAttribute(k_train_warp<7, false, WPC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)bytes);
  cudaFuncSetAttribute(k_train_warp<7, true, WPC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)bytes);
  int nb = 0;
  if (exact)
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_train_warp<7, true, WPC>, WPC * 32, bytes);
  else
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_train_warp<7, false, WPC>, WPC * 32, bytes);
  return nb;
}

int train_warp_occupancy(uint32_t Wpmax, uint32_t Bmin, uint32_t Bmax, uint32_t smax, int wpc,
                         size_t *smem_bytes) {
  const uint32_t ovf_cap = smax / 4 > 0 ? smax / 4 : 1;
  const size_t bytes = (size_t)wpc * warp_slice_words(Wpmax, Bmax, Wpmax, ovf_cap) * 4;
  *smem_bytes = bytes;
  const bool exact = Bmin == 8 && Bmax == 8;
  return wpc == 1 ? warp_occ<1>(exact, bytes) : warp_occ<4>(exact, bytes);
}

template <int WPC>
static void warp_launch(bool exact, int grid, size_t bytes, cudaStream_t st,
                        const TrainDev *machines, const WorkItem *work, uint32_t nwork,
                        uint32_t *counter, uint32_t e_begin, uint32_t e_end, uint32_t slice,
                        uint32_t Wpmax, uint32_t ovf_cap, uint32_t stride,
                        unsigned long long *pairs) {
  if (exact)
    k_train_warp<7, true, WPC><<<grid, WPC * 32, bytes, st>>>(
        machines, work, nwork, counter, e_begin, e_end, slice, Wpmax, ovf_cap, stride, pairs);
  else
    k_train_warp<7, false, WPC><<<grid, WPC * 32, bytes, st>>>(
        machines, work, nwork, counter, e_begin, e_end, slice, Wpmax, ovf_cap, stride, pairs);
}

cudaError_t launch_train_warp(const TrainDev *machines, const WorkItem *work, uint32_t nwork,
                              uint32_t *counter, uint32_t e_begin, uint32_t e_end, uint32_t Wpmax,
                              uint32_t Bmin, uint32_t Bmax, uint32_t smax, int wpc, int grid,
                              cudaStream_t st, unsigned long long *pairs) {
  const uint32_t ovf_cap = smax / 4 > 0 ? smax / 4 : 1;
  const uint32_t slice = 8 * Bmax * Wpmax;
  const uint32_t stride = warp_slice_words(Wpmax, Bmax, Wpmax, ovf_cap);
  const size_t bytes = (size_t)wpc * stride * 4;
  const bool exact = Bmin == 8 && Bmax == 8;
  if (wpc == 1)
    warp_launch<1>(exact, grid, bytes, st, machines, work, nwork, counter, e_begin, e_end, slice,
                   Wpmax, ovf_cap, stride, pairs);
  else
    warp_launch<4>(exact, grid, bytes, st, machines, work, nwork, counter, e_begin, e_end, slice,
                   Wpmax, ovf_cap, stride, pairs);
  return cudaGetLastError();
}

template <bool S, bool P, int BM, bool EX = false, int CPW = 1>
static int occ_of(const TrainSmem &lay) {
  cudaFuncSetAttribute(k_train<S, P, BM, EX, CPW>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       lay.total);
  if (!P) {
    int nb = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_train<S, P, BM, EX, CPW>,
                                                  TM_TRAIN_THREADS / CPW, lay.total);
    return nb;
  }
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = 2;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.gridDim = dim3(2, 1, 1);
  cfg.blockDim = dim3(2 * TM_TRAIN_THREADS, 1, 1);
  cfg.dynamicSmemBytes = lay.total;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  int nc = 0;
  if (cudaOccupancyMaxActiveClusters(&nc, k_train<S, P, BM>, &cfg) != cudaSuccess) return 0;
  return nc;
}

int train_threads(int mode, int cpw) {
  return mode == TM_MODE_PAIR ? 2 * TM_TRAIN_THREADS : TM_TRAIN_THREADS / cpw;
}

// Single: co-resident CTAs per SM.  Pair: co-resident clusters per device.
// cpw > 1 (clauses per warp) exists for 8 state bits only.
int train_occupancy(const TrainSmem &lay, int mode, uint32_t Bmin, uint32_t Bmax, int cpw) {
  const bool small = Bmax <= 8, exact = Bmin == 8 && Bmax == 8;
  if (cpw != 1 && (!exact || mode == TM_MODE_PAIR)) return 0;
  if (mode == TM_MODE_PAIR) return occ_of<true, true, 7>(lay);
  if (mode == TM_MODE_SMEM) {
    if (exact)
      return cpw == 4 ? occ_of<true, false, 7, true, 4>(lay)
                      : (cpw == 2 ? occ_of<true, false, 7, true, 2>(lay)
                                  : occ_of<true, false, 7, true>(lay));
    return small ? occ_of<true, false, 7>(lay) : occ_of<true, false, 31>(lay);
  }
  if (exact)
    return cpw == 4 ? occ_of<false, false, 7, true, 4>(lay)
                    : (cpw == 2 ? occ_of<false, false, 7, true, 2>(lay)
                                : occ_of<false, false, 7, true>(lay));
  return small ? occ_of<false, false, 7>(lay) : occ_of<false, false, 31>(lay);
}

cudaError_t launch_train(const TrainDev *machines, const WorkItem *work, uint32_t nwork,
                         uint32_t *counter, uint32_t e_begin, uint32_t e_end, const TrainSmem &lay,
                         int mode, uint32_t Bmin, uint32_t Bmax, int cpw, int grid,
                         uint32_t *err, cudaStream_t st) {
  const bool small = Bmax <= 8, exact = Bmin == 8 && Bmax == 8;
  if (cpw != 1 && (!exact || mode == TM_MODE_PAIR)) return cudaErrorInvalidValue;
  if (mode == TM_MODE_PAIR) {
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = 2;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(grid, 1, 1);
    cfg.blockDim = dim3(2 * TM_TRAIN_THREADS, 1, 1);
    cfg.dynamicSmemBytes = lay.total;
    cfg.stream = st;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k_train<true, true, 7>, machines, work, nwork, counter,
                              e_begin, e_end, lay, err);
  }
#define TM_LAUNCH(S, BM, EX, CW)                                                             \
  k_train<S, false, BM, EX, CW><<<grid, TM_TRAIN_THREADS / CW, lay.total, st>>>(            \
      machines, work, nwork, counter, e_begin, e_end, lay, err)
  if (mode == TM_MODE_SMEM) {
    if (exact && cpw == 4) TM_LAUNCH(true, 7, true, 4);
    else if (exact && cpw == 2) TM_LAUNCH(true, 7, true, 2);
    else if (exact) TM_LAUNCH(true, 7, true, 1);
    else if (small) TM_LAUNCH(true, 7, false, 1);
    else TM_LAUNCH(true, 31, false, 1);
  } else {
    if (exact && cpw == 4) TM_LAUNCH(false, 7, true, 4);
    else if (exact && cpw == 2) TM_LAUNCH(false, 7, true, 2);
    else if (exact) TM_LAUNCH(false, 7, true, 1);
    else if (small) TM_LAUNCH(false, 7, false, 1);
    else TM_LAUNCH(false, 31, false, 1);
  }
#undef TM_LAUNCH
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Literal counts (capi.c:103-108): one warp per clause row.
// ---------------------------------------------------------------------------
__global__ void k_lits(const uint32_t *__restrict__ act, const ClassDev *__restrict__ cls,
                       uint32_t clauses, int32_t *__restrict__ lits,
                       const uint32_t *__restrict__ gate) {
  if (gate && *gate == 0) return;
  const ClassDev C = cls[blockIdx.y];
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t c = warp; c < clauses; c += nw) {
    const uint32_t *row = act + C.act_off + (uint64_t)c * C.Wp;
    uint32_t l = 0;
    for (uint32_t w = lane; w < C.W; w += 32) {
      uint32_t a = row[w];
      if (w + 1 == C.W) a &= C.emask;
      l += __popc(a);
    }
    l = __reduce_add_sync(0xFFFFFFFFu, l);
    if (lane == 0) lits[(uint64_t)blockIdx.y * clauses + c] = (int32_t)l;
  }
}

cudaError_t launch_lits_gated(const uint32_t *act, const ClassDev *cls, uint32_t classes,
                              uint32_t clauses, int32_t *lits, const uint32_t *gate,
                              cudaStream_t st) {
  dim3 grid((clauses + 7) / 8 < 64 ? (clauses + 7) / 8 : 64, classes);
  k_lits<<<grid, 256, 0, st>>>(act, cls, clauses, lits, gate);
  return cudaGetLastError();
}

cudaError_t launch_lits(const uint32_t *act, const ClassDev *cls, uint32_t classes,
                        uint32_t clauses, int32_t *lits, cudaStream_t st) {
  return launch_lits_gated(act, cls, classes, clauses, lits, nullptr, st);
}

// ---------------------------------------------------------------------------
// Predict: a (64 samples) x (64 clauses of one class) tile per CTA; the
// words of both rows stream through shared memory in 32-word chunks.  Each
// thread accumulates failed-literal counts popc(a & ~x) for 4 clauses x 4
// samples; the epilogue turns them into votes (capi.c:110-118), signs them
// by clause parity (:148-161) and adds the tile's per-class partial sums.
// ---------------------------------------------------------------------------
constexpr int PT_S = 64, PT_C = 64, PT_K = 32, PT_LD = PT_K + 4;

// 16-byte asynchronous global -> shared copy; `valid` false zero-fills the
// destination without reading the source.
__device__ __forceinline__ void cp_async16(void *dst, const void *src, bool valid) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src),
               "r"(valid ? 16 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// One (64 samples) x (64 clauses of class h) tile: samples s0.., clauses c0..
__device__ __forceinline__ void predict_tile(const uint32_t *__restrict__ act,
                                             const int32_t *__restrict__ lits, const ClassDev &C,
                                             uint32_t h, uint32_t c0, uint32_t s0,
                                             uint32_t clauses, uint32_t tol,
                                             const uint32_t *__restrict__ x, uint32_t n,
                                             uint32_t classes, int32_t *__restrict__ sums) {
  // two buffers: the next 32-word chunk streams in while this one is used
  __shared__ __align__(16) uint32_t As[2][PT_C * PT_LD];
  __shared__ __align__(16) uint32_t Xs[2][PT_S * PT_LD];
  __shared__ int32_t red[16][PT_S + 1];
  const uint32_t tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  // Failed-literal counts popc(a & ~x) per (clause, sample).  Five of every
  // eight 4-word steps go through carry-save adders: `ones` and `twos` hold
  // bit-sliced partial counts and only the weight-4 carries are popcounted
  // (one POPC per four words, ten logic ops); the other three steps
  // popcount their words directly (four POPC, four logic ops, two 3-input
  // adds).  POPC and the logic ops issue on separate pipes (measured on
  // B200: they overlap fully), and this mix balances them.  acc is the exact count of everything
  // already reduced: count = acc + 2 * popc(twos) + popc(ones).
  uint32_t acc[4][4], ones[4][4], twos[4][4];
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 4; b++) acc[a][b] = ones[a][b] = twos[a][b] = 0;
  const uint32_t *arow = act + C.act_off;
  const uint32_t *xrow = x + C.x_off;
  auto stage = [&](uint32_t k0, int buf) {
#pragma unroll
    for (int v = 0; v < 2; v++) {
      const uint32_t idx = tid + 256 * v, r = idx >> 3, c4 = (idx & 7) * 4;
      const uint32_t kw = k0 + c4;
      const bool va = c0 + r < clauses && kw < C.Wp, vx = s0 + r < n && kw < C.Wp;
      cp_async16(&As[buf][r * PT_LD + c4], va ? arow + (uint64_t)(c0 + r) * C.Wp + kw : arow, va);
      cp_async16(&Xs[buf][r * PT_LD + c4], vx ? xrow + (uint64_t)(s0 + r) * C.Wp + kw : xrow, vx);
    }
    cp_async_commit();
  };
  const uint32_t nch = (C.Wp + PT_K - 1) / PT_K;
  stage(0, 0);
  for (uint32_t ch = 0; ch < nch; ch++) {
    const uint32_t k0 = ch * PT_K;
    const int buf = ch & 1;
    if (ch + 1 < nch) {
      stage(k0 + PT_K, buf ^ 1);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    if (k0 <= C.W - 1 && C.W - 1 < k0 + PT_K) {
      // evaluation mask on the last word (capi.c:104-106)
      if (tid < PT_C) As[buf][tid * PT_LD + (C.W - 1 - k0)] &= C.emask;
      __syncthreads();
    }
    const uint32_t *Ab = As[buf], *Xb = Xs[buf];
#pragma unroll
    for (int kk = 0; kk < PT_K; kk += 4) {
      uint4 a4[4], x4[4];
#pragma unroll
      for (int c = 0; c < 4; c++) a4[c] = *(const uint4 *)(Ab + (ty + 16 * c) * PT_LD + kk);
#pragma unroll
      for (int i = 0; i < 4; i++) x4[i] = *(const uint4 *)(Xb + (tx + 16 * i) * PT_LD + kk);
#pragma unroll
      for (int c = 0; c < 4; c++)
#pragma unroll
        for (int i = 0; i < 4; i++) {
          const uint32_t t0 = a4[c].x & ~x4[i].x, t1 = a4[c].y & ~x4[i].y;
          const uint32_t t2 = a4[c].z & ~x4[i].z, t3 = a4[c].w & ~x4[i].w;
          if (kk == 8 || kk == 20 || kk == 28) {
            // steps 2, 5 and 7 of 8: direct popcounts
            acc[c][i] += __popc(t0) + __popc(t1) + __popc(t2) + __popc(t3);
          } else {
            uint32_t o = ones[c][i];
            // carry-save adders: (sum, carry) = (a ^ b ^ c, majority(a, b, c))
            const uint32_t h1 = (o & t0) | (o & t1) | (t0 & t1);
            o ^= t0 ^ t1;
            const uint32_t h2 = (o & t2) | (o & t3) | (t2 & t3);
            o ^= t2 ^ t3;
            const uint32_t tw = twos[c][i];
            const uint32_t f4 = (tw & h1) | (tw & h2) | (h1 & h2);
            twos[c][i] = tw ^ h1 ^ h2;
            ones[c][i] = o;
            acc[c][i] += 4 * __popc(f4);
          }
        }
    }
    __syncthreads();
  }
#pragma unroll
  for (int c = 0; c < 4; c++)
#pragma unroll
    for (int i = 0; i < 4; i++)
      acc[c][i] += 2 * __popc(twos[c][i]) + __popc(ones[c][i]);
  int32_t part[4] = {0, 0, 0, 0};
#pragma unroll
  for (int c = 0; c < 4; c++) {
    const uint32_t cl = c0 + ty + 16 * c;
    if (cl < clauses) {
      const int32_t L = lits[(uint64_t)h * clauses + cl];
#pragma unroll
      for (int i = 0; i < 4; i++) {
        int32_t vote;
        if (L == 0)
          vote = (int32_t)tol;
        else {
          vote = (L < (int32_t)tol ? L : (int32_t)tol) - (int32_t)acc[c][i];
          vote = vote < 0 ? 0 : vote;
        }
        part[i] += (cl & 1) ? -vote : vote;
      }
    }
  }
#pragma unroll
  for (int i = 0; i < 4; i++) red[ty][tx + 16 * i] = part[i];
  __syncthreads();
  if (tid < PT_S && s0 + tid < n) {
    int32_t t = 0;
#pragma unroll
    for (int r = 0; r < 16; r++) t += red[r][tid];
    atomicAdd(&sums[(uint64_t)(s0 + tid) * classes + h], t);
  }
}


__global__ void __launch_bounds__(256, 2)
    k_predict(const uint32_t *__restrict__ act, const int32_t *__restrict__ lits,
              const ClassDev *__restrict__ cls, uint32_t clauses, uint32_t tiles_per_class,
              uint32_t tol, const uint32_t *__restrict__ x, uint32_t n, uint32_t classes,
              int32_t *__restrict__ sums) {
  const uint32_t h = blockIdx.y / tiles_per_class;
  const ClassDev C = cls[h];
  predict_tile(act, lits, C, h, (blockIdx.y % tiles_per_class) * PT_C, blockIdx.x * PT_S, clauses,
               tol, x, n, classes, sums);
}

// Many predict jobs (machines and sample sets of any size) in one launch:
// block b runs tile b - jobs[j].tile0 of the job j whose tiles contain b
// (jobs in ascending tile0); a job whose gate reads 0 is skipped.
__global__ void __launch_bounds__(256, 2)
    k_predict_multi(const PredictJob *__restrict__ jobs, uint32_t njobs) {
  uint32_t lo = 0, hi = njobs;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (jobs[mid].tile0 <= blockIdx.x) lo = mid;
    else hi = mid;
  }
  const PredictJob J = jobs[lo];
  if (J.gate && *J.gate == 0) return;
  const uint32_t t = blockIdx.x - J.tile0;
  const uint32_t st = t % J.stiles, ct = t / J.stiles;
  const uint32_t h = ct / J.tpc;
  const ClassDev C = J.cls[h];
  predict_tile(J.act, J.lits, C, h, (ct % J.tpc) * PT_C, st * PT_S, J.clauses, J.tol, J.x, J.n,
               J.classes, J.sums);
}

// ---------------------------------------------------------------------------
// Small-batch predict (at most 16 samples per launch).  A warp evaluates one
// clause row at a time: the row streams once through the warp in 128-bit
// loads that do not allocate in L1 (every action word is read once per
// launch: the HBM-bound regime of a serving request), up to 8 loads per
// lane issued before any is used so that a warp keeps up to 4 KB of the row
// in flight, and each word is tested against all the launch's samples,
// whose rows the CTAs re-read through L1.  From 4 samples on, the failed-
// literal counts popc(a & ~x) go through carry-save adders on every other
// 4-word step (one POPC per four words there, the logic ops on the other
// pipe), since POPC throughput, not HBM, bounds those launches.  Lane s
// keeps sample s's vote sum (capi.c:110-118 votes, signed by clause parity
// as in capi.c:148-161) and adds it to sums at the end of each class.  The
// same integer votes as k_predict, so the same sums bit for bit.
// ---------------------------------------------------------------------------
constexpr uint32_t TM_SMALL_CPB = 32;  // clauses per CTA of the multi-job kernel
// 128-bit loads per lane in flight: fewer as more samples' rows are tested
// against each word (their loads and counters take the registers)
template <int NS>
__host__ __device__ constexpr int small_lpl() { return NS <= 2 ? 8 : (NS <= 8 ? 4 : 2); }

__device__ __forceinline__ uint4 ld_stream16(const void *p) {
  uint4 v;
  asm("ld.global.nc.L1::no_allocate.v4.u32 {%0, %1, %2, %3}, [%4];"
      : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
      : "l"(p));
  return v;
}

// Lane-partial failed-literal counts of one clause row `ar` for the ns
// samples whose padded rows start at xr (Q 4-word groups per row); the
// caller reduces them over the warp.
template <int NS>
__device__ __forceinline__ void small_clause(const uint4 *__restrict__ ar,
                                             const uint4 *__restrict__ xr, const ClassDev &C,
                                             uint32_t ns, uint32_t lane, uint32_t (&f)[NS]) {
  const uint32_t Q = C.Wp >> 2, qlast = (C.W - 1) >> 2, klast = (C.W - 1) & 3;
  constexpr bool CSA = NS >= 4;
  uint32_t ones[NS], twos[NS];
#pragma unroll
  for (int s = 0; s < NS; s++) f[s] = ones[s] = twos[s] = 0;
  constexpr int LPL = small_lpl<NS>();
  for (uint32_t q0 = 0; q0 < Q; q0 += 32 * LPL) {
    uint4 a[LPL];
#pragma unroll
    for (int k = 0; k < LPL; k++) {
      const uint32_t q = q0 + k * 32 + lane;
      a[k] = q < Q ? ld_stream16(ar + q) : make_uint4(0u, 0u, 0u, 0u);
    }
#pragma unroll
    for (int k = 0; k < LPL; k++) {
      const uint32_t q = q0 + k * 32 + lane;
      if (q == qlast) {  // evaluation mask on word W-1 (capi.c:104-106)
        if (klast == 0) a[k].x &= C.emask;
        if (klast == 1) a[k].y &= C.emask;
        if (klast == 2) a[k].z &= C.emask;
        if (klast == 3) a[k].w &= C.emask;
      }
      const uint32_t qs = q < Q ? q : 0;  // past the row: a[k] is zero, any x word will do
#pragma unroll
      for (int s = 0; s < NS; s++) {
        if ((uint32_t)s < ns) {
          const uint4 v = __ldg(xr + (uint64_t)s * Q + qs);
          const uint32_t t0 = a[k].x & ~v.x, t1 = a[k].y & ~v.y;
          const uint32_t t2 = a[k].z & ~v.z, t3 = a[k].w & ~v.w;
          if (CSA && (k & 1) == 0) {
            // (ones, twos) hold bit-sliced partial counts of weight 1 and 2;
            // only the weight-4 carries are popcounted
            uint32_t o = ones[s];
            const uint32_t h1 = (o & t0) | (o & t1) | (t0 & t1);
            o ^= t0 ^ t1;
            const uint32_t h2 = (o & t2) | (o & t3) | (t2 & t3);
            o ^= t2 ^ t3;
            const uint32_t tw = twos[s];
            const uint32_t f4 = (tw & h1) | (tw & h2) | (h1 & h2);
            twos[s] = tw ^ h1 ^ h2;
            ones[s] = o;
            f[s] += 4 * __popc(f4);
          } else {
            f[s] += __popc(t0) + __popc(t1) + __popc(t2) + __popc(t3);
          }
        }
      }
    }
  }
  if (CSA) {
#pragma unroll
    for (int s = 0; s < NS; s++) f[s] += 2 * __popc(twos[s]) + __popc(ones[s]);
  }
}

// Warp-reduces the counts of clause c (literal count L) and adds each
// sample's signed vote to lane s's `part`.
template <int NS>
__device__ __forceinline__ void small_vote(const uint32_t (&f)[NS], int32_t L, uint32_t c,
                                           uint32_t tol, uint32_t ns, uint32_t lane,
                                           int32_t &part) {
#pragma unroll
  for (int s = 0; s < NS; s++) {
    if ((uint32_t)s < ns) {
      const int32_t F = (int32_t)__reduce_add_sync(0xFFFFFFFFu, f[s]);
      if (lane == (uint32_t)s) {
        int32_t vote;
        if (L == 0)
          vote = (int32_t)tol;
        else {
          vote = (L < (int32_t)tol ? L : (int32_t)tol) - F;
          vote = vote < 0 ? 0 : vote;
        }
        part += (c & 1) ? -vote : vote;
      }
    }
  }
}

// Multi-job form: the CTA's 8 warps take the clauses of one block of
// TM_SMALL_CPB clauses of class h in turn, add their votes in shared memory
// and send one atomic per sample to sums.
template <int NS>
__device__ __forceinline__ void predict_small_body(const uint32_t *__restrict__ act,
                                                   const int32_t *__restrict__ lits,
                                                   const ClassDev &C, uint32_t h, uint32_t cblock,
                                                   uint32_t clauses, uint32_t tol,
                                                   const uint32_t *__restrict__ x, uint32_t s0,
                                                   uint32_t ns, uint32_t classes,
                                                   int32_t *__restrict__ sums) {
  __shared__ int32_t red[8][NS];
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t cb = cblock * TM_SMALL_CPB;
  const uint32_t ce = cb + TM_SMALL_CPB < clauses ? cb + TM_SMALL_CPB : clauses;
  const uint4 *xr = (const uint4 *)(x + C.x_off + (uint64_t)s0 * C.Wp);
  int32_t part = 0;  // lane s < ns: sample s0 + s
  for (uint32_t c = cb + warp; c < ce; c += 8) {
    const uint4 *ar = (const uint4 *)(act + C.act_off + (uint64_t)c * C.Wp);
    const int32_t L = lits[(uint64_t)h * clauses + c];
    uint32_t f[NS];
    small_clause<NS>(ar, xr, C, ns, lane, f);
    small_vote<NS>(f, L, c, tol, ns, lane, part);
  }
  if (lane < (uint32_t)NS) red[warp][lane] = part;
  __syncthreads();
  if (warp == 0 && lane < ns) {
    int32_t t = 0;
#pragma unroll
    for (int w = 0; w < 8; w++) t += red[w][lane];
    if (t != 0) atomicAdd(&sums[(uint64_t)(s0 + lane) * classes + h], t);
  }
}

// One machine: warp w evaluates the contiguous clause range
// [w * per_warp, (w + 1) * per_warp) of the flattened (class, clause)
// order, so that the grid is one balanced wave of resident warps; a warp
// sends its votes to sums when its range leaves a class and at its end.
template <int NS>
__global__ void __launch_bounds__(256, NS <= 2 ? 3 : 2)
    k_predict_small(const uint32_t *__restrict__ act, const int32_t *__restrict__ lits,
                    const ClassDev *__restrict__ cls, uint32_t classes, uint32_t clauses,
                    uint32_t tol, const uint32_t *__restrict__ x, uint32_t s0, uint32_t ns,
                    uint32_t per_warp, int32_t *__restrict__ sums) {
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t total = (uint64_t)classes * clauses;
  uint64_t q = (((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * per_warp;
  if (q >= total) return;  // the whole warp
  const uint64_t qe = q + per_warp < total ? q + per_warp : total;
  uint32_t h = (uint32_t)(q / clauses), c = (uint32_t)(q - (uint64_t)h * clauses);
  ClassDev C = cls[h];
  const uint4 *xr = (const uint4 *)(x + C.x_off + (uint64_t)s0 * C.Wp);
  int32_t part = 0;  // lane s < ns: sample s0 + s
  for (; q < qe; q++, c++) {
    if (c == clauses) {
      if (lane < ns && part != 0) atomicAdd(&sums[(uint64_t)(s0 + lane) * classes + h], part);
      part = 0;
      h++;
      c = 0;
      C = cls[h];
      xr = (const uint4 *)(x + C.x_off + (uint64_t)s0 * C.Wp);
    }
    const uint4 *ar = (const uint4 *)(act + C.act_off + (uint64_t)c * C.Wp);
    uint32_t f[NS];
    small_clause<NS>(ar, xr, C, ns, lane, f);
    small_vote<NS>(f, lits[(uint64_t)h * clauses + c], c, tol, ns, lane, part);
  }
  if (lane < ns && part != 0) atomicAdd(&sums[(uint64_t)(s0 + lane) * classes + h], part);
}

// Many small predict jobs (at most 16 samples each, any machines) in one
// launch: block b serves (class, clause block) b - jobs[j].block0 of the job
// j whose blocks contain b (jobs in ascending block0).
__global__ void __launch_bounds__(256, 2)
    k_predict_small_multi(const SmallJob *__restrict__ jobs, uint32_t njobs) {
  uint32_t lo = 0, hi = njobs;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (jobs[mid].block0 <= blockIdx.x) lo = mid;
    else hi = mid;
  }
  const SmallJob J = jobs[lo];
  const uint32_t t = blockIdx.x - J.block0;
  const uint32_t h = t / J.cblocks;
  const ClassDev C = J.cls[h];
  predict_small_body<16>(J.act, J.lits, C, h, t % J.cblocks, J.clauses, J.tol, J.x, J.s0, J.ns,
                         J.classes, J.sums);
}

// Launch shape of k_predict_small<NS>: one wave of resident warps, each
// with an equal share of the machine's clauses.
template <int NS>
static cudaError_t small_launch(cudaStream_t st, const uint32_t *act, const int32_t *lits,
                                const ClassDev *cls, uint32_t classes, uint32_t clauses,
                                uint32_t tol, const uint32_t *x, uint32_t s0, uint32_t ns,
                                int32_t *sums) {
  static int per_sm[64];  // resident CTAs per SM, per device (0: not yet asked)
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  int sms = 0;
  e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  int &occ = per_sm[dev & 63];
  if (occ <= 0) {
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_predict_small<NS>, 256, 0);
    if (e != cudaSuccess) return e;
    if (occ <= 0) occ = 1;
  }
  const uint64_t total = (uint64_t)classes * clauses;
  const uint64_t resident = (uint64_t)sms * occ * 8;
  const uint64_t warps = total < resident ? total : resident;
  const uint32_t per_warp = (uint32_t)((total + warps - 1) / warps);
  const uint64_t used = (total + per_warp - 1) / per_warp;
  k_predict_small<NS><<<(unsigned)((used + 7) / 8), 256, 0, st>>>(act, lits, cls, classes, clauses,
                                                                  tol, x, s0, ns, per_warp, sums);
  return cudaGetLastError();
}

cudaError_t launch_predict(const uint32_t *act, const int32_t *lits, const ClassDev *cls,
                           const ClassDev *cls_host, uint32_t classes, uint32_t clauses,
                           uint32_t tol, const uint32_t *x, uint32_t n, int32_t *sums,
                           cudaStream_t st) {
  (void)cls_host;
  if (!n) return cudaSuccess;
  if (n <= TM_SMALL_N_MAX) {
    for (uint32_t s0 = 0; s0 < n; s0 += 16) {
      const uint32_t ns = n - s0 < 16 ? n - s0 : 16;
      cudaError_t e;
      if (ns <= 1) e = small_launch<1>(st, act, lits, cls, classes, clauses, tol, x, s0, ns, sums);
      else if (ns <= 2) e = small_launch<2>(st, act, lits, cls, classes, clauses, tol, x, s0, ns, sums);
      else if (ns <= 4) e = small_launch<4>(st, act, lits, cls, classes, clauses, tol, x, s0, ns, sums);
      else if (ns <= 8) e = small_launch<8>(st, act, lits, cls, classes, clauses, tol, x, s0, ns, sums);
      else e = small_launch<16>(st, act, lits, cls, classes, clauses, tol, x, s0, ns, sums);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  }
  const uint32_t tpc = (clauses + PT_C - 1) / PT_C;
  dim3 grid((n + PT_S - 1) / PT_S, classes * tpc);
  k_predict<<<grid, 256, 0, st>>>(act, lits, cls, clauses, tpc, tol, x, n, classes, sums);
  return cudaGetLastError();
}

uint32_t small_job_blocks(uint32_t classes, uint32_t clauses, uint32_t *cblocks) {
  *cblocks = (clauses + TM_SMALL_CPB - 1) / TM_SMALL_CPB;
  return *cblocks * classes;
}

cudaError_t launch_predict_small_multi(const SmallJob *jobs_dev, uint32_t njobs,
                                       uint32_t total_blocks, cudaStream_t st) {
  if (!njobs || !total_blocks) return cudaSuccess;
  k_predict_small_multi<<<total_blocks, 256, 0, st>>>(jobs_dev, njobs);
  return cudaGetLastError();
}

// Per request of a serving launch (grid.y = request): its reference byte
// rows -> padded words (k_repack's rule), and its vote sums -> classes or
// code bits (k_finalize's rule, capi.c:934-942, 982-990).
__global__ void k_repack_multi(const ServeJob *__restrict__ jobs) {
  const ServeJob J = jobs[blockIdx.y];
  const uint64_t total = (uint64_t)J.n * J.Wp;
  for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t r = t / J.Wp;
    const uint64_t b0 = (t - r * J.Wp) * 4;
    const uint8_t *row = J.raw + r * J.row_bytes;
    uint32_t v = 0;
#pragma unroll
    for (int b = 0; b < 4; b++)
      if (b0 + b < J.row_bytes) v |= (uint32_t)row[b0 + b] << (8 * b);
    J.x[t] = v;
  }
}

__global__ void k_finalize_multi(const ServeJob *__restrict__ jobs) {
  const ServeJob J = jobs[blockIdx.y];
  for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < J.n; s += gridDim.x * blockDim.x) {
    const int32_t *r = J.sums + (uint64_t)s * J.classes;
    if (J.type == 0) {
      int32_t best = r[0];
      uint32_t bc = 0;
      for (uint32_t h = 1; h < J.classes; h++)
        if (r[h] > best) {
          best = r[h];
          bc = h;
        }
      ((int64_t *)J.out)[s] = bc;
    } else {
      const uint32_t nb = (J.classes + 7) >> 3;
      for (uint32_t b = 0; b < nb; b++) {
        uint32_t byte = 0;
        for (uint32_t q = 0; q < 8 && b * 8 + q < J.classes; q++)
          byte |= (r[b * 8 + q] > 0 ? 1u : 0u) << q;
        J.out[(uint64_t)s * nb + b] = (uint8_t)byte;
      }
    }
  }
}

cudaError_t launch_serve_repack(const ServeJob *jobs_dev, uint32_t njobs, cudaStream_t st) {
  if (!njobs) return cudaSuccess;
  k_repack_multi<<<dim3(64, njobs), 256, 0, st>>>(jobs_dev);
  return cudaGetLastError();
}

cudaError_t launch_serve_finalize(const ServeJob *jobs_dev, uint32_t njobs, cudaStream_t st) {
  if (!njobs) return cudaSuccess;
  k_finalize_multi<<<dim3(16, njobs), 256, 0, st>>>(jobs_dev);
  return cudaGetLastError();
}

uint32_t predict_job_tiles(uint32_t n, uint32_t classes, uint32_t clauses, uint32_t *stiles,
                           uint32_t *tpc) {
  *stiles = (n + PT_S - 1) / PT_S;
  *tpc = (clauses + PT_C - 1) / PT_C;
  return *stiles * classes * *tpc;
}

cudaError_t launch_predict_multi(const PredictJob *jobs_dev, uint32_t njobs, uint32_t total_tiles,
                                 cudaStream_t st) {
  if (!njobs || !total_tiles) return cudaSuccess;
  k_predict_multi<<<total_tiles, 256, 0, st>>>(jobs_dev, njobs);
  return cudaGetLastError();
}

// capi.c:934-942 (argmax, strict >, ties to the lowest class) and :982-990
// (code bit h = votes[h] > 0, LSB-first).
__global__ void k_finalize(const int32_t *__restrict__ sums, uint32_t n, uint32_t classes,
                           int32_t type, int64_t *__restrict__ out_classes,
                           uint8_t *__restrict__ out_codes, int64_t *__restrict__ out_scores) {
  for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    const int32_t *r = sums + (uint64_t)s * classes;
    if (out_scores)
      for (uint32_t h = 0; h < classes; h++) out_scores[(uint64_t)s * classes + h] = r[h];
    if (type == 0 && out_classes) {
      int64_t best = -INT64_MAX;
      uint32_t bc = 0;
      for (uint32_t h = 0; h < classes; h++)
        if ((int64_t)r[h] > best) {
          best = r[h];
          bc = h;
        }
      out_classes[s] = bc;
    }
    if (type == 1 && out_codes) {
      const uint32_t nb = (classes + 7) >> 3;
      for (uint32_t b = 0; b < nb; b++) {
        uint32_t byte = 0;
        for (uint32_t q = 0; q < 8 && b * 8 + q < classes; q++)
          byte |= (r[b * 8 + q] > 0 ? 1u : 0u) << q;
        out_codes[(uint64_t)s * nb + b] = (uint8_t)byte;
      }
    }
  }
}

cudaError_t launch_finalize(const int32_t *sums, uint32_t n, uint32_t classes, int32_t type,
                            int64_t *out_classes, uint8_t *out_codes, int64_t *out_scores,
                            cudaStream_t st) {
  if (!n) return cudaSuccess;
  const int blocks = (int)std::min<uint32_t>((n + 255) / 256, 148u * 8);
  k_finalize<<<blocks, 256, 0, st>>>(sums, n, classes, type, out_classes, out_codes, out_scores);
  return cudaGetLastError();
}

}  // namespace tmb
