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
#include <cub/cub.cuh>

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
__device__ __forceinline__ void tma_row(uint64_t *bar, void *dst, const void *src,
                                        uint32_t bytes) {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
// Bounded wait for the phase with the given parity; false on time-out.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  for (uint32_t it = 0; it < (1u << 22); it++) {
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
// Layout kernels
// ---------------------------------------------------------------------------
__global__ void k_repack(const uint8_t *__restrict__ src, uint64_t n, uint64_t row_bytes,
                         uint64_t src_stride, uint32_t *__restrict__ dst, uint32_t dst_words) {
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
                          uint32_t *dst, uint32_t dst_words, cudaStream_t st) {
  const uint64_t total = n * dst_words;
  if (!total) return cudaSuccess;
  const int blocks = (int)std::min<uint64_t>((total + 255) / 256, 148ull * 32);
  k_repack<<<blocks, 256, 0, st>>>(src, n, row_bytes, src_stride, dst, dst_words);
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
                            uint32_t *idx) {
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
                        size_t scratch_bytes, cudaStream_t st) {
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
  k_perm_keys<<<blocks, 256, 0, st>>>(seed, epoch, n, k_in, v_in);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return cub::DeviceRadixSort::SortPairs(tmp, temp, k_in, k_out, v_in, out, (int)n, 0, 64, st);
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

// ---------------------------------------------------------------------------
// k_train: one CTA trains one unit (8 clauses of one class of one machine)
// at a time, pulling units from a work list.  Warp j owns clause j.
//
// Per batch of TM_BATCH sample positions of the epoch order, every thread
// examines one position: negative-sampling skip (capi.c:215) and the eight
// chance draws (capi.c:232-239) are independent of the automata, so they
// are drawn up front and the surviving samples are compacted into a list.
// Per surviving sample:
//   1. its padded row arrives in a 4-slot shared-memory ring by TMA bulk
//      copy (issued 3 samples ahead, completion on an mbarrier);
//   2. warp j evaluates clause j (popcounts reduced with __reduce_add_sync)
//      and publishes its vote;
//   3. one CTA barrier; every warp forms the clamped chunk vote and decides
//      its own clause's feedback from the pre-drawn chance values;
//   4. warp j applies Type Ia / Ib / II feedback to clause j alone, so no
//      further barrier is needed before the next sample.
// ---------------------------------------------------------------------------
template <bool SMEM_STATE, int BM>
__global__ void __launch_bounds__(TM_TRAIN_THREADS)
    k_train(const TrainDev *__restrict__ machines, const WorkItem *__restrict__ work,
            uint32_t nwork, uint32_t *__restrict__ counter, uint32_t e_begin, uint32_t e_end,
            TrainSmem lay, uint32_t *__restrict__ err) {
  extern __shared__ __align__(128) uint8_t smem[];
  const uint32_t tid = threadIdx.x, lane = tid & 31, j = tid >> 5;
  uint32_t *ring = (uint32_t *)(smem + lay.ring_off);
  uint64_t *bars = (uint64_t *)(smem + lay.bar_off);
  uint32_t *list_s = (uint32_t *)(smem + lay.list_off);
  uint32_t *list_d = list_s + TM_BATCH;
  int32_t *votes = (int32_t *)(smem + lay.votes_off);
  uint32_t *lev0 = (uint32_t *)(smem + lay.ib_off) + (size_t)j * 2 * lay.ib_words;
  uint32_t *lev1 = lev0 + lay.ib_words;
  uint32_t *ovf = (uint32_t *)(smem + lay.ovf_off) + (size_t)j * lay.ovf_cap;
  uint32_t *misc = (uint32_t *)(smem + lay.misc_off);
  // misc: [0] unit, [1..8] warp active counts, [9] abort, [16..23] overflow counts

  if (tid == 0) {
    for (int r = 0; r < TM_RING; r++) mbar_init(&bars[r], 1);
    mbar_fence_init();
    misc[9] = 0;
  }
  for (uint32_t i = tid; i < 16 * lay.ib_words; i += blockDim.x)
    ((uint32_t *)(smem + lay.ib_off))[i] = 0;
  if (tid < 8) misc[16 + tid] = 0;
  __syncthreads();

  uint32_t gs = 0;  // rows issued to the ring so far (slot/phase of row k: k % R, k / R)
  uint32_t issued = 0;
  bool aborted = false;

  while (true) {
    if (tid == 0) misc[0] = atomicAdd(counter, 1u);
    __syncthreads();
    const uint32_t u = misc[0];
    if (u >= nwork) break;
    const WorkItem wi = work[u];
    const TrainDev &M = machines[wi.m];
    const ClassDev C = M.cls[wi.h];
    const uint32_t m = M.B - 1;
    const uint32_t Wp = C.Wp, W = C.W;
    const uint32_t g = wi.h * M.clause_chunks + wi.k;
    uint32_t *gact = M.act + C.act_off + (uint64_t)wi.k * 8 * Wp;
    uint32_t *gcnt = M.cnt + C.cnt_off + (uint64_t)wi.k * 8 * m * Wp;
    uint32_t *act, *cnt;
    if (SMEM_STATE) {
      act = (uint32_t *)(smem + lay.state_off);
      cnt = act + 8 * Wp;
      const uint32_t na4 = 2 * Wp, nc4 = 2 * m * Wp;  // uint4 counts
      for (uint32_t i = tid; i < na4; i += blockDim.x)
        ((uint4 *)act)[i] = ((const uint4 *)gact)[i];
      for (uint32_t i = tid; i < nc4; i += blockDim.x)
        ((uint4 *)cnt)[i] = ((const uint4 *)gcnt)[i];
      __syncthreads();
    } else {
      act = gact;
      cnt = gcnt;
    }
    uint32_t *act_j = act + j * Wp;
    uint32_t *cnt_j = cnt + (size_t)j * m * Wp;
    const uint32_t T = M.T;
    const uint64_t T2 = 2ull * T;
    const uint32_t ep_end = e_end < M.epochs ? e_end : M.epochs;
    const uint32_t row_bytes = Wp * 4;
    const uint32_t *xbase = M.x + C.x_off;

    for (uint32_t e = e_begin; e < ep_end && !aborted; e++) {
      const uint32_t ee = M.epoch_base + e;
      const uint32_t *perm = M.perm + (uint64_t)(e - e_begin) * M.n;
      for (uint32_t base = 0; base < M.n && !aborted; base += TM_BATCH) {
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
        if (lane == 0) misc[1 + j] = __popc(bal);
        __syncthreads();
        uint32_t off = 0, nact = 0;
#pragma unroll
        for (uint32_t w = 0; w < 8; w++) {
          const uint32_t c = misc[1 + w];
          off += w < j ? c : 0;
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
          if (!mbar_wait(&bars[sl], (k / TM_RING) & 1u)) {
            misc[9] = 1;
            atomicOr(err, 1u);
          }
          const uint32_t *xr = ring + sl * lay.ring_words;
          const uint32_t ent = list_s[a];
          const uint32_t pa = ent >> 31;

          // clause j: literal count L and failed count F (capi.c:97-122)
          uint32_t l = 0, f = 0;
          for (uint32_t w = lane; w < W; w += 32) {
            uint32_t av = act_j[w];
            if (w + 1 == W) av &= C.emask;
            l += __popc(av);
            f += __popc(av & ~xr[w]);
          }
          const uint32_t L = __reduce_add_sync(0xFFFFFFFFu, l);
          const uint32_t F = __reduce_add_sync(0xFFFFFFFFu, f);
          int32_t vote;
          if (L == 0)
            vote = (int32_t)M.tol;
          else {
            vote = (int32_t)(L < M.tol ? L : M.tol) - (int32_t)F;
            vote = vote < 0 ? 0 : vote;
          }
          if (lane == 0) votes[(a & 1) * 8 + j] = vote;
          __syncthreads();
          if (misc[9]) {
            aborted = true;
            break;
          }
          if (tid == 0 && a + TM_RING - 1 < nact) {
            const uint32_t k2 = gs + a + TM_RING - 1, sl2 = k2 % TM_RING;
            tma_row(&bars[sl2], ring + sl2 * lay.ring_words,
                    xbase + (uint64_t)(list_s[a + TM_RING - 1] & 0x7FFFFFFFu) * Wp, row_bytes);
            issued = k2 + 1;
          }
          // chunk vote, clamp, feedback probability (capi.c:217-225)
          const int32_t *vv = votes + (a & 1) * 8;
          int32_t v = vv[0] - vv[1] + vv[2] - vv[3] + vv[4] - vv[5] + vv[6] - vv[7];
          v = v > (int32_t)T ? (int32_t)T : v;
          v = v < -(int32_t)T ? -(int32_t)T : v;
          const uint64_t av = (uint64_t)(pa ? (int64_t)T - v : (int64_t)T + v);
          // clause j's pair and role (capi.c:226-242)
          const uint32_t pr = j >> 1, odd = j & 1u;
          const bool type1 = pa ? !odd : odd;
          const uint32_t dr = list_d[a * 8 + 2 * pr + (type1 ? 0 : 1)];
          if (bounded64(dr, T2) >= av) continue;
          if (type1 && vote == 0) {
            // Type Ib (capi.c:181-190): s single-automaton decrements with
            // replacement, counted per bit in binary (two levels in shared
            // memory, larger counts as overflow entries of 4 each), then
            // applied as saturating subtractions -- order-free, so equal to
            // the reference's sequential decrements.
            const uint32_t sp = ent & 0x7FFFFFFFu;
            const uint32_t npk = C.s_picks;
            const uint32_t nq = (npk + 3) >> 2;
            for (uint32_t q = lane; q < nq; q += 32) {
              uint32_t o[4];
              philox(sp, ee, g, ST_IB | (j << 20) | q, M.seed, o);
#pragma unroll
              for (uint32_t r = 0; r < 4; r++) {
                if (4 * q + r < npk) {
                  const uint32_t bit = __umulhi(o[r], C.input_bits);
                  const uint32_t w = bit >> 5, mk = 1u << (bit & 31);
                  if (atomicXor(&lev0[w], mk) & mk) {
                    if (atomicXor(&lev1[w], mk) & mk) {
                      const uint32_t at = atomicAdd(&misc[16 + j], 1u);
                      if (at < lay.ovf_cap) ovf[at] = bit;
                    }
                  }
                }
              }
            }
            __syncwarp();
            for (uint32_t w0 = lane; w0 < W; w0 += 64) {
              const uint32_t w1 = w0 + 32;
              const uint32_t a0m = lev0[w0], a1m = lev1[w0];
              const uint32_t b0m = w1 < W ? lev0[w1] : 0u, b1m = w1 < W ? lev1[w1] : 0u;
              uint32_t pa[BM], pb[BM], aa = 0, ab = 0;
              const bool ua = (a0m | a1m) != 0, ub = (b0m | b1m) != 0;
              if (ua) {
                lev0[w0] = 0;
                lev1[w0] = 0;
                ld_word<BM>(act_j, cnt_j, Wp, m, w0, pa, aa);
              }
              if (ub) {
                lev0[w1] = 0;
                lev1[w1] = 0;
                ld_word<BM>(act_j, cnt_j, Wp, m, w1, pb, ab);
              }
              if (ua) {
                const uint32_t am = w0 + 1 == W ? C.amask : 0xFFFFFFFFu;
                rg_sub_pow2<BM>(pa, aa, m, 0, a0m, am);
                rg_sub_pow2<BM>(pa, aa, m, 1, a1m, am);
                st_word<BM>(act_j, cnt_j, Wp, m, w0, pa, aa);
              }
              if (ub) {
                const uint32_t am = w1 + 1 == W ? C.amask : 0xFFFFFFFFu;
                rg_sub_pow2<BM>(pb, ab, m, 0, b0m, am);
                rg_sub_pow2<BM>(pb, ab, m, 1, b1m, am);
                st_word<BM>(act_j, cnt_j, Wp, m, w1, pb, ab);
              }
            }
            __syncwarp();
            const uint32_t no = misc[16 + j];
            for (uint32_t t = 0; t < no && t < lay.ovf_cap; t++) {
              const uint32_t bit = ovf[t], w = bit >> 5;
              if ((w & 31) == lane) {
                const uint32_t am = w + 1 == W ? C.amask : 0xFFFFFFFFu;
                uint32_t pp[BM], aq;
                ld_word<BM>(act_j, cnt_j, Wp, m, w, pp, aq);
                rg_sub_pow2<BM>(pp, aq, m, 2, 1u << (bit & 31), am);
                st_word<BM>(act_j, cnt_j, Wp, m, w, pp, aq);
              }
            }
            __syncwarp();
            if (lane == 0) misc[16 + j] = 0;
            __syncwarp();
          } else if (vote > 0) {
            // Type Ia (capi.c:177-180): inc where x=1 (if L <= maximum),
            // dec where x=0 and not included.  Type II (capi.c:192-196): inc
            // where x=0 and not included.
            const bool inc_x = type1 && L <= M.maxlit;
            for (uint32_t w0 = lane; w0 < W; w0 += 64) {
              const uint32_t w1 = w0 + 32;
              const uint32_t vma = w0 + 1 == W ? C.vmask : 0xFFFFFFFFu;
              const uint32_t vmb = w1 + 1 == W ? C.vmask : (w1 < W ? 0xFFFFFFFFu : 0u);
              const uint32_t xa = xr[w0], xb = w1 < W ? xr[w1] : 0xFFFFFFFFu;
              // Type II changes nothing where every literal is 1
              const bool ua = type1 || (~xa & vma) != 0;
              const bool ub = w1 < W && (type1 || (~xb & vmb) != 0);
              uint32_t pa[BM], pb[BM], aa = 0, ab = 0;
              if (ua) ld_word<BM>(act_j, cnt_j, Wp, m, w0, pa, aa);
              if (ub) ld_word<BM>(act_j, cnt_j, Wp, m, w1, pb, ab);
              if (ua) {
                const uint32_t am = w0 + 1 == W ? C.amask : 0xFFFFFFFFu;
                const uint32_t nx = ~xa & ~rg_included<BM>(pa, aa, m, M.ib) & vma;
                if (type1)
                  rg_add<BM>(pa, aa, m, inc_x ? (xa & vma) : 0u, nx, am);
                else
                  rg_add<BM>(pa, aa, m, nx, 0u, am);
                st_word<BM>(act_j, cnt_j, Wp, m, w0, pa, aa);
              }
              if (ub) {
                const uint32_t am = w1 + 1 == W ? C.amask : 0xFFFFFFFFu;
                const uint32_t nx = ~xb & ~rg_included<BM>(pb, ab, m, M.ib) & vmb;
                if (type1)
                  rg_add<BM>(pb, ab, m, inc_x ? (xb & vmb) : 0u, nx, am);
                else
                  rg_add<BM>(pb, ab, m, nx, 0u, am);
                st_word<BM>(act_j, cnt_j, Wp, m, w1, pb, ab);
              }
            }
          }
        }
        gs += nact;
        __syncthreads();
      }
    }
    if (aborted) break;
    if (SMEM_STATE) {
      __syncthreads();
      const uint32_t na4 = 2 * Wp, nc4 = 2 * m * Wp;
      for (uint32_t i = tid; i < na4; i += blockDim.x)
        ((uint4 *)gact)[i] = ((const uint4 *)act)[i];
      for (uint32_t i = tid; i < nc4; i += blockDim.x)
        ((uint4 *)gcnt)[i] = ((const uint4 *)cnt)[i];
    }
    __syncthreads();
  }
  if (aborted && tid == 0) {
    // wait (bounded) for this CTA's copies still in flight before exiting
    for (uint32_t k = gs; k < issued; k++) mbar_wait(&bars[k % TM_RING], (k / TM_RING) & 1u);
  }
}

template <bool S, int BM>
static int occ_of(const TrainSmem &lay) {
  int nb = 0;
  cudaFuncSetAttribute(k_train<S, BM>, cudaFuncAttributeMaxDynamicSharedMemorySize, lay.total);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_train<S, BM>, TM_TRAIN_THREADS, lay.total);
  return nb;
}

int train_occupancy(const TrainSmem &lay, bool smem_state, uint32_t Bmax) {
  const bool small = Bmax <= 8;
  if (smem_state) return small ? occ_of<true, 7>(lay) : occ_of<true, 31>(lay);
  return small ? occ_of<false, 7>(lay) : occ_of<false, 31>(lay);
}

cudaError_t launch_train(const TrainDev *machines, const WorkItem *work, uint32_t nwork,
                         uint32_t *counter, uint32_t e_begin, uint32_t e_end, const TrainSmem &lay,
                         bool smem_state, uint32_t Bmax, int grid, uint32_t *err, cudaStream_t st) {
  const bool small = Bmax <= 8;
#define TM_LAUNCH(S, BM)                                                                   \
  k_train<S, BM><<<grid, TM_TRAIN_THREADS, lay.total, st>>>(machines, work, nwork, counter, \
                                                          e_begin, e_end, lay, err)
  if (smem_state) {
    if (small) TM_LAUNCH(true, 7);
    else TM_LAUNCH(true, 31);
  } else {
    if (small) TM_LAUNCH(false, 7);
    else TM_LAUNCH(false, 31);
  }
#undef TM_LAUNCH
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Literal counts (capi.c:103-108): one warp per clause row.
// ---------------------------------------------------------------------------
__global__ void k_lits(const uint32_t *__restrict__ act, const ClassDev *__restrict__ cls,
                       uint32_t clauses, int32_t *__restrict__ lits) {
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

cudaError_t launch_lits(const uint32_t *act, const ClassDev *cls, uint32_t classes,
                        uint32_t clauses, int32_t *lits, cudaStream_t st) {
  dim3 grid((clauses + 7) / 8 < 64 ? (clauses + 7) / 8 : 64, classes);
  k_lits<<<grid, 256, 0, st>>>(act, cls, clauses, lits);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Predict: a (64 samples) x (64 clauses of one class) tile per CTA; the
// words of both rows stream through shared memory in 32-word chunks.  Each
// thread accumulates failed-literal counts popc(a & ~x) for 4 clauses x 4
// samples; the epilogue turns them into votes (capi.c:110-118), signs them
// by clause parity (:148-161) and adds the tile's per-class partial sums.
// ---------------------------------------------------------------------------
constexpr int PT_S = 64, PT_C = 64, PT_K = 32, PT_LD = PT_K + 4;

__global__ void __launch_bounds__(256)
    k_predict(const uint32_t *__restrict__ act, const int32_t *__restrict__ lits,
              const ClassDev *__restrict__ cls, uint32_t clauses, uint32_t tiles_per_class,
              uint32_t tol, const uint32_t *__restrict__ x, uint32_t n, uint32_t classes,
              int32_t *__restrict__ sums) {
  __shared__ __align__(16) uint32_t As[PT_C * PT_LD];
  __shared__ __align__(16) uint32_t Xs[PT_S * PT_LD];
  __shared__ int32_t red[16][PT_S + 1];
  const uint32_t h = blockIdx.y / tiles_per_class;
  const uint32_t c0 = (blockIdx.y % tiles_per_class) * PT_C;
  const uint32_t s0 = blockIdx.x * PT_S;
  const ClassDev C = cls[h];
  const uint32_t tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  uint32_t acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 4; b++) acc[a][b] = 0;
  const uint32_t *arow = act + C.act_off;
  const uint32_t *xrow = x + C.x_off;
  for (uint32_t k0 = 0; k0 < C.Wp; k0 += PT_K) {
#pragma unroll
    for (int v = 0; v < 2; v++) {
      const uint32_t idx = tid + 256 * v, r = idx >> 3, c4 = (idx & 7) * 4;
      const uint32_t kw = k0 + c4;
      uint4 av = make_uint4(0, 0, 0, 0), xv = make_uint4(0, 0, 0, 0);
      if (c0 + r < clauses && kw < C.Wp) {
        av = *(const uint4 *)(arow + (uint64_t)(c0 + r) * C.Wp + kw);
        // evaluation mask on the last word (capi.c:104-106)
        if (kw <= C.W - 1 && C.W - 1 < kw + 4) {
          const uint32_t q = C.W - 1 - kw;
          if (q == 0) av.x &= C.emask;
          if (q == 1) av.y &= C.emask;
          if (q == 2) av.z &= C.emask;
          if (q == 3) av.w &= C.emask;
        }
      }
      if (s0 + r < n && kw < C.Wp) xv = *(const uint4 *)(xrow + (uint64_t)(s0 + r) * C.Wp + kw);
      *(uint4 *)(As + r * PT_LD + c4) = av;
      *(uint4 *)(Xs + r * PT_LD + c4) = xv;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < PT_K; kk += 4) {
      uint4 a4[4], x4[4];
#pragma unroll
      for (int c = 0; c < 4; c++) a4[c] = *(const uint4 *)(As + (ty + 16 * c) * PT_LD + kk);
#pragma unroll
      for (int i = 0; i < 4; i++) x4[i] = *(const uint4 *)(Xs + (tx + 16 * i) * PT_LD + kk);
#pragma unroll
      for (int c = 0; c < 4; c++)
#pragma unroll
        for (int i = 0; i < 4; i++)
          acc[c][i] += __popc(a4[c].x & ~x4[i].x) + __popc(a4[c].y & ~x4[i].y) +
                       __popc(a4[c].z & ~x4[i].z) + __popc(a4[c].w & ~x4[i].w);
    }
    __syncthreads();
  }
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

cudaError_t launch_predict(const uint32_t *act, const int32_t *lits, const ClassDev *cls,
                           const ClassDev *cls_host, uint32_t classes, uint32_t clauses,
                           uint32_t tol, const uint32_t *x, uint32_t n, int32_t *sums,
                           cudaStream_t st) {
  (void)cls_host;
  if (!n) return cudaSuccess;
  const uint32_t tpc = (clauses + PT_C - 1) / PT_C;
  dim3 grid((n + PT_S - 1) / PT_S, classes * tpc);
  k_predict<<<grid, 256, 0, st>>>(act, lits, cls, clauses, tpc, tol, x, n, classes, sums);
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
