// k_train_wpt: the fused train kernel with one CTA per unit of 8 clauses in
// which every thread owns WPT consecutive words of all eight clauses
// (capi.c:85-243 evaluation and feedback, automata.h:88-742 updates).
//
// The action plane and the lowest RP count planes of the thread's words
// live in its registers; the other 7 - RP count planes in shared memory.  A
// unit's automata therefore never leave the SM while it trains (the
// global-plane variant of k_train reads and writes every fed-back clause's
// count planes through L2 on every sample), and because each thread updates
// only its own words, no barrier separates one sample's feedback from the
// next sample's evaluation.  Per active sample:
//   1. the row arrives in a 3-slot shared-memory ring by TMA bulk copy
//      (issued 2 samples ahead, mbarrier completion, no multicast);
//   2. every thread counts its words' failed (and, for clauses updated
//      since, included) literals of the eight clauses, warps reduce them
//      and write one partial per warp; barrier;
//   3. warp 0 sums the partials, forms votes, the clamped chunk vote and the
//      eight feedback decisions from the pre-drawn chance values (the
//      draw contract of k_train), writes four decision masks; barrier;
//   4. Type Ib clauses (at most one per clause pair): all threads draw the
//      picks into per-clause binary level counters in shared memory; barrier;
//   5. every thread applies Type Ia / Ib / II to its own words of every
//      fed-back clause, register and shared planes alike.
// The same rules and draws as k_train, so the same automata bit for bit.
#include "tm_device.cuh"

namespace tmb {


template <int WPT>
struct WVec;
template <>
struct WVec<1> {
  __device__ static void ld(const uint32_t *p, uint32_t (&v)[1]) { v[0] = *p; }
  __device__ static void st(uint32_t *p, const uint32_t (&v)[1]) { *p = v[0]; }
};
template <>
struct WVec<2> {
  __device__ static void ld(const uint32_t *p, uint32_t (&v)[2]) {
    const uint2 t = *(const uint2 *)p;
    v[0] = t.x;
    v[1] = t.y;
  }
  __device__ static void st(uint32_t *p, const uint32_t (&v)[2]) {
    *(uint2 *)p = make_uint2(v[0], v[1]);
  }
};
template <>
struct WVec<4> {
  __device__ static void ld(const uint32_t *p, uint32_t (&v)[4]) {
    const uint4 t = *(const uint4 *)p;
    v[0] = t.x;
    v[1] = t.y;
    v[2] = t.z;
    v[3] = t.w;
  }
  __device__ static void st(uint32_t *p, const uint32_t (&v)[4]) {
    *(uint4 *)p = make_uint4(v[0], v[1], v[2], v[3]);
  }
};

// Shared-memory layout of one launch (byte offsets; planes are
// [plane - RP][clause][Wp] words)
__host__ __device__ inline void wpt_layout(uint32_t Wp, uint32_t NT, int RP, int IBS,
                                           uint32_t ovf_cap, uint32_t *o) {
  uint32_t at = 0;
  auto take = [&](uint32_t bytes) {
    const uint32_t r = at;
    at += (bytes + 127) / 128 * 128;
    return r;
  };
  o[0] = take((7 - RP) * 8 * Wp * 4);               // planes
  o[1] = take(TM_RING * Wp * 4);                    // ring
  o[2] = take(TM_RING * 8);                         // barriers
  o[3] = take(NT * 4);                              // list_s
  o[4] = take(NT * 8 * 4);                          // list_d
  o[5] = take((NT / 32) * 16 * 4);                  // partials
  o[6] = take(IBS * 2 * Wp * 4);                    // Type Ib levels
  o[7] = take(IBS * ovf_cap * 4);                   // Type Ib overflow entries
  o[8] = take(64 * 4);                              // misc
  o[9] = at;                                        // total
}

// misc: [0] unit, [1..32] warp live counts, [40..43] decision masks,
// [44] abort, [48..51] overflow counts
// NT threads per unit, WPT words per thread, RP count planes in registers,
// MINB CTAs per SM the registers are sized for, IBS Type Ib level-counter
// slots (a sample with more Ib clauses takes further rounds)
template <int NT, int WPT, int RP, int MINB, int IBS>
__global__ void __launch_bounds__(NT, MINB)
    k_train_wpt(const TrainDev *__restrict__ machines, const WorkItem *__restrict__ work,
                uint32_t nwork, uint32_t *__restrict__ counter, uint32_t e_begin, uint32_t e_end,
                uint32_t Wpmax, uint32_t ovf_cap, uint32_t wait_limit, uint32_t *__restrict__ err) {
  constexpr int NW = NT / 32;
  constexpr int M7 = 7;  // count planes (8 state bits)
  extern __shared__ __align__(128) uint8_t smem[];
  uint32_t o[10];
  wpt_layout(Wpmax, NT, RP, IBS, ovf_cap, o);
  uint32_t *splanes = (uint32_t *)(smem + o[0]);
  uint32_t *ring = (uint32_t *)(smem + o[1]);
  uint64_t *bars = (uint64_t *)(smem + o[2]);
  uint32_t *list_s = (uint32_t *)(smem + o[3]);
  uint32_t *list_d = (uint32_t *)(smem + o[4]);
  uint32_t *partial = (uint32_t *)(smem + o[5]);
  uint32_t *lev = (uint32_t *)(smem + o[6]);
  uint32_t *ovf = (uint32_t *)(smem + o[7]);
  uint32_t *misc = (uint32_t *)(smem + o[8]);
  const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t w0 = tid * WPT;  // this thread's first word
  if (tid == 0) {
    for (int r = 0; r < TM_RING; r++) mbar_init(&bars[r], 1);
    mbar_fence_init();
    misc[44] = 0;
  }
  for (uint32_t i = tid; i < IBS * 2 * Wpmax; i += NT) lev[i] = 0;
  if (tid < IBS) misc[48 + tid] = 0;
  __syncthreads();
  uint32_t gs = 0, issued = 0;
  bool aborted = false;
  while (true) {
    if (tid == 0) {
      // the next unit, passing over those of machines whose gate is closed
      uint32_t v = atomicAdd(counter, 1u);
      while (v < nwork) {
        const uint32_t *gt = machines[work[v].m].gate;
        if (!gt || *gt) break;
        v = atomicAdd(counter, 1u);
      }
      misc[0] = v;
    }
    __syncthreads();
    const uint32_t u = misc[0];
    if (u >= nwork) break;
    const WorkItem wi = work[u];
    const TrainDev &M = machines[wi.m];
    const ClassDev C = M.cls[wi.h];
    const uint32_t Wp = C.Wp, W = C.W;
    const uint32_t g = wi.h * M.clause_chunks + wi.k;
    uint32_t *gact = M.act + C.act_off + (uint64_t)wi.k * 8 * Wp;
    uint32_t *gcnt = M.cnt + C.cnt_off + (uint64_t)wi.k * 8 * M7 * Wp;
    // ---- the unit's automata onto the SM ------------------------------------
    uint32_t act[8][WPT], pl[8][RP > 0 ? RP : 1][WPT];
    const bool mine = w0 < Wp;  // Wp is a multiple of 4 and of WPT
#pragma unroll
    for (int c = 0; c < 8; c++) {
      if (mine) {
        WVec<WPT>::ld(gact + c * Wp + w0, act[c]);
#pragma unroll
        for (int b = 0; b < RP; b++) WVec<WPT>::ld(gcnt + (c * M7 + b) * Wp + w0, pl[c][b]);
      } else {
#pragma unroll
        for (int k = 0; k < WPT; k++) {
          act[c][k] = 0;
#pragma unroll
          for (int b = 0; b < RP; b++) pl[c][b][k] = 0;
        }
      }
    }
    for (uint32_t i = tid; i < (uint32_t)(M7 - RP) * 8 * Wp; i += NT) {
      const uint32_t bb = i / (8 * Wp), rem = i - bb * 8 * Wp, c = rem / Wp, w = rem - c * Wp;
      splanes[i] = gcnt[(c * M7 + RP + bb) * Wp + w];
    }
    uint32_t vm[WPT], em[WPT], am[WPT];
#pragma unroll
    for (int k = 0; k < WPT; k++) {
      vm[k] = word_mask(w0 + k, W, C.vmask);
      em[k] = word_mask(w0 + k, W, C.emask);
      am[k] = word_mask(w0 + k, W, C.amask);
    }
    __syncthreads();
    const uint32_t T = M.T;
    const uint64_t T2 = 2ull * T;
    const uint32_t ep_end = e_end < M.epochs ? e_end : M.epochs;
    const uint32_t *xbase = M.x + C.x_off;
    uint32_t dirty = 0xFFu;  // clauses whose literal counts must be recounted
    uint32_t lcache = 0;     // warp 0, lane c < 8: literal count of clause c
    // the count planes of this thread's words of clause c: registers for
    // planes below RP, shared memory for the others
    auto gather = [&](int c, uint32_t (&p)[WPT][M7]) {
#pragma unroll
      for (int b = 0; b < M7; b++) {
        if (b < RP) {
#pragma unroll
          for (int q = 0; q < WPT; q++) p[q][b] = pl[c][b < RP ? b : 0][q];
        } else {
          uint32_t t[WPT];
          WVec<WPT>::ld(splanes + ((b - RP) * 8 + c) * Wp + w0, t);
#pragma unroll
          for (int q = 0; q < WPT; q++) p[q][b] = t[q];
        }
      }
    };
    auto scatter = [&](int c, const uint32_t (&p)[WPT][M7]) {
#pragma unroll
      for (int b = 0; b < M7; b++) {
        if (b < RP) {
#pragma unroll
          for (int q = 0; q < WPT; q++) pl[c][b < RP ? b : 0][q] = p[q][b];
        } else {
          uint32_t t[WPT];
#pragma unroll
          for (int q = 0; q < WPT; q++) t[q] = p[q][b];
          WVec<WPT>::st(splanes + ((b - RP) * 8 + c) * Wp + w0, t);
        }
      }
    };

    for (uint32_t e = e_begin; e < ep_end && !aborted; e++) {
      const uint32_t ee = M.epoch_base + e;
      const uint32_t *perm = M.perm + (uint64_t)(e - e_begin) * M.n;
      for (uint32_t base = 0; base < M.n && !aborted; base += NT) {
        // ---- batch phase: skip decisions and chance draws (as k_train) -------
        const uint32_t i = base + tid;
        bool live = false;
        uint32_t s = 0, pos = 0;
        if (i < M.n) {
          s = perm[i];
          if (M.type == 0) {
            pos = (uint32_t)M.labels[s] == wi.h;
            live = pos;
            if (!pos) {
              uint32_t r[4];
              philox(s, ee, g, ST_NEG, M.seed, r);
              live = (uint64_t)r[0] >= M.thr_neg;
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
        for (uint32_t w = 0; w < (uint32_t)NW; w++) {
          const uint32_t cnt = misc[1 + w];
          off += w < warp ? cnt : 0;
          nact += cnt;
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
            tma_row(&bars[sl], ring + sl * Wpmax, xbase + (uint64_t)(list_s[a] & 0x7FFFFFFFu) * Wp,
                    Wp * 4);
          }
          issued = gs + pre;
          if (nact) atomicAdd((unsigned long long *)(err + 2), (unsigned long long)nact);
        }
        // ---- sequential per-sample steps ------------------------------------
        for (uint32_t a = 0; a < nact; a++) {
          const uint32_t k = gs + a, sl = k % TM_RING;
          if (!mbar_wait(&bars[sl], (k / TM_RING) & 1u, wait_limit)) {
            misc[44] = 1;
            atomicOr(err, 1u);
          }
          uint32_t x[WPT];
          if (mine) WVec<WPT>::ld(ring + sl * Wpmax + w0, x);
          else
#pragma unroll
            for (int q = 0; q < WPT; q++) x[q] = 0xFFFFFFFFu;
          // failed literal counts (and literal counts of dirty clauses)
#pragma unroll
          for (int c = 0; c < 8; c++) {
            uint32_t f = 0, l = 0;
#pragma unroll
            for (int q = 0; q < WPT; q++) {
              const uint32_t aw = act[c][q] & em[q];
              f += __popc(aw & ~x[q]);
              l += __popc(aw);
            }
            f = __reduce_add_sync(0xFFFFFFFFu, f);
            if ((dirty >> c) & 1u) l = __reduce_add_sync(0xFFFFFFFFu, l);
            if (lane == 0) {
              partial[warp * 16 + c] = f;
              partial[warp * 16 + 8 + c] = l;
            }
          }
          __syncthreads();
          if (misc[44]) {
            aborted = true;
            gs += a;
            break;
          }
          if (tid == 0) {
            for (int q = 0; q < IBS; q++) misc[48 + q] = 0;  // previous sample's overflow lists
            if (a + TM_RING - 1 < nact) {
              const uint32_t k2 = gs + a + TM_RING - 1, sl2 = k2 % TM_RING;
              tma_row(&bars[sl2], ring + sl2 * Wpmax,
                      xbase + (uint64_t)(list_s[a + TM_RING - 1] & 0x7FFFFFFFu) * Wp, Wp * 4);
              issued = k2 + 1;
            }
          }
          const uint32_t ent = list_s[a];
          if (warp == 0) {
            // votes (capi.c:110-118), chunk vote, clamp, p (capi.c:217-225),
            // decisions (capi.c:226-242), lane c deciding clause c
            uint32_t sum = 0;
            if (lane < 16)
              for (uint32_t w = 0; w < (uint32_t)NW; w++) sum += partial[w * 16 + lane];
            const uint32_t Ls = __shfl_sync(0xFFFFFFFFu, sum, (lane & 7) + 8);
            if (lane < 8 && ((dirty >> lane) & 1u)) lcache = Ls;
            const uint32_t Lq = lane < 8 ? lcache : 0u;
            int32_t vq = 0;
            if (lane < 8) {
              if (Lq == 0)
                vq = (int32_t)M.tol;
              else {
                vq = (int32_t)(Lq < M.tol ? Lq : M.tol) - (int32_t)sum;
                vq = vq < 0 ? 0 : vq;
              }
            }
            int32_t v = __reduce_add_sync(0xFFFFFFFFu, (lane & 1) ? -vq : vq);
            v = v > (int32_t)T ? (int32_t)T : v;
            v = v < -(int32_t)T ? -(int32_t)T : v;
            const uint32_t pa = ent >> 31;
            const uint64_t av = (uint64_t)(pa ? (int64_t)T - v : (int64_t)T + v);
            const uint32_t c = lane & 7;
            const bool type1 = pa ? !(c & 1u) : (c & 1u);
            const uint64_t drv = bounded64(list_d[a * 8 + 2 * (c >> 1) + (type1 ? 0 : 1)], T2);
            const bool fire = lane < 8 && drv < av;
            const uint32_t ibm = __ballot_sync(0xFFFFFFFFu, fire && type1 && vq == 0);
            const uint32_t fbm = __ballot_sync(0xFFFFFFFFu, fire && vq > 0);
            const uint32_t t1m = __ballot_sync(0xFFFFFFFFu, fire && type1 && vq > 0);
            const uint32_t incm =
                __ballot_sync(0xFFFFFFFFu, fire && type1 && vq > 0 && Lq <= M.maxlit);
            if (lane == 0) {
              misc[40] = ibm;
              misc[41] = fbm;
              misc[42] = t1m;
              misc[43] = incm;
            }
          }
          __syncthreads();
          const uint32_t ibm = misc[40], fbm = misc[41], t1m = misc[42], incm = misc[43];
          dirty = ibm | fbm;
          const uint32_t sp_s = ent & 0x7FFFFFFFu;
          // ---- Type Ib (capi.c:181-190), in rounds of IBS clauses: the picks
          // of each clause counted per bit in two binary levels, larger counts
          // as overflow entries worth 4 each (saturating subtraction is
          // order-free), then applied by the owners of the words ----------------
          for (uint32_t rest = ibm; rest;) {
            uint32_t grp = 0;
            for (int q = 0; q < IBS && rest; q++) {
              grp |= rest & (0u - rest);
              rest &= rest - 1u;
            }
            const uint32_t npk = C.s_picks, nq = (npk + 3) >> 2;
            uint32_t slot = 0;
            for (uint32_t cm = grp; cm; cm &= cm - 1, slot++) {
              const uint32_t c = __ffs(cm) - 1;
              uint32_t *l0 = lev + slot * 2 * Wpmax, *l1 = l0 + Wpmax;
              for (uint32_t q = tid; q < nq; q += NT) {
                uint32_t r[4];
                philox(sp_s, ee, g, ST_IB | (c << 20) | q, M.seed, r);
#pragma unroll
                for (uint32_t z = 0; z < 4; z++) {
                  if (4 * q + z < npk) {
                    const uint32_t bit = __umulhi(r[z], C.input_bits);
                    const uint32_t w = bit >> 5, mk = 1u << (bit & 31);
                    if (atomicXor(&l0[w], mk) & mk) {
                      if (atomicXor(&l1[w], mk) & mk) {
                        const uint32_t at = atomicAdd(&misc[48 + slot], 1u);
                        if (at < ovf_cap) ovf[slot * ovf_cap + at] = bit;
                      }
                    }
                  }
                }
              }
            }
            __syncthreads();
#pragma unroll
            for (int c = 0; c < 8; c++) {
              if (!((grp >> c) & 1u) || !mine) continue;
              uint32_t p[WPT][M7];
              gather(c, p);
              const uint32_t sl2 = __popc(grp & ((1u << c) - 1u));
              uint32_t *l0 = lev + sl2 * 2 * Wpmax + w0, *l1 = l0 + Wpmax;
              uint32_t m0[WPT], m1[WPT], zero[WPT];
              WVec<WPT>::ld(l0, m0);
              WVec<WPT>::ld(l1, m1);
#pragma unroll
              for (int q = 0; q < WPT; q++) zero[q] = 0;
              WVec<WPT>::st(l0, zero);
              WVec<WPT>::st(l1, zero);
#pragma unroll
              for (int q = 0; q < WPT; q++) {
                rg_sub_pow2<M7>(p[q], act[c][q], M7, 0, m0[q], am[q]);
                rg_sub_pow2<M7>(p[q], act[c][q], M7, 1, m1[q], am[q]);
              }
              const uint32_t no = min(misc[48 + sl2], ovf_cap);
              for (uint32_t t = 0; t < no; t++) {
                const uint32_t bit = ovf[sl2 * ovf_cap + t], w = bit >> 5;
#pragma unroll
                for (int q = 0; q < WPT; q++)
                  if (w == w0 + q) rg_sub_pow2<M7>(p[q], act[c][q], M7, 2, 1u << (bit & 31), am[q]);
              }
              scatter(c, p);
            }
            if (rest) {
              // another round reuses the slots: every thread has read the
              // overflow counts before they are reset
              __syncthreads();
              if (tid < IBS) misc[48 + tid] = 0;
              __syncthreads();
            }
          }
          // ---- Type Ia / II of this thread's words of every fed-back clause --
#pragma unroll
          for (int c = 0; c < 8; c++) {
            if (!((fbm >> c) & 1u) || !mine) continue;
            uint32_t p[WPT][M7];
            gather(c, p);
            const bool t1 = (t1m >> c) & 1u, incx = (incm >> c) & 1u;
#pragma unroll
            for (int q = 0; q < WPT; q++) {
              // Type Ia (capi.c:177-180): inc where x=1 (if L <= maximum),
              // dec where x=0 and not included.  Type II (capi.c:192-196):
              // inc where x=0 and not included.
              const uint32_t nx = ~x[q] & ~rg_included<M7>(p[q], act[c][q], M7, M.ib) & vm[q];
              if (t1 && incx)
                rg_add<M7>(p[q], act[c][q], M7, x[q] & vm[q], nx, am[q]);
              else if (t1)
                rg_dec<M7>(p[q], act[c][q], M7, nx, am[q]);
              else
                rg_inc<M7>(p[q], act[c][q], M7, nx, am[q]);
            }
            scatter(c, p);
          }
        }
        if (!aborted) gs += nact;
        __syncthreads();
      }
    }
    if (aborted) break;
    // ---- the unit's automata back to global memory ----------------------------
#pragma unroll
    for (int c = 0; c < 8; c++) {
      if (mine) {
        WVec<WPT>::st(gact + c * Wp + w0, act[c]);
#pragma unroll
        for (int b = 0; b < RP; b++) WVec<WPT>::st(gcnt + (c * M7 + b) * Wp + w0, pl[c][b]);
      }
    }
    for (uint32_t i = tid; i < (uint32_t)(M7 - RP) * 8 * Wp; i += NT) {
      const uint32_t bb = i / (8 * Wp), rem = i - bb * 8 * Wp, c = rem / Wp, w = rem - c * Wp;
      gcnt[(c * M7 + RP + bb) * Wp + w] = splanes[i];
    }
    __syncthreads();
  }
  if (aborted && tid == 0) {
    // wait (bounded) for this CTA's copies still in flight before exiting
    for (uint32_t k = gs; k < issued; k++) mbar_wait(&bars[k % TM_RING], (k / TM_RING) & 1u);
  }
  __syncthreads();
}

// ---- configurations ----------------------------------------------------------
// id (1-based): threads per unit, words per thread, register planes, CTAs
// per SM the registers are sized for, Type Ib slots
#define TM_WPT_CONFIGS(X)   \
  X(1, 512, 2, 2, 1, 2)     \
  X(2, 256, 1, 0, 3, 2)     \
  X(3, 256, 2, 2, 2, 2)     \
  X(4, 128, 2, 1, 4, 2)     \
  X(5, 64, 1, 0, 8, 2)      \
  X(6, 32, 2, 0, 14, 2)     \
  X(7, 32, 2, 1, 14, 2)

struct WptConfig {
  int nt, wpt, rp, minb, ibs;
};
static const WptConfig kWpt[] = {
#define TM_WPT_ROW(ID, NT, WPT, RP, MINB, IBS) {NT, WPT, RP, MINB, IBS},
    TM_WPT_CONFIGS(TM_WPT_ROW)
#undef TM_WPT_ROW
};
constexpr int kWptCount = (int)(sizeof(kWpt) / sizeof(kWpt[0]));

int wpt_configs() { return kWptCount; }

static uint32_t wpt_ovf_cap(uint32_t smax) { return smax / 4 > 0 ? smax / 4 : 1; }

template <int NT, int WPT, int RP, int MINB, int IBS>
static int wpt_occ(size_t bytes) {
  cudaFuncSetAttribute(k_train_wpt<NT, WPT, RP, MINB, IBS>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  int nb = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_train_wpt<NT, WPT, RP, MINB, IBS>, NT,
                                                bytes);
  return nb;
}

// Resident CTAs (units) per SM of configuration `id` for rows of at most
// Wpmax words (0 when it cannot hold them), and its shared memory.
int train_wpt_occupancy(int id, uint32_t Wpmax, uint32_t smax, size_t *smem_bytes) {
  if (id < 1 || id > kWptCount) return 0;
  const WptConfig &k = kWpt[id - 1];
  if (Wpmax > (uint32_t)(k.nt * k.wpt) || Wpmax % k.wpt) return 0;
  uint32_t o[10];
  wpt_layout(Wpmax, k.nt, k.rp, k.ibs, wpt_ovf_cap(smax), o);
  *smem_bytes = o[9];
  switch (id) {
#define TM_WPT_OCC(ID, NT, WPT, RP, MINB, IBS) \
  case ID: return wpt_occ<NT, WPT, RP, MINB, IBS>(o[9]);
    TM_WPT_CONFIGS(TM_WPT_OCC)
#undef TM_WPT_OCC
  }
  return 0;
}

cudaError_t launch_train_wpt(int id, const TrainDev *machines, const WorkItem *work,
                             uint32_t nwork, uint32_t *counter, uint32_t e_begin, uint32_t e_end,
                             uint32_t Wpmax, uint32_t smax, uint32_t wait_limit, int grid,
                             uint32_t *err, cudaStream_t st) {
  if (id < 1 || id > kWptCount) return cudaErrorInvalidValue;
  const WptConfig &k = kWpt[id - 1];
  const uint32_t ovf_cap = wpt_ovf_cap(smax);
  uint32_t o[10];
  wpt_layout(Wpmax, k.nt, k.rp, k.ibs, ovf_cap, o);
  switch (id) {
#define TM_WPT_LAUNCH(ID, NT, WPT, RP, MINB, IBS)                                            \
  case ID:                                                                                   \
    k_train_wpt<NT, WPT, RP, MINB, IBS><<<grid, NT, o[9], st>>>(                             \
        machines, work, nwork, counter, e_begin, e_end, Wpmax, ovf_cap, wait_limit, err);    \
    break;
    TM_WPT_CONFIGS(TM_WPT_LAUNCH)
#undef TM_WPT_LAUNCH
  }
  return cudaGetLastError();
}

}  // namespace tmb
