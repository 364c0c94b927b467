// Device-side neighbours of the hot path: the evaluator metrics the
// reference's search driver computes after every epoch, and the packing of
// set-bit lists into flip-interleaved sample rows.
//
//   tm_class_accuracy     evaluator/capi.c:119-202 (per-class precision,
//                         recall, F1 and their macro averages)
//   tm_encoding_accuracy  evaluator/capi.c:497-574 (bitwise Hamming
//                         agreement of codes: mean, min, max, std of the
//                         per-bit error rates)
//   tm_bits_to_cvec       santoku-matrix's bits_to_cvec(n, F, flip), the
//                         packing the reference's tests apply to their
//                         inputs (doc/sth.md:70-78)
//   tm_bits_to_cvec_ind   santoku-matrix's bits_to_cvec_ind: the
//                         individualized layout, one block of rows per
//                         class / code bit (doc/sth.md:42-54, consumed at
//                         capi.c:1020-1023, 1344-1354, 1440-1451)
//
// Counting runs in kernels; the per-class / per-bit finish (a few hundred
// doubles) runs in one small kernel in the reference's summation order, so
// the results are the reference's to the last bit.
#include <math.h>
#include <stdint.h>

#include <vector>

#include "../../include/tsetlin_b200.h"
#include "tm_internal.h"

namespace {

struct DevScratch {
  void *p = nullptr;
  size_t cap = 0;
  cudaError_t ensure(size_t n) {
    if (n <= cap) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    cudaError_t e = tmb_dev_malloc(&p, n);
    if (e == cudaSuccess) cap = n;
    return e;
  }
  ~DevScratch() {
    if (p) cudaFree(p);
  }
};

// capi.c:141-153 of the evaluator: TP/FP/FN per class; samples whose
// predicted or true class is out of range are skipped.
__global__ void k_class_counts(const int64_t *__restrict__ pred, const int64_t *__restrict__ truth,
                               uint64_t n, uint32_t classes, unsigned long long *__restrict__ tp,
                               unsigned long long *__restrict__ fp,
                               unsigned long long *__restrict__ fn) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t yp = (uint32_t)pred[i], yt = (uint32_t)truth[i];
    if (yp >= classes || yt >= classes) continue;
    if (yp == yt) {
      atomicAdd(&tp[yt], 1ull);
    } else {
      atomicAdd(&fp[yp], 1ull);
      atomicAdd(&fn[yt], 1ull);
    }
  }
}

}  // namespace

namespace tmb {
// Precision, recall and F1 of one class from its counts (evaluator
// capi.c:155-160), with explicit round-to-nearest operations: no fused
// multiply-add, so each operation rounds as in a plain IEEE evaluation of
// the formula and the result equals the reference's double arithmetic.
__device__ __forceinline__ void class_prf(unsigned long long t, unsigned long long f,
                                          unsigned long long g, double &p, double &r,
                                          double &f1) {
  p = (t + f) > 0 ? __ddiv_rn((double)t, (double)(t + f)) : 0.0;
  r = (t + g) > 0 ? __ddiv_rn((double)t, (double)(t + g)) : 0.0;
  const double pr = __dadd_rn(p, r);
  f1 = pr > 0 ? __ddiv_rn(__dmul_rn(__dmul_rn(2.0, p), r), pr) : 0.0;
}
}  // namespace tmb

namespace {

// capi.c:155-172 of the evaluator, in its order: out = [precision, recall,
// f1 (macro), then per class precision, recall, f1]
__global__ void k_class_finish(const unsigned long long *__restrict__ tp,
                               const unsigned long long *__restrict__ fp,
                               const unsigned long long *__restrict__ fn, uint32_t classes,
                               double *__restrict__ out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double pa = 0.0, ra = 0.0, fa = 0.0;
  for (uint32_t c = 0; c < classes; c++) {
    double p, r, f1;
    tmb::class_prf(tp[c], fp[c], fn[c], p, r, f1);
    out[3 + 3 * c] = p;
    out[3 + 3 * c + 1] = r;
    out[3 + 3 * c + 2] = f1;
    pa = __dadd_rn(pa, p);
    ra = __dadd_rn(ra, r);
    fa = __dadd_rn(fa, f1);
  }
  out[0] = __ddiv_rn(pa, (double)classes);
  out[1] = __ddiv_rn(ra, (double)classes);
  out[2] = __ddiv_rn(fa, (double)classes);
}

// capi.c:520-535 of the evaluator: per-bit disagreements.  One thread per
// (sample, code byte).
__global__ void k_code_diffs(const uint8_t *__restrict__ pred, const uint8_t *__restrict__ truth,
                             uint64_t n, uint32_t hidden, unsigned long long *__restrict__ bdiff) {
  const uint32_t nb = (hidden + 7) / 8;
  const uint64_t total = n * nb;
  for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t b = (uint32_t)(t % nb);
    uint32_t d = (uint32_t)(pred[t] ^ truth[t]);
    while (d) {
      const uint32_t k = __ffs(d) - 1;
      d &= d - 1;
      const uint32_t j = b * 8 + k;
      if (j < hidden) atomicAdd(&bdiff[j], 1ull);
    }
  }
}

// capi.c:544-570 of the evaluator: out = [mean_hamming, ber_min, ber_max,
// ber_std, then per-bit error rate]
__global__ void k_code_finish(const unsigned long long *__restrict__ bdiff, uint64_t n,
                              uint32_t hidden, double *__restrict__ out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double mn = 1.0, mx = 0.0;
  unsigned long long total = 0;
  for (uint32_t j = 0; j < hidden; j++) {
    const double t = __ddiv_rn((double)bdiff[j], (double)n);
    if (t < mn) mn = t;
    if (t > mx) mx = t;
    out[4 + j] = t;
    total += bdiff[j];
  }
  const double mean = __ddiv_rn((double)total, (double)(n * hidden));
  double var = 0.0;
  for (uint32_t j = 0; j < hidden; j++) {
    const double d = __dsub_rn(__ddiv_rn((double)bdiff[j], (double)n), mean);
    var = __dadd_rn(var, __dmul_rn(d, d));
  }
  out[0] = __dsub_rn(1.0, mean);
  out[1] = __dsub_rn(1.0, mn);
  out[2] = __dsub_rn(1.0, mx);
  out[3] = hidden > 1 ? __dsqrt_rn(__ddiv_rn(var, (double)(hidden - 1))) : 0.0;
}

// bits_to_cvec: set bit f of sample s for every listed index s * F + f;
// with flip, bit F + f of sample s is set when bit f is not.
__global__ void k_scatter_bits(const int64_t *__restrict__ idx, uint64_t n_idx, uint64_t n,
                               uint32_t features, uint32_t row_bits, uint32_t row_words,
                               uint32_t *__restrict__ rows) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_idx;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const int64_t v = idx[i];
    if (v < 0) continue;
    const uint64_t s = (uint64_t)v / features, f = (uint64_t)v % features;
    if (s >= n) continue;
    atomicOr(&rows[s * row_words + (uint32_t)(f >> 5)], 1u << (f & 31));
    (void)row_bits;
  }
}

__global__ void k_flip_bits(uint64_t n, uint32_t features, uint32_t row_words,
                            uint32_t *__restrict__ rows) {
  const uint64_t total = n * features;
  for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t s = t / features;
    const uint32_t f = (uint32_t)(t % features);
    uint32_t *row = rows + s * row_words;
    const bool on = (row[f >> 5] >> (f & 31)) & 1u;
    if (!on) {
      const uint32_t g = features + f;
      atomicOr(&row[g >> 5], 1u << (g & 31));
    }
  }
}

// 32-bit word rows -> byte rows of nb bytes (little-endian words)
__global__ void k_words_to_bytes(const uint32_t *__restrict__ rows, uint64_t n, uint32_t row_words,
                                 uint32_t nb, uint8_t *__restrict__ out) {
  const uint64_t total = n * nb;
  for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t s = t / nb;
    const uint32_t b = (uint32_t)(t % nb);
    out[t] = (uint8_t)(rows[s * row_words + (b >> 2)] >> (8 * (b & 3)));
  }
}

// bits_to_cvec_ind, step 1: set bit f of row s of dimension h's staging
// block for every entry s * k_h + f of dimension h's list.  meta holds four
// int64 arrays of dims + 1 entries: list offsets, feature offsets, staging
// word offsets, output byte offsets.
__device__ __forceinline__ uint32_t find_block(const int64_t *__restrict__ off, uint32_t dims,
                                               int64_t v) {
  // largest h with off[h] <= v (off nondecreasing, off[0] <= v < off[dims])
  uint32_t lo = 0, hi = dims;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (off[mid] <= v) lo = mid;
    else hi = mid;
  }
  return lo;
}

__global__ void k_scatter_bits_ind(const int64_t *__restrict__ idx, const int64_t *__restrict__ meta,
                                   uint32_t dims, uint64_t n, uint32_t *__restrict__ stage) {
  const int64_t *lists = meta, *feats = meta + (dims + 1), *woff = meta + 2 * (dims + 1);
  const uint64_t first = (uint64_t)lists[0], total = (uint64_t)lists[dims] - first;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const int64_t v = idx[i];
    if (v < 0) continue;
    const uint32_t h = find_block(lists, dims, (int64_t)(first + i));
    const uint64_t k = (uint64_t)(feats[h + 1] - feats[h]);
    if (k == 0) continue;
    const uint64_t s = (uint64_t)v / k, f = (uint64_t)v % k;
    if (s >= n) continue;
    const uint64_t rw = (k + 31) / 32;
    atomicOr(&stage[woff[h] + s * rw + (f >> 5)], 1u << (f & 31));
  }
}

// 8 bits of a staged row starting at bit o; bits outside [0, 32 rw) read 0
__device__ __forceinline__ uint32_t row_byte_at(const uint32_t *__restrict__ row, uint64_t rw,
                                                int64_t o) {
  if (o <= -8) return 0;
  const uint32_t lead = o < 0 ? (uint32_t)(-o) : 0u;  // bits below 0 read 0
  const uint64_t q = o < 0 ? 0 : (uint64_t)o;
  const uint64_t w = q >> 5;
  if (w >= rw) return 0;
  uint64_t v = row[w];
  if (w + 1 < rw) v |= (uint64_t)row[w + 1] << 32;
  return ((uint32_t)(v >> (q & 31)) << lead) & 0xffu;
}

// step 2: byte b of row s of block h: bits 0..k_h-1 are the staged bits,
// with flip bits k_h..2k_h-1 their complements, padding bits 0.
__global__ void k_pack_bytes_ind(const uint32_t *__restrict__ stage, const int64_t *__restrict__ meta,
                                 uint32_t dims, uint64_t n, int32_t flip, uint8_t *__restrict__ out) {
  const int64_t *feats = meta + (dims + 1), *woff = meta + 2 * (dims + 1),
                *boff = meta + 3 * (dims + 1);
  const uint64_t total = (uint64_t)boff[dims];
  for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t h = find_block(boff, dims, (int64_t)t);
    const uint64_t k = (uint64_t)(feats[h + 1] - feats[h]);
    const uint64_t nb = ((flip ? 2 * k : k) + 7) / 8, rw = (k + 31) / 32;
    const uint64_t local = t - (uint64_t)boff[h];
    const uint64_t s = local / nb, b = local % nb;
    const uint32_t *row = stage + woff[h] + s * rw;
    const int64_t p0 = (int64_t)(8 * b);
    uint32_t lo_mask = 0, fl_mask = 0;
#pragma unroll
    for (int j = 0; j < 8; j++) {
      const int64_t p = p0 + j;
      if (p < (int64_t)k) lo_mask |= 1u << j;
      else if (flip && p < 2 * (int64_t)k) fl_mask |= 1u << j;
    }
    uint32_t v = row_byte_at(row, rw, p0) & lo_mask;
    if (fl_mask) v |= ~row_byte_at(row, rw, p0 - (int64_t)k) & fl_mask;
    out[t] = (uint8_t)v;
  }
}

int grid_for(uint64_t work) {
  const uint64_t g = (work + 255) / 256;
  return (int)(g < 148ull * 16 ? (g ? g : 1) : 148ull * 16);
}

}  // namespace

namespace tmb {

// The score of one machine per CTA: predictions from the vote sums (argmax
// with ties to the lowest class, capi.c:934-942, or code bits h = sum > 0,
// capi.c:982-990), the evaluator's counts (class_accuracy,
// evaluator/capi.c:141-153; encoding_accuracy, :520-535), then the metric
// and the epoch logic of the reference's train_tm (optimize.lua:599-625):
// a score above best + tolerance becomes the best (and is checkpointed when
// patience > 0); `patience` epochs without one, or the last iteration,
// stop the machine.  final_pass scores the machines holding a checkpoint
// after the restore and only records the score.
__global__ void k_search_score(const ScoreJob *__restrict__ jobs, SearchState *__restrict__ state,
                               double *__restrict__ scores, uint32_t max_epochs, int final_pass) {
  extern __shared__ uint32_t cnt[];
  SearchState *S = state + blockIdx.x;
  if (!(final_pass ? S->has_ckpt : S->live)) return;
  const ScoreJob J = jobs[blockIdx.x];
  const uint32_t C = J.classes, tid = threadIdx.x;
  const uint32_t ncnt = J.type == 0 ? 3 * C : C;
  for (uint32_t i = tid; i < ncnt; i += blockDim.x) cnt[i] = 0;
  __syncthreads();
  if (J.type == 0) {
    for (uint32_t s = tid; s < J.n; s += blockDim.x) {
      int32_t *r = J.sums + (uint64_t)s * C;
      int32_t best = r[0];
      uint32_t bc = 0;
      r[0] = 0;
      for (uint32_t h = 1; h < C; h++) {
        const int32_t v = r[h];
        r[h] = 0;
        if (v > best) {
          best = v;
          bc = h;
        }
      }
      const uint32_t yt = (uint32_t)J.labels[s];
      if (yt >= C) continue;
      if (bc == yt) {
        atomicAdd(&cnt[yt], 1u);
      } else {
        atomicAdd(&cnt[C + bc], 1u);
        atomicAdd(&cnt[2 * C + yt], 1u);
      }
    }
  } else {
    const uint32_t nb = (C + 7) >> 3;
    for (uint32_t s = tid; s < J.n; s += blockDim.x) {
      int32_t *r = J.sums + (uint64_t)s * C;
      const uint8_t *code = J.codes + (uint64_t)s * nb;
      for (uint32_t h = 0; h < C; h++) {
        const uint32_t p = r[h] > 0 ? 1u : 0u;
        r[h] = 0;
        if (p != ((code[h >> 3] >> (h & 7)) & 1u)) atomicAdd(&cnt[h], 1u);
      }
    }
  }
  __syncthreads();
  if (tid != 0) return;
  double score;
  if (J.type == 0 && J.metric == 0) {  // macro F1 (evaluator capi.c:155-172)
    double fa = 0.0;
    for (uint32_t c = 0; c < C; c++) {
      double p, r, f1;
      class_prf(cnt[c], cnt[C + c], cnt[2 * C + c], p, r, f1);
      fa = __dadd_rn(fa, f1);
    }
    score = __ddiv_rn(fa, (double)C);
  } else if (J.type == 0) {  // accuracy: correct / n
    unsigned long long t = 0;
    for (uint32_t c = 0; c < C; c++) t += cnt[c];
    score = J.n ? __ddiv_rn((double)t, (double)J.n) : 0.0;
  } else {  // mean_hamming = 1 - mean bit error rate (evaluator capi.c:557-566)
    unsigned long long t = 0;
    for (uint32_t h = 0; h < C; h++) t += cnt[h];
    score = __dsub_rn(1.0, __ddiv_rn((double)t, (double)((uint64_t)J.n * C)));
  }
  if (final_pass) {
    S->last = score;
    return;
  }
  const uint32_t e = S->epochs_run;
  if (scores && e < max_epochs) scores[(uint64_t)blockIdx.x * max_epochs + e] = score;
  S->epochs_run = e + 1;
  S->last = score;
  if (score > __dadd_rn(S->best, S->tolerance)) {
    S->best = score;
    S->since = 0;
    S->best_epoch = e + 1;
    S->ckpt_now = S->patience ? 1u : 0u;
    if (S->patience) S->has_ckpt = 1;
  } else {
    S->since++;
    S->ckpt_now = 0;
  }
  if ((S->patience && S->since >= S->patience) || e + 1 >= S->iterations) S->live = 0;
}

cudaError_t launch_search_score(const ScoreJob *jobs, SearchState *state, double *scores,
                                uint32_t max_epochs, uint32_t njobs, uint32_t max_classes,
                                int final_pass, cudaStream_t st) {
  if (!njobs) return cudaSuccess;
  const size_t smem = (size_t)3 * max_classes * 4;
  k_search_score<<<njobs, 256, smem, st>>>(jobs, state, scores, max_epochs, final_pass);
  return cudaGetLastError();
}

// capi.c:103-108 literal counts for many machines: grid (64, classes, job)
__global__ void k_lits_multi(const LitsJob *__restrict__ jobs) {
  const LitsJob J = jobs[blockIdx.z];
  if (J.gate && *J.gate == 0) return;
  if (blockIdx.y >= J.classes) return;
  const ClassDev C = J.cls[blockIdx.y];
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t c = warp; c < J.clauses; c += nw) {
    const uint32_t *row = J.act + C.act_off + (uint64_t)c * C.Wp;
    uint32_t l = 0;
    for (uint32_t w = lane; w < C.W; w += 32) {
      uint32_t a = row[w];
      if (w + 1 == C.W) a &= C.emask;
      l += __popc(a);
    }
    l = __reduce_add_sync(0xFFFFFFFFu, l);
    if (lane == 0) J.lits[(uint64_t)blockIdx.y * J.clauses + c] = (int32_t)l;
  }
}

cudaError_t launch_lits_multi(const LitsJob *jobs, uint32_t njobs, uint32_t max_classes,
                              cudaStream_t st) {
  if (!njobs || !max_classes) return cudaSuccess;
  k_lits_multi<<<dim3(64, max_classes, njobs), 256, 0, st>>>(jobs);
  return cudaGetLastError();
}

// grid (blocks, job): 16-byte copies while the job's flag is set
__global__ void k_copy_multi(const CopyJob *__restrict__ jobs) {
  const CopyJob J = jobs[blockIdx.y];
  if (!J.flag || *J.flag == 0) return;
  const uint64_t n4 = J.words >> 2;
  const uint4 *src = (const uint4 *)J.src;
  uint4 *dst = (uint4 *)J.dst;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n4;
       i += (uint64_t)gridDim.x * blockDim.x)
    dst[i] = src[i];
}

cudaError_t launch_copy_multi(const CopyJob *jobs, uint32_t njobs, cudaStream_t st) {
  if (!njobs) return cudaSuccess;
  k_copy_multi<<<dim3(32, njobs), 256, 0, st>>>(jobs);
  return cudaGetLastError();
}

__global__ void k_tick(uint32_t *counter) { *counter += 1; }

__global__ void k_tick_machines(TrainDev *machines, uint32_t count) {
  for (uint32_t i = threadIdx.x; i < count; i += blockDim.x) machines[i].epoch_base += 1;
}

cudaError_t launch_tick_machines(TrainDev *machines, uint32_t count, cudaStream_t st) {
  if (!count) return cudaSuccess;
  k_tick_machines<<<1, 256, 0, st>>>(machines, count);
  return cudaGetLastError();
}

cudaError_t launch_tick(uint32_t *counter, cudaStream_t st) {
  k_tick<<<1, 1, 0, st>>>(counter);
  return cudaGetLastError();
}

}  // namespace tmb

#define CKU(call)                                                                \
  do {                                                                           \
    cudaError_t e_ = (call);                                                     \
    if (e_ != cudaSuccess) return tmb_fail(TM_ERR_CUDA, cudaGetErrorString(e_)); \
  } while (0)

extern "C" int tm_class_accuracy(const int64_t *predicted, const int64_t *expected, uint64_t n,
                                 uint32_t classes, int32_t on_device, int32_t device, double *out) {
  if (!out || (n && (!predicted || !expected))) return tmb_fail(TM_ERR_ARG, "class_accuracy: bad arguments");
  if (classes == 0) return tmb_fail(TM_ERR_ARG, "class_accuracy: n_classes must be > 0");
  tmb::DevGuard guard(device);
  CKU(guard.err);
  DevScratch buf;
  const size_t cnt = 3 * (size_t)classes * 8, outb = (3 + 3 * (size_t)classes) * 8;
  const size_t inb = on_device ? 0 : 2 * n * 8;
  CKU(buf.ensure(cnt + outb + inb + 64));
  unsigned long long *tp = (unsigned long long *)buf.p, *fp = tp + classes, *fn = fp + classes;
  double *dout = (double *)((uint8_t *)buf.p + cnt);
  const int64_t *dp = predicted, *de = expected;
  if (!on_device && n) {
    int64_t *st = (int64_t *)((uint8_t *)buf.p + cnt + outb);
    CKU(cudaMemcpy(st, predicted, n * 8, cudaMemcpyHostToDevice));
    CKU(cudaMemcpy(st + n, expected, n * 8, cudaMemcpyHostToDevice));
    dp = st;
    de = st + n;
  }
  CKU(cudaMemset(tp, 0, cnt));
  if (n) k_class_counts<<<grid_for(n), 256>>>(dp, de, n, classes, tp, fp, fn);
  k_class_finish<<<1, 32>>>(tp, fp, fn, classes, dout);
  CKU(cudaGetLastError());
  CKU(cudaMemcpy(out, dout, outb, cudaMemcpyDeviceToHost));
  return TM_OK;
}

extern "C" int tm_encoding_accuracy(const uint8_t *predicted, const uint8_t *expected, uint64_t n,
                                    uint32_t hidden, int32_t on_device, int32_t device, double *out) {
  if (!out || !n || !predicted || !expected) return tmb_fail(TM_ERR_ARG, "encoding_accuracy: bad arguments");
  if (hidden == 0) return tmb_fail(TM_ERR_ARG, "encoding_accuracy: n_hidden must be > 0");
  tmb::DevGuard guard(device);
  CKU(guard.err);
  const uint64_t nb = (hidden + 7) / 8;
  DevScratch buf;
  const size_t cnt = (size_t)hidden * 8, outb = (4 + (size_t)hidden) * 8;
  const size_t inb = on_device ? 0 : 2 * n * nb;
  CKU(buf.ensure(cnt + outb + inb + 64));
  unsigned long long *bd = (unsigned long long *)buf.p;
  double *dout = (double *)((uint8_t *)buf.p + cnt);
  const uint8_t *dp = predicted, *de = expected;
  if (!on_device) {
    uint8_t *st = (uint8_t *)buf.p + cnt + outb;
    CKU(cudaMemcpy(st, predicted, n * nb, cudaMemcpyHostToDevice));
    CKU(cudaMemcpy(st + n * nb, expected, n * nb, cudaMemcpyHostToDevice));
    dp = st;
    de = st + n * nb;
  }
  CKU(cudaMemset(bd, 0, cnt));
  k_code_diffs<<<grid_for(n * nb), 256>>>(dp, de, n, hidden, bd);
  k_code_finish<<<1, 32>>>(bd, n, hidden, dout);
  CKU(cudaGetLastError());
  CKU(cudaMemcpy(out, dout, outb, cudaMemcpyDeviceToHost));
  return TM_OK;
}

extern "C" int tm_bits_to_cvec(const int64_t *set_bits, uint64_t n_set, uint64_t n,
                               uint32_t features, int32_t flip, int32_t on_device, int32_t device,
                               uint8_t *out) {
  if (!out || (n_set && !set_bits) || features == 0) return tmb_fail(TM_ERR_ARG, "bits_to_cvec: bad arguments");
  tmb::DevGuard guard(device);
  CKU(guard.err);
  const uint64_t row_bits = flip ? 2ull * features : features;
  const uint32_t nb = (uint32_t)((row_bits + 7) / 8);
  const uint32_t rw = (uint32_t)((row_bits + 31) / 32);
  DevScratch buf;
  const size_t rows_b = n * rw * 4, idx_b = on_device ? 0 : n_set * 8, out_b = on_device ? 0 : n * nb;
  CKU(buf.ensure(rows_b + idx_b + out_b + 256));
  uint32_t *rows = (uint32_t *)buf.p;
  const int64_t *di = set_bits;
  uint8_t *dout = out;
  if (!on_device) {
    int64_t *st = (int64_t *)((uint8_t *)buf.p + ((rows_b + 7) & ~(size_t)7));
    if (n_set) CKU(cudaMemcpy(st, set_bits, n_set * 8, cudaMemcpyHostToDevice));
    di = st;
    dout = (uint8_t *)st + idx_b;
  }
  CKU(cudaMemset(rows, 0, rows_b ? rows_b : 4));
  if (n_set) k_scatter_bits<<<grid_for(n_set), 256>>>(di, n_set, n, features, (uint32_t)row_bits, rw, rows);
  if (flip && n) k_flip_bits<<<grid_for(n * features), 256>>>(n, features, rw, rows);
  if (n) k_words_to_bytes<<<grid_for(n * nb), 256>>>(rows, n, rw, nb, dout);
  CKU(cudaGetLastError());
  if (!on_device && n) CKU(cudaMemcpy(out, dout, n * nb, cudaMemcpyDeviceToHost));
  else CKU(cudaDeviceSynchronize());
  return TM_OK;
}

extern "C" int tm_bits_to_cvec_ind(const int64_t *set_bits, const int64_t *ind_offsets,
                                   const int64_t *feat_offsets, uint32_t dims, uint64_t n,
                                   int32_t flip, int32_t on_device, int32_t device, uint8_t *out,
                                   uint64_t out_cap, int64_t *dim_offsets) {
  if (!ind_offsets || !feat_offsets || !dim_offsets || dims == 0)
    return tmb_fail(TM_ERR_ARG, "bits_to_cvec_ind: bad arguments");
  if (ind_offsets[0] < 0 || feat_offsets[0] < 0)
    return tmb_fail(TM_ERR_ARG, "bits_to_cvec_ind: offsets must be >= 0");
  // host side: validate the offsets, lay out staging words and output blocks
  std::vector<int64_t> meta(4 * ((size_t)dims + 1));
  int64_t *lists = meta.data(), *feats = lists + dims + 1, *woff = feats + dims + 1,
          *boff = woff + dims + 1;
  uint64_t words = 0, bytes = 0;
  for (uint32_t h = 0; h <= dims; h++) {
    lists[h] = ind_offsets[h];
    feats[h] = feat_offsets[h];
    woff[h] = (int64_t)words;
    boff[h] = (int64_t)bytes;
    if (h == dims) break;
    if (ind_offsets[h + 1] < ind_offsets[h] || feat_offsets[h + 1] < feat_offsets[h])
      return tmb_fail(TM_ERR_ARG, "bits_to_cvec_ind: offsets must be nondecreasing");
    const uint64_t k = (uint64_t)(feat_offsets[h + 1] - feat_offsets[h]);
    words += n * ((k + 31) / 32);
    bytes += n * (((flip ? 2 * k : k) + 7) / 8);
  }
  for (uint32_t h = 0; h <= dims; h++) dim_offsets[h] = boff[h];
  if (!out) return TM_OK;  // sizing call: dim_offsets only
  if (out_cap < bytes) return tmb_fail(TM_ERR_ARG, "bits_to_cvec_ind: output too small");
  const uint64_t n_set = (uint64_t)(ind_offsets[dims] - ind_offsets[0]);
  if (n_set && !set_bits) return tmb_fail(TM_ERR_ARG, "bits_to_cvec_ind: bad arguments");
  tmb::DevGuard guard(device);
  CKU(guard.err);
  DevScratch buf;
  const size_t meta_b = meta.size() * 8, stage_b = ((words * 4 + 255) / 256) * 256;
  const size_t idx_b = on_device ? 0 : n_set * 8, out_b = on_device ? 0 : bytes;
  CKU(buf.ensure(meta_b + stage_b + idx_b + out_b + 512));
  uint8_t *base = (uint8_t *)buf.p;
  int64_t *dmeta = (int64_t *)base;
  uint32_t *stage = (uint32_t *)(base + ((meta_b + 255) / 256) * 256);
  uint8_t *tail = (uint8_t *)stage + stage_b;
  const int64_t *di = set_bits;
  uint8_t *dout = out;
  if (!on_device) {
    int64_t *st = (int64_t *)tail;
    if (n_set) CKU(cudaMemcpy(st, set_bits, n_set * 8, cudaMemcpyHostToDevice));
    di = st;
    dout = tail + idx_b;
  }
  CKU(cudaMemcpy(dmeta, meta.data(), meta_b, cudaMemcpyHostToDevice));
  if (words) CKU(cudaMemset(stage, 0, words * 4));
  if (n_set) k_scatter_bits_ind<<<grid_for(n_set), 256>>>(di, dmeta, dims, n, stage);
  if (bytes) k_pack_bytes_ind<<<grid_for(bytes), 256>>>(stage, dmeta, dims, n, flip, dout);
  CKU(cudaGetLastError());
  if (!on_device && bytes) CKU(cudaMemcpy(out, dout, bytes, cudaMemcpyDeviceToHost));
  else CKU(cudaDeviceSynchronize());
  return TM_OK;
}
