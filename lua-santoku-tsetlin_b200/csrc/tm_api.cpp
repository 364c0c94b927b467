// Host side of the C ABI (include/tsetlin_b200.h): machine lifecycle, data
// staging, training orchestration, predict, persistence.  Device work is in
// tm_kernels.cu; this file never computes a result on the CPU.
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <functional>
#include <map>
#include <tuple>
#include <atomic>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/tsetlin_b200.h"
#include "tm_internal.h"

using namespace tmb;

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
static thread_local std::string g_err;

static int fail(int code, const char *fmt, ...) __attribute__((format(printf, 2, 3)));
static int fail(int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

#define CK(call)                                                                      \
  do {                                                                                \
    cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess)                                                            \
      return fail(e_ == cudaErrorMemoryAllocation ? TM_ERR_OOM : TM_ERR_CUDA,         \
                  "%s failed: %s", #call, cudaGetErrorString(e_));                    \
  } while (0)

// Every device allocation of the library goes through here.  A failure
// injected by tm_debug_fail_alloc makes the chosen allocation report
// cudaErrorMemoryAllocation without calling cudaMalloc, so the error paths
// of create / train / predict can be tested without exhausting a GPU.
static std::atomic<int64_t> g_fail_alloc{-1};

cudaError_t tmb_dev_malloc(void **p, size_t n) {
  int64_t c = g_fail_alloc.load();
  while (c >= 0 && !g_fail_alloc.compare_exchange_weak(c, c - 1)) {
  }
  if (c == 0) {
    *p = nullptr;
    return cudaErrorMemoryAllocation;
  }
  return cudaMalloc(p, n);
}

extern "C" int tm_debug_fail_alloc(int64_t after) {
  g_fail_alloc.store(after < 0 ? -1 : after);
  return TM_OK;
}

extern "C" const char *tm_last_error(void) { return g_err.c_str(); }
extern "C" uint32_t tm_align(void) { return 8; }
extern "C" void tm_free(void *p) { free(p); }

// Grow-only device buffer.
struct DevBuf {
  void *p = nullptr;
  size_t cap = 0;
  cudaError_t ensure(size_t n) {
    if (n <= cap) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    size_t want = n < 256 ? 256 : n;
    cudaError_t e = tmb_dev_malloc(&p, want);
    if (e == cudaSuccess) cap = want;
    return e;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
  template <class T>
  T *as() const { return (T *)p; }
};

// ---------------------------------------------------------------------------
// machine
// ---------------------------------------------------------------------------
struct tm_machine {
  int32_t type = TM_CLASSIFIER;
  bool individualized = false, reusable = false, has_state = false, trained = false;
  uint32_t classes = 0, features = 0, clauses = 0, tol = 0, maxlit = 0, target = 0;
  uint32_t B = 8, ib = 1, input_bits = 0, input_chunks = 0, clause_chunks = 0;
  uint32_t class_chunks = 0, state_chunks = 0, action_chunks = 0;
  uint8_t tail_mask = 0xFF;
  double negative = 0, specificity = 1;
  uint64_t seed = 0;
  int device = 0;
  std::vector<uint64_t> feat_sizes;   // individualized
  std::vector<uint32_t> n_chunks;     // per class reference row bytes
  std::vector<ClassDev> cls;          // host copy of the class layout
  uint64_t act_words = 0, cnt_words = 0;
  uint32_t *d_act = nullptr, *d_cnt = nullptr;
  ClassDev *d_cls = nullptr;
  int32_t *d_lits = nullptr;
  bool lits_valid = false;
  cudaStream_t st = nullptr;
  bool timing = false;
  bool pair = false;      // TSETLIN_B200_PAIR=1: split units too large for one SM over a
                          // 2-CTA cluster instead of keeping their automata in global memory
  bool no_warp = false;   // TSETLIN_B200_NO_WARP=1: never train a unit with one warp
  uint32_t row_wait = TM_WAIT_LIMIT;  // TSETLIN_B200_ROW_WAIT: try-wait iterations per
                                      // sample row (tests shorten it to see TM_ERR_DEVICE)
  int force_mode = -1;    // >= 0: train with this variant (tm_force_variant)
  int force_cpw = 1;
  int autotune = 1;       // 0 heuristic variant choice, 1 tuned (cached per shape),
                          // 2 tuned afresh on every train call; TSETLIN_B200_AUTOTUNE
  int last_mode = -1;     // k_train variant of the last launch
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  tm_stats stats{};
  // tx: training rows (kept for all epochs of a train call); x: predict rows.
  // Separate, so that a predict inside an `each` callback does not replace
  // the rows the next epoch trains on.
  DevBuf x, tx, raw, labels, codes, perm, perm_scratch, sums, outc, work, tdev, cls_job, errf;
  // device-resident search round: checkpoint of the actions, and (owner of
  // the round) its tables and the staged holdout truth
  DevBuf ckpt, search, search_truth;
  // large-batch predict as a GEMM: the action bytes (valid while act8_valid,
  // in the encoding of act8_kind), a chunk of sample bytes, the chunk's
  // clause x sample products and the library's workspace
  DevBuf act8, x8, gemm_c, gemm_ws;
  bool act8_valid = false;
  int act8_kind = 0;
  // (owner of a search round) the GEMM predict's action-byte scratch, shared
  // by the round's machines one after another, and the holdout bytes of
  // each distinct holdout row layout
  DevBuf search_act8;
  std::vector<DevBuf> search_x8;
  // the autotuner's snapshot of the automata between its trials
  DevBuf tune_snap;
  // pinned staging of small host requests (TM_PIN_STAGE bytes each way):
  // inputs go host -> pin -> device, outputs device -> pin -> host, so that
  // a one-sample predict makes no pageable (synchronously staged) copy.
  // pin_ev marks the end of the last copy out of the input half.
  uint8_t *pin = nullptr;
  cudaEvent_t pin_ev = nullptr;
  bool pin_pending = false;
};

// The automata changed: the literal counts and the action bytes of the GEMM
// predict are stale.
static void invalidate_derived(tm_machine *m) {
  m->lits_valid = false;
  m->act8_valid = false;
}

// ---- large-batch predict as a GEMM ------------------------------------------
// The 8-bit encoding the GEMM uses on each device: 0 not yet tried, a
// TM_GEMM_* kind, or -1 when the library offers neither (the bitwise
// kernels then serve every size).  TSETLIN_B200_GEMM=off|int8|fp8 overrides
// the choice at the first large predict of the process.
static std::mutex g_gemm_mu;
static int g_gemm_kind[64];

static int gemm_kind_of(int dev) {
  std::lock_guard<std::mutex> lk(g_gemm_mu);
  if (dev < 0 || dev >= 64) return -1;
  if (g_gemm_kind[dev] == 0) {
    const char *e = getenv("TSETLIN_B200_GEMM");
    if (e && !strcmp(e, "off")) g_gemm_kind[dev] = -1;
    else if (e && !strcmp(e, "fp8")) g_gemm_kind[dev] = TM_GEMM_FP8;
    else g_gemm_kind[dev] = TM_GEMM_INT8;
  }
  return g_gemm_kind[dev];
}


constexpr uint64_t TM_PIN_STAGE = 256 << 10;

// The input half of the machine's pinned staging buffer, ready to be
// written, or null when the request is too large for it (or pinned memory
// cannot be had: the caller then copies from the pageable source).
static uint8_t *pin_stage(tm_machine *m, uint64_t bytes) {
  if (bytes > TM_PIN_STAGE) return nullptr;
  if (!m->pin) {
    if (cudaHostAlloc((void **)&m->pin, 2 * TM_PIN_STAGE, cudaHostAllocDefault) != cudaSuccess) {
      cudaGetLastError();
      m->pin = nullptr;
      return nullptr;
    }
    if (cudaEventCreateWithFlags(&m->pin_ev, cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError();
      cudaFreeHost(m->pin);
      m->pin = nullptr;
      return nullptr;
    }
  }
  if (m->pin_pending) {
    if (cudaEventSynchronize(m->pin_ev) != cudaSuccess) return nullptr;
    m->pin_pending = false;
  }
  return m->pin;
}

// Kernels launched by a CUB 64-bit radix sort of pairs: upsweep histogram,
// exclusive scan and one onesweep pass per 8-bit digit.
static const uint64_t kSortKernels = 10;

static void note_launch(tm_machine *m, uint64_t k) { m->stats.kernel_launches += k; }

static uint32_t derive_target(uint32_t clauses, uint32_t tol, double targetf) {
  // capi.c:480-483 (fmaxf: single precision)
  double t;
  if (targetf < 0)
    t = sqrt((double)clauses / 2.0) * (double)tol;
  else
    t = ceil(targetf >= 1 ? targetf : (double)fmaxf(1.0f, (float)((double)clauses * targetf)));
  return (uint32_t)t;
}

// Per-class device layout (see ClassDev).
static void layout_classes(tm_machine *m) {
  const uint32_t C = m->classes;
  m->cls.assign(C, ClassDev{});
  m->n_chunks.assign(C, 0);
  uint64_t ao = 0, co = 0;
  const uint32_t mpl = m->B - 1;
  for (uint32_t h = 0; h < C; h++) {
    const uint64_t F = m->individualized ? m->feat_sizes[h] : m->features;
    const uint64_t ibits = 2 * F;
    const uint32_t nch = (uint32_t)((ibits + 7) / 8);
    ClassDev &c = m->cls[h];
    c.W = (nch + 3) / 4;
    c.Wp = (c.W + 3) / 4 * 4;
    c.input_bits = (uint32_t)ibits;
    c.s_picks = (uint32_t)((double)(2 * F) / m->specificity);  // capi.c:181 / :347
    const uint32_t lb = nch - 4 * (c.W - 1);
    c.vmask = lb >= 4 ? 0xFFFFFFFFu : ((1u << (8 * lb)) - 1);
    const uint32_t sh = 8 * (lb - 1);
    const uint32_t tb = (uint32_t)(ibits & 7);
    const uint32_t tmask = tb ? ((1u << tb) - 1) : 0xFFu;
    c.emask = (c.vmask & ~(0xFFu << sh)) | (tmask << sh);
    // the reference masks the action carry of the tail byte only on its byte
    // path, which handles the tail when input_chunks % 16 != 0
    c.amask = (nch % 16 != 0) ? c.emask : c.vmask;
    c.act_off = ao;
    c.cnt_off = co;
    c.x_off = 0;
    ao += (uint64_t)m->clauses * c.Wp;
    co += (uint64_t)m->clauses * mpl * c.Wp;
    m->n_chunks[h] = nch;
  }
  m->act_words = ao;
  m->cnt_words = co;
  uint64_t ta = 0;
  for (uint32_t h = 0; h < C; h++) ta += (uint64_t)m->clauses * m->n_chunks[h];
  m->action_chunks = (uint32_t)ta;
  m->state_chunks = (uint32_t)(ta * mpl);
}

static void free_device(tm_machine *m) {
  if (m->d_act) cudaFree(m->d_act);
  if (m->d_cnt) cudaFree(m->d_cnt);
  if (m->d_cls) cudaFree(m->d_cls);
  if (m->d_lits) cudaFree(m->d_lits);
  m->d_act = m->d_cnt = nullptr;
  m->d_cls = nullptr;
  m->d_lits = nullptr;
}

static int alloc_device(tm_machine *m, bool with_state) {
  free_device(m);
  CK(tmb_dev_malloc((void **)&m->d_act, std::max<uint64_t>(m->act_words, 4) * 4));
  CK(cudaMemsetAsync(m->d_act, 0, std::max<uint64_t>(m->act_words, 4) * 4, m->st));
  if (with_state) {
    CK(tmb_dev_malloc((void **)&m->d_cnt, std::max<uint64_t>(m->cnt_words, 4) * 4));
    CK(cudaMemsetAsync(m->d_cnt, 0, std::max<uint64_t>(m->cnt_words, 4) * 4, m->st));
  }
  CK(tmb_dev_malloc((void **)&m->d_cls, std::max<size_t>(m->classes, 1) * sizeof(ClassDev)));
  CK(cudaMemcpyAsync(m->d_cls, m->cls.data(), m->classes * sizeof(ClassDev),
                     cudaMemcpyHostToDevice, m->st));
  CK(tmb_dev_malloc((void **)&m->d_lits, std::max<uint64_t>((uint64_t)m->classes * m->clauses, 1) * 4));
  invalidate_derived(m);
  m->has_state = with_state;
  return TM_OK;
}

extern "C" void tm_params_init(tm_params *p) {
  memset(p, 0, sizeof(*p));
  p->state_bits = 8;
  p->include_bits = 1;
  p->target = -1;
  p->negative = -1;
}

static int check_limits(tm_machine *m) {
  for (uint32_t h = 0; h < m->classes; h++) {
    const uint64_t F = m->individualized ? m->feat_sizes[h] : m->features;
    if (F == 0) return fail(TM_ERR_ARG, "class %u has no features", h);
    if (2 * F >= (1ull << 31)) return fail(TM_ERR_ARG, "too many features");
    if ((uint64_t)m->clauses * m->tol >= (1ull << 31))
      return fail(TM_ERR_ARG, "clauses * clause_tolerance must stay below 2^31");
  }
  if (m->B > 32) return fail(TM_ERR_ARG, "state above 32 bits is not supported");
  return TM_OK;
}

// A train-kernel variant a caller may pin: modes 0-3 with 1, 2 or 4
// clauses per warp, or mode 4 with one of its configurations.
static bool variant_ok(int mode, int cpw) {
  if (mode == TM_MODE_WPT) return cpw >= 1 && cpw <= wpt_configs();
  return mode >= -1 && mode <= TM_MODE_WARP && (cpw == 1 || cpw == 2 || cpw == 4);
}

extern "C" int tm_create(const tm_params *p, tm_machine **out) {
  if (!p || !out) return fail(TM_ERR_ARG, "null argument");
  *out = nullptr;
  // capi.c:463-472
  if (!p->classes) return fail(TM_ERR_ARG, "create: classes must be greater than 1");
  if (!p->clauses) return fail(TM_ERR_ARG, "create: clauses must be greater than 0");
  if (!p->clause_tolerance) return fail(TM_ERR_ARG, "create: clause_tolerance must be greater than 0");
  if (!p->clause_maximum) return fail(TM_ERR_ARG, "create: clause_maximum must be greater than 0");
  const uint32_t sb = p->state_bits ? p->state_bits : 8;
  if (sb < 2) return fail(TM_ERR_ARG, "create: bits must be greater than 1");
  if (!(p->specificity > 0)) return fail(TM_ERR_ARG, "create: specificity must be positive");
  if (p->type != TM_CLASSIFIER && p->type != TM_ENCODER)
    return fail(TM_ERR_ARG, "unexpected tsetlin machine type in create");
  if (p->individualized && !p->feat_offsets)
    return fail(TM_ERR_ARG, "create: feat_offsets must have classes + 1 elements");
  tm_machine *m = new tm_machine();
  m->type = p->type;
  m->individualized = p->individualized != 0;
  m->reusable = p->reusable != 0;
  m->negative = p->negative < 0 ? 1.0 / (double)p->classes : p->negative;  // capi.c:474
  m->classes = p->classes;
  m->class_chunks = (p->classes + 7) / 8;
  m->clauses = (p->clauses + 7) / 8 * 8;                                    // capi.c:477
  m->tol = p->clause_tolerance;
  m->maxlit = p->clause_maximum;
  m->target = derive_target(m->clauses, m->tol, p->target);
  m->B = sb;
  m->ib = p->include_bits ? p->include_bits : 1;
  m->specificity = p->specificity;
  m->clause_chunks = m->clauses / 8;
  m->seed = p->seed;
  m->device = p->device;
  {
    const char *e = getenv("TSETLIN_B200_PAIR");
    m->pair = e && e[0] == '1';
    const char *w = getenv("TSETLIN_B200_NO_WARP");
    m->no_warp = w && w[0] == '1';
    const char *t = getenv("TSETLIN_B200_AUTOTUNE");
    m->autotune = t && t[0] >= '0' && t[0] <= '2' ? t[0] - '0' : 1;
    // TSETLIN_B200_VARIANT=mode:cpw pins the train-kernel variant, as
    // tm_force_variant does (for measurements from the command line)
    // TSETLIN_B200_ROW_WAIT=k: a thread gives up on a sample row after k
    // try-waits and the train call reports TM_ERR_DEVICE (0: at once).  For
    // tests of the device error path; copies in flight are still drained.
    const char *rw = getenv("TSETLIN_B200_ROW_WAIT");
    if (rw && rw[0] >= '0' && rw[0] <= '9') m->row_wait = (uint32_t)strtoul(rw, nullptr, 10);
    const char *v = getenv("TSETLIN_B200_VARIANT");
    int vm = -1, vc = 1;
    if (v && sscanf(v, "%d:%d", &vm, &vc) >= 1 && vm >= 0 && variant_ok(vm, vc)) {
      m->force_mode = vm;
      m->force_cpw = vc;
    }
  }
  if (m->individualized) {
    // capi.c:528-606 leaves features, input_bits, input_chunks and tail_mask
    // of an individualized machine unset (zero); they are persisted as such
    m->tail_mask = 0;
    for (uint32_t h = 0; h < m->classes; h++) {
      const int64_t k = p->feat_offsets[h + 1] - p->feat_offsets[h];
      if (k <= 0) {
        delete m;
        return fail(TM_ERR_ARG, "create: feat_offsets must be increasing");
      }
      m->feat_sizes.push_back((uint64_t)k);
    }
  } else {
    m->features = p->features;
    m->input_bits = 2 * m->features;                                         // capi.c:487
    const uint32_t tb = m->input_bits & 7;
    m->tail_mask = tb ? (uint8_t)((1u << tb) - 1) : 0xFF;
    m->input_chunks = (m->input_bits + 7) / 8;
  }
  int rc = check_limits(m);
  if (rc) {
    delete m;
    return rc;
  }
  layout_classes(m);
  DevGuard g(m->device);
  if (cudaStreamCreateWithFlags(&m->st, cudaStreamNonBlocking) != cudaSuccess) {
    delete m;
    return fail(TM_ERR_CUDA, "stream creation failed");
  }
  rc = alloc_device(m, true);
  if (!rc) {
    cudaError_t e = launch_setup(m->d_act, m->d_cnt, m->d_cls, m->classes, m->clauses, m->B,
                                 m->act_words, m->st);
    note_launch(m, 1);
    if (e == cudaSuccess) e = cudaStreamSynchronize(m->st);
    if (e != cudaSuccess) rc = fail(TM_ERR_CUDA, "setup: %s", cudaGetErrorString(e));
  }
  if (rc) {
    tm_destroy(m);
    return rc;
  }
  *out = m;
  return TM_OK;
}

extern "C" void tm_destroy(tm_machine *m) {
  if (!m) return;
  DevGuard g(m->device);
  if (m->st) cudaStreamSynchronize(m->st);
  free_device(m);
  for (DevBuf *b : {&m->x, &m->tx, &m->raw, &m->labels, &m->codes, &m->perm, &m->perm_scratch, &m->sums,
                    &m->outc, &m->work, &m->tdev, &m->cls_job, &m->errf, &m->ckpt, &m->search,
                    &m->search_truth, &m->act8, &m->x8, &m->gemm_c, &m->gemm_ws,
                    &m->search_act8, &m->tune_snap})
    b->release();
  for (DevBuf &b : m->search_x8) b.release();
  if (m->ev0) cudaEventDestroy(m->ev0);
  if (m->ev1) cudaEventDestroy(m->ev1);
  if (m->pin_ev) cudaEventDestroy(m->pin_ev);
  if (m->pin) cudaFreeHost(m->pin);
  if (m->st) cudaStreamDestroy(m->st);
  delete m;
}

extern "C" int tm_force_variant(tm_machine *m, int32_t mode, int32_t cpw) {
  if (!m) return fail(TM_ERR_ARG, "null machine");
  if (!variant_ok(mode, cpw))
    return fail(TM_ERR_ARG, "force_variant: mode -1..3 with clauses per warp 1, 2 or 4, or mode 4 "
                            "with a configuration 1..%d", wpt_configs());
  m->force_mode = mode;
  m->force_cpw = cpw;
  return TM_OK;
}

extern "C" int tm_set_autotune(tm_machine *m, int32_t mode) {
  if (!m) return fail(TM_ERR_ARG, "null machine");
  if (mode < 0 || mode > 2) return fail(TM_ERR_ARG, "autotune: mode must be 0, 1 or 2");
  m->autotune = mode;
  return TM_OK;
}

extern "C" int tm_stats_enable(tm_machine *m, int32_t on) {
  if (!m) return fail(TM_ERR_ARG, "null machine");
  DevGuard g(m->device);
  if (on && !m->ev0) {
    CK(cudaEventCreate(&m->ev0));
    CK(cudaEventCreate(&m->ev1));
  }
  m->timing = on != 0;
  return TM_OK;
}

extern "C" int tm_get_stats(const tm_machine *m, tm_stats *out) {
  if (!m || !out) return fail(TM_ERR_ARG, "null argument");
  *out = m->stats;
  return TM_OK;
}

extern "C" int tm_reset_stats(tm_machine *m) {
  if (!m) return fail(TM_ERR_ARG, "null machine");
  m->stats = tm_stats{};
  return TM_OK;
}

extern "C" int tm_type(const tm_machine *m) { return m ? m->type : TM_ERR_ARG; }

extern "C" int tm_get_info(const tm_machine *m, uint64_t *o) {
  if (!m || !o) return fail(TM_ERR_ARG, "null argument");
  o[0] = (uint64_t)m->type; o[1] = m->classes; o[2] = m->features; o[3] = m->clauses;
  o[4] = m->tol; o[5] = m->maxlit; o[6] = m->target; o[7] = m->B; o[8] = m->ib;
  o[9] = m->input_bits; o[10] = m->input_chunks; o[11] = m->clause_chunks;
  o[12] = m->class_chunks; o[13] = m->state_chunks; o[14] = m->action_chunks;
  o[15] = m->tail_mask; o[16] = m->individualized; o[17] = m->reusable; o[18] = m->has_state;
  return TM_OK;
}

// ---------------------------------------------------------------------------
// staging of samples: reference byte rows -> padded device words
// ---------------------------------------------------------------------------
// Sets cls[h].x_off for an n-sample upload and returns the words needed.
static uint64_t x_layout(tm_machine *m, uint64_t n, std::vector<ClassDev> &cls) {
  cls = m->cls;
  if (!m->individualized) return n * cls[0].Wp;
  uint64_t off = 0;
  for (uint32_t h = 0; h < m->classes; h++) {
    cls[h].x_off = off;
    off += n * cls[h].Wp;
  }
  return off;
}

static int stage_rows(tm_machine *m, DevBuf &dst, const uint8_t *src, const int64_t *dim_offsets,
                      uint64_t n, bool on_device, std::vector<ClassDev> &cls,
                      uint32_t *zero = nullptr, uint64_t zero_words = 0) {
  const uint64_t words = x_layout(m, n, cls);
  CK(dst.ensure(std::max<uint64_t>(words, 4) * 4));
  const uint32_t nblk = m->individualized ? m->classes : 1;
  for (uint32_t h = 0; h < nblk; h++) {
    const uint64_t nch = m->n_chunks[h];
    const uint8_t *s = src + (m->individualized ? (uint64_t)dim_offsets[h] : 0);
    const uint8_t *dsrc = s;
    if (!on_device) {
      CK(m->raw.ensure(std::max<uint64_t>(n * nch, 16)));
      if (uint8_t *pb = pin_stage(m, n * nch)) {
        memcpy(pb, s, n * nch);
        CK(cudaMemcpyAsync(m->raw.p, pb, n * nch, cudaMemcpyHostToDevice, m->st));
        CK(cudaEventRecord(m->pin_ev, m->st));
        m->pin_pending = true;
      } else {
        CK(cudaMemcpyAsync(m->raw.p, s, n * nch, cudaMemcpyHostToDevice, m->st));
      }
      dsrc = m->raw.as<uint8_t>();
    }
    CK(launch_repack(dsrc, n, nch, nch, dst.as<uint32_t>() + cls[h].x_off, cls[h].Wp, m->st,
                     h == 0 ? zero : nullptr, h == 0 ? zero_words : 0));
    note_launch(m, 1);
    if (!on_device && m->individualized) CK(cudaStreamSynchronize(m->st));  // raw reuse
  }
  return TM_OK;
}

static int upload_cls(tm_machine *m, ClassDev *d, const std::vector<ClassDev> &cls) {
  CK(cudaMemcpyAsync(d, cls.data(), cls.size() * sizeof(ClassDev), cudaMemcpyHostToDevice, m->st));
  return TM_OK;
}

// ---------------------------------------------------------------------------
// training
// ---------------------------------------------------------------------------
static uint64_t neg_threshold(double negative) {
  const double q = (1.0 - negative) * 4294967296.0;
  if (!(q > 0)) return 0;
  if (q >= 4294967296.0) return 4294967296ull;
  return (uint64_t)floor(q);
}

struct TrainJob {
  tm_machine *m;
  const tm_train_args *a;
  std::vector<ClassDev> cls;  // with x offsets
  ClassDev *d_cls = nullptr;  // per-job class table (device)
  uint32_t *d_x = nullptr;
  int32_t *d_labels = nullptr;
  uint8_t *d_codes = nullptr;
  uint64_t seed = 0;
};

static TrainSmem plan_smem(uint32_t Wpmax, uint32_t Bmax, uint32_t smax, int mode, int cpw = 1) {
  TrainSmem L{};
  uint32_t o = 0;
  auto take = [&](uint32_t bytes) {
    const uint32_t at = o;
    o += (bytes + 127) / 128 * 128;
    return at;
  };
  const uint32_t cpc = mode == TM_MODE_PAIR ? 4 : 8;  // clauses held by one CTA
  // GLOBAL: the action plane only (count planes stay in global memory)
  L.state_words = mode == TM_MODE_GLOBAL ? cpc * Wpmax : cpc * Bmax * Wpmax;
  L.state_off = take(L.state_words * 4);
  L.ring_words = Wpmax;
  L.ring_off = take(TM_RING * Wpmax * 4);
  L.bar_off = take(TM_RING * 8);
  L.list_off = take(train_threads(mode, cpw) * 4 * 9);  // one entry per thread
  L.votes_off = take(128 * 4);
  L.ib_words = Wpmax;
  // Type Ib levels and overflow lists: TM_IB_SLOTS slots
  L.ib_off = take(2 * TM_IB_SLOTS * Wpmax * 4);
  L.ovf_cap = std::max<uint32_t>(1, smax / 4);
  L.ovf_off = take(TM_IB_SLOTS * L.ovf_cap * 4);
  L.misc_off = take(32 * 4);
  L.total = o;
  L.wait_limit = TM_WAIT_LIMIT;
  return L;
}

static int num_sms(int dev) {
  int v = 0;
  cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
  return v > 0 ? v : 1;
}

static int max_smem_optin(int dev) {
  int v = 0;
  cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  return v > 0 ? v : 48 * 1024;
}

static int validate_train(tm_machine *m, const tm_train_args *a) {
  if (!m || !a) return fail(TM_ERR_ARG, "null argument");
  if (a->class_end && (a->class_begin >= a->class_end || a->class_end > m->classes))
    return fail(TM_ERR_ARG, "train: class range [%u, %u) outside [0, %u)", a->class_begin,
                a->class_end, m->classes);
  if (!m->has_state || !m->d_cnt)
    return fail(TM_ERR_STATE, "can't train a model loaded without state");
  if (a->samples >= (1ull << 31)) return fail(TM_ERR_ARG, "train: too many samples");
  if (a->samples && !a->problems) return fail(TM_ERR_ARG, "train: problems missing");
  if (m->type == TM_CLASSIFIER && a->samples && !a->solutions)
    return fail(TM_ERR_ARG, "train: solutions missing");
  if (m->type == TM_ENCODER && a->samples && !a->codes)
    return fail(TM_ERR_ARG, "train: codes missing");
  if (m->individualized && a->samples && !a->dim_offsets)
    return fail(TM_ERR_ARG, "train: dim_offsets missing");
  return TM_OK;
}

// ---------------------------------------------------------------------------
// Train kernel variants.  All end in the same automaton state (every random
// draw is a Philox output keyed by seed, epoch, sample and unit, so no draw
// depends on which thread or variant takes it), so the choice is a matter of
// speed only: a
// heuristic by resident CTAs per SM, or an autotuner that times the
// feasible variants on a short trial of the actual launch and caches the
// fastest per launch shape for the life of the process.
// ---------------------------------------------------------------------------
struct TrainShape {
  uint32_t Wpmax, Bmin, Bmax, smax, units;
  int optin, sms;
};

struct TrainPlan {
  int mode = TM_MODE_GLOBAL;
  int cpw = 1;  // clauses per warp (single-CTA variants, 8 state bits)
  TrainSmem lay{};
  int grid = 0;
};

// Fills `p` for `mode` (and `cpw` clauses per warp) when that variant can
// run this launch.
// Units per CTA of the one-warp-per-unit kernel for its variant number
// (cpw): 1 four units per CTA, 2 one unit per CTA.
static int warp_units_per_cta(int cpw) { return cpw == 2 ? 1 : 4; }

static bool plan_mode(int mode, const TrainShape &sh, TrainPlan &p, int cpw = 1) {
  p = TrainPlan{};
  p.mode = mode;
  p.cpw = cpw;
  if (mode == TM_MODE_WPT) {
    // cpw is the configuration id; the automata of 8-bit units only
    if (sh.Bmin != 8 || sh.Bmax != 8) return false;
    size_t bytes = 0;
    const int occ = train_wpt_occupancy(cpw, sh.Wpmax, sh.smax, &bytes);
    if (occ <= 0 || (int)bytes > sh.optin) return false;
    p.grid = (int)std::min<uint64_t>(sh.units, (uint64_t)sh.sms * occ);
    return true;
  }
  if (mode == TM_MODE_WARP) {
    // cpw selects the units per CTA: 1 -> four, 2 -> one (8-bit automata)
    if (sh.Wpmax > 64 || sh.Bmax > 8 || (cpw != 1 && cpw != 2)) return false;
    if (cpw == 2 && (sh.Bmin != 8 || sh.Bmax != 8)) return false;
    const int wpc = warp_units_per_cta(cpw);
    size_t wsm = 0;
    const int occ = train_warp_occupancy(sh.Wpmax, sh.Bmin, sh.Bmax, sh.smax, wpc, &wsm);
    if (occ <= 0 || (int)wsm > sh.optin) return false;
    p.grid = (int)std::min<uint64_t>((sh.units + wpc - 1) / wpc, (uint64_t)sh.sms * occ);
    return true;
  }
  if (cpw != 1 && (mode == TM_MODE_PAIR || sh.Bmin != 8 || sh.Bmax != 8)) return false;
  if (mode == TM_MODE_PAIR && sh.Bmax > 8) return false;
  p.lay = plan_smem(sh.Wpmax, sh.Bmax, sh.smax, mode, cpw);
  if ((int)p.lay.total > sh.optin) return false;
  const int occ = train_occupancy(p.lay, mode, sh.Bmin, sh.Bmax, cpw);
  if (occ <= 0) return false;
  p.grid = mode == TM_MODE_PAIR ? 2 * (int)std::min<uint64_t>(sh.units, (uint64_t)occ)
                                : (int)std::min<uint64_t>(sh.units, (uint64_t)sh.sms * occ);
  return true;
}

static int heuristic_plan(const TrainShape &sh, const tm_machine *m0, TrainPlan &out) {
  // short rows: one warp per unit
  if (!m0->no_warp && plan_mode(TM_MODE_WARP, sh, out)) return TM_OK;
  // all planes in shared memory when a unit fits one SM, unless global
  // planes give more resident CTAs (measured on B200: 8,192-feature rows
  // train 26 % faster with global planes at two CTAs per SM than with shared
  // planes at one); a 2-CTA cluster only on request (its per-sample cluster
  // barrier costs more than the L2 round trips it saves)
  TrainPlan s, g, c;
  const bool hs = plan_mode(TM_MODE_SMEM, sh, s);
  const bool hg = plan_mode(TM_MODE_GLOBAL, sh, g);
  if (!hs && m0->pair && plan_mode(TM_MODE_PAIR, sh, c)) {
    out = c;
    return TM_OK;
  }
  if (hs && (!hg || s.grid >= g.grid)) {
    out = s;
    return TM_OK;
  }
  if (hg) {
    out = g;
    return TM_OK;
  }
  return fail(TM_ERR_ARG, "train: rows too wide for one CTA (%u words, %u state bits)", sh.Wpmax,
              sh.Bmax);
}

// Units a launch of `p` holds at once: a warp per unit (4 or 1 per CTA), a CTA
// per unit, or a 2-CTA cluster per unit.
static uint64_t resident_units(const TrainPlan &p) {
  if (p.mode == TM_MODE_WARP) return (uint64_t)p.grid * warp_units_per_cta(p.cpw);
  if (p.mode == TM_MODE_WPT) return (uint64_t)p.grid;
  if (p.mode == TM_MODE_PAIR) return (uint64_t)p.grid / 2;
  return (uint64_t)p.grid;
}

// Uploads the machine table and work list and launches `p` over epochs
// [e0, e1).  `ms` (optional) receives the kernel's device time.
static int launch_plan(const TrainPlan &p, const TrainShape &sh, const std::vector<TrainDev> &td,
                       const std::vector<WorkItem> &work, uint32_t e0, uint32_t e1,
                       tm_machine *m0, float *ms, uint32_t *herr) {
  cudaStream_t st = m0->st;
  const size_t tb = td.size() * sizeof(TrainDev);
  const size_t wb = work.size() * sizeof(WorkItem);
  const size_t off_w = (tb + 255) & ~(size_t)255;
  const size_t off_c = (off_w + wb + 255) & ~(size_t)255;
  CK(m0->tdev.ensure(off_c + 256));
  uint8_t *base = m0->tdev.as<uint8_t>();
  CK(cudaMemcpyAsync(base, td.data(), tb, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(base + off_w, work.data(), wb, cudaMemcpyHostToDevice, st));
  // [0] work counter, [2] status bits, [4..5] active (unit, sample) steps
  CK(cudaMemsetAsync(base + off_c, 0, 32, st));
  uint32_t *counter = (uint32_t *)(base + off_c);
  uint32_t *err = counter + 2;
  TrainSmem lay = p.lay;
  lay.wait_limit = m0->row_wait;
  if (ms) CK(cudaEventRecord(m0->ev0, st));
  if (p.mode == TM_MODE_WARP)
    CK(launch_train_warp((const TrainDev *)base, (const WorkItem *)(base + off_w),
                         (uint32_t)work.size(), counter, e0, e1, sh.Wpmax, sh.Bmin, sh.Bmax,
                         sh.smax, warp_units_per_cta(p.cpw), p.grid, st,
                         (unsigned long long *)(err + 2)));
  else if (p.mode == TM_MODE_WPT)
    CK(launch_train_wpt(p.cpw, (const TrainDev *)base, (const WorkItem *)(base + off_w),
                        (uint32_t)work.size(), counter, e0, e1, sh.Wpmax, sh.smax, m0->row_wait,
                        p.grid, err, st));
  else
    CK(launch_train((const TrainDev *)base, (const WorkItem *)(base + off_w),
                    (uint32_t)work.size(), counter, e0, e1, lay, p.mode, sh.Bmin, sh.Bmax,
                    p.cpw, p.grid, err, st));
  if (ms) CK(cudaEventRecord(m0->ev1, st));
  note_launch(m0, 1);
  uint32_t hc[4] = {0, 0, 0, 0};
  CK(cudaMemcpyAsync(hc, err, 16, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  *herr = hc[0];
  m0->stats.train_active_pairs += (uint64_t)hc[2] | ((uint64_t)hc[3] << 32);
  if (ms) CK(cudaEventElapsedTime(ms, m0->ev0, m0->ev1));
  return TM_OK;
}

// Process-wide cache of tuned variants, keyed by launch shape.
static std::mutex g_tune_mu;
static std::map<std::string, std::pair<int, int>> g_tuned;  // -> (mode, clauses per warp)

static std::string tune_key(const TrainShape &sh, const tm_machine *m0) {
  char k[160];
  // units bucketed by powers of two: the wave count matters, not the exact count
  uint32_t ub = 0;
  while ((1u << ub) < sh.units && ub < 31) ub++;
  snprintf(k, sizeof k, "%d:%u:%u:%u:%u:%u:%d:%d", m0->device, sh.Wpmax, sh.Bmin, sh.Bmax, sh.smax,
           ub, m0->no_warp ? 1 : 0, m0->pair ? 1 : 0);
  return k;
}

static bool lookup_tuned(const TrainShape &sh, const tm_machine *m0, TrainPlan &out) {
  std::pair<int, int> v;
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tuned.find(tune_key(sh, m0));
    if (it == g_tuned.end()) return false;
    v = it->second;
  }
  return plan_mode(v.first, sh, out, v.second);
}

// Times every feasible variant on the first samples of epoch 0 of a
// sample of the launch's units, keeps the fastest, and resets the automata
// of every job to their initial state.
static int autotune_plan(std::vector<TrainJob> &jobs, const std::vector<TrainDev> &td,
                         const std::vector<WorkItem> &work, const TrainShape &sh,
                         tm_machine *m0, TrainPlan &out, bool &tuned) {
  tuned = false;
  if (m0->autotune == 1 && lookup_tuned(sh, m0, out)) {
    tuned = true;
    return TM_OK;
  }
  if (!m0->ev0) {
    CK(cudaEventCreate(&m0->ev0));
    CK(cudaEventCreate(&m0->ev1));
  }
  std::vector<TrainPlan> cand;
  for (int mode : {TM_MODE_WARP, TM_MODE_SMEM, TM_MODE_GLOBAL, TM_MODE_PAIR, TM_MODE_WPT}) {
    if (mode == TM_MODE_WARP && m0->no_warp) continue;
    if (mode == TM_MODE_WPT) {
      for (int id = 1; id <= wpt_configs(); id++) {
        TrainPlan p;
        if (plan_mode(mode, sh, p, id)) cand.push_back(p);
      }
      continue;
    }
    for (int cpw : {1, 2, 4}) {
      TrainPlan p;
      if (plan_mode(mode, sh, p, cpw)) cand.push_back(p);
    }
  }
  if (cand.size() < 2) return TM_OK;  // nothing to choose: the heuristic plan
  // Two trials, each on automata reset to the initial state (capi.c:1136-
  // 1146; a trial on automata that earlier trials trained would see another
  // feedback mix).  The first times every candidate on up to 2,048 samples
  // of epoch 0 and up to 32 units per SM, taken evenly from the cost-ordered
  // work list -- enough units that every candidate's grid is full, so that
  // occupancy counts as in the real launch.  The second times the three
  // fastest again on up to 8,192 samples and 64 units per SM, where wave
  // tails and start-up costs weigh less, and decides.
  auto trial_units = [&](size_t per_sm) {
    const size_t nu = std::min<size_t>(work.size(), (size_t)sh.sms * per_sm);
    std::vector<WorkItem> tw;
    tw.reserve(nu);
    for (size_t i = 0; i < nu; i++) tw.push_back(work[i * work.size() / nu]);
    return tw;
  };
  auto trial_rows = [&](uint32_t cap) {
    std::vector<TrainDev> tt = td;
    for (auto &t : tt) t.n = std::min<uint32_t>(t.n, cap);
    return tt;
  };
  auto reset = [&]() -> int {
    for (auto &J : jobs) {
      tm_machine *m = J.m;
      cudaError_t e = launch_setup(m->d_act, m->d_cnt, m->d_cls, m->classes, m->clauses, m->B,
                                   m->act_words, m0->st);
      if (e != cudaSuccess) return fail(TM_ERR_CUDA, "setup: %s", cudaGetErrorString(e));
      note_launch(m0, 1);
    }
    return TM_OK;
  };
  // TSETLIN_B200_TUNE_LOG=1: each candidate's trial time on stderr
  const char *tl = getenv("TSETLIN_B200_TUNE_LOG");
  const bool tune_log = tl && tl[0] == '1';
  // the trials' (unit, sample) steps are not the caller's training
  const uint64_t pairs0 = m0->stats.train_active_pairs;
  // the automata every trial starts from: reset (the initial state) or a
  // snapshot taken part-way into epoch 0
  std::function<int()> prepare = reset;
  auto timed = [&](size_t i, const std::vector<TrainDev> &tt, const std::vector<WorkItem> &tw,
                   int stage, float &tmin) -> int {
    TrainShape tsh = sh;
    tsh.units = (uint32_t)tw.size();
    TrainPlan p;
    tmin = -1;
    if (!plan_mode(cand[i].mode, tsh, p, cand[i].cpw)) return TM_OK;
    float t = 0;
    for (int rep = 0; rep < 2; rep++) {
      int rc = prepare();
      if (rc) return rc;
      uint32_t herr = 0;
      rc = launch_plan(p, tsh, tt, tw, 0, 1, m0, &t, &herr);
      if (rc) return rc;
      if (herr) return fail(TM_ERR_DEVICE, "train: a sample copy did not complete (status %u)", herr);
      tmin = rep == 0 ? t : std::min(tmin, t);
    }
    if (tune_log)
      fprintf(stderr, "tsetlin_b200 tune %d: variant %d:%d  %.3f ms  (%zu units, grid %d)\n",
              stage, cand[i].mode, cand[i].cpw, tmin, tw.size(), p.grid);
    return TM_OK;
  };
  std::vector<std::pair<float, size_t>> first;
  {
    const std::vector<TrainDev> tt = trial_rows(2048);
    const std::vector<WorkItem> tw = trial_units(32);
    for (size_t i = 0; i < cand.size(); i++) {
      float tmin = -1;
      int rc = timed(i, tt, tw, 1, tmin);
      if (rc) return rc;
      if (tmin >= 0) first.emplace_back(tmin, i);
    }
  }
  std::sort(first.begin(), first.end());
  int best = first.empty() ? -1 : (int)first[0].second;
  if (first.size() > 1) {
    // The second trial times positions [W, W + T) of epoch 0 from the
    // automata as the first W positions leave them (any variant gives the
    // same automata): past the first samples, whose empty clauses make for
    // another mix of feedback than the rest of an epoch.  Launches of fewer
    // than W + T samples time the first T from the initial state.
    const uint32_t W = 8192, T = 8192;
    const std::vector<WorkItem> tw = trial_units(64);
    std::vector<TrainDev> tt;
    uint32_t nmax = 0;
    for (const auto &t : td) nmax = std::max(nmax, t.n);
    uint64_t snap_bytes = 0;
    for (const auto &J : jobs) snap_bytes += ((uint64_t)J.m->act_words + J.m->cnt_words) * 4;
    bool steady = nmax >= W + T && snap_bytes > 0;
    if (steady) {
      TrainShape tsh = sh;
      tsh.units = (uint32_t)tw.size();
      TrainPlan p0;
      steady = plan_mode(cand[first[0].second].mode, tsh, p0, cand[first[0].second].cpw) &&
               m0->tune_snap.ensure(snap_bytes) == cudaSuccess;
      if (!steady) cudaGetLastError();
      if (steady) {
        int rc = reset();
        if (rc) return rc;
        uint32_t herr = 0;
        float tw0 = 0;
        rc = launch_plan(p0, tsh, trial_rows(W), tw, 0, 1, m0, &tw0, &herr);
        if (rc) return rc;
        if (herr) return fail(TM_ERR_DEVICE, "train: a sample copy did not complete (status %u)", herr);
        uint64_t o = 0;
        for (auto &J : jobs) {
          const uint64_t ab = (uint64_t)J.m->act_words * 4, cb = (uint64_t)J.m->cnt_words * 4;
          CK(cudaMemcpyAsync(m0->tune_snap.as<uint8_t>() + o, J.m->d_act, ab,
                             cudaMemcpyDeviceToDevice, m0->st));
          if (cb)
            CK(cudaMemcpyAsync(m0->tune_snap.as<uint8_t>() + o + ab, J.m->d_cnt, cb,
                               cudaMemcpyDeviceToDevice, m0->st));
          o += ab + cb;
        }
        prepare = [&]() -> int {
          uint64_t q = 0;
          for (auto &J : jobs) {
            const uint64_t ab = (uint64_t)J.m->act_words * 4, cb = (uint64_t)J.m->cnt_words * 4;
            CK(cudaMemcpyAsync(J.m->d_act, m0->tune_snap.as<uint8_t>() + q, ab,
                               cudaMemcpyDeviceToDevice, m0->st));
            if (cb)
              CK(cudaMemcpyAsync(J.m->d_cnt, m0->tune_snap.as<uint8_t>() + q + ab, cb,
                                 cudaMemcpyDeviceToDevice, m0->st));
            q += ab + cb;
          }
          return TM_OK;
        };
        tt = td;
        for (auto &t : tt) {
          t.perm += W;
          t.n = t.n > W ? std::min<uint32_t>(t.n - W, T) : 0;
        }
      }
    }
    if (!steady) tt = trial_rows(T);
    float best_ms = -1;
    for (size_t r = 0; r < first.size() && r < 3; r++) {
      float tmin = -1;
      int rc = timed(first[r].second, tt, tw, 2, tmin);
      if (rc) return rc;
      if (tmin >= 0 && (best_ms < 0 || tmin < best_ms)) {
        best_ms = tmin;
        best = (int)first[r].second;
      }
    }
  }
  m0->stats.train_active_pairs = pairs0;
  m0->tune_snap.release();
  // back to the initial state
  {
    int rc = reset();
    if (rc) return rc;
  }
  if (best < 0) return TM_OK;
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tuned[tune_key(sh, m0)] = std::make_pair(cand[best].mode, cand[best].cpw);
  }
  if (!plan_mode(cand[best].mode, sh, out, cand[best].cpw)) return TM_OK;
  tuned = true;
  return TM_OK;
}

// Machine table and cost-ordered work list of one launch over local epochs
// [e0, e1); job i's epoch orders start at word joff[i] of the owner's
// permutation buffer.
static void build_tables(std::vector<TrainJob> &jobs, uint32_t e0, uint32_t e1, tm_machine *m0,
                         const std::vector<uint64_t> &joff, std::vector<TrainDev> &td,
                         std::vector<WorkItem> &work, TrainShape &sh) {
  td.assign(jobs.size(), TrainDev{});
  work.clear();
  uint32_t Wpmax = 4, Bmin = 32, Bmax = 2, smax = 0;
  for (size_t i = 0; i < jobs.size(); i++) {
    TrainJob &J = jobs[i];
    tm_machine *m = J.m;
    TrainDev &t = td[i];
    t.act = m->d_act;
    t.cnt = m->d_cnt;
    t.x = J.d_x;
    t.labels = J.d_labels;
    t.codes = J.d_codes;
    t.perm = m0->perm.as<uint32_t>() + joff[i];
    t.cls = J.d_cls;
    t.seed = J.seed;
    t.thr_neg = neg_threshold(m->negative);
    t.n = (uint32_t)J.a->samples;
    t.classes = m->classes;
    t.clause_chunks = m->clause_chunks;
    t.B = m->B;
    t.ib = m->ib;
    t.tol = m->tol;
    t.maxlit = m->maxlit;
    t.T = m->target;
    t.type = (uint32_t)m->type;
    t.code_bytes = m->class_chunks;
    t.epochs = std::min<uint32_t>(J.a->iterations, e1);
    t.epoch_base = 0;
    if (t.n == 0 || t.epochs <= e0) continue;
    const uint32_t hb = J.a->class_end ? J.a->class_begin : 0;
    const uint32_t he = J.a->class_end ? std::min(J.a->class_end, m->classes) : m->classes;
    for (uint32_t h = hb; h < he; h++) {
      const ClassDev &c = J.cls[h];
      Wpmax = std::max(Wpmax, c.Wp);
      smax = std::max(smax, c.s_picks);
      const double frac =
          m->type == TM_CLASSIFIER ? std::min(1.0, 1.0 / m->classes + m->negative) : 1.0;
      const double cost = (double)t.n * (t.epochs - e0) * frac * c.Wp * m->B *
                          (1.0 + c.s_picks / (32.0 * c.W));
      for (uint32_t k = 0; k < m->clause_chunks; k++)
        work.push_back(WorkItem{(uint32_t)i, h, k, (uint32_t)std::min(cost / 64.0, 4e9)});
    }
    Bmax = std::max(Bmax, m->B);
    Bmin = std::min(Bmin, m->B);
  }
  std::stable_sort(work.begin(), work.end(),
                   [](const WorkItem &a, const WorkItem &b) { return a.cost > b.cost; });
  const int dev = m0->device;
  sh = TrainShape{Wpmax, Bmin, Bmax, smax, (uint32_t)work.size(), max_smem_optin(dev),
                  num_sms(dev)};
}

// The train-kernel variant of a launch: pinned, tuned (trials at epoch 0,
// on the freshly reset automata) or by the heuristic.
static int choose_plan(std::vector<TrainJob> &jobs, const std::vector<TrainDev> &td,
                       const std::vector<WorkItem> &work, const TrainShape &sh, uint32_t e0,
                       tm_machine *m0, TrainPlan &plan, bool &tuned) {
  tuned = false;
  if (m0->force_mode >= 0) {
    if (!plan_mode(m0->force_mode, sh, plan, m0->force_cpw))
      return fail(TM_ERR_ARG, "train: variant %d with %d clauses per warp cannot run this launch",
                  m0->force_mode, m0->force_cpw);
  } else if (m0->autotune && e0 == 0) {
    // the automata hold their initial state here (every train call starts
    // from it), so trial launches may run on them and a setup restores them
    int rc = autotune_plan(jobs, td, work, sh, m0, plan, tuned);
    if (rc) return rc;
  }
  if (!tuned && m0->force_mode < 0) {
    if (m0->autotune && lookup_tuned(sh, m0, plan)) {
      tuned = true;
    } else {
      int rc = heuristic_plan(sh, m0, plan);
      if (rc) return rc;
    }
  }
  return TM_OK;
}

// Runs local epochs [e0, e1) of every job in one launch (units of all jobs
// share the grid).  Permutations are built per job for those epochs.
static int run_epochs(std::vector<TrainJob> &jobs, uint32_t e0, uint32_t e1, tm_machine *owner) {
  tm_machine *m0 = owner;
  cudaStream_t st = m0->st;
  // distinct (seed, n) -> permutation block
  std::map<std::pair<uint64_t, uint64_t>, uint64_t> pidx;
  uint64_t pwords = 0;
  std::vector<uint64_t> joff(jobs.size());
  for (size_t i = 0; i < jobs.size(); i++) {
    auto key = std::make_pair(jobs[i].seed, (uint64_t)jobs[i].a->samples);
    auto it = pidx.find(key);
    if (it == pidx.end()) {
      pidx[key] = pwords;
      joff[i] = pwords;
      pwords += (uint64_t)(e1 - e0) * jobs[i].a->samples;
    } else {
      joff[i] = it->second;
    }
  }
  CK(m0->perm.ensure(std::max<uint64_t>(pwords, 4) * 4));
  uint32_t maxn = 0;
  for (auto &j : jobs) maxn = std::max<uint32_t>(maxn, (uint32_t)j.a->samples);
  const size_t psb = perm_scratch_bytes(std::max<uint32_t>(maxn, 1));
  CK(m0->perm_scratch.ensure(psb));
  for (auto &kv : pidx) {
    const uint64_t seed = kv.first.first, n = kv.first.second;
    for (uint32_t e = e0; e < e1; e++) {
      // the draw-contract epoch index is local epoch e (epoch_base 0)
      CK(launch_perm(seed, e, (uint32_t)n, m0->perm.as<uint32_t>() + kv.second + (e - e0) * n,
                     m0->perm_scratch.p, m0->perm_scratch.cap, st));
      note_launch(m0, 1 + kSortKernels);
    }
  }
  std::vector<TrainDev> td;
  std::vector<WorkItem> work;
  TrainShape sh{};
  build_tables(jobs, e0, e1, m0, joff, td, work, sh);
  if (work.empty()) return TM_OK;
  TrainPlan plan;
  bool tuned = false;
  int prc = choose_plan(jobs, td, work, sh, e0, m0, plan, tuned);
  if (prc) return prc;
  m0->last_mode = plan.mode;
  m0->stats.train_mode = plan.mode;
  m0->stats.train_autotuned = tuned ? 1 : 0;
  m0->stats.train_cpw = plan.cpw;
  m0->stats.train_resident = resident_units(plan);
  float ms = 0;
  uint32_t herr = 0;
  int rc = launch_plan(plan, sh, td, work, e0, e1, m0, m0->timing ? &ms : nullptr, &herr);
  if (rc) return rc;
  m0->stats.train_launches++;
  for (auto &J : jobs)
    m0->stats.train_unit_steps += (uint64_t)(J.a->class_end ? std::min(J.a->class_end, J.m->classes) -
                                                                  J.a->class_begin
                                                            : J.m->classes) *
                                  J.m->clause_chunks * J.a->samples *
                                  (std::min<uint32_t>(J.a->iterations, e1) > e0
                                       ? std::min<uint32_t>(J.a->iterations, e1) - e0 : 0);
  if (m0->timing) m0->stats.train_kernel_ms += ms;
  if (herr) return fail(TM_ERR_DEVICE, "train: a sample copy did not complete (status %u)", herr);
  return TM_OK;
}

static int prepare_job(TrainJob &J, DevBuf &xbuf, DevBuf &lbuf, DevBuf &cbuf, DevBuf &clsbuf) {
  tm_machine *m = J.m;
  const tm_train_args *a = J.a;
  const uint64_t n = a->samples;
  J.seed = a->has_seed ? a->seed : m->seed;
  int rc = stage_rows(m, xbuf, a->problems, a->dim_offsets, n, a->on_device != 0, J.cls);
  if (rc) return rc;
  J.d_x = xbuf.as<uint32_t>();
  CK(clsbuf.ensure(std::max<size_t>(m->classes, 1) * sizeof(ClassDev)));
  J.d_cls = clsbuf.as<ClassDev>();
  rc = upload_cls(m, J.d_cls, J.cls);
  if (rc) return rc;
  if (m->type == TM_CLASSIFIER) {
    const uint64_t lab32 = (std::max<uint64_t>(n, 1) * 4 + 255) & ~255ull;
    CK(lbuf.ensure(lab32 + std::max<uint64_t>(n, 1) * 8));
    const int64_t *src = a->solutions;
    int64_t *stage = (int64_t *)((uint8_t *)lbuf.p + lab32);
    if (!a->on_device) {
      CK(cudaMemcpyAsync(stage, src, n * 8, cudaMemcpyHostToDevice, m->st));
      src = stage;
    }
    CK(launch_labels(src, lbuf.as<int32_t>(), n, m->st));
    note_launch(m, 1);
    J.d_labels = lbuf.as<int32_t>();
  } else {
    const uint64_t cb = n * m->class_chunks;
    if (a->on_device) {
      J.d_codes = (uint8_t *)a->codes;
    } else {
      CK(cbuf.ensure(std::max<uint64_t>(cb, 16)));
      CK(cudaMemcpyAsync(cbuf.p, a->codes, cb, cudaMemcpyHostToDevice, m->st));
      J.d_codes = cbuf.as<uint8_t>();
    }
  }
  return TM_OK;
}

static int finish_train(tm_machine *m) {
  invalidate_derived(m);
  m->trained = true;
  if (!m->reusable) {
    // capi.c:1187-1188 / :718-723: a non-reusable machine drops its state
    CK(cudaStreamSynchronize(m->st));
    if (m->d_cnt) cudaFree(m->d_cnt);
    m->d_cnt = nullptr;
    m->has_state = false;
  }
  return TM_OK;
}

extern "C" int tm_train(tm_machine *m, const tm_train_args *a) {
  int rc = validate_train(m, a);
  if (rc) return rc;
  DevGuard g(m->device);
  std::vector<TrainJob> jobs(1);
  jobs[0].m = m;
  jobs[0].a = a;
  rc = prepare_job(jobs[0], m->tx, m->labels, m->codes, m->cls_job);
  if (rc) return rc;
  // capi.c:1136-1146: every train call starts from the initial state
  cudaError_t e = launch_setup(m->d_act, m->d_cnt, m->d_cls, m->classes, m->clauses, m->B,
                               m->act_words, m->st);
  if (e != cudaSuccess) return fail(TM_ERR_CUDA, "setup: %s", cudaGetErrorString(e));
  note_launch(m, 1);
  const uint32_t E = a->iterations;
  if (!a->each) {
    // all epochs resident in one launch, in groups that bound the
    // permutation buffer
    const uint64_t n = std::max<uint64_t>(a->samples, 1);
    const uint32_t group = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(E, (256ull << 20) / (4 * n)));
    for (uint32_t e0 = 0; e0 < E; e0 += group) {
      rc = run_epochs(jobs, e0, std::min(E, e0 + group), m);
      if (rc) return rc;
    }
  } else {
    for (uint32_t e0 = 0; e0 < E; e0++) {
      rc = run_epochs(jobs, e0, e0 + 1, m);
      if (rc) return rc;
      invalidate_derived(m);
      // capi.c:1168-1182: `each(epoch)`; false (non-zero here) stops
      if (a->each(a->each_user, e0 + 1) != 0) break;
    }
  }
  return finish_train(m);
}

static int train_batch_impl(tm_machine *const *ms, const tm_train_args *args, uint32_t count,
                            tm_batch_epoch_cb each, void *user);

extern "C" int tm_train_batch(tm_machine *const *ms, const tm_train_args *args, uint32_t count) {
  return train_batch_impl(ms, args, count, nullptr, nullptr);
}

extern "C" int tm_train_batch_each(tm_machine *const *ms, const tm_train_args *args, uint32_t count,
                                   tm_batch_epoch_cb each, void *user) {
  if (!each) return fail(TM_ERR_ARG, "train_batch_each: callback missing");
  return train_batch_impl(ms, args, count, each, user);
}

// Validates a batch, stages every job's inputs (identical inputs once) and
// resets every machine's automata (capi.c:1136-1146).
static int stage_batch(tm_machine *const *ms, const tm_train_args *args, uint32_t count,
                       std::vector<TrainJob> &jobs) {
  if (!ms || !args) return fail(TM_ERR_ARG, "null argument");
  tm_machine *m0 = ms[0];
  for (uint32_t i = 0; i < count; i++) {
    int rc = validate_train(ms[i], &args[i]);
    if (rc) return rc;
    if (ms[i]->device != m0->device) return fail(TM_ERR_ARG, "train_batch: machines on different devices");
    if (args[i].each) return fail(TM_ERR_ARG, "train_batch: per-epoch callbacks are not supported");
    for (uint32_t k = 0; k < i; k++)
      if (ms[k] == ms[i]) return fail(TM_ERR_ARG, "train_batch: machine listed twice");
  }
  jobs.assign(count, TrainJob{});
  // identical inputs (same pointers, layout and size) are staged once
  std::vector<int> same_x(count, -1);
  for (uint32_t i = 0; i < count; i++) {
    jobs[i].m = ms[i];
    jobs[i].a = &args[i];
    for (uint32_t k = 0; k < i; k++) {
      const tm_train_args &A = args[k], &Bq = args[i];
      if (A.problems == Bq.problems && A.samples == Bq.samples &&
          A.dim_offsets == Bq.dim_offsets && A.on_device == Bq.on_device &&
          !ms[k]->individualized && !ms[i]->individualized &&
          ms[k]->input_chunks == ms[i]->input_chunks && ms[k]->type == ms[i]->type &&
          A.solutions == Bq.solutions && A.codes == Bq.codes &&
          ms[k]->class_chunks == ms[i]->class_chunks) {
        same_x[i] = (int)k;
        break;
      }
    }
  }
  for (uint32_t i = 0; i < count; i++) {
    tm_machine *m = ms[i];
    if (m->st != m0->st) CK(cudaStreamSynchronize(m->st));
    TrainJob &J = jobs[i];
    if (same_x[i] >= 0) {
      const TrainJob &S = jobs[same_x[i]];
      J.seed = args[i].has_seed ? args[i].seed : m->seed;
      J.cls = m->cls;  // x offsets 0 (dense)
      J.d_x = S.d_x;
      J.d_labels = S.d_labels;
      J.d_codes = S.d_codes;
      CK(m->cls_job.ensure(std::max<size_t>(m->classes, 1) * sizeof(ClassDev)));
      J.d_cls = m->cls_job.as<ClassDev>();
      CK(cudaMemcpyAsync(J.d_cls, J.cls.data(), m->classes * sizeof(ClassDev),
                         cudaMemcpyHostToDevice, m0->st));
    } else {
      // stage on machine i's buffers, ordered on the owner stream
      cudaStream_t keep = m->st;
      m->st = m0->st;
      int rc = prepare_job(J, m->tx, m->labels, m->codes, m->cls_job);
      m->st = keep;
      if (rc) return rc;
    }
    cudaError_t e = launch_setup(m->d_act, m->d_cnt, m->d_cls, m->classes, m->clauses, m->B,
                                 m->act_words, m0->st);
    if (e != cudaSuccess) return fail(TM_ERR_CUDA, "setup: %s", cudaGetErrorString(e));
    note_launch(m0, 1);
  }
  return TM_OK;
}

static int train_batch_impl(tm_machine *const *ms, const tm_train_args *args, uint32_t count,
                            tm_batch_epoch_cb each, void *user) {
  if (!ms || !args) return fail(TM_ERR_ARG, "null argument");
  if (count == 0) return TM_OK;
  if (!ms[0]) return fail(TM_ERR_ARG, "null machine");
  tm_machine *m0 = ms[0];
  DevGuard g(m0->device);
  std::vector<TrainJob> jobs;
  int src = stage_batch(ms, args, count, jobs);
  if (src) return src;
  uint32_t E = 0;
  uint64_t maxn = 1;
  for (uint32_t i = 0; i < count; i++) {
    E = std::max(E, args[i].iterations);
    maxn = std::max<uint64_t>(maxn, args[i].samples);
  }
  if (!each) {
    const uint32_t group = (uint32_t)std::max<uint64_t>(
        1, std::min<uint64_t>(E, (512ull << 20) / (4 * maxn * std::max<uint32_t>(count, 1))));
    for (uint32_t e0 = 0; e0 < E; e0 += group) {
      int rc = run_epochs(jobs, e0, std::min(E, e0 + group), m0);
      if (rc) return rc;
    }
  } else {
    // one epoch per launch; stopped machines leave the launch
    std::vector<int32_t> stop(count, 0);
    for (uint32_t e0 = 0; e0 < E; e0++) {
      std::vector<TrainJob> live;
      for (uint32_t i = 0; i < count; i++)
        if (!stop[i] && e0 < args[i].iterations) live.push_back(jobs[i]);
      if (live.empty()) break;
      int rc = run_epochs(live, e0, e0 + 1, m0);
      if (rc) return rc;
      for (uint32_t i = 0; i < count; i++) invalidate_derived(ms[i]);
      std::vector<int32_t> req(count, 0);
      const int all = each(user, e0 + 1, req.data(), count);
      for (uint32_t i = 0; i < count; i++)
        if (req[i] || e0 + 1 >= args[i].iterations) stop[i] = 1;
      if (all) break;
    }
  }
  for (uint32_t i = 0; i < count; i++) {
    int rc = finish_train(ms[i]);
    if (rc) return rc;
  }
  return TM_OK;
}

// ---------------------------------------------------------------------------
// Device-resident search round: the trials of one round of the reference's
// search (optimize.lua:424-471), each with train_tm's per-epoch logic
// (optimize.lua:586-653), for all machines at once.  One epoch is one CUDA
// graph -- the epoch orders, the fused train kernel over every live
// machine's units, literal counts, predict of the holdout for every machine
// (k_predict_multi), the scores and early-stop decisions
// (k_search_score), the checkpoint copies, the epoch counter and a copy of
// the per-machine states to pinned host memory -- replayed once per epoch
// with one host synchronisation.  Every kernel reads the machine's `live`
// flag, so stopped machines drop out of the replays without a new graph.
// ---------------------------------------------------------------------------
static int search_round(tm_machine *const *ms, const tm_train_args *args, uint32_t count,
                        const tm_search_args *sa) {
  tm_machine *m0 = ms[0];
  const int32_t type = m0->type;
  const uint64_t nt = sa->test_samples;
  if (nt == 0 || nt >= (1ull << 31)) return fail(TM_ERR_ARG, "search: test_samples out of range");
  if (!sa->test_problems && !sa->test_each)
    return fail(TM_ERR_ARG, "search: test problems missing");
  if (type == TM_CLASSIFIER) {
    if (sa->metric != TM_METRIC_F1 && sa->metric != TM_METRIC_ACCURACY)
      return fail(TM_ERR_ARG, "search: classifiers are scored by TM_METRIC_F1 or TM_METRIC_ACCURACY");
    if (!sa->test_solutions) return fail(TM_ERR_ARG, "search: test solutions missing");
  } else {
    if (sa->metric != TM_METRIC_HAMMING)
      return fail(TM_ERR_ARG, "search: encoders are scored by TM_METRIC_HAMMING");
    if (!sa->test_codes) return fail(TM_ERR_ARG, "search: test codes missing");
  }
  uint32_t E = 0, maxC = 1;
  for (uint32_t i = 0; i < count; i++) {
    tm_machine *m = ms[i];
    if (!m) return fail(TM_ERR_ARG, "null machine");
    if (m->type != type) return fail(TM_ERR_ARG, "search: classifiers and encoders mixed");
    if (type == TM_ENCODER && m->classes != m0->classes)
      return fail(TM_ERR_ARG, "search: encoders of different hidden sizes");
    if (m->classes > TM_SEARCH_MAX_CLASSES)
      return fail(TM_ERR_ARG, "search: more than %u classes", TM_SEARCH_MAX_CLASSES);
    if (m->individualized && !sa->test_dim_offsets)
      return fail(TM_ERR_ARG, "search: test dim_offsets missing");
    if (sa->test_each && !sa->test_each[i] && !sa->test_problems)
      return fail(TM_ERR_ARG, "search: test problems of machine %u missing", i);
    E = std::max(E, args[i].iterations);
    maxC = std::max(maxC, m->classes);
  }
  std::vector<TrainJob> jobs;
  int rc = stage_batch(ms, args, count, jobs);
  if (rc) return rc;
  cudaStream_t st = m0->st;
  const uint32_t Es = std::max<uint32_t>(E, 1);
  // ---- holdout: truth once, padded rows per machine ------------------------
  const uint64_t tb = type == TM_CLASSIFIER ? nt * 8 : nt * m0->class_chunks;
  const int64_t *d_lab = nullptr;
  const uint8_t *d_cod = nullptr;
  if (sa->on_device) {
    d_lab = sa->test_solutions;
    d_cod = sa->test_codes;
  } else {
    CK(m0->search_truth.ensure(tb));
    CK(cudaMemcpyAsync(m0->search_truth.p,
                       type == TM_CLASSIFIER ? (const void *)sa->test_solutions
                                             : (const void *)sa->test_codes,
                       tb, cudaMemcpyHostToDevice, st));
    if (type == TM_CLASSIFIER) d_lab = m0->search_truth.as<int64_t>();
    else d_cod = m0->search_truth.as<uint8_t>();
  }
  for (uint32_t i = 0; i < count; i++) {
    tm_machine *m = ms[i];
    std::vector<ClassDev> tcls;
    const uint8_t *tp = sa->test_each && sa->test_each[i] ? sa->test_each[i] : sa->test_problems;
    cudaStream_t keep = m->st;
    m->st = st;
    rc = stage_rows(m, m->x, tp, sa->test_dim_offsets, nt, sa->on_device != 0, tcls);
    if (!rc) rc = upload_cls(m, m->d_cls, tcls);
    m->st = keep;
    if (rc) return rc;
    CK(m->sums.ensure(nt * m->classes * 4));
    CK(cudaMemsetAsync(m->sums.p, 0, nt * m->classes * 4, st));
    if (sa->patience) CK(m->ckpt.ensure(std::max<uint64_t>(m->act_words, 4) * 4));
  }
  // ---- the holdout predict of large dense machines as the 8-bit GEMM ---------
  // Their holdout rows are expanded to bytes once; in every epoch the graph
  // expands the trained actions and runs the products and the vote epilogue
  // (gated by the machine's live flag, like the bitwise predict).  Each
  // product width is tried once here, outside the capture: a machine whose
  // shape the library cannot take keeps the bitwise predict.
  const int gkind = gemm_kind_of(m0->device);
  const size_t gws = 32u << 20;
  std::vector<char> use_gemm(count, 0);
  std::vector<uint64_t> gchunk(count, 0);
  std::vector<uint8_t *> gx8(count, nullptr);
  {
    uint64_t cmax = 0;
    for (uint32_t i = 0; i < count; i++) {
      tm_machine *m = ms[i];
      const ClassDev &c0 = m->cls[0];
      const uint64_t M = (uint64_t)m->classes * m->clauses;
      if (gkind <= 0 || m->individualized || nt <= TM_SMALL_N_MAX ||
          M * nt * c0.W < (1ull << 28))
        continue;
      uint64_t nc = ((512ull << 20) / (4 * M)) / 64 * 64;
      nc = std::max<uint64_t>(nc, 64);
      gchunk[i] = nc;
      cmax = std::max<uint64_t>(cmax, gemm_bucket(std::min<uint64_t>(nc, nt), nc) * M * 4);
      use_gemm[i] = 1;
    }
    uint64_t amax = 0;
    for (uint32_t i = 0; i < count; i++)
      if (use_gemm[i])
        amax = std::max<uint64_t>(amax, (uint64_t)ms[i]->classes * ms[i]->clauses *
                                            ms[i]->cls[0].W * 32);
    if (cmax) {
      CK(m0->gemm_c.ensure(cmax));
      CK(m0->gemm_ws.ensure(gws));
      CK(m0->search_act8.ensure(amax));
    }
    // one byte copy of the holdout per distinct row layout (the machines'
    // staged rows of one source, feature count and row width are the same)
    std::map<std::tuple<const void *, uint64_t, uint32_t, uint32_t>, size_t> x8_of;
    for (uint32_t i = 0; i < count; i++) {
      if (!use_gemm[i]) continue;
      tm_machine *m = ms[i];
      const ClassDev &c0 = m->cls[0];
      const uint64_t K = (uint64_t)c0.W * 32;
      const void *src = sa->test_each && sa->test_each[i] ? (const void *)sa->test_each[i]
                                                          : (const void *)sa->test_problems;
      const auto key = std::make_tuple(src, (uint64_t)m->features, c0.Wp, c0.W);
      if (x8_of.count(key)) continue;
      const size_t at = x8_of.size();
      x8_of[key] = at;
      if (m0->search_x8.size() <= at) m0->search_x8.resize(at + 1);
      // rows past nt: the last product's bucket reads them (its columns
      // there are not used); sized for the largest chunk of any machine
      uint64_t pad = 0;
      for (uint32_t j = 0; j < count; j++)
        if (use_gemm[j])
          pad = std::max<uint64_t>(pad, gemm_bucket(std::min<uint64_t>(gchunk[j], nt), gchunk[j]));
      CK(m0->search_x8[at].ensure((nt + pad) * K));
      CK(launch_expand_bits(m->x.as<uint32_t>(), nt, c0.Wp, c0.W, 0xFFFFFFFFu, gkind,
                            m0->search_x8[at].as<uint8_t>(), st));
    }
    for (uint32_t i = 0; i < count; i++) {
      if (!use_gemm[i]) continue;
      tm_machine *m = ms[i];
      const ClassDev &c0 = m->cls[0];
      const void *src = sa->test_each && sa->test_each[i] ? (const void *)sa->test_each[i]
                                                          : (const void *)sa->test_problems;
      gx8[i] = m0->search_x8[x8_of[std::make_tuple(src, (uint64_t)m->features, c0.Wp, c0.W)]]
                   .as<uint8_t>();
      const uint64_t M = (uint64_t)m->classes * m->clauses, K = (uint64_t)c0.W * 32;
      const uint64_t nc = gchunk[i];
      for (uint64_t s0 = 0; s0 < nt && use_gemm[i]; s0 += nc) {
        const uint64_t k = std::min<uint64_t>(nc, nt - s0);
        const int g = gemm_clause_products(m0->device, gkind, m0->search_act8.as<uint8_t>(),
                                           gx8[i] + s0 * K, m0->gemm_c.p, M, gemm_bucket(k, nc),
                                           K, m0->gemm_ws.p, gws, st);
        if (g < 0) use_gemm[i] = 0;
        else if (g > 0) return fail(TM_ERR_CUDA, "search: cuBLASLt matmul failed (status %d)", g);
      }
    }
    CK(cudaStreamSynchronize(st));
  }
  // ---- device tables ---------------------------------------------------------
  auto al = [](size_t v) { return (v + 255) & ~(size_t)255; };
  const size_t o_scores = al(count * sizeof(SearchState));
  const size_t o_pj = al(o_scores + (size_t)count * Es * 8);
  const size_t o_pjf = al(o_pj + count * sizeof(PredictJob));
  const size_t o_lj = al(o_pjf + count * sizeof(PredictJob));
  const size_t o_ljf = al(o_lj + count * sizeof(LitsJob));
  const size_t o_sj = al(o_ljf + count * sizeof(LitsJob));
  const size_t o_cj = al(o_sj + count * sizeof(ScoreJob));
  const size_t o_rj = al(o_cj + count * sizeof(CopyJob));
  const size_t o_ctr = al(o_rj + count * sizeof(CopyJob));
  CK(m0->search.ensure(o_ctr + 256));
  uint8_t *base = m0->search.as<uint8_t>();
  SearchState *d_state = (SearchState *)base;
  double *d_scores = (double *)(base + o_scores);
  // [0] epoch, [2] status bits of the train kernel, [4..5] its active steps
  uint32_t *d_epoch = (uint32_t *)(base + o_ctr), *d_err = d_epoch + 2;
  std::vector<SearchState> hs(count);
  std::vector<PredictJob> pj(count), pjf(count);
  std::vector<LitsJob> lj(count), ljf(count);
  std::vector<ScoreJob> sj(count);
  std::vector<CopyJob> cj(count), rj(count);
  uint32_t tiles = 0, tiles_f = 0;  // per-epoch predict (GEMM machines apart), final pass
  for (uint32_t i = 0; i < count; i++) {
    tm_machine *m = ms[i];
    SearchState &S = hs[i];
    S = SearchState{};
    S.live = args[i].iterations > 0 && args[i].samples > 0 ? 1u : 0u;
    S.patience = sa->patience;
    S.iterations = args[i].iterations;
    S.best = -INFINITY;
    S.last = -INFINITY;
    S.tolerance = sa->tolerance;
    PredictJob &P = pj[i];
    P = PredictJob{};
    P.act = m->d_act;
    P.lits = m->d_lits;
    P.cls = m->d_cls;
    P.x = m->x.as<uint32_t>();
    P.sums = m->sums.as<int32_t>();
    P.gate = &d_state[i].live;
    P.clauses = m->clauses;
    P.tol = m->tol;
    P.n = (uint32_t)nt;
    P.classes = m->classes;
    const uint32_t jt = predict_job_tiles((uint32_t)nt, m->classes, m->clauses, &P.stiles, &P.tpc);
    P.tile0 = tiles;
    if (!use_gemm[i]) tiles += jt;  // a GEMM machine's job has no tiles: never picked
    pjf[i] = P;
    pjf[i].tile0 = tiles_f;
    tiles_f += jt;
    pjf[i].gate = &d_state[i].has_ckpt;
    lj[i] = LitsJob{m->d_act, m->d_cls, m->d_lits, &d_state[i].live, m->classes, m->clauses};
    ljf[i] = lj[i];
    ljf[i].gate = &d_state[i].has_ckpt;
    sj[i] = ScoreJob{m->sums.as<int32_t>(), d_lab, d_cod, (uint32_t)nt, m->classes,
                     (uint32_t)type, (uint32_t)sa->metric};
    const uint64_t aw = (m->act_words + 3) & ~3ull;
    cj[i] = CopyJob{m->d_act, sa->patience ? m->ckpt.as<uint32_t>() : nullptr, aw,
                    sa->patience ? &d_state[i].ckpt_now : nullptr};
    rj[i] = CopyJob{sa->patience ? m->ckpt.as<uint32_t>() : nullptr, m->d_act, aw,
                    sa->patience ? &d_state[i].has_ckpt : nullptr};
  }
  CK(cudaMemcpyAsync(d_state, hs.data(), count * sizeof(SearchState), cudaMemcpyHostToDevice, st));
  CK(cudaMemsetAsync(d_scores, 0xFF, (size_t)count * Es * 8, st));  // NaN
  CK(cudaMemcpyAsync(base + o_pj, pj.data(), count * sizeof(PredictJob), cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(base + o_pjf, pjf.data(), count * sizeof(PredictJob), cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(base + o_lj, lj.data(), count * sizeof(LitsJob), cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(base + o_ljf, ljf.data(), count * sizeof(LitsJob), cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(base + o_sj, sj.data(), count * sizeof(ScoreJob), cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(base + o_cj, cj.data(), count * sizeof(CopyJob), cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(base + o_rj, rj.data(), count * sizeof(CopyJob), cudaMemcpyHostToDevice, st));
  CK(cudaMemsetAsync(d_epoch, 0, 32, st));
  // ---- one epoch's train launch ----------------------------------------------
  std::map<std::pair<uint64_t, uint64_t>, uint64_t> pidx;
  uint64_t pwords = 0;
  std::vector<uint64_t> joff(count);
  uint32_t maxn = 1;
  for (uint32_t i = 0; i < count; i++) {
    auto key = std::make_pair(jobs[i].seed, (uint64_t)args[i].samples);
    auto it = pidx.find(key);
    if (it == pidx.end()) {
      pidx[key] = pwords;
      joff[i] = pwords;
      pwords += args[i].samples;
    } else {
      joff[i] = it->second;
    }
    maxn = std::max<uint32_t>(maxn, (uint32_t)args[i].samples);
  }
  CK(m0->perm.ensure(std::max<uint64_t>(pwords, 4) * 4));
  CK(m0->perm_scratch.ensure(perm_scratch_bytes(maxn)));
  std::vector<TrainDev> td;
  std::vector<WorkItem> work;
  TrainShape sh{};
  build_tables(jobs, 0, 1, m0, joff, td, work, sh);
  for (uint32_t i = 0; i < count; i++) td[i].gate = &d_state[i].live;
  // epoch 0's orders: the tuner's trial launches read them (the graph
  // rebuilds them for every epoch from the device epoch counter)
  for (auto &kv : pidx)
    CK(launch_perm(kv.first.first, 0, (uint32_t)kv.first.second,
                   m0->perm.as<uint32_t>() + kv.second, m0->perm_scratch.p, m0->perm_scratch.cap,
                   st, d_epoch));
  // Units of rows of at most 32 words train in a launch of their own, next
  // to the others' (two kernels of one graph at once): a launch's shared
  // memory slices are sized by its widest row, so narrow units in the same
  // launch as wide ones would hold as few units per SM as the wide ones.
  std::vector<WorkItem> work_n;
  TrainShape sh_n = sh;
  {
    std::vector<WorkItem> wide;
    for (const WorkItem &wi : work)
      (jobs[wi.m].cls[wi.h].Wp <= 32 ? work_n : wide).push_back(wi);
    if (!work_n.empty() && !wide.empty()) {
      auto shape_of = [&](const std::vector<WorkItem> &w, TrainShape &out) {
        out = sh;
        out.Wpmax = 4;
        out.Bmin = 32;
        out.Bmax = 2;
        out.smax = 0;
        for (const WorkItem &wi : w) {
          const ClassDev &c = jobs[wi.m].cls[wi.h];
          const uint32_t B = jobs[wi.m].m->B;
          out.Wpmax = std::max(out.Wpmax, c.Wp);
          out.smax = std::max(out.smax, c.s_picks);
          out.Bmin = std::min(out.Bmin, B);
          out.Bmax = std::max(out.Bmax, B);
        }
        out.units = (uint32_t)w.size();
      };
      shape_of(work_n, sh_n);
      shape_of(wide, sh);
      work.swap(wide);
    } else {
      work_n.clear();
    }
  }
  TrainPlan plan, plan_n;
  bool tuned = false, tuned_n = false;
  if (!work.empty()) {
    // trial launches of the tuner also read the gates and the epoch counter
    CK(cudaStreamSynchronize(st));
    rc = choose_plan(jobs, td, work, sh, 0, m0, plan, tuned);
    if (rc) return rc;
    if (!work_n.empty()) {
      rc = choose_plan(jobs, td, work_n, sh_n, 0, m0, plan_n, tuned_n);
      if (rc) return rc;
      // planning sets each kernel's dynamic shared-memory limit; when both
      // launches use one kernel it must end at the wide rows' size
      TrainPlan again;
      if (!plan_mode(plan_n.mode, sh_n, again, plan_n.cpw) ||
          !plan_mode(plan.mode, sh, again, plan.cpw))
        return fail(TM_ERR_STATE, "search: a train variant no longer fits its launch");
    }
    m0->last_mode = plan.mode;
    m0->stats.train_mode = plan.mode;
    m0->stats.train_autotuned = tuned ? 1 : 0;
    m0->stats.train_cpw = plan.cpw;
    m0->stats.train_resident = resident_units(plan) + (work_n.empty() ? 0 : resident_units(plan_n));
  }
  const size_t tbytes = td.size() * sizeof(TrainDev);
  const size_t off_w = (tbytes + 255) & ~(size_t)255;
  const size_t off_wn = (off_w + work.size() * sizeof(WorkItem) + 255) & ~(size_t)255;
  const size_t off_c = (off_wn + work_n.size() * sizeof(WorkItem) + 255) & ~(size_t)255;
  CK(m0->tdev.ensure(off_c + 256));
  uint8_t *tbase = m0->tdev.as<uint8_t>();
  CK(cudaMemcpyAsync(tbase, td.data(), tbytes, cudaMemcpyHostToDevice, st));
  if (!work.empty())
    CK(cudaMemcpyAsync(tbase + off_w, work.data(), work.size() * sizeof(WorkItem),
                       cudaMemcpyHostToDevice, st));
  if (!work_n.empty())
    CK(cudaMemcpyAsync(tbase + off_wn, work_n.data(), work_n.size() * sizeof(WorkItem),
                       cudaMemcpyHostToDevice, st));
  uint32_t *counter = (uint32_t *)(tbase + off_c), *counter_n = counter + 1;
  TrainSmem lay = plan.lay;
  lay.wait_limit = m0->row_wait;
  TrainSmem lay_n = plan_n.lay;
  lay_n.wait_limit = m0->row_wait;
  // the second launch's stream and the events that fork it off and join it
  cudaStream_t st_n = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  if (!work_n.empty()) {
    if (cudaStreamCreateWithFlags(&st_n, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming) != cudaSuccess) {
      if (st_n) cudaStreamDestroy(st_n);
      if (ev_fork) cudaEventDestroy(ev_fork);
      if (ev_join) cudaEventDestroy(ev_join);
      return fail(TM_ERR_CUDA, "search: stream creation failed");
    }
  }
  // one train launch of a plan over a work list
  auto launch_group = [&](const TrainPlan &pl, const TrainShape &shp, const TrainSmem &ly,
                          const WorkItem *wk, uint32_t nw, uint32_t *ctr,
                          cudaStream_t s_) -> cudaError_t {
    if (pl.mode == TM_MODE_WARP)
      return launch_train_warp((const TrainDev *)tbase, wk, nw, ctr, 0, 1, shp.Wpmax, shp.Bmin,
                               shp.Bmax, shp.smax, warp_units_per_cta(pl.cpw), pl.grid, s_,
                               (unsigned long long *)(d_err + 2));
    if (pl.mode == TM_MODE_WPT)
      return launch_train_wpt(pl.cpw, (const TrainDev *)tbase, wk, nw, ctr, 0, 1, shp.Wpmax,
                              shp.smax, m0->row_wait, pl.grid, d_err, s_);
    return launch_train((const TrainDev *)tbase, wk, nw, ctr, 0, 1, ly, pl.mode, shp.Bmin,
                        shp.Bmax, pl.cpw, pl.grid, d_err, s_);
  };
  // ---- pinned mirror of the states, events around the train kernel -----------
  SearchState *h_state = nullptr;
  CK(cudaHostAlloc((void **)&h_state, count * sizeof(SearchState) + 64, cudaHostAllocDefault));
  uint32_t *h_err = (uint32_t *)(h_state + count);
  const bool timing = m0->timing && m0->ev0 && m0->ev1;
  cudaEvent_t tk0 = nullptr, tk1 = nullptr;
  if (timing && (cudaEventCreate(&tk0) != cudaSuccess || cudaEventCreate(&tk1) != cudaSuccess)) {
    cudaFreeHost(h_state);
    if (st_n) cudaStreamDestroy(st_n);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    return fail(TM_ERR_CUDA, "search: event creation failed");
  }
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  auto drop = [&]() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
    if (tk0) cudaEventDestroy(tk0);
    if (tk1) cudaEventDestroy(tk1);
    tk0 = tk1 = nullptr;
    if (h_state) cudaFreeHost(h_state);
    h_state = nullptr;
    if (st_n) cudaStreamDestroy(st_n);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    st_n = nullptr;
    ev_fork = ev_join = nullptr;
  };
  // ---- capture one epoch ------------------------------------------------------
  uint64_t launches = 0;
  cudaError_t ce = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
  if (ce == cudaSuccess) {
    for (auto &kv : pidx) {
      if (ce != cudaSuccess) break;
      ce = launch_perm(kv.first.first, 0, (uint32_t)kv.first.second,
                       m0->perm.as<uint32_t>() + kv.second, m0->perm_scratch.p,
                       m0->perm_scratch.cap, st, d_epoch);
      launches += 1 + kSortKernels;
    }
    if (ce == cudaSuccess) ce = cudaMemsetAsync(counter, 0, 8, st);  // both work counters
    // external event records: real events inside the graph, so that the
    // train kernels' time can be read after each replay
    if (ce == cudaSuccess && timing) ce = cudaEventRecordWithFlags(tk0, st, cudaEventRecordExternal);
    if (ce == cudaSuccess && !work_n.empty()) {
      // the narrow rows' launch on a second stream of the capture
      ce = cudaEventRecord(ev_fork, st);
      if (ce == cudaSuccess) ce = cudaStreamWaitEvent(st_n, ev_fork, 0);
      if (ce == cudaSuccess)
        ce = launch_group(plan_n, sh_n, lay_n, (const WorkItem *)(tbase + off_wn),
                          (uint32_t)work_n.size(), counter_n, st_n);
      if (ce == cudaSuccess) ce = cudaEventRecord(ev_join, st_n);
      launches++;
    }
    if (ce == cudaSuccess && !work.empty()) {
      ce = launch_group(plan, sh, lay, (const WorkItem *)(tbase + off_w), (uint32_t)work.size(),
                        counter, st);
      launches++;
    }
    if (ce == cudaSuccess && !work_n.empty()) ce = cudaStreamWaitEvent(st, ev_join, 0);
    if (ce == cudaSuccess && timing) ce = cudaEventRecordWithFlags(tk1, st, cudaEventRecordExternal);
    if (ce == cudaSuccess)
      ce = launch_lits_multi((const LitsJob *)(base + o_lj), count, maxC, st);
    if (ce == cudaSuccess && tiles)
      ce = launch_predict_multi((const PredictJob *)(base + o_pj), count, tiles, st);
    for (uint32_t i = 0; i < count && ce == cudaSuccess; i++) {
      if (!use_gemm[i]) continue;
      tm_machine *m = ms[i];
      const ClassDev &c0 = m->cls[0];
      const uint64_t M = (uint64_t)m->classes * m->clauses, K = (uint64_t)c0.W * 32;
      const uint64_t nc = gchunk[i];
      ce = launch_expand_bits(m->d_act + c0.act_off, M, c0.Wp, c0.W, c0.emask, gkind,
                              m0->search_act8.as<uint8_t>(), st);
      launches++;
      for (uint64_t s0 = 0; s0 < nt && ce == cudaSuccess; s0 += nc) {
        const uint64_t k = std::min<uint64_t>(nc, nt - s0);
        const int g = gemm_clause_products(m0->device, gkind, m0->search_act8.as<uint8_t>(),
                                           gx8[i] + s0 * K, m0->gemm_c.p, M,
                                           gemm_bucket(k, nc), K, m0->gemm_ws.p, gws, st);
        if (g != 0) {
          ce = cudaErrorUnknown;
          break;
        }
        ce = launch_gemm_votes(m0->gemm_c.p, gkind, m->d_lits, m->classes, m->clauses, m->tol,
                               (uint32_t)k, m->sums.as<int32_t>() + s0 * m->classes, st,
                               &d_state[i].live);
        launches++;  // the epilogue (the GEMM is the library's)
      }
    }
    if (ce == cudaSuccess)
      ce = launch_search_score((const ScoreJob *)(base + o_sj), d_state, d_scores, Es, count,
                               maxC, 0, st);
    if (ce == cudaSuccess && sa->patience)
      ce = launch_copy_multi((const CopyJob *)(base + o_cj), count, st);
    if (ce == cudaSuccess) ce = launch_tick(d_epoch, st);
    if (ce == cudaSuccess) ce = launch_tick_machines((TrainDev *)tbase, count, st);
    if (ce == cudaSuccess)
      ce = cudaMemcpyAsync(h_state, d_state, count * sizeof(SearchState), cudaMemcpyDeviceToHost,
                           st);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(h_err, d_err, 4, cudaMemcpyDeviceToHost, st);
    launches += 5 + (sa->patience ? 1 : 0);
    cudaError_t ee = cudaStreamEndCapture(st, &graph);
    if (ce == cudaSuccess) ce = ee;
  }
  if (ce == cudaSuccess) ce = cudaGraphInstantiate(&exec, graph, 0);
  if (ce != cudaSuccess) {
    drop();
    return fail(TM_ERR_CUDA, "search: epoch graph: %s", cudaGetErrorString(ce));
  }
  // ---- epochs -----------------------------------------------------------------
  std::vector<double> last(count);
  std::vector<int32_t> live(count), stop(count);
  for (uint32_t e = 0; e < E; e++) {
    ce = timing ? cudaEventRecord(m0->ev0, st) : cudaSuccess;
    if (ce == cudaSuccess) ce = cudaGraphLaunch(exec, st);
    if (ce == cudaSuccess && timing) ce = cudaEventRecord(m0->ev1, st);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
    if (ce != cudaSuccess) {
      drop();
      return fail(TM_ERR_CUDA, "search: epoch %u: %s", e + 1, cudaGetErrorString(ce));
    }
    if (timing) {
      float ms = 0, tms = 0;
      if (cudaEventElapsedTime(&ms, m0->ev0, m0->ev1) == cudaSuccess) m0->stats.search_epoch_ms += ms;
      if (!work.empty() && cudaEventElapsedTime(&tms, tk0, tk1) == cudaSuccess) {
        m0->stats.search_train_ms += tms;
        m0->stats.train_kernel_ms += tms;
      }
      cudaGetLastError();  // a failed timing query leaves no error behind
      m0->stats.search_epochs++;
    }
    m0->stats.kernel_launches += launches;
    m0->stats.train_launches += work.empty() ? 0 : 1;
    if (*h_err) {
      const uint32_t he = *h_err;
      drop();
      return fail(TM_ERR_DEVICE, "train: a sample copy did not complete (status %u)", he);
    }
    bool any = false;
    for (uint32_t i = 0; i < count; i++) {
      live[i] = (int32_t)h_state[i].live;
      last[i] = h_state[i].epochs_run == e + 1 ? h_state[i].last : NAN;
      stop[i] = 0;
    }
    if (sa->each) {
      const int all = sa->each(sa->each_user, e + 1, last.data(), live.data(), stop.data(), count);
      for (uint32_t i = 0; i < count; i++) {
        if ((all || stop[i]) && live[i]) {
          static const uint32_t zero = 0;
          ce = cudaMemcpyAsync(&d_state[i].live, &zero, 4, cudaMemcpyHostToDevice, st);
          if (ce != cudaSuccess) {
            drop();
            return fail(TM_ERR_CUDA, "search: %s", cudaGetErrorString(ce));
          }
          live[i] = 0;
        }
      }
      ce = cudaStreamSynchronize(st);
      if (ce != cudaSuccess) {
        drop();
        return fail(TM_ERR_CUDA, "search: %s", cudaGetErrorString(ce));
      }
    }
    for (uint32_t i = 0; i < count; i++) any = any || live[i];
    if (!any) break;
  }
  drop();
  // ---- restore each machine's best checkpoint and score it ---------------------
  if (sa->patience) {
    CK(launch_copy_multi((const CopyJob *)(base + o_rj), count, st));
    CK(launch_lits_multi((const LitsJob *)(base + o_ljf), count, maxC, st));
    CK(launch_predict_multi((const PredictJob *)(base + o_pjf), count, tiles_f, st));
    CK(launch_search_score((const ScoreJob *)(base + o_sj), d_state, d_scores, Es, count, maxC, 1,
                           st));
    m0->stats.kernel_launches += 4;
  }
  std::vector<double> scores((size_t)count * Es);
  uint32_t hc[4] = {0, 0, 0, 0};
  CK(cudaMemcpyAsync(hc, d_err, 16, cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(hs.data(), d_state, count * sizeof(SearchState), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(scores.data(), d_scores, scores.size() * 8, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  m0->stats.train_active_pairs += (uint64_t)hc[2] | ((uint64_t)hc[3] << 32);
  for (uint32_t i = 0; i < count; i++) {
    if (sa->final_scores) sa->final_scores[i] = hs[i].last;
    if (sa->best_scores) sa->best_scores[i] = hs[i].best;
    if (sa->epochs_run) sa->epochs_run[i] = hs[i].epochs_run;
    if (sa->best_epochs) sa->best_epochs[i] = hs[i].best_epoch;
    if (sa->scores)
      for (uint32_t e = 0; e < E; e++) sa->scores[(size_t)i * E + e] = scores[(size_t)i * Es + e];
    tm_machine *m = ms[i];
    m0->stats.train_unit_steps +=
        (uint64_t)m->classes * m->clause_chunks * args[i].samples * hs[i].epochs_run;
    if (m->individualized) {
      rc = upload_cls(m, m->d_cls, m->cls);
      if (rc) return rc;
    }
  }
  CK(cudaStreamSynchronize(st));
  for (uint32_t i = 0; i < count; i++) {
    rc = finish_train(ms[i]);
    if (rc) return rc;
  }
  return TM_OK;
}

extern "C" int tm_train_batch_search(tm_machine *const *ms, const tm_train_args *args,
                                     uint32_t count, const tm_search_args *sa) {
  if (!ms || !args || !sa) return fail(TM_ERR_ARG, "null argument");
  if (count == 0) return TM_OK;
  if (!ms[0]) return fail(TM_ERR_ARG, "null machine");
  DevGuard g(ms[0]->device);
  return search_round(ms, args, count, sa);
}

// ---------------------------------------------------------------------------
// predict
// ---------------------------------------------------------------------------
static int ensure_lits(tm_machine *m) {
  if (m->lits_valid) return TM_OK;
  CK(launch_lits(m->d_act, m->d_cls, m->classes, m->clauses, m->d_lits, m->st));
  note_launch(m, 1);
  m->lits_valid = true;
  return TM_OK;
}

// Whether a predict of n samples goes through the GEMM: dense machines,
// past the small-batch kernel's sizes, and enough bitwise work (clauses x
// samples x row words >= 2^28, about 50 µs of the bitwise kernel) to pay
// for the byte expansions and the library call.
static bool gemm_wanted(tm_machine *m, uint64_t n) {
  if (m->individualized || n <= TM_SMALL_N_MAX) return false;
  const uint64_t M = (uint64_t)m->classes * m->clauses;
  if (M * n * m->cls[0].W < (1ull << 28)) return false;
  return gemm_kind_of(m->device) > 0;
}

// The action bytes of a dense machine in `kind`'s encoding (queued on the
// machine's stream).
static int ensure_act8(tm_machine *m, int kind) {
  if (m->act8_valid && m->act8_kind == kind) return TM_OK;
  const ClassDev &c0 = m->cls[0];
  const uint64_t M = (uint64_t)m->classes * m->clauses, K = (uint64_t)c0.W * 32;
  CK(m->act8.ensure(M * K));
  // dense machines: the classes' clause rows follow each other
  CK(launch_expand_bits(m->d_act + c0.act_off, M, c0.Wp, c0.W, c0.emask, kind,
                        m->act8.as<uint8_t>(), m->st));
  note_launch(m, 1);
  m->act8_valid = true;
  m->act8_kind = kind;
  return TM_OK;
}

// The vote sums of the n staged rows (m->x) through the GEMM.  Returns
// TM_OK, a TM_ERR_* code, or 1 when the library has no algorithm for this
// shape in either encoding (no vote sum was written; the caller uses the
// bitwise kernels).
static int predict_gemm(tm_machine *m, uint64_t n) {
  const ClassDev &c0 = m->cls[0];
  const uint64_t M = (uint64_t)m->classes * m->clauses, K = (uint64_t)c0.W * 32;
  int kind = gemm_kind_of(m->device);
  while (true) {
    if (kind <= 0) return 1;
    int rc = ensure_act8(m, kind);
    if (rc) return rc;
    // samples per chunk: products of at most 512 MB, in multiples of 64;
    // each product's width rounded up to a bucket (gemm_bucket), whose
    // columns past the chunk's samples are not read
    uint64_t nc = ((512ull << 20) / (4 * M)) / 64 * 64;
    nc = std::max<uint64_t>(nc, 64);
    const uint64_t cap = gemm_bucket(std::min<uint64_t>(nc, n), nc);
    const size_t ws_bytes = 32u << 20;
    CK(m->x8.ensure(cap * K));
    CK(m->gemm_c.ensure(cap * M * 4));
    CK(m->gemm_ws.ensure(ws_bytes));
    bool retry = false;
    for (uint64_t s0 = 0; s0 < n; s0 += nc) {
      const uint64_t k = std::min<uint64_t>(nc, n - s0);
      CK(launch_expand_bits(m->x.as<uint32_t>() + s0 * c0.Wp, k, c0.Wp, c0.W, 0xFFFFFFFFu, kind,
                            m->x8.as<uint8_t>(), m->st));
      const int g = gemm_clause_products(m->device, kind, m->act8.as<uint8_t>(),
                                         m->x8.as<uint8_t>(), m->gemm_c.p, M,
                                         gemm_bucket(k, nc), K, m->gemm_ws.p, ws_bytes, m->st);
      if (g < 0 && s0 == 0) {  // no algorithm: the other encoding, then the bitwise kernels
        kind = kind == TM_GEMM_INT8 ? TM_GEMM_FP8 : -1;
        retry = true;
        break;
      }
      if (g != 0) return fail(TM_ERR_CUDA, "predict: cuBLASLt matmul failed (status %d)", g);
      CK(launch_gemm_votes(m->gemm_c.p, kind, m->d_lits, m->classes, m->clauses, m->tol,
                           (uint32_t)k, m->sums.as<int32_t>() + s0 * m->classes, m->st));
      note_launch(m, 2);  // the expansion and the epilogue (the GEMM is the library's)
    }
    if (!retry) return TM_OK;
  }
}

static int predict_common(tm_machine *m, const uint8_t *problems, const int64_t *dim_offsets,
                          uint64_t n, int64_t *out_classes, uint8_t *out_codes,
                          int64_t *out_scores, bool on_device) {
  if (!m) return fail(TM_ERR_ARG, "null machine");
  if (n && !problems) return fail(TM_ERR_ARG, "predict: problems missing");
  if (m->individualized && n && !dim_offsets) return fail(TM_ERR_ARG, "predict: dim_offsets missing");
  if (n >= (1ull << 31)) return fail(TM_ERR_ARG, "predict: too many samples");
  if (n == 0) return TM_OK;
  DevGuard g(m->device);
  std::vector<ClassDev> cls;
  const uint64_t sb = n * m->classes * 4;
  CK(m->sums.ensure(sb));
  // the repack launch also clears the vote sums
  int rc = stage_rows(m, m->x, problems, dim_offsets, n, on_device, cls, m->sums.as<uint32_t>(),
                      sb / 4);
  if (rc) return rc;
  // a dense machine's rows start at offset 0 for every class: its resident
  // class table already describes them
  if (m->individualized) {
    rc = upload_cls(m, m->d_cls, cls);
    if (rc) return rc;
  }
  rc = ensure_lits(m);
  if (rc) return rc;
  if (m->timing) CK(cudaEventRecord(m->ev0, m->st));
  int gr = gemm_wanted(m, n) ? predict_gemm(m, n) : 1;
  if (gr < 0) return gr;
  m->stats.predict_gemm = gr == 0 ? m->act8_kind : 0;
  if (gr == 1) {
    CK(launch_predict(m->d_act, m->d_lits, m->d_cls, nullptr, m->classes, m->clauses, m->tol,
                      m->x.as<uint32_t>(), (uint32_t)n, m->sums.as<int32_t>(), m->st));
    note_launch(m, n <= TM_SMALL_N_MAX ? (n + 15) / 16 : 1);
  }
  if (m->timing) CK(cudaEventRecord(m->ev1, m->st));
  m->stats.predict_launches++;
  // outputs
  int64_t *dcls = nullptr, *dsc = nullptr;
  uint8_t *dcod = nullptr;
  const uint64_t clsb = n * 8, codb = n * m->class_chunks, scb = n * m->classes * 8;
  if (on_device) {
    dcls = out_classes;
    dcod = out_codes;
    dsc = out_scores;
  } else {
    CK(m->outc.ensure(clsb + codb + scb + 64));
    uint8_t *p = m->outc.as<uint8_t>();
    if (out_classes) dcls = (int64_t *)p;
    if (out_codes) dcod = p + clsb;
    if (out_scores) dsc = (int64_t *)(p + ((clsb + codb + 7) & ~7ull));
  }
  CK(launch_finalize(m->sums.as<int32_t>(), (uint32_t)n, m->classes, m->type, dcls, dcod, dsc,
                     m->st));
  note_launch(m, 1);
  // small results come back through the output half of the pinned buffer
  uint8_t *po = nullptr;
  const uint64_t outb = (out_classes ? clsb : 0) + (out_codes ? codb : 0) + (out_scores ? scb : 0);
  if (!on_device && outb <= TM_PIN_STAGE && pin_stage(m, 0)) po = m->pin + TM_PIN_STAGE;
  if (!on_device) {
    uint8_t *q = po;
    auto back = [&](void *dst, const void *src, uint64_t b) -> cudaError_t {
      if (!po) return cudaMemcpyAsync(dst, src, b, cudaMemcpyDeviceToHost, m->st);
      const cudaError_t e = cudaMemcpyAsync(q, src, b, cudaMemcpyDeviceToHost, m->st);
      q += b;
      return e;
    };
    if (out_classes) CK(back(out_classes, dcls, clsb));
    if (out_codes) CK(back(out_codes, dcod, codb));
    if (out_scores) CK(back(out_scores, dsc, scb));
  }
  CK(cudaStreamSynchronize(m->st));
  if (po) {
    const uint8_t *q = po;
    if (out_classes) memcpy(out_classes, q, clsb), q += clsb;
    if (out_codes) memcpy(out_codes, q, codb), q += codb;
    if (out_scores) memcpy(out_scores, q, scb);
  }
  if (m->timing) {
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, m->ev0, m->ev1));
    m->stats.predict_kernel_ms += ms;
  }
  // restore the resident class table (x offsets of dense machines are 0)
  if (m->individualized) {
    rc = upload_cls(m, m->d_cls, m->cls);
    if (rc) return rc;
  }
  return TM_OK;
}

int tmb_fail(int code, const char *msg) { return fail(code, "%s", msg); }

int tmb_machine_act8(tm_machine *m, MachineView *v) {
  v->act8 = nullptr;
  v->act8_kind = 0;
  if (!m || m->individualized) return TM_OK;
  const int kind = gemm_kind_of(m->device);
  if (kind <= 0) return TM_OK;
  DevGuard g(m->device);
  int rc = ensure_act8(m, kind);
  if (rc) return rc;
  CK(cudaStreamSynchronize(m->st));
  v->act8 = m->act8.as<uint8_t>();
  v->act8_kind = kind;
  return TM_OK;
}

int tmb_machine_view(tm_machine *m, MachineView *v, const char *who) {
  if (!m || !v) return fail(TM_ERR_ARG, "null argument");
  if (m->individualized)
    return fail(TM_ERR_ARG, "%s takes dense (non-individualized) machines",
                who ? who : "this call");
  DevGuard g(m->device);
  // A dense machine's resident class table never changes after it is laid
  // out, so nothing is uploaded here.  The literal counts are recomputed
  // only after the automata changed (train, restore, import), and only then
  // is the machine's stream drained so that callers on other streams see
  // them: a view of an unchanged machine costs no copy and no wait.
  const bool fresh = !m->lits_valid;
  int rc = ensure_lits(m);
  if (rc) return rc;
  if (fresh) CK(cudaStreamSynchronize(m->st));
  v->act = m->d_act;
  v->lits = m->d_lits;
  v->cls = m->d_cls;
  v->classes = m->classes;
  v->clauses = m->clauses;
  v->tol = m->tol;
  v->type = (uint32_t)m->type;
  v->input_chunks = m->input_chunks;
  v->Wp = m->cls[0].Wp;
  v->W = m->cls[0].W;
  v->act8 = nullptr;
  v->act8_kind = 0;
  v->class_chunks = m->class_chunks;
  v->device = m->device;
  v->st = m->st;
  return TM_OK;
}

extern "C" int tm_predict(tm_machine *m, const uint8_t *problems, const int64_t *dim_offsets,
                          uint64_t n, int64_t *out_classes, uint8_t *out_codes, int32_t on_device) {
  if (!m) return fail(TM_ERR_ARG, "null machine");
  if (m->type == TM_CLASSIFIER && !out_classes) return fail(TM_ERR_ARG, "predict: out_classes missing");
  if (m->type == TM_ENCODER && !out_codes) return fail(TM_ERR_ARG, "predict: out_codes missing");
  return predict_common(m, problems, dim_offsets, n, m->type == TM_CLASSIFIER ? out_classes : nullptr,
                        m->type == TM_ENCODER ? out_codes : nullptr, nullptr, on_device != 0);
}

extern "C" int tm_predict_scores(tm_machine *m, const uint8_t *problems, const int64_t *dim_offsets,
                                 uint64_t n, int64_t *out_scores, int32_t on_device) {
  if (!out_scores) return fail(TM_ERR_ARG, "predict_scores: out_scores missing");
  return predict_common(m, problems, dim_offsets, n, nullptr, nullptr, out_scores, on_device != 0);
}

// ---------------------------------------------------------------------------
// state in the reference byte layout
// ---------------------------------------------------------------------------
static int copy_rows(tm_machine *m, bool to_host, uint8_t *host, bool counts) {
  const uint32_t planes = counts ? m->B - 1 : 1;
  uint64_t ho = 0;
  for (uint32_t h = 0; h < m->classes; h++) {
    const ClassDev &c = m->cls[h];
    const uint64_t rows = (uint64_t)m->clauses * planes;
    uint32_t *dev = (counts ? m->d_cnt + c.cnt_off : m->d_act + c.act_off);
    const size_t width = m->n_chunks[h];
    if (to_host)
      CK(cudaMemcpy2DAsync(host + ho, width, dev, (size_t)c.Wp * 4, width, rows,
                           cudaMemcpyDeviceToHost, m->st));
    else
      CK(cudaMemcpy2DAsync(dev, (size_t)c.Wp * 4, host + ho, width, width, rows,
                           cudaMemcpyHostToDevice, m->st));
    ho += rows * width;
  }
  return TM_OK;
}

// For dense machines the per-class loop above covers classes * clauses rows
// in one copy: the class blocks are contiguous with the same stride.
static int copy_all(tm_machine *m, bool to_host, uint8_t *host, bool counts) {
  if (m->individualized) return copy_rows(m, to_host, host, counts);
  const uint32_t planes = counts ? m->B - 1 : 1;
  const ClassDev &c = m->cls[0];
  const uint64_t rows = (uint64_t)m->classes * m->clauses * planes;
  uint32_t *dev = counts ? m->d_cnt : m->d_act;
  const size_t width = m->input_chunks;
  if (to_host)
    CK(cudaMemcpy2DAsync(host, width, dev, (size_t)c.Wp * 4, width, rows, cudaMemcpyDeviceToHost,
                         m->st));
  else
    CK(cudaMemcpy2DAsync(dev, (size_t)c.Wp * 4, host, width, width, rows, cudaMemcpyHostToDevice,
                         m->st));
  return TM_OK;
}

extern "C" int tm_export_state(tm_machine *m, uint8_t *actions, uint8_t *state) {
  if (!m) return fail(TM_ERR_ARG, "null machine");
  DevGuard g(m->device);
  if (actions) {
    int rc = copy_all(m, true, actions, false);
    if (rc) return rc;
  }
  if (state) {
    if (!m->d_cnt) return fail(TM_ERR_STATE, "machine has no state");
    int rc = copy_all(m, true, state, true);
    if (rc) return rc;
  }
  CK(cudaStreamSynchronize(m->st));
  return TM_OK;
}

extern "C" int tm_import_state(tm_machine *m, const uint8_t *actions, const uint8_t *state) {
  if (!m) return fail(TM_ERR_ARG, "null machine");
  DevGuard g(m->device);
  if (actions) {
    int rc = copy_all(m, false, (uint8_t *)actions, false);
    if (rc) return rc;
    invalidate_derived(m);
  }
  if (state) {
    if (!m->d_cnt) return fail(TM_ERR_STATE, "machine has no state");
    int rc = copy_all(m, false, (uint8_t *)state, true);
    if (rc) return rc;
  }
  CK(cudaStreamSynchronize(m->st));
  return TM_OK;
}

// Classes [lo, hi) of the actions (counts = false) or count planes, in the
// reference byte layout, to or from `buf` (host, or device memory of the
// machine's device when on_device).  Class h's rows start where the classes
// before it end, so the range is one contiguous byte slice of the full
// layout; for a dense machine it is also one strided device block.
static int copy_classes(tm_machine *m, uint32_t lo, uint32_t hi, bool to_buf, uint8_t *buf,
                        bool counts, bool on_device) {
  const uint32_t planes = counts ? m->B - 1 : 1;
  const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice
                                        : (to_buf ? cudaMemcpyDeviceToHost : cudaMemcpyHostToDevice);
  uint64_t bo = 0;
  for (uint32_t h = lo; h < hi;) {
    // dense machines: every class from h on in one copy
    const uint32_t h1 = m->individualized ? h + 1 : hi;
    const ClassDev &c = m->cls[h];
    const uint64_t rows = (uint64_t)(h1 - h) * m->clauses * planes;
    uint32_t *dev = counts ? m->d_cnt + c.cnt_off : m->d_act + c.act_off;
    const size_t width = m->n_chunks[h];
    if (to_buf)
      CK(cudaMemcpy2DAsync(buf + bo, width, dev, (size_t)c.Wp * 4, width, rows, kind, m->st));
    else
      CK(cudaMemcpy2DAsync(dev, (size_t)c.Wp * 4, buf + bo, width, width, rows, kind, m->st));
    bo += rows * width;
    h = h1;
  }
  return TM_OK;
}

static int classes_io(tm_machine *m, uint32_t lo, uint32_t hi, bool to_buf, uint8_t *actions,
                      uint8_t *state, int32_t on_device) {
  if (!m) return fail(TM_ERR_ARG, "null machine");
  if (lo > hi || hi > m->classes)
    return fail(TM_ERR_ARG, "class range [%u, %u) outside [0, %u)", lo, hi, m->classes);
  if (state && !m->d_cnt) return fail(TM_ERR_STATE, "machine has no state");
  DevGuard g(m->device);
  if (actions) {
    int rc = copy_classes(m, lo, hi, to_buf, actions, false, on_device != 0);
    if (rc) return rc;
    if (!to_buf) invalidate_derived(m);
  }
  if (state) {
    int rc = copy_classes(m, lo, hi, to_buf, state, true, on_device != 0);
    if (rc) return rc;
  }
  CK(cudaStreamSynchronize(m->st));
  return TM_OK;
}

extern "C" int tm_export_classes(tm_machine *m, uint32_t class_begin, uint32_t class_end,
                                 uint8_t *actions, uint8_t *state, int32_t on_device) {
  return classes_io(m, class_begin, class_end, true, actions, state, on_device);
}

extern "C" int tm_import_classes(tm_machine *m, uint32_t class_begin, uint32_t class_end,
                                 const uint8_t *actions, const uint8_t *state, int32_t on_device) {
  return classes_io(m, class_begin, class_end, false, (uint8_t *)actions, (uint8_t *)state,
                    on_device);
}

// capi.c:1564-1576
extern "C" int tm_checkpoint(tm_machine *m, uint8_t *buf, uint64_t cap, uint64_t *len) {
  if (!m) return fail(TM_ERR_ARG, "null machine");
  if (len) *len = m->action_chunks;
  if (!buf) return TM_OK;
  if (cap < m->action_chunks) return fail(TM_ERR_ARG, "failed to resize checkpoint buffer");
  return tm_export_state(m, buf, nullptr);
}

// capi.c:1578-1588
extern "C" int tm_restore(tm_machine *m, const uint8_t *buf, uint64_t len) {
  if (!m || !buf) return fail(TM_ERR_ARG, "null argument");
  if (len != m->action_chunks)
    return fail(TM_ERR_ARG, "checkpoint size mismatch: expected %u bytes, got %llu",
                m->action_chunks, (unsigned long long)len);
  return tm_import_state(m, buf, nullptr);
}

// ---------------------------------------------------------------------------
// persist / load (capi.c:1509-1562, 1675-1772) -- byte-identical layout
// ---------------------------------------------------------------------------
static int serialize(tm_machine *m, std::vector<uint8_t> &out) {
  out.clear();
  auto put = [&](const void *p, size_t n) {
    const uint8_t *b = (const uint8_t *)p;
    out.insert(out.end(), b, b + n);
  };
  const int32_t type = m->type;
  put(&type, 4);
  put(&m->classes, 4); put(&m->features, 4); put(&m->clauses, 4); put(&m->tol, 4);
  put(&m->maxlit, 4); put(&m->target, 4); put(&m->B, 4); put(&m->ib, 4);
  put(&m->input_bits, 4); put(&m->input_chunks, 4); put(&m->clause_chunks, 4);
  put(&m->state_chunks, 4); put(&m->action_chunks, 4); put(&m->specificity, 8);
  put(&m->tail_mask, 1);
  const size_t at = out.size();
  out.resize(at + m->action_chunks);
  int rc = tm_export_state(m, out.data() + at, nullptr);
  if (rc) return rc;
  const uint8_t ind = m->individualized ? 1 : 0;
  put(&ind, 1);
  if (m->individualized) put(m->feat_sizes.data(), 8 * (size_t)m->classes);
  return TM_OK;
}

extern "C" int tm_persist(tm_machine *m, const char *path) {
  if (!m || !path) return fail(TM_ERR_ARG, "null argument");
  std::vector<uint8_t> d;
  int rc = serialize(m, d);
  if (rc) return rc;
  FILE *f = fopen(path, "wb");
  if (!f) return fail(TM_ERR_IO, "persist: cannot open %s", path);
  const size_t w = fwrite(d.data(), 1, d.size(), f);
  const int c = fclose(f);
  if (w != d.size() || c != 0) return fail(TM_ERR_IO, "persist: write failed");
  return TM_OK;
}

extern "C" int tm_persist_buf(tm_machine *m, uint8_t **data, uint64_t *len) {
  if (!m || !data || !len) return fail(TM_ERR_ARG, "null argument");
  std::vector<uint8_t> d;
  int rc = serialize(m, d);
  if (rc) return rc;
  *data = (uint8_t *)malloc(d.size() ? d.size() : 1);
  if (!*data) return fail(TM_ERR_OOM, "persist: out of memory");
  memcpy(*data, d.data(), d.size());
  *len = d.size();
  return TM_OK;
}

// Parses one record in the reference's persisted layout and builds the
// machine on `device`; with_state also allocates count planes (left for the
// caller to fill).
static int load_record(const uint8_t *data, uint64_t len, int32_t device, bool with_state,
                       tm_machine **out) {
  *out = nullptr;
  size_t o = 0;
  auto get = [&](void *p, size_t n) {
    if (o + n > len) return false;
    memcpy(p, data + o, n);
    o += n;
    return true;
  };
  int32_t type;
  tm_machine tmp;
  uint32_t f4[13];
  double spec;
  uint8_t tail, ind;
  if (!get(&type, 4)) return fail(TM_ERR_IO, "load: truncated model data");
  if (type != TM_CLASSIFIER && type != TM_ENCODER)
    return fail(TM_ERR_ARG, "unexpected tsetlin machine type in load");
  for (int i = 0; i < 13; i++)
    if (!get(&f4[i], 4)) return fail(TM_ERR_IO, "load: truncated model data");
  if (!get(&spec, 8) || !get(&tail, 1)) return fail(TM_ERR_IO, "load: truncated model data");
  const uint32_t ach = f4[12];
  if (o + ach > len) return fail(TM_ERR_IO, "load: truncated model data");
  const uint8_t *acts = data + o;
  o += ach;
  if (!get(&ind, 1)) return fail(TM_ERR_IO, "load: truncated model data");
  tm_machine *m = new tm_machine();
  m->type = type;
  m->classes = f4[0]; m->features = f4[1]; m->clauses = f4[2]; m->tol = f4[3];
  m->maxlit = f4[4]; m->target = f4[5]; m->B = f4[6]; m->ib = f4[7] ? f4[7] : 1;
  m->input_bits = f4[8]; m->input_chunks = f4[9]; m->clause_chunks = f4[10];
  m->specificity = spec;
  m->tail_mask = tail;
  m->class_chunks = (m->classes + 7) / 8;
  m->individualized = ind != 0;
  m->device = device;
  m->negative = m->classes ? 1.0 / m->classes : 0;
  if (m->B < 2 || m->B > 32 || !m->classes || m->clauses % 8 || m->clause_chunks * 8 != m->clauses) {
    delete m;
    return fail(TM_ERR_ARG, "load: inconsistent model header");
  }
  if (m->individualized) {
    m->feat_sizes.resize(m->classes);
    for (uint32_t h = 0; h < m->classes; h++)
      if (!get(&m->feat_sizes[h], 8)) {
        delete m;
        return fail(TM_ERR_IO, "load: truncated model data");
      }
  }
  layout_classes(m);
  if (m->action_chunks != ach || m->state_chunks != f4[11]) {
    delete m;
    return fail(TM_ERR_ARG, "load: inconsistent model sizes");
  }
  DevGuard g(m->device);
  if (cudaStreamCreateWithFlags(&m->st, cudaStreamNonBlocking) != cudaSuccess) {
    delete m;
    return fail(TM_ERR_CUDA, "stream creation failed");
  }
  // capi.c:1696: the state is not persisted; a loaded machine predicts only
  int rc = alloc_device(m, with_state);
  if (!rc) rc = tm_import_state(m, acts, nullptr);
  if (rc) {
    tm_destroy(m);
    return rc;
  }
  m->trained = true;
  *out = m;
  return TM_OK;
}

// ---------------------------------------------------------------------------
// versioned container (no counterpart in the reference, whose persisted
// record has no version and no state, capi.c:1509-1531, 1696):
//   0  "STMV"            magic (a reference record starts with type 0 or 1)
//   4  u32 version       1
//   8  u32 flags         1 = count planes present, 2 = reusable
//  12  u32 reserved      0
//  16  f64 negative      (not in the reference record)
//  24  u64 seed          default training seed
//  32  u64 record_len    then the reference record, byte for byte
//      [u64 state_len, state_len bytes]   count planes, reference layout
//      u64 FNV-1a 64 of every byte before it
// ---------------------------------------------------------------------------
static const uint8_t kMagic[4] = {'S', 'T', 'M', 'V'};
static const uint32_t kVersion = 1;

static uint64_t fnv1a64(const uint8_t *p, size_t n) {
  uint64_t h = 0xcbf29ce484222325ull;
  for (size_t i = 0; i < n; i++) {
    h ^= p[i];
    h *= 0x100000001b3ull;
  }
  return h;
}

static int save_container(tm_machine *m, uint32_t flags, std::vector<uint8_t> &out) {
  if (!m) return fail(TM_ERR_ARG, "null machine");
  if (flags & ~(uint32_t)TM_SAVE_STATE) return fail(TM_ERR_ARG, "save: unknown flags");
  const bool st = (flags & TM_SAVE_STATE) != 0;
  if (st && (!m->has_state || !m->d_cnt)) return fail(TM_ERR_STATE, "save: machine has no state");
  std::vector<uint8_t> rec;
  int rc = serialize(m, rec);
  if (rc) return rc;
  out.clear();
  auto put = [&](const void *p, size_t n) {
    const uint8_t *b = (const uint8_t *)p;
    out.insert(out.end(), b, b + n);
  };
  const uint32_t fl = (st ? 1u : 0u) | (m->reusable ? 2u : 0u), zero = 0;
  const uint64_t rl = rec.size();
  put(kMagic, 4); put(&kVersion, 4); put(&fl, 4); put(&zero, 4);
  put(&m->negative, 8); put(&m->seed, 8); put(&rl, 8);
  put(rec.data(), rec.size());
  if (st) {
    const uint64_t sl = m->state_chunks;
    put(&sl, 8);
    const size_t at = out.size();
    out.resize(at + sl);
    rc = tm_export_state(m, nullptr, out.data() + at);
    if (rc) return rc;
  }
  const uint64_t h = fnv1a64(out.data(), out.size());
  put(&h, 8);
  return TM_OK;
}

extern "C" int tm_save(tm_machine *m, const char *path, uint32_t flags) {
  if (!m || !path) return fail(TM_ERR_ARG, "null argument");
  std::vector<uint8_t> d;
  int rc = save_container(m, flags, d);
  if (rc) return rc;
  FILE *f = fopen(path, "wb");
  if (!f) return fail(TM_ERR_IO, "save: cannot open %s", path);
  const size_t w = fwrite(d.data(), 1, d.size(), f);
  const int c = fclose(f);
  if (w != d.size() || c != 0) return fail(TM_ERR_IO, "save: write failed");
  return TM_OK;
}

extern "C" int tm_save_buf(tm_machine *m, uint32_t flags, uint8_t **data, uint64_t *len) {
  if (!m || !data || !len) return fail(TM_ERR_ARG, "null argument");
  std::vector<uint8_t> d;
  int rc = save_container(m, flags, d);
  if (rc) return rc;
  *data = (uint8_t *)malloc(d.size());
  if (!*data) return fail(TM_ERR_OOM, "save: out of memory");
  memcpy(*data, d.data(), d.size());
  *len = d.size();
  return TM_OK;
}

static int load_container(const uint8_t *data, uint64_t len, int32_t device, tm_machine **out) {
  if (len < 48) return fail(TM_ERR_IO, "load: truncated model data");
  uint32_t version, flags, reserved;
  double negative;
  uint64_t seed, rl, h;
  memcpy(&version, data + 4, 4);
  memcpy(&flags, data + 8, 4);
  memcpy(&reserved, data + 12, 4);
  if (version == 0 || version > kVersion)
    return fail(TM_ERR_ARG, "load: unsupported format version %u (this library reads 1)", version);
  memcpy(&h, data + len - 8, 8);
  if (fnv1a64(data, len - 8) != h) return fail(TM_ERR_IO, "load: checksum mismatch (corrupt model data)");
  if ((flags & ~3u) || reserved) return fail(TM_ERR_ARG, "load: unknown flags");
  memcpy(&negative, data + 16, 8);
  memcpy(&seed, data + 24, 8);
  memcpy(&rl, data + 32, 8);
  const uint64_t body = len - 8;
  if (rl > body - 40) return fail(TM_ERR_IO, "load: truncated model data");
  const bool st = flags & 1u;
  uint64_t o = 40 + rl, sl = 0;
  if (st) {
    if (body - o < 8) return fail(TM_ERR_IO, "load: truncated model data");
    memcpy(&sl, data + o, 8);
    o += 8;
    if (sl > body - o) return fail(TM_ERR_IO, "load: truncated model data");
  }
  if (o + sl != body) return fail(TM_ERR_IO, "load: trailing bytes in model data");
  tm_machine *m = nullptr;
  int rc = load_record(data + 40, rl, device, st, &m);
  if (rc) return rc;
  m->negative = negative;
  m->seed = seed;
  m->reusable = (flags & 2u) != 0;
  if (st) {
    if (sl != m->state_chunks) {
      tm_destroy(m);
      return fail(TM_ERR_ARG, "load: state size mismatch: expected %u bytes, got %llu",
                  m->state_chunks, (unsigned long long)sl);
    }
    rc = tm_import_state(m, nullptr, data + o);
    if (rc) {
      tm_destroy(m);
      return rc;
    }
  }
  *out = m;
  return TM_OK;
}

extern "C" int tm_load(const uint8_t *data, uint64_t len, int32_t from_string, int32_t device,
                       tm_machine **out) {
  if (!data || !out) return fail(TM_ERR_ARG, "null argument");
  *out = nullptr;
  std::vector<uint8_t> file;
  if (!from_string) {
    FILE *f = fopen((const char *)data, "rb");
    if (!f) return fail(TM_ERR_IO, "load: cannot open %s", (const char *)data);
    uint8_t buf[1 << 16];
    size_t r;
    while ((r = fread(buf, 1, sizeof(buf), f)) > 0) file.insert(file.end(), buf, buf + r);
    fclose(f);
    data = file.data();
    len = file.size();
  }
  if (len >= 4 && memcmp(data, kMagic, 4) == 0) return load_container(data, len, device, out);
  return load_record(data, len, device, false, out);
}

// ---------------------------------------------------------------------------
// reconfigure (capi.c:1590-1673) and restrict (capi.c:752-901)
// ---------------------------------------------------------------------------
extern "C" int tm_reconfigure(tm_machine *m, const tm_reconfig *r) {
  if (!m || !r) return fail(TM_ERR_ARG, "null argument");
  if (!m->reusable) return fail(TM_ERR_STATE, "reconfigure requires reusable=true at creation time");
  if (!r->clauses || !r->clause_tolerance || !r->clause_maximum || !(r->specificity > 0))
    return fail(TM_ERR_ARG, "reconfigure: clauses, clause_tolerance, clause_maximum and specificity are required");
  DevGuard g(m->device);
  cudaStreamSynchronize(m->st);
  tm_machine saved = *m;  // only the scalar fields are restored on failure
  m->clauses = (r->clauses + 7) / 8 * 8;
  m->clause_chunks = m->clauses / 8;
  m->tol = r->clause_tolerance;
  m->maxlit = r->clause_maximum;
  const int64_t ib = r->include_bits < 0 ? (int64_t)m->ib : r->include_bits;
  m->ib = ib ? (uint32_t)ib : 1;
  m->specificity = r->specificity;
  m->target = derive_target(m->clauses, m->tol, r->target);
  int rc = check_limits(m);
  if (rc) {
    m->clauses = saved.clauses; m->clause_chunks = saved.clause_chunks; m->tol = saved.tol;
    m->maxlit = saved.maxlit; m->ib = saved.ib; m->specificity = saved.specificity;
    m->target = saved.target;
    return rc;
  }
  layout_classes(m);
  rc = alloc_device(m, true);  // actions zero (capi.c:1625), fresh state
  if (rc) return rc;
  m->trained = false;
  CK(cudaStreamSynchronize(m->st));
  return TM_OK;
}

extern "C" int tm_restrict(tm_machine *m, const int64_t *dims, uint64_t n) {
  if (!m) return fail(TM_ERR_ARG, "null machine");
  if (!m->individualized) return fail(TM_ERR_STATE, "restrict only supported for individualized TMs");
  if (n == 0 || !dims) return fail(TM_ERR_ARG, "selected_dims cannot be empty");
  for (uint64_t i = 0; i < n; i++) {
    if (dims[i] < 0 || (uint64_t)dims[i] >= m->classes)
      return fail(TM_ERR_ARG, "selected_dims[%d] = %d out of range [0, %d)", (int)i, (int)dims[i],
                  (int)m->classes);
    for (uint64_t j = i + 1; j < n; j++)
      if (dims[i] == dims[j]) return fail(TM_ERR_ARG, "duplicate dimension %d in selected_dims", (int)dims[i]);
  }
  DevGuard g(m->device);
  cudaStreamSynchronize(m->st);
  const std::vector<ClassDev> old = m->cls;
  uint32_t *oact = m->d_act, *ocnt = m->d_cnt;
  m->d_act = nullptr;
  m->d_cnt = nullptr;
  const bool had_state = m->has_state && ocnt;
  std::vector<uint64_t> nf(n);
  for (uint64_t i = 0; i < n; i++) nf[i] = m->feat_sizes[dims[i]];
  m->feat_sizes = nf;
  m->classes = (uint32_t)n;
  m->class_chunks = (m->classes + 7) / 8;
  layout_classes(m);
  int rc = alloc_device(m, had_state);
  if (!rc) {
    for (uint64_t i = 0; i < n; i++) {
      const ClassDev &o = old[dims[i]], &c = m->cls[i];
      cudaError_t e = cudaMemcpyAsync(m->d_act + c.act_off, oact + o.act_off,
                                      (size_t)m->clauses * c.Wp * 4, cudaMemcpyDeviceToDevice, m->st);
      if (e == cudaSuccess && had_state)
        e = cudaMemcpyAsync(m->d_cnt + c.cnt_off, ocnt + o.cnt_off,
                            (size_t)m->clauses * (m->B - 1) * c.Wp * 4, cudaMemcpyDeviceToDevice,
                            m->st);
      if (e != cudaSuccess) {
        rc = fail(TM_ERR_CUDA, "restrict: %s", cudaGetErrorString(e));
        break;
      }
    }
  }
  cudaStreamSynchronize(m->st);
  if (oact) cudaFree(oact);
  if (ocnt) cudaFree(ocnt);
  return rc;
}
