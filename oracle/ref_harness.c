/*
 * Reference-code harness.  TEST INFRASTRUCTURE ONLY, built only where the
 * reference tree exists (oracle/Makefile, target `ref`), output in _ref/.
 *
 * It compiles the reference's own lib/santoku/tsetlin/capi.c (and through
 * it automata.h) from where they lie, against the shim headers in
 * ref_shim/, and drives the reference's static functions directly:
 *   tk_tsetlin_init_classifier / _ind      (capi.c:449-606)
 *   tk_automata_setup                      (automata.h:72-86)
 *   tk_tsetlin_calculate / _ind, tm_update / tm_update_ind, apply_feedback
 *                                          (capi.c:85-402)
 *   tk_tsetlin_init_shuffle                (capi.c:245-256)
 *   _tk_tsetlin_persist_classifier / _tk_tsetlin_load_classifier
 *                                          (capi.c:1509-1531, 1675-1737)
 * The loops around them restate the Lua-bound drivers (capi.c:1112-1482,
 * 903-1086) with the Lua calls removed.
 *
 * The reference's generator (tk_fast_seed / tk_fast_random / tk_fast_chance,
 * from the un-vendored santoku rock) is supplied here in two modes:
 *   REF_PHILOX     routes each call to the keyed Philox draw contract, using
 *                  the (sample, epoch, unit) context the driver loop sets
 *                  before every step, so that the reference's code consumes
 *                  exactly the draws the CUDA kernels consume;
 *   REF_REFSTRUCT  a per-thread multiplicative congruential generator seeded
 *                  by thread id (the same stand-in the C oracle uses).
 */
#include <santoku/lua/utils.h>

#include TM_REF_CAPI

#include <omp.h>

void tm_shim_abort(const char *f) { tm_shim_unreachable(f); }

#define REF_PHILOX 0
#define REF_REFSTRUCT 1

/* ---- Philox4x32-10 (Salmon et al., SC'11), same contract as the oracle -- */
static void hphilox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint64_t key,
                    uint32_t *out) {
  uint32_t k0 = (uint32_t)key, k1 = (uint32_t)(key >> 32);
  for (int r = 0; r < 10; r++) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
    uint32_t n1 = (uint32_t)p1;
    uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
    uint32_t n3 = (uint32_t)p0;
    c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

typedef struct {
  int mode;
  uint64_t seed;
  uint32_t s, e, g;
  int pos;            /* chunk_class == sample_class && target_vote */
  int neg_pending;    /* next chance() is the negative-sampling draw */
  uint64_t T2;        /* 2 * target */
  uint64_t input_bits;
  uint32_t d[8];      /* chance draws of this step */
  int chance_idx;
  uint32_t ib_clause, pick;
  uint64_t mcg;
} hctx_t;
static __thread hctx_t hctx;

static void tk_fast_seed(uint64_t s) {
  uint64_t z = (s ^ hctx.seed) + 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  hctx.mcg = z | 1;
}
static inline uint32_t h_mcg(void) {
  hctx.mcg *= 0xDA942042E4DD58B5ull;
  return (uint32_t)(hctx.mcg >> 32);
}
static uint64_t tk_fast_random(void) {
  if (hctx.mode == REF_REFSTRUCT) return h_mcg();
  /* Philox: only Type Ib picks call this (apply_feedback, capi.c:185) */
  uint32_t r = hctx.pick++;
  uint32_t o[4];
  hphilox(hctx.s, hctx.e, hctx.g, 0x01000000u | (hctx.ib_clause << 20) | (r >> 2), hctx.seed, o);
  return (uint64_t)(((uint64_t)o[r & 3] * hctx.input_bits) >> 32);
}
static bool tk_fast_chance(double p) {
  if (hctx.mode == REF_REFSTRUCT)
    return (double)h_mcg() * (1.0 / 4294967296.0) < p;
  if (hctx.neg_pending) {
    /* capi.c:215 / :1449: chance(1 - negative) */
    hctx.neg_pending = 0;
    uint32_t o[4];
    hphilox(hctx.s, hctx.e, hctx.g, 0, hctx.seed, o);
    double q = p * 4294967296.0;
    uint64_t thr = !(q > 0) ? 0 : (q >= 4294967296.0 ? 4294967296ull : (uint64_t)floor(q));
    return (uint64_t)o[0] < thr;
  }
  int k = hctx.chance_idx++;
  uint64_t a = (uint64_t)llround(p * (double)hctx.T2);   /* p = a / 2T exactly */
  uint64_t t = ((uint64_t)hctx.d[k] * hctx.T2) >> 32;
  bool r = t < a;
  if ((k & 1) == 0 && r) {        /* Type I draw: picks that follow are for this clause */
    hctx.ib_clause = hctx.pos ? (uint32_t)k : (uint32_t)k + 1;
    hctx.pick = 0;
  }
  return r;
}

static void step_ctx(uint32_t s, uint32_t e, uint32_t g, int pos, int neg, uint64_t T,
                     uint64_t input_bits) {
  hctx.s = s; hctx.e = e; hctx.g = g; hctx.pos = pos; hctx.neg_pending = neg;
  hctx.T2 = 2 * T; hctx.input_bits = input_bits; hctx.chance_idx = 0;
  if (hctx.mode == REF_PHILOX) {
    hphilox(s, e, g, 1, hctx.seed, hctx.d);
    hphilox(s, e, g, 2, hctx.seed, hctx.d + 4);
  }
}

/* permutation contract (same as the oracle): sort by 64-bit Philox key */
typedef struct { uint64_t k; uint32_t i; } hkey;
static int hkey_cmp(const void *a, const void *b) {
  const hkey *x = a, *y = b;
  if (x->k != y->k) return x->k < y->k ? -1 : 1;
  return x->i < y->i ? -1 : (x->i > y->i);
}
static void h_perm(uint64_t seed, uint32_t e, uint64_t n, uint32_t *out) {
  hkey *k = malloc((n ? n : 1) * sizeof(hkey));
  for (uint64_t i = 0; i < n; i++) {
    uint32_t o[4];
    hphilox((uint32_t)i, e, 0, 0xFFFFFFFFu, seed, o);
    k[i].k = ((uint64_t)o[0] << 32) | o[1];
    k[i].i = (uint32_t)i;
  }
  qsort(k, n, sizeof(hkey), hkey_cmp);
  for (uint64_t i = 0; i < n; i++) out[i] = k[i].i;
  free(k);
}

/* ------------------------------------------------------------------------ */
void *ref_create(int type, uint32_t classes, uint32_t features, uint32_t clauses,
                 uint32_t tol, uint32_t maxl, uint32_t state_bits, uint32_t ib,
                 double target, double negative, double specificity, int reusable,
                 int individualized, const int64_t *feat_offsets) {
  tk_tsetlin_t *tm = calloc(1, sizeof(tk_tsetlin_t));
  tm->type = type ? TM_ENCODER : TM_CLASSIFIER;
  tm->has_state = true;
  if (individualized) {
    tk_ivec_t fo = { classes + 1, classes + 1, (int64_t *)feat_offsets };
    tk_tsetlin_init_classifier_ind(NULL, tm, classes, &fo, clauses, tol, maxl, state_bits, ib,
                                   target, negative, specificity);
  } else {
    tk_tsetlin_init_classifier(NULL, tm, classes, features, clauses, tol, maxl, state_bits, ib,
                               target, negative, specificity);
  }
  tm->reusable = reusable ? true : false;
  return tm;
}

void ref_destroy(void *p) {
  tk_tsetlin_t *tm = p;
  _tk_tsetlin_destroy(tm);
  free(tm);
}

void ref_info(void *p, uint64_t *o) {
  tk_tsetlin_t *tm = p;
  o[0] = tm->type; o[1] = tm->classes; o[2] = tm->features; o[3] = tm->clauses;
  o[4] = tm->clause_tolerance; o[5] = tm->clause_maximum; o[6] = tm->target;
  o[7] = tm->state_bits; o[8] = tm->include_bits; o[9] = tm->input_bits;
  o[10] = tm->input_chunks; o[11] = tm->clause_chunks; o[12] = tm->class_chunks;
  o[13] = tm->state_chunks; o[14] = tm->action_chunks; o[15] = tm->tail_mask;
  o[16] = tm->individualized; o[17] = tm->reusable; o[18] = tm->state != NULL;
}

double ref_negative(void *p) { return ((tk_tsetlin_t *)p)->negative; }

void ref_export(void *p, uint8_t *actions, uint8_t *state) {
  tk_tsetlin_t *tm = p;
  if (actions) memcpy(actions, tm->actions, tm->action_chunks);
  if (state && tm->state) memcpy(state, tm->state, tm->state_chunks);
}

void ref_import(void *p, const uint8_t *actions, const uint8_t *state) {
  tk_tsetlin_t *tm = p;
  if (actions) memcpy(tm->actions, actions, tm->action_chunks);
  if (state && tm->state) memcpy(tm->state, state, tm->state_chunks);
}

static void setup_all(tk_tsetlin_t *tm) {
  if (!tm->individualized) {
    for (unsigned int c = 0; c < tm->clause_chunks * tm->classes; c++)
      tk_automata_setup(&tm->automata, (uint64_t)c * 8, (uint64_t)c * 8 + 7);
  } else {
    for (unsigned int h = 0; h < tm->classes; h++)
      for (unsigned int c = 0; c < tm->clause_chunks; c++)
        tk_automata_setup(&tm->automata_arr[h], (uint64_t)c * 8, (uint64_t)c * 8 + 7);
  }
}

void ref_setup(void *p) { setup_all(p); }

int ref_train(void *p, const uint8_t *x, const int64_t *labels, const uint8_t *codes,
              const int64_t *dim_offsets, uint64_t n, uint32_t epochs, uint64_t seed,
              uint32_t epoch_base, int mode, int nthreads) {
  tk_tsetlin_t *tm = p;
  if (nthreads <= 0) nthreads = omp_get_max_threads();
  char *ps = (char *)x;
  unsigned int cc = tm->clause_chunks;
  unsigned int total = cc * tm->classes;
  if (mode == REF_PHILOX) {
    hctx.mode = REF_PHILOX;
    hctx.seed = seed;
    setup_all(tm);
    uint32_t *perm = malloc((n ? n : 1) * sizeof(uint32_t));
    for (uint32_t it = 0; it < epochs; it++) {
      uint32_t e = epoch_base + it;
      h_perm(seed, e, n, perm);
      unsigned int lit[8], vot[8];
      if (!tm->individualized) {
        for (unsigned int chunk = 0; chunk < total; chunk++) {
          unsigned int cls = chunk / cc;
          for (uint64_t i = 0; i < n; i++) {
            unsigned int s = perm[i];
            char *input = ps + (uint64_t)s * tm->input_chunks;
            if (tm->type == TM_CLASSIFIER) {
              unsigned int label = (unsigned int)labels[s];
              step_ctx(s, e, chunk, label == cls, label != cls, tm->target, tm->input_bits);
              uint8_t out = tk_tsetlin_calculate(tm, input, lit, vot, chunk);
              tm_update(tm, input, out, lit, vot, s, label, 1, cls, chunk, 0);
            } else {
              bool tv = (codes[(uint64_t)s * tm->class_chunks + cls / 8] & (1 << (cls % 8))) > 0;
              step_ctx(s, e, chunk, tv, 0, tm->target, tm->input_bits);
              uint8_t out = tk_tsetlin_calculate(tm, input, lit, vot, chunk);
              tm_update(tm, input, out, lit, vot, s, cls, tv, cls, chunk, 0);
            }
          }
        }
      } else {
        for (unsigned int h = 0; h < tm->classes; h++) {
          tk_automata_t *aut = &tm->automata_arr[h];
          uint64_t ich = tm->input_chunks_ind[h];
          for (unsigned int chunk = 0; chunk < cc; chunk++) {
            unsigned int g = h * cc + chunk;
            for (uint64_t i = 0; i < n; i++) {
              unsigned int s = perm[i];
              char *input = ps + (uint64_t)dim_offsets[h] + (uint64_t)s * ich;
              bool tv;
              if (tm->type == TM_CLASSIFIER) {
                unsigned int label = (unsigned int)labels[s];
                step_ctx(s, e, g, h == label, h != label, tm->target, 2 * tm->feat_sizes[h]);
                /* capi.c:1449-1450 */
                if (h != label && tk_fast_chance(1 - tm->negative)) continue;
                tv = h == label;
              } else {
                tv = (codes[(uint64_t)s * tm->class_chunks + h / 8] & (1 << (h % 8))) > 0;
                step_ctx(s, e, g, tv, 0, tm->target, 2 * tm->feat_sizes[h]);
              }
              uint8_t out = tk_tsetlin_calculate_ind(aut, input, lit, vot, chunk, ich,
                                                     tm->tail_masks_ind[h], tm->clause_tolerance);
              tm_update_ind(aut, input, out, lit, vot, tv, chunk, (long int)tm->target,
                            tm->type == TM_CLASSIFIER ? tm->negative : 0.0, tm->feat_sizes[h],
                            ich, tm->specificity, tm->clause_maximum);
            }
          }
        }
      }
    }
    free(perm);
    return 0;
  }
  /* REF_REFSTRUCT: capi.c:1134-1167 with the Lua callback removed */
  unsigned int **shuffles = malloc((size_t)nthreads * sizeof(unsigned int *));
  for (int t = 0; t < nthreads; t++) shuffles[t] = malloc((n ? n : 1) * sizeof(unsigned int));
  #pragma omp parallel num_threads(nthreads)
  {
    hctx.mode = REF_REFSTRUCT;
    hctx.seed = seed;
    tk_fast_seed((uint64_t)omp_get_thread_num());
  }
  setup_all(tm);
  for (uint32_t it = 0; it < epochs; it++) {
    #pragma omp parallel num_threads(nthreads)
    {
      int tid = omp_get_thread_num();
      unsigned int *shuffle = shuffles[tid];
      unsigned int lit[8], vot[8];
      tk_tsetlin_init_shuffle(shuffle, (unsigned int)n);
      if (!tm->individualized) {
        #pragma omp for schedule(static)
        for (unsigned int chunk = 0; chunk < total; chunk++) {
          unsigned int cls = chunk / cc;
          for (unsigned int i = 0; i < n; i++) {
            unsigned int s = shuffle[i];
            char *input = ps + (uint64_t)s * tm->input_chunks;
            uint8_t out = tk_tsetlin_calculate(tm, input, lit, vot, chunk);
            if (tm->type == TM_CLASSIFIER) {
              unsigned int label = (unsigned int)labels[s];
              tm_update(tm, input, out, lit, vot, s, label, 1, cls, chunk, (unsigned int)tid);
            } else {
              bool tv = (codes[(uint64_t)s * tm->class_chunks + cls / 8] & (1 << (cls % 8))) > 0;
              tm_update(tm, input, out, lit, vot, s, cls, tv, cls, chunk, (unsigned int)tid);
            }
          }
        }
      } else {
        #pragma omp for schedule(static)
        for (unsigned int h = 0; h < tm->classes; h++) {
          tk_automata_t *aut = &tm->automata_arr[h];
          uint64_t ich = tm->input_chunks_ind[h];
          for (unsigned int chunk = 0; chunk < cc; chunk++) {
            for (unsigned int i = 0; i < n; i++) {
              unsigned int s = shuffle[i];
              bool tv;
              if (tm->type == TM_CLASSIFIER) {
                unsigned int label = (unsigned int)labels[s];
                if (h != label && tk_fast_chance(1 - tm->negative)) continue;
                tv = h == label;
              } else {
                tv = (codes[(uint64_t)s * tm->class_chunks + h / 8] & (1 << (h % 8))) > 0;
              }
              char *input = ps + (uint64_t)dim_offsets[h] + (uint64_t)s * ich;
              uint8_t out = tk_tsetlin_calculate_ind(aut, input, lit, vot, chunk, ich,
                                                     tm->tail_masks_ind[h], tm->clause_tolerance);
              tm_update_ind(aut, input, out, lit, vot, tv, chunk, (long int)tm->target,
                            tm->type == TM_CLASSIFIER ? tm->negative : 0.0, tm->feat_sizes[h],
                            ich, tm->specificity, tm->clause_maximum);
            }
          }
        }
      }
    }
  }
  for (int t = 0; t < nthreads; t++) free(shuffles[t]);
  free(shuffles);
  return 0;
}

/* capi.c:903-1086 without the Lua result vectors */
int ref_predict(void *p, const uint8_t *x, const int64_t *dim_offsets, uint64_t n,
                int64_t *out_classes, uint8_t *out_codes, int64_t *out_scores, int nthreads) {
  tk_tsetlin_t *tm = p;
  if (nthreads <= 0) nthreads = omp_get_max_threads();
  unsigned int classes = tm->classes, cc = tm->clause_chunks;
  #pragma omp parallel for schedule(static) num_threads(nthreads)
  for (uint64_t s = 0; s < n; s++) {
    long int sums[classes];
    unsigned int lit[8], vot[8];
    for (unsigned int h = 0; h < classes; h++) sums[h] = 0;
    if (!tm->individualized) {
      char *input = (char *)x + s * tm->input_chunks;
      for (unsigned int chunk = 0; chunk < cc * classes; chunk++) {
        uint8_t out = tk_tsetlin_calculate(tm, input, lit, vot, chunk);
        sums[chunk / cc] += tk_tsetlin_sums(tm, out, vot);
      }
    } else {
      for (unsigned int h = 0; h < classes; h++) {
        uint64_t ich = tm->input_chunks_ind[h];
        char *input = (char *)x + (uint64_t)dim_offsets[h] + s * ich;
        for (unsigned int chunk = 0; chunk < cc; chunk++) {
          uint8_t out = tk_tsetlin_calculate_ind(&tm->automata_arr[h], input, lit, vot, chunk,
                                                 ich, tm->tail_masks_ind[h], tm->clause_tolerance);
          sums[h] += tk_tsetlin_sums_ind(out, vot);
        }
      }
    }
    if (out_scores) for (unsigned int h = 0; h < classes; h++) out_scores[s * classes + h] = sums[h];
    if (out_classes) {
      long int maxval = -INT64_MAX;
      unsigned int maxclass = 0;
      for (unsigned int h = 0; h < classes; h++)
        if (sums[h] > maxval) { maxval = sums[h]; maxclass = h; }
      out_classes[s] = maxclass;
    }
    if (out_codes) {
      uint8_t *e = out_codes + s * tm->class_chunks;
      for (unsigned int h = 0; h < classes; h++) {
        if (sums[h] > 0) e[h / 8] |= (uint8_t)(1 << (h % 8));
        else e[h / 8] &= (uint8_t)~(1 << (h % 8));
      }
    }
  }
  return 0;
}

/* tk_tsetlin_persist (capi.c:1538-1562) with the Lua string result replaced
 * by a caller buffer */
int ref_persist(void *p, uint8_t *buf, uint64_t cap, uint64_t *len) {
  tk_tsetlin_t *tm = p;
  char *data = NULL;
  size_t sz = 0;
  FILE *fh = open_memstream(&data, &sz);
  tk_lua_fwrite(NULL, &tm->type, sizeof(tk_tsetlin_type_t), 1, fh);
  tk_tsetlin_persist_classifier(NULL, tm, fh);
  fclose(fh);
  *len = sz;
  int rc = 0;
  if (sz <= cap) memcpy(buf, data, sz);
  else rc = -1;
  free(data);
  return rc;
}

/* tk_tsetlin_load (capi.c:1751-1772) */
void *ref_load(const uint8_t *buf, uint64_t len) {
  FILE *fh = fmemopen((void *)buf, len, "r");
  tk_tsetlin_type_t type;
  tk_lua_fread(NULL, &type, sizeof(type), 1, fh);
  tk_tsetlin_t *tm = calloc(1, sizeof(tk_tsetlin_t));
  tm->type = type;
  tm->has_state = true;
  _tk_tsetlin_load_classifier(NULL, tm, fh);
  fclose(fh);
  return tm;
}
