/*
 * CPU oracle for the santoku.tsetlin Tsetlin-machine hot path (see
 * tm_oracle.h).  TEST INFRASTRUCTURE ONLY: the product never links this.
 *
 * Layout used internally: every clause row of the reference's byte layout
 * (`input_chunks` bytes, automata.h:17-31) is held as little-endian 64-bit
 * words, so bit i of a row is bit (i % 64) of word i / 64 -- the reference's
 * LSB-first bit order (capi.c:488-489).  Rows are zero padded to whole
 * words; three masks on the last word keep the padding out of every result:
 *   vmask  bytes that exist in the reference row,
 *   emask  vmask with the tail byte ANDed with tail_mask (evaluation,
 *          capi.c:104-106),
 *   amask  the mask the reference applies to the carry/borrow into the
 *          action plane of the tail byte.  The reference applies tail_mask
 *          there only on its byte path (automata.h:97,128); its 128-bit path
 *          (automata.h:163-194 and siblings) covers the tail byte unmasked
 *          when input_chunks is a multiple of 16.
 */
#include "tm_oracle.h"

#include <math.h>
#include <omp.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define CVEC_BITS 8

static __thread char orc_err[256];
const char *orc_last_error(void) { return orc_err; }
static int fail(const char *msg) {
  snprintf(orc_err, sizeof(orc_err), "%s", msg);
  return -1;
}

/* ------------------------------------------------------------------------ */
/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw: "Parallel random numbers: as  */
/* easy as 1, 2, 3", SC'11).                                                */
/* ------------------------------------------------------------------------ */
void orc_philox(const uint32_t *ctr, uint64_t key, uint32_t *out) {
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
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

static inline void ph(uint32_t a, uint32_t b, uint32_t c, uint32_t d, uint64_t key,
                      uint32_t *out) {
  uint32_t ctr[4] = { a, b, c, d };
  orc_philox(ctr, key, out);
}

/* Counter words: (sample, epoch, unit, stream).  unit = class *
 * clause_chunks + chunk.  Streams: */
#define ST_NEG 0u            /* negative-sampling draw: output 0 */
#define ST_CH0 1u            /* chance draws 0..3 */
#define ST_CH1 2u            /* chance draws 4..7 */
#define ST_IB 0x01000000u    /* | clause << 20 | pick / 4 */
#define ST_PERM 0xFFFFFFFFu  /* permutation keys: (i, epoch, 0, ST_PERM) */

/* bounded draw in [0, range): multiply-shift */
static inline uint32_t bounded(uint32_t u, uint64_t range) {
  return (uint32_t)(((uint64_t)u * range) >> 32);
}

typedef struct { uint64_t k; uint32_t i; } perm_key;
static int perm_cmp(const void *a, const void *b) {
  const perm_key *x = a, *y = b;
  if (x->k != y->k) return x->k < y->k ? -1 : 1;
  return x->i < y->i ? -1 : (x->i > y->i);
}

/* The epoch's sample order: samples sorted by a 64-bit Philox key, ties by
 * index.  Stands in for the per-thread Fisher-Yates of capi.c:245-256: any
 * uniformly random order has the reference's meaning, and one order per
 * (seed, epoch) shared by all units replaces the per-thread orders. */
void orc_perm(uint64_t seed, uint32_t epoch, uint64_t n, uint32_t *out) {
  perm_key *keys = malloc(n * sizeof(perm_key));
  for (uint64_t i = 0; i < n; i++) {
    uint32_t o[4];
    ph((uint32_t)i, epoch, 0, ST_PERM, seed, o);
    keys[i].k = ((uint64_t)o[0] << 32) | o[1];
    keys[i].i = (uint32_t)i;
  }
  qsort(keys, n, sizeof(perm_key), perm_cmp);
  for (uint64_t i = 0; i < n; i++) out[i] = keys[i].i;
  free(keys);
}

/* ------------------------------------------------------------------------ */
/* Stand-in for the reference's per-thread generator (refstruct mode only). */
/* ------------------------------------------------------------------------ */
static __thread uint64_t mcg_state = 1;
static inline void mcg_seed(uint64_t s) {
  uint64_t z = s + 0x9E3779B97F4A7C15ull;          /* splitmix64 finaliser */
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  mcg_state = z | 1;
}
static inline uint32_t mcg_next(void) {
  mcg_state *= 0xDA942042E4DD58B5ull;
  return (uint32_t)(mcg_state >> 32);
}
static inline int mcg_chance(double p) {
  return (double)mcg_next() * (1.0 / 4294967296.0) < p;
}

/* ------------------------------------------------------------------------ */
/* Machine                                                                  */
/* ------------------------------------------------------------------------ */
typedef struct {
  uint64_t rows;        /* clauses held */
  uint64_t W;           /* 64-bit words per row */
  uint64_t n_chunks;    /* bytes per row in the reference layout */
  uint64_t input_bits;  /* 2 * features */
  uint32_t s_picks;     /* Type Ib picks per event */
  uint64_t vmask, emask, amask;
  uint64_t *act;        /* [rows][W] */
  uint64_t *cnt;        /* [rows][m][W] */
} aut_t;

struct orc_tm {
  int type, individualized, reusable, has_state;
  uint32_t classes, features, clauses, clause_tolerance, clause_maximum, target;
  uint32_t state_bits, include_bits, input_bits, input_chunks, clause_chunks;
  uint32_t class_chunks, state_chunks, action_chunks;
  uint8_t tail_mask;
  double negative, specificity;
  uint64_t *feat_sizes; /* individualized: per class */
  uint32_t n_aut;
  aut_t *aut;           /* 1 (classes * clauses rows) or one per class */
};

static inline uint64_t atl1(uint64_t v) { return v ? v : 1; }

static uint64_t bytes_mask(uint64_t nbytes) {
  return nbytes >= 8 ? ~0ull : ((1ull << (8 * nbytes)) - 1);
}

/* capi.c:480-483: target derivation (note fmaxf: single precision). */
static uint32_t derive_target(uint32_t clauses, uint32_t tol, double targetf) {
  double t;
  if (targetf < 0)
    t = sqrt((double)clauses / 2.0) * (double)tol;
  else
    t = ceil(targetf >= 1 ? targetf
                          : (double)fmaxf(1.0f, (float)((double)clauses * targetf)));
  return (uint32_t)t;
}

static void aut_layout(aut_t *a, uint64_t rows, uint64_t features, uint32_t state_bits,
                       double specificity) {
  a->rows = rows;
  a->input_bits = 2 * features;
  a->n_chunks = (a->input_bits + CVEC_BITS - 1) / CVEC_BITS;
  a->W = (a->n_chunks + 7) / 8;
  if (a->W == 0) a->W = 1;
  /* capi.c:181 / :347: s = (unsigned)((double)(2F) / specificity) */
  a->s_picks = (uint32_t)((double)(2 * features) / specificity);
  uint64_t tail_bits = a->input_bits & (CVEC_BITS - 1);
  uint8_t tail_mask = tail_bits ? (uint8_t)((1u << tail_bits) - 1) : 0xFF;
  uint64_t last_bytes = a->n_chunks - 8 * (a->W - 1);
  a->vmask = a->n_chunks ? bytes_mask(last_bytes) : 0;
  uint64_t tail_sh = a->n_chunks ? 8 * (last_bytes - 1) : 0;
  uint64_t tm64 = a->n_chunks ? (0xFFull << tail_sh) : 0;
  uint64_t tail_eval = ((uint64_t)tail_mask << tail_sh) | (a->vmask & ~tm64);
  a->emask = tail_eval;
  a->amask = (a->n_chunks % 16 != 0) ? tail_eval : a->vmask;
  (void)state_bits;
}

static int aut_alloc(aut_t *a, uint32_t state_bits) {
  uint64_t m = state_bits - 1;
  a->act = calloc(atl1(a->rows * a->W), 8);
  a->cnt = calloc(atl1(a->rows * m * a->W), 8);
  return (a->act && a->cnt) ? 0 : -1;
}

static void aut_free(aut_t *a) {
  free(a->act); free(a->cnt);
  a->act = a->cnt = NULL;
}

/* automata.h:72-86: counts all ones, actions zero. */
static void aut_setup(aut_t *a, uint32_t state_bits) {
  uint64_t m = state_bits - 1;
  memset(a->act, 0, a->rows * a->W * 8);
  for (uint64_t r = 0; r < a->rows; r++)
    for (uint64_t b = 0; b < m; b++)
      for (uint64_t w = 0; w < a->W; w++)
        a->cnt[(r * m + b) * a->W + w] = (w == a->W - 1) ? a->vmask : ~0ull;
}

void orc_setup(orc_tm *tm) {
  for (uint32_t h = 0; h < tm->n_aut; h++) aut_setup(&tm->aut[h], tm->state_bits);
}

orc_tm *orc_create(int type, uint32_t classes, uint32_t features, uint32_t clauses,
                   uint32_t clause_tolerance, uint32_t clause_maximum,
                   uint32_t state_bits, uint32_t include_bits, double target,
                   double negative, double specificity, int reusable,
                   int individualized, const int64_t *feat_offsets) {
  /* capi.c:463-472 */
  if (!classes) { fail("classes must be greater than 1"); return NULL; }
  if (!clauses) { fail("clauses must be greater than 0"); return NULL; }
  if (!clause_tolerance) { fail("clause_tolerance must be greater than 0"); return NULL; }
  if (!clause_maximum) { fail("clause_maximum must be greater than 0"); return NULL; }
  if (state_bits < 2) { fail("bits must be greater than 1"); return NULL; }
  if (state_bits > 32) { fail("state_bits above 32 unsupported"); return NULL; }
  orc_tm *tm = calloc(1, sizeof(orc_tm));
  tm->type = type;
  tm->individualized = individualized ? 1 : 0;
  tm->reusable = reusable ? 1 : 0;
  tm->has_state = 1;
  tm->negative = negative < 0 ? 1.0 / (double)classes : negative;   /* :474 */
  tm->classes = classes;
  tm->class_chunks = (classes + CVEC_BITS - 1) / CVEC_BITS;
  tm->clauses = ((clauses + CVEC_BITS - 1) / CVEC_BITS) * CVEC_BITS; /* :477 */
  tm->clause_tolerance = clause_tolerance;
  tm->clause_maximum = clause_maximum;
  tm->target = derive_target(tm->clauses, clause_tolerance, target);
  tm->state_bits = state_bits;
  tm->include_bits = include_bits ? include_bits : 1;
  tm->specificity = specificity;
  tm->clause_chunks = tm->clauses / CVEC_BITS;
  if (!individualized) {
    /* capi.c:486-493 */
    tm->features = features;
    tm->input_bits = 2 * features;
    uint64_t tail_bits = tm->input_bits & (CVEC_BITS - 1);
    tm->tail_mask = tail_bits ? (uint8_t)((1u << tail_bits) - 1) : 0xFF;
    tm->input_chunks = (tm->input_bits + CVEC_BITS - 1) / CVEC_BITS;
    tm->state_chunks = tm->classes * tm->clauses * (tm->state_bits - 1) * tm->input_chunks;
    tm->action_chunks = tm->classes * tm->clauses * tm->input_chunks;
    tm->n_aut = 1;
    tm->aut = calloc(1, sizeof(aut_t));
    aut_layout(&tm->aut[0], (uint64_t)classes * tm->clauses, features, state_bits, specificity);
  } else {
    /* capi.c:528-606 */
    tm->n_aut = classes;
    tm->aut = calloc(classes, sizeof(aut_t));
    tm->feat_sizes = calloc(classes, sizeof(uint64_t));
    uint64_t ts = 0, ta = 0;
    for (uint32_t h = 0; h < classes; h++) {
      uint64_t k = (uint64_t)(feat_offsets[h + 1] - feat_offsets[h]);
      tm->feat_sizes[h] = k;
      aut_layout(&tm->aut[h], tm->clauses, k, state_bits, specificity);
      ts += tm->clauses * tm->aut[h].n_chunks * (state_bits - 1);
      ta += tm->clauses * tm->aut[h].n_chunks;
    }
    tm->state_chunks = (uint32_t)ts;
    tm->action_chunks = (uint32_t)ta;
  }
  for (uint32_t h = 0; h < tm->n_aut; h++)
    if (aut_alloc(&tm->aut[h], state_bits)) { fail("oom"); orc_destroy(tm); return NULL; }
  orc_setup(tm);
  return tm;
}

void orc_destroy(orc_tm *tm) {
  if (!tm) return;
  for (uint32_t h = 0; h < tm->n_aut; h++) aut_free(&tm->aut[h]);
  free(tm->aut);
  free(tm->feat_sizes);
  free(tm);
}

void orc_info(const orc_tm *tm, uint64_t *o) {
  o[0] = (uint64_t)tm->type; o[1] = tm->classes; o[2] = tm->features;
  o[3] = tm->clauses; o[4] = tm->clause_tolerance; o[5] = tm->clause_maximum;
  o[6] = tm->target; o[7] = tm->state_bits; o[8] = tm->include_bits;
  o[9] = tm->input_bits; o[10] = tm->input_chunks; o[11] = tm->clause_chunks;
  o[12] = tm->class_chunks; o[13] = tm->state_chunks; o[14] = tm->action_chunks;
  o[15] = tm->tail_mask; o[16] = (uint64_t)tm->individualized;
  o[17] = (uint64_t)tm->reusable; o[18] = (uint64_t)tm->has_state;
}
double orc_negative(const orc_tm *tm) { return tm->negative; }
double orc_specificity(const orc_tm *tm) { return tm->specificity; }

/* ------------------------------------------------------------------------ */
/* Bit-sliced automata (automata.h)                                         */
/* ------------------------------------------------------------------------ */
static inline uint64_t amask_of(const aut_t *a, uint64_t w) {
  return w == a->W - 1 ? a->amask : ~0ull;
}
static inline uint64_t vmask_of(const aut_t *a, uint64_t w) {
  return w == a->W - 1 ? a->vmask : ~0ull;
}
static inline uint64_t emask_of(const aut_t *a, uint64_t w) {
  return w == a->W - 1 ? a->emask : ~0ull;
}

/* Saturating +1 on the automata selected by `carry` in word w of row r:
 * ripple carry through the count planes, into the action plane (masked),
 * then saturate at all ones (automata.h:88-117, 147-232). */
static inline void w_inc(aut_t *a, uint64_t m, uint64_t r, uint64_t w, uint64_t carry) {
  if (!carry) return;
  uint64_t *cnt = a->cnt + r * m * a->W;
  uint64_t *act = a->act + r * a->W;
  for (uint64_t b = 0; b < m; b++) {
    uint64_t v = cnt[b * a->W + w];
    uint64_t nc = v & carry;
    cnt[b * a->W + w] = v ^ carry;
    carry = nc;
  }
  uint64_t cm = carry & amask_of(a, w);
  uint64_t nc = act[w] & cm;
  act[w] ^= cm;
  carry = nc;
  if (carry) {
    for (uint64_t b = 0; b < m; b++) cnt[b * a->W + w] |= carry;
    act[w] |= carry;
  }
}

/* Saturating -1 (automata.h:118-146, 234-318). */
static inline void w_dec(aut_t *a, uint64_t m, uint64_t r, uint64_t w, uint64_t borrow) {
  if (!borrow) return;
  uint64_t *cnt = a->cnt + r * m * a->W;
  uint64_t *act = a->act + r * a->W;
  for (uint64_t b = 0; b < m; b++) {
    uint64_t v = cnt[b * a->W + w];
    uint64_t nb = ~v & borrow;
    cnt[b * a->W + w] = v ^ borrow;
    borrow = nb;
  }
  uint64_t bm = borrow & amask_of(a, w);
  uint64_t nb = ~act[w] & bm;
  act[w] ^= bm;
  borrow = nb;
  if (borrow) {
    for (uint64_t b = 0; b < m; b++) cnt[b * a->W + w] &= ~borrow;
    act[w] &= ~borrow;
  }
}

/* automata.h:499-512: action AND the top include_bits-1 count planes. */
static inline uint64_t w_included(const aut_t *a, uint64_t m, uint64_t ib, uint64_t r,
                                  uint64_t w) {
  const uint64_t *cnt = a->cnt + r * m * a->W;
  uint64_t inc = a->act[r * a->W + w];
  for (uint64_t i = 1; i < ib && i <= m; i++) inc &= cnt[(m - i) * a->W + w];
  return inc;
}

/* tk_automata_inc (automata.h:147-232) */
static void aut_inc(aut_t *a, uint64_t m, uint64_t r, const uint64_t *x) {
  for (uint64_t w = 0; w < a->W; w++) w_inc(a, m, r, w, x[w] & vmask_of(a, w));
}
/* tk_automata_dec_not_excluded (automata.h:538-640) */
static void aut_dec_not_excluded(aut_t *a, uint64_t m, uint64_t ib, uint64_t r,
                                 const uint64_t *x) {
  for (uint64_t w = 0; w < a->W; w++) {
    uint64_t inc = w_included(a, m, ib, r, w);
    w_dec(a, m, r, w, ~x[w] & ~inc & vmask_of(a, w));
  }
}
/* tk_automata_inc_not_excluded (automata.h:642-742) */
static void aut_inc_not_excluded(aut_t *a, uint64_t m, uint64_t ib, uint64_t r,
                                 const uint64_t *x) {
  for (uint64_t w = 0; w < a->W; w++) {
    uint64_t inc = w_included(a, m, ib, r, w);
    w_inc(a, m, r, w, ~x[w] & ~inc & vmask_of(a, w));
  }
}

/* ------------------------------------------------------------------------ */
/* Clause evaluation (capi.c:85-146, 258-315) and chunk vote (:148-161)      */
/* ------------------------------------------------------------------------ */
static inline uint8_t eval_chunk(const aut_t *a, uint64_t row0, const uint64_t *x,
                                 uint32_t tol, uint32_t *lit, uint32_t *vot) {
  uint8_t out = 0;
  for (uint32_t j = 0; j < CVEC_BITS; j++) {
    const uint64_t *act = a->act + (row0 + j) * a->W;
    uint32_t L = 0, F = 0;
    for (uint64_t w = 0; w < a->W; w++) {
      uint64_t av = act[w] & emask_of(a, w);
      L += (uint32_t)__builtin_popcountll(av);
      F += (uint32_t)__builtin_popcountll(av & ~x[w]);
    }
    long v;
    if (L == 0) v = (long)tol;
    else {
      v = (L < tol ? (long)L : (long)tol) - (long)F;
      if (v < 0) v = 0;
    }
    if (v > 0) out |= (uint8_t)(1u << j);
    lit[j] = L;
    vot[j] = (uint32_t)v;
  }
  return out;
}

static inline long chunk_sum(uint8_t out, const uint32_t *vot) {
  long s = 0;
  for (uint32_t j = 0; j < CVEC_BITS; j += 2) if (out & (1u << j)) s += (long)vot[j];
  for (uint32_t j = 1; j < CVEC_BITS; j += 2) if (out & (1u << j)) s -= (long)vot[j];
  return s;
}

/* ------------------------------------------------------------------------ */
/* Feedback (capi.c:163-243, 326-402)                                        */
/* ------------------------------------------------------------------------ */
typedef struct {
  int mode;
  uint64_t seed;
  uint32_t s, e, g;     /* philox counter words */
} rng_ctx;

static void type_i(const orc_tm *tm, aut_t *a, uint64_t m, uint64_t row0, uint32_t j,
                   const uint64_t *x, const uint32_t *lit, const uint32_t *vot,
                   const rng_ctx *rc) {
  uint64_t r = row0 + j;
  if (vot[j] > 0) {
    /* Type Ia: capi.c:177-180 */
    if (lit[j] <= tm->clause_maximum) aut_inc(a, m, r, x);
    aut_dec_not_excluded(a, m, tm->include_bits, r, x);
  } else {
    /* Type Ib: capi.c:181-190 -- s single-automaton decrements, with
     * replacement */
    uint32_t s = a->s_picks;
    uint32_t o[4];
    for (uint32_t p = 0; p < s; p++) {
      uint32_t bit;
      if (rc->mode == ORC_RNG_PHILOX) {
        if ((p & 3) == 0) ph(rc->s, rc->e, rc->g, ST_IB | (j << 20) | (p >> 2), rc->seed, o);
        bit = bounded(o[p & 3], a->input_bits);
      } else {
        bit = (uint32_t)(mcg_next() % a->input_bits);
      }
      w_dec(a, m, r, bit >> 6, 1ull << (bit & 63));
    }
  }
}

static void type_ii(const orc_tm *tm, aut_t *a, uint64_t m, uint64_t row0, uint32_t j,
                    const uint64_t *x, const uint32_t *vot) {
  /* capi.c:192-196 */
  if (vot[j] > 0) aut_inc_not_excluded(a, m, tm->include_bits, row0 + j, x);
}

/* One (unit, sample) step: evaluation + tm_update (capi.c:201-243).  `pos` is
 * the reference's `chunk_class == sample_class && target_vote`.  In philox
 * mode the draws are keyed; in refstruct mode they are consumed from the
 * thread's stream in the reference's order.  The negative-sampling skip is
 * decided by the caller. */
static void unit_step(const orc_tm *tm, aut_t *a, uint64_t row0, const uint64_t *x, int pos,
                      const rng_ctx *rc) {
  uint64_t m = tm->state_bits - 1;
  uint32_t lit[8], vot[8];
  uint8_t out = eval_chunk(a, row0, x, tm->clause_tolerance, lit, vot);
  long T = (long)tm->target;
  long v = chunk_sum(out, vot);
  if (v > T) v = T;
  if (v < -T) v = -T;
  uint64_t av = (uint64_t)(pos ? T - v : T + v);
  uint32_t d[8];
  if (rc->mode == ORC_RNG_PHILOX) {
    ph(rc->s, rc->e, rc->g, ST_CH0, rc->seed, d);
    ph(rc->s, rc->e, rc->g, ST_CH1, rc->seed, d + 4);
  }
  double p = (double)av / (2.0 * (double)T);
  for (uint32_t pr = 0; pr < 4; pr++) {
    uint32_t ji = pos ? 2 * pr : 2 * pr + 1;   /* Type I clause */
    uint32_t jii = pos ? 2 * pr + 1 : 2 * pr;  /* Type II clause */
    int c1, c2;
    if (rc->mode == ORC_RNG_PHILOX) {
      c1 = bounded(d[2 * pr], 2 * (uint64_t)T) < av;
      if (c1) type_i(tm, a, m, row0, ji, x, lit, vot, rc);
      c2 = bounded(d[2 * pr + 1], 2 * (uint64_t)T) < av;
      if (c2) type_ii(tm, a, m, row0, jii, x, vot);
    } else {
      c1 = mcg_chance(p);
      if (c1) type_i(tm, a, m, row0, ji, x, lit, vot, rc);
      c2 = mcg_chance(p);
      if (c2) type_ii(tm, a, m, row0, jii, x, vot);
    }
  }
}

/* ------------------------------------------------------------------------ */
/* Train drivers (capi.c:1112-1482)                                          */
/* ------------------------------------------------------------------------ */
static uint64_t *pack_rows(const uint8_t *x, uint64_t n, uint64_t n_chunks, uint64_t W) {
  uint64_t *o = calloc(atl1(n * W), 8);
  for (uint64_t s = 0; s < n; s++) memcpy(o + s * W, x + s * n_chunks, n_chunks);
  return o;
}

static uint64_t neg_threshold(double negative) {
  double q = (1.0 - negative) * 4294967296.0;
  if (!(q > 0)) return 0;
  if (q >= 4294967296.0) return 4294967296ull;
  return (uint64_t)floor(q);
}

int orc_train(orc_tm *tm, const uint8_t *x, const int64_t *labels, const uint8_t *codes,
              const int64_t *dim_offsets, uint64_t n, uint32_t epochs, uint64_t seed,
              uint32_t epoch_base, int rng_mode, int nthreads) {
  if (!tm->has_state) return fail("can't train a model loaded without state");
  if (tm->type == ORC_CLASSIFIER && !labels) return fail("missing solutions");
  if (tm->type == ORC_ENCODER && !codes) return fail("missing codes");
  if (tm->individualized && !dim_offsets) return fail("missing dim_offsets");
  if (nthreads <= 0) nthreads = omp_get_max_threads();
  /* packed per-aut sample rows */
  uint64_t **rows = calloc(tm->n_aut, sizeof(uint64_t *));
  for (uint32_t h = 0; h < tm->n_aut; h++) {
    const uint8_t *base = x + (tm->individualized ? (uint64_t)dim_offsets[h] : 0);
    rows[h] = pack_rows(base, n, tm->aut[h].n_chunks, tm->aut[h].W);
  }
  const uint32_t cc = tm->clause_chunks;
  const uint64_t total = (uint64_t)tm->classes * cc;
  const uint64_t thr = neg_threshold(tm->negative);
  orc_setup(tm); /* capi.c:1136-1146: every train starts from scratch */
  uint32_t *perm = malloc((n ? n : 1) * sizeof(uint32_t));
  for (uint32_t it = 0; it < epochs; it++) {
    uint32_t e = epoch_base + it;
    if (rng_mode == ORC_RNG_PHILOX) {
      orc_perm(seed, e, n, perm);
      #pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
      for (uint64_t u = 0; u < total; u++) {
        uint32_t h = (uint32_t)(u / cc), k = (uint32_t)(u % cc);
        aut_t *a = tm->individualized ? &tm->aut[h] : &tm->aut[0];
        uint64_t row0 = tm->individualized ? (uint64_t)k * 8 : u * 8;
        const uint64_t *xr = tm->individualized ? rows[h] : rows[0];
        rng_ctx rc = { ORC_RNG_PHILOX, seed, 0, e, (uint32_t)u };
        for (uint64_t i = 0; i < n; i++) {
          uint32_t s = perm[i];
          rc.s = s;
          int pos;
          if (tm->type == ORC_CLASSIFIER) {
            uint32_t label = (uint32_t)labels[s];
            pos = label == h;
            if (!pos) {
              uint32_t o[4];
              ph(s, e, (uint32_t)u, ST_NEG, seed, o);
              if ((uint64_t)o[0] < thr) continue;
            }
          } else {
            pos = (codes[(uint64_t)s * tm->class_chunks + h / 8] >> (h % 8)) & 1;
          }
          unit_step(tm, a, row0, xr + (uint64_t)s * a->W, pos, &rc);
        }
      }
    }
  }
  if (rng_mode == ORC_RNG_REFSTRUCT) {
    /* capi.c:1134-1167 (dense), :1314-1361 (enc-ind), :1410-1458 (cls-ind) */
    uint32_t **shuffles = calloc((size_t)nthreads, sizeof(uint32_t *));
    for (int t = 0; t < nthreads; t++) shuffles[t] = malloc((n ? n : 1) * sizeof(uint32_t));
    #pragma omp parallel num_threads(nthreads)
    mcg_seed((uint64_t)omp_get_thread_num() ^ seed);
    for (uint32_t it = 0; it < epochs; it++) {
      #pragma omp parallel num_threads(nthreads)
      {
        int tid = omp_get_thread_num();
        uint32_t *sh = shuffles[tid];
        /* capi.c:245-256 */
        for (uint64_t i = 0; i < n; i++) {
          sh[i] = (uint32_t)i;
          uint64_t j = i == 0 ? 0 : mcg_next() % (i + 1);
          uint32_t t = sh[i]; sh[i] = sh[j]; sh[j] = t;
        }
        rng_ctx rc = { ORC_RNG_REFSTRUCT, 0, 0, 0, 0 };
        if (!tm->individualized) {
          #pragma omp for schedule(static)
          for (uint64_t u = 0; u < total; u++) {
            uint32_t h = (uint32_t)(u / cc);
            aut_t *a = &tm->aut[0];
            for (uint64_t i = 0; i < n; i++) {
              uint32_t s = sh[i];
              int pos;
              if (tm->type == ORC_CLASSIFIER) {
                pos = (uint32_t)labels[s] == h;
                /* capi.c:215: chance(1-negative) drawn after evaluation;
                 * evaluation has no side effects, so drawing first is the
                 * same */
                if (!pos && mcg_chance(1 - tm->negative)) continue;
              } else {
                pos = (codes[(uint64_t)s * tm->class_chunks + h / 8] >> (h % 8)) & 1;
              }
              unit_step(tm, a, u * 8, rows[0] + (uint64_t)s * a->W, pos, &rc);
            }
          }
        } else {
          #pragma omp for schedule(static)
          for (uint64_t h = 0; h < tm->classes; h++) {
            aut_t *a = &tm->aut[h];
            for (uint32_t k = 0; k < cc; k++) {
              for (uint64_t i = 0; i < n; i++) {
                uint32_t s = sh[i];
                int pos;
                if (tm->type == ORC_CLASSIFIER) {
                  pos = (uint32_t)labels[s] == h;
                  if (!pos && mcg_chance(1 - tm->negative)) continue;
                } else {
                  pos = (codes[(uint64_t)s * tm->class_chunks + h / 8] >> (h % 8)) & 1;
                }
                unit_step(tm, a, (uint64_t)k * 8, rows[h] + (uint64_t)s * a->W, pos, &rc);
              }
            }
          }
        }
      }
    }
    for (int t = 0; t < nthreads; t++) free(shuffles[t]);
    free(shuffles);
  }
  free(perm);
  for (uint32_t h = 0; h < tm->n_aut; h++) free(rows[h]);
  free(rows);
  return 0;
}

/* ------------------------------------------------------------------------ */
/* Predict (capi.c:903-1086)                                                 */
/* ------------------------------------------------------------------------ */
int orc_predict(const orc_tm *tm, const uint8_t *x, const int64_t *dim_offsets, uint64_t n,
                int64_t *out_classes, uint8_t *out_codes, int64_t *out_scores,
                int nthreads) {
  if (tm->individualized && !dim_offsets) return fail("missing dim_offsets");
  if (nthreads <= 0) nthreads = omp_get_max_threads();
  const uint32_t C = tm->classes, cc = tm->clause_chunks;
  uint64_t maxW = 1;
  for (uint32_t h = 0; h < tm->n_aut; h++) if (tm->aut[h].W > maxW) maxW = tm->aut[h].W;
  #pragma omp parallel num_threads(nthreads)
  {
    uint64_t *xr = malloc(maxW * 8);
    long *sums = malloc((C ? C : 1) * sizeof(long));
    #pragma omp for schedule(static)
    for (uint64_t s = 0; s < n; s++) {
      uint32_t lit[8], vot[8];
      for (uint32_t h = 0; h < C; h++) {
        const aut_t *a = tm->individualized ? &tm->aut[h] : &tm->aut[0];
        const uint8_t *base = x + (tm->individualized ? (uint64_t)dim_offsets[h] : 0);
        memset(xr, 0, a->W * 8);
        memcpy(xr, base + s * a->n_chunks, a->n_chunks);
        long sum = 0;
        for (uint32_t k = 0; k < cc; k++) {
          uint64_t row0 = tm->individualized ? (uint64_t)k * 8 : ((uint64_t)h * cc + k) * 8;
          uint8_t out = eval_chunk(a, row0, xr, tm->clause_tolerance, lit, vot);
          sum += chunk_sum(out, vot);
        }
        sums[h] = sum;
      }
      if (out_scores)
        for (uint32_t h = 0; h < C; h++) out_scores[s * C + h] = sums[h];
      if (out_classes) {
        /* capi.c:934-942: strict > from -INT64_MAX, ties to the lowest class */
        long maxval = -INT64_MAX;
        uint32_t maxc = 0;
        for (uint32_t h = 0; h < C; h++)
          if (sums[h] > maxval) { maxval = sums[h]; maxc = h; }
        out_classes[s] = maxc;
      }
      if (out_codes) {
        /* capi.c:982-990: bit h = votes[h] > 0, LSB-first */
        uint8_t *e = out_codes + s * tm->class_chunks;
        memset(e, 0, tm->class_chunks);
        for (uint32_t h = 0; h < C; h++)
          if (sums[h] > 0) e[h / 8] |= (uint8_t)(1u << (h % 8));
      }
    }
    free(xr);
    free(sums);
  }
  return 0;
}

int orc_clause_eval(const orc_tm *tm, const uint8_t *x, const int64_t *dim_offsets,
                    uint64_t n, uint32_t *literals, uint32_t *votes) {
  const uint32_t C = tm->classes, cc = tm->clause_chunks;
  const uint64_t ncl = (uint64_t)C * tm->clauses;
  for (uint64_t s = 0; s < n; s++) {
    for (uint32_t h = 0; h < C; h++) {
      const aut_t *a = tm->individualized ? &tm->aut[h] : &tm->aut[0];
      uint64_t *xr = calloc(a->W, 8);
      const uint8_t *base = x + (tm->individualized ? (uint64_t)dim_offsets[h] : 0);
      memcpy(xr, base + s * a->n_chunks, a->n_chunks);
      for (uint32_t k = 0; k < cc; k++) {
        uint64_t row0 = tm->individualized ? (uint64_t)k * 8 : ((uint64_t)h * cc + k) * 8;
        uint32_t lit[8], vot[8];
        eval_chunk(a, row0, xr, tm->clause_tolerance, lit, vot);
        for (uint32_t j = 0; j < 8; j++) {
          uint64_t c = ((uint64_t)h * cc + k) * 8 + j;
          literals[s * ncl + c] = lit[j];
          votes[s * ncl + c] = vot[j];
        }
      }
      free(xr);
    }
  }
  return 0;
}

/* ------------------------------------------------------------------------ */
/* Reference byte layouts                                                    */
/* ------------------------------------------------------------------------ */
uint64_t orc_action_bytes(const orc_tm *tm) {
  uint64_t t = 0;
  for (uint32_t h = 0; h < tm->n_aut; h++) t += tm->aut[h].rows * tm->aut[h].n_chunks;
  return t;
}
uint64_t orc_state_bytes(const orc_tm *tm) {
  return orc_action_bytes(tm) * (tm->state_bits - 1);
}

void orc_export(const orc_tm *tm, uint8_t *actions, uint8_t *state) {
  uint64_t m = tm->state_bits - 1;
  uint64_t ao = 0, so = 0;
  for (uint32_t h = 0; h < tm->n_aut; h++) {
    const aut_t *a = &tm->aut[h];
    for (uint64_t r = 0; r < a->rows; r++) {
      if (actions) memcpy(actions + ao + r * a->n_chunks, a->act + r * a->W, a->n_chunks);
      if (state)
        for (uint64_t b = 0; b < m; b++)
          memcpy(state + so + (r * m + b) * a->n_chunks, a->cnt + (r * m + b) * a->W,
                 a->n_chunks);
    }
    ao += a->rows * a->n_chunks;
    so += a->rows * m * a->n_chunks;
  }
}

int orc_import(orc_tm *tm, const uint8_t *actions, const uint8_t *state) {
  uint64_t m = tm->state_bits - 1;
  uint64_t ao = 0, so = 0;
  for (uint32_t h = 0; h < tm->n_aut; h++) {
    aut_t *a = &tm->aut[h];
    for (uint64_t r = 0; r < a->rows; r++) {
      if (actions) {
        a->act[r * a->W + a->W - 1] = 0;
        memcpy(a->act + r * a->W, actions + ao + r * a->n_chunks, a->n_chunks);
      }
      if (state && a->cnt)
        for (uint64_t b = 0; b < m; b++) {
          a->cnt[(r * m + b) * a->W + a->W - 1] = 0;
          memcpy(a->cnt + (r * m + b) * a->W, state + so + (r * m + b) * a->n_chunks,
                 a->n_chunks);
        }
    }
    ao += a->rows * a->n_chunks;
    so += a->rows * m * a->n_chunks;
  }
  return 0;
}

/* ------------------------------------------------------------------------ */
/* Persist / load (capi.c:1509-1562, 1675-1772)                              */
/* ------------------------------------------------------------------------ */
uint64_t orc_persist_size(const orc_tm *tm) {
  return 4 + 13 * 4 + 8 + 1 + tm->action_chunks + 1 +
         (tm->individualized ? 8ull * tm->classes : 0);
}

#define PUT(v) do { memcpy(buf + o, &(v), sizeof(v)); o += sizeof(v); } while (0)
int orc_persist(const orc_tm *tm, uint8_t *buf, uint64_t cap, uint64_t *len) {
  uint64_t need = orc_persist_size(tm);
  if (len) *len = need;
  if (cap < need) return fail("buffer too small");
  uint64_t o = 0;
  int32_t type = tm->type;
  PUT(type);
  PUT(tm->classes); PUT(tm->features); PUT(tm->clauses); PUT(tm->clause_tolerance);
  PUT(tm->clause_maximum); PUT(tm->target); PUT(tm->state_bits); PUT(tm->include_bits);
  PUT(tm->input_bits); PUT(tm->input_chunks); PUT(tm->clause_chunks);
  PUT(tm->state_chunks); PUT(tm->action_chunks); PUT(tm->specificity); PUT(tm->tail_mask);
  orc_export(tm, buf + o, NULL);
  o += tm->action_chunks;
  uint8_t ind = (uint8_t)tm->individualized;
  PUT(ind);
  if (tm->individualized)
    for (uint32_t h = 0; h < tm->classes; h++) PUT(tm->feat_sizes[h]);
  return 0;
}

#define GET(v) do { if (o + sizeof(v) > len) goto short_read; \
  memcpy(&(v), buf + o, sizeof(v)); o += sizeof(v); } while (0)
orc_tm *orc_load(const uint8_t *buf, uint64_t len) {
  uint64_t o = 0;
  int32_t type;
  uint32_t classes, features, clauses, tol, maxl, target, sb, ib, ibits, ichunks, cch, sch, ach;
  double spec;
  uint8_t tail, ind;
  GET(type);
  if (type != ORC_CLASSIFIER && type != ORC_ENCODER) {
    fail("unexpected tsetlin machine type in load");
    return NULL;
  }
  GET(classes); GET(features); GET(clauses); GET(tol); GET(maxl); GET(target); GET(sb);
  GET(ib); GET(ibits); GET(ichunks); GET(cch); GET(sch); GET(ach); GET(spec); GET(tail);
  if (o + ach > len) goto short_read;
  const uint8_t *acts = buf + o;
  o += ach;
  GET(ind);
  {
    orc_tm *tm = calloc(1, sizeof(orc_tm));
    tm->type = type; tm->classes = classes; tm->features = features; tm->clauses = clauses;
    tm->clause_tolerance = tol; tm->clause_maximum = maxl; tm->target = target;
    tm->state_bits = sb; tm->include_bits = ib ? ib : 1; tm->input_bits = ibits;
    tm->input_chunks = ichunks; tm->clause_chunks = cch; tm->state_chunks = sch;
    tm->action_chunks = ach; tm->specificity = spec; tm->tail_mask = tail;
    tm->class_chunks = (classes + 7) / 8;
    tm->individualized = ind ? 1 : 0;
    tm->has_state = 0;   /* capi.c:1696: state is not persisted */
    tm->negative = 1.0 / (double)classes;
    if (!ind) {
      tm->n_aut = 1;
      tm->aut = calloc(1, sizeof(aut_t));
      aut_layout(&tm->aut[0], (uint64_t)classes * clauses, features, sb, spec);
    } else {
      tm->n_aut = classes;
      tm->aut = calloc(classes, sizeof(aut_t));
      tm->feat_sizes = calloc(classes, sizeof(uint64_t));
      for (uint32_t h = 0; h < classes; h++) {
        if (o + 8 > len) { orc_destroy(tm); goto short_read; }
        memcpy(&tm->feat_sizes[h], buf + o, 8);
        o += 8;
        aut_layout(&tm->aut[h], clauses, tm->feat_sizes[h], sb, spec);
      }
    }
    for (uint32_t h = 0; h < tm->n_aut; h++) aut_alloc(&tm->aut[h], sb);
    orc_import(tm, acts, NULL);
    return tm;
  }
short_read:
  fail("truncated model data");
  return NULL;
}

/* ------------------------------------------------------------------------ */
/* reconfigure (capi.c:1590-1673) and restrict (capi.c:752-901)              */
/* ------------------------------------------------------------------------ */
int orc_reconfigure(orc_tm *tm, uint32_t clauses, uint32_t tol, uint32_t maxl,
                    int64_t include_bits, double target, double specificity) {
  if (!tm->reusable) return fail("reconfigure requires reusable=true at creation time");
  uint32_t nc = ((clauses + 7) / 8) * 8;
  uint32_t ib = include_bits < 0 ? tm->include_bits : (uint32_t)include_bits;
  tm->clauses = nc;
  tm->clause_chunks = nc / 8;
  tm->clause_tolerance = tol;
  tm->clause_maximum = maxl;
  tm->include_bits = ib ? ib : 1;
  tm->specificity = specificity;
  tm->target = derive_target(nc, tol, target);
  uint64_t ta = 0;
  for (uint32_t h = 0; h < tm->n_aut; h++) {
    aut_t *a = &tm->aut[h];
    aut_free(a);
    uint64_t feats = a->input_bits / 2;
    aut_layout(a, tm->individualized ? nc : (uint64_t)tm->classes * nc, feats,
               tm->state_bits, specificity);
    if (aut_alloc(a, tm->state_bits)) return fail("oom");
    ta += a->rows * a->n_chunks;
  }
  tm->action_chunks = (uint32_t)ta;
  tm->state_chunks = (uint32_t)(ta * (tm->state_bits - 1));
  tm->has_state = 1;
  return 0;
}

int orc_restrict(orc_tm *tm, const int64_t *dims, uint64_t n) {
  if (!tm->individualized) return fail("restrict only supported for individualized TMs");
  if (n == 0) return fail("selected_dims cannot be empty");
  for (uint64_t i = 0; i < n; i++) {
    if (dims[i] < 0 || (uint64_t)dims[i] >= tm->classes) return fail("selected_dims out of range");
    for (uint64_t j = i + 1; j < n; j++)
      if (dims[i] == dims[j]) return fail("duplicate dimension in selected_dims");
  }
  aut_t *na = calloc(n, sizeof(aut_t));
  uint64_t *nf = calloc(n, sizeof(uint64_t));
  int *used = calloc(tm->classes, sizeof(int));
  for (uint64_t i = 0; i < n; i++) {
    na[i] = tm->aut[dims[i]];
    nf[i] = tm->feat_sizes[dims[i]];
    used[dims[i]] = 1;
  }
  for (uint32_t h = 0; h < tm->classes; h++) if (!used[h]) aut_free(&tm->aut[h]);
  free(used);
  free(tm->aut);
  free(tm->feat_sizes);
  tm->aut = na;
  tm->feat_sizes = nf;
  tm->n_aut = (uint32_t)n;
  tm->classes = (uint32_t)n;
  tm->class_chunks = (tm->classes + 7) / 8;
  uint64_t ta = 0;
  for (uint64_t i = 0; i < n; i++) ta += na[i].rows * na[i].n_chunks;
  tm->action_chunks = (uint32_t)ta;
  tm->state_chunks = (uint32_t)(ta * (tm->state_bits - 1));
  return 0;
}
