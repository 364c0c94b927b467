/*
 * CPU oracle for the santoku.tsetlin Tsetlin-machine hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links, loads or
 * calls this code.  It is used by tests/ (as the checker), by
 * __graft_entry__.smoke() (as the checker) and by bench.py's cpu_baseline
 * leg (as the timed CPU reference).
 *
 * It restates, in plain C, the algorithm of
 *   lib/santoku/tsetlin/capi.c      (clause evaluation, feedback, train,
 *                                    predict, persist/load, reconfigure,
 *                                    restrict)
 *   lib/santoku/tsetlin/automata.h  (bit-sliced saturating automata)
 * Each function cites the reference lines it follows.
 *
 * Two random-number modes:
 *   ORC_RNG_PHILOX    the keyed Philox4x32-10 draw contract shared with the
 *                     CUDA kernels (bit-exact replay; units are independent,
 *                     so OpenMP over units does not change results).
 *   ORC_RNG_REFSTRUCT the reference's own structure: one RNG stream per
 *                     OpenMP thread seeded by thread id, one Fisher-Yates
 *                     shuffle per thread per epoch, draws in the reference's
 *                     sequential order (capi.c:1136-1167).  The reference's
 *                     generator (tk_fast_random, from the un-vendored santoku
 *                     rock) is unknown; a 64-bit multiplicative congruential
 *                     generator stands in for it.  Results depend on the
 *                     thread count, exactly as the reference's do.
 */
#ifndef TM_ORACLE_H
#define TM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_CLASSIFIER 0
#define ORC_ENCODER 1

#define ORC_RNG_PHILOX 0
#define ORC_RNG_REFSTRUCT 1

typedef struct orc_tm orc_tm;

/* Derived parameters, in this order (orc_info):
 *  0 type, 1 classes, 2 features, 3 clauses, 4 clause_tolerance,
 *  5 clause_maximum, 6 target, 7 state_bits, 8 include_bits, 9 input_bits,
 *  10 input_chunks, 11 clause_chunks, 12 class_chunks, 13 state_chunks,
 *  14 action_chunks, 15 tail_mask, 16 individualized, 17 reusable,
 *  18 has_state */
#define ORC_INFO_N 19

orc_tm *orc_create(int type, uint32_t classes, uint32_t features, uint32_t clauses,
                   uint32_t clause_tolerance, uint32_t clause_maximum,
                   uint32_t state_bits, uint32_t include_bits, double target,
                   double negative, double specificity, int reusable,
                   int individualized, const int64_t *feat_offsets);
void orc_destroy(orc_tm *tm);
void orc_info(const orc_tm *tm, uint64_t *out);
double orc_negative(const orc_tm *tm);
double orc_specificity(const orc_tm *tm);
const char *orc_last_error(void);

int orc_train(orc_tm *tm, const uint8_t *x, const int64_t *labels,
              const uint8_t *codes, const int64_t *dim_offsets, uint64_t n,
              uint32_t epochs, uint64_t seed, uint32_t epoch_base, int rng_mode,
              int nthreads);

int orc_predict(const orc_tm *tm, const uint8_t *x, const int64_t *dim_offsets,
                uint64_t n, int64_t *out_classes, uint8_t *out_codes,
                int64_t *out_scores, int nthreads);

/* per-(sample, clause) literal counts / votes / outputs, for clause-level
 * parity checks (capi.c:85-146) */
int orc_clause_eval(const orc_tm *tm, const uint8_t *x, const int64_t *dim_offsets,
                    uint64_t n, uint32_t *literals, uint32_t *votes);

/* Reference byte layouts (automata.h:17-31; ind: capi.c:568-597). */
uint64_t orc_action_bytes(const orc_tm *tm);
uint64_t orc_state_bytes(const orc_tm *tm);
void orc_export(const orc_tm *tm, uint8_t *actions, uint8_t *state);
int orc_import(orc_tm *tm, const uint8_t *actions, const uint8_t *state);
void orc_setup(orc_tm *tm);

uint64_t orc_persist_size(const orc_tm *tm);
int orc_persist(const orc_tm *tm, uint8_t *buf, uint64_t cap, uint64_t *len);
orc_tm *orc_load(const uint8_t *buf, uint64_t len);

int orc_reconfigure(orc_tm *tm, uint32_t clauses, uint32_t clause_tolerance,
                    uint32_t clause_maximum, int64_t include_bits, double target,
                    double specificity);
int orc_restrict(orc_tm *tm, const int64_t *dims, uint64_t n);

/* The draw contract, exposed for tests. */
void orc_philox(const uint32_t *ctr, uint64_t key, uint32_t *out);
void orc_perm(uint64_t seed, uint32_t epoch, uint64_t n, uint32_t *out);

#ifdef __cplusplus
}
#endif
#endif
