/*
 * tsetlin_b200 -- C ABI of the B200 (sm_100a) Tsetlin-machine classifier and
 * encoder.
 *
 * Each entry point replaces one method of the reference's Lua module
 * `santoku.tsetlin` (lib/santoku/tsetlin/capi.c).  The Lua binding a
 * maintainer adds calls these with the same argument meaning and order; the
 * citation beside each declaration names the reference function it stands
 * in for.
 *
 * Conventions
 *   - Every function returns TM_OK (0) or a negative TM_ERR_* code; the
 *     message of the calling thread's last failure is tm_last_error().
 *     Nothing longjmps (the reference raises Lua errors instead).
 *   - Sizes are uint64_t.  Bit order is LSB-first within each byte and
 *     features are aligned to tm_align() == 8 bits, as in the reference.
 *   - Buffers belong to the caller.  `on_device` = 1 means the pointers are
 *     CUDA device pointers on the machine's device; 0 means host memory.
 *   - A machine lives on one device.  Calls on one machine are not
 *     thread-safe; calls on different machines are.  Every entry point
 *     leaves the calling thread's current CUDA device as it found it.
 */
#ifndef TSETLIN_B200_H
#define TSETLIN_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TM_OK 0
#define TM_ERR_ARG (-1)      /* bad argument / size mismatch */
#define TM_ERR_STATE (-2)    /* operation not valid for this machine */
#define TM_ERR_CUDA (-3)     /* CUDA runtime failure */
#define TM_ERR_OOM (-4)      /* allocation failed (host or device) */
#define TM_ERR_IO (-5)       /* file or stream error */
#define TM_ERR_DEVICE (-6)   /* a kernel reported an error status */
#define TM_ERR_BUSY (-7)     /* the server's queue is full: retry later */

#define TM_CLASSIFIER 0
#define TM_ENCODER 1

typedef struct tm_machine tm_machine;

/* Creation parameters (capi.c:627-699).  For an encoder `classes` is
 * `hidden` and `features` is `visible`. */
typedef struct tm_params {
  int32_t type;              /* TM_CLASSIFIER or TM_ENCODER */
  uint32_t classes;          /* classes / hidden */
  uint32_t features;         /* features / visible (unused when individualized) */
  uint32_t clauses;          /* per class; rounded up to a multiple of 8 */
  uint32_t clause_tolerance;
  uint32_t clause_maximum;
  uint32_t state_bits;       /* "state"; 0 means the default, 8 */
  uint32_t include_bits;     /* 0 means the default, 1 */
  double target;             /* < 0: sqrt(clauses / 2) * clause_tolerance */
  double negative;           /* < 0: 1 / classes */
  double specificity;
  int32_t reusable;
  int32_t individualized;
  const int64_t *feat_offsets; /* classes + 1 entries when individualized */
  uint64_t seed;             /* key of the Philox draw contract */
  int32_t device;            /* CUDA device ordinal */
} tm_params;

/* Per-epoch callback: the reference's `each(epoch)` (capi.c:1168-1182).
 * Return 0 to continue, non-zero to stop training (the reference stops on
 * `false` or on an error raised by the callback). */
typedef int (*tm_epoch_cb)(void *user, uint32_t epoch);

/* Train arguments (capi.c:1116-1126, 1197-1214, 1288-1297, 1388-1398). */
typedef struct tm_train_args {
  uint64_t samples;
  const uint8_t *problems;     /* classifier `problems` / encoder `sentences` */
  const int64_t *solutions;    /* classifier labels */
  const uint8_t *codes;        /* encoder target codes, ceil(hidden/8) B/sample */
  const int64_t *dim_offsets;  /* individualized: byte offset of class h's block */
  uint32_t iterations;
  tm_epoch_cb each;
  void *each_user;
  int32_t on_device;           /* problems/solutions/codes are device pointers */
  int32_t has_seed;            /* 1: use `seed` instead of the machine's */
  uint64_t seed;
  /* Train only the units of classes [class_begin, class_end) (0, 0: all).
   * Units are independent and every draw is keyed, so ranks that each train
   * a class range and then exchange those classes' automata hold exactly
   * the single-GPU result (the multi-GPU split of one machine).  No
   * counterpart in the reference. */
  uint32_t class_begin;
  uint32_t class_end;
} tm_train_args;

/* Reconfigure arguments (capi.c:1590-1673). */
typedef struct tm_reconfig {
  uint32_t clauses;
  uint32_t clause_tolerance;
  uint32_t clause_maximum;
  int64_t include_bits;        /* < 0: keep the current value */
  double target;               /* < 0: default */
  double specificity;
} tm_reconfig;

/* Fills defaults: state_bits 8, include_bits 1, target -1, negative -1. */
void tm_params_init(tm_params *p);

/* tsetlin.create("classifier"|"encoder", tbl): capi.c:701-716 */
int tm_create(const tm_params *p, tm_machine **out);

/* machine:train(tbl): capi.c:1484-1507 */
int tm_train(tm_machine *m, const tm_train_args *a);

/* Trains `count` independent machines in one persistent launch per epoch
 * group.  Each machine trains exactly as tm_train would train it alone.
 * Has no single counterpart in the reference: it batches the trials of one
 * search round (optimize.lua:424-471, which calls capi.c:1484-1507 once per
 * trial).  `args[i]` belongs to `machines[i]`; callbacks are not allowed
 * here (use tm_train for per-epoch control). */
int tm_train_batch(tm_machine *const *machines, const tm_train_args *args, uint32_t count);

/* Per-epoch callback of a batch: after local epoch `epoch` (1-based) of the
 * machines still training, set stop[i] = 1 to stop machine i (it keeps its
 * state as of that epoch); return non-zero to stop every machine.  Plays
 * the role of each trial's `each` in the reference's search driver
 * (optimize.lua:586-653). */
typedef int (*tm_batch_epoch_cb)(void *user, uint32_t epoch, int32_t *stop, uint32_t count);

/* tm_train_batch with per-epoch control: every machine ends exactly as
 * tm_train would leave it with an `each` that stops it at the same epoch.
 * No single counterpart in the reference (see tm_train_batch). */
int tm_train_batch_each(tm_machine *const *machines, const tm_train_args *args, uint32_t count,
                        tm_batch_epoch_cb each, void *user);

/* ---- device-resident search round ----------------------------------------
 * One round of the reference's hyper-parameter search for `count` machines
 * at once: every trial trains with train_tm's per-epoch logic
 * (optimize.lua:586-653) -- after each epoch the machine is scored on a
 * holdout, a score above best + tolerance is kept (and, with patience > 0,
 * the actions are checkpointed), `patience` epochs without one stop the
 * machine, and at the end a machine with a checkpoint is restored to it
 * and scored again.  The search metric is computed on the device: the
 * reference's usual search_metric, evaluator.class_accuracy(...).f1
 * (evaluator/capi.c:119-202), the fraction of correct classes, or
 * encoding_accuracy(...).mean_hamming for encoders (:497-574).  Each epoch
 * of all machines is one CUDA graph replay and one host synchronisation.
 * Every machine ends exactly as tm_train with the same `each` logic would
 * leave it.  No single counterpart in the reference. */
#define TM_METRIC_F1 0        /* classifier: macro F1 of class_accuracy */
#define TM_METRIC_ACCURACY 1  /* classifier: correct / test_samples */
#define TM_METRIC_HAMMING 2   /* encoder: mean_hamming of encoding_accuracy */

/* After each epoch: scores[i] is machine i's score this epoch (NaN if it
 * did not train), training[i] whether it trains on; set stop[i] = 1 to stop
 * machine i, return non-zero to stop all. */
typedef int (*tm_search_epoch_cb)(void *user, uint32_t epoch, const double *scores,
                                  const int32_t *training, int32_t *stop, uint32_t count);

typedef struct tm_search_args {
  uint64_t test_samples;
  const uint8_t *test_problems;       /* classifier problems / encoder sentences */
  const int64_t *test_solutions;      /* classifier labels */
  const uint8_t *test_codes;          /* encoder codes */
  const int64_t *test_dim_offsets;    /* individualized machines */
  const uint8_t *const *test_each;    /* optional: machine i's own holdout rows (machines whose
                                         literal layouts differ), else test_problems for all */
  int32_t on_device;                  /* test buffers are device pointers */
  int32_t metric;                     /* TM_METRIC_* */
  uint32_t patience;                  /* search_patience; 0: no early stop, no checkpoint */
  double tolerance;                   /* search_tolerance */
  tm_search_epoch_cb each;            /* optional */
  void *each_user;
  /* outputs (host arrays, each may be NULL) */
  double *scores;          /* [count * max iterations] per-epoch scores, NaN where untrained */
  double *final_scores;    /* [count] score of the machine as it ends */
  double *best_scores;     /* [count] */
  uint32_t *epochs_run;    /* [count] */
  uint32_t *best_epochs;   /* [count] 1-based epoch of the best score */
} tm_search_args;

int tm_train_batch_search(tm_machine *const *machines, const tm_train_args *args, uint32_t count,
                          const tm_search_args *search);

/* machine:predict(problems, n) / (problems, dim_offsets, n): capi.c:1088-1110.
 * Classifier: out_classes[n] (int64, argmax, ties to the lowest class).
 * Encoder: out_codes[n * ceil(hidden/8)].
 * Up to 32 samples run a kernel that reads every clause row once; large
 * predicts of dense machines run as an 8-bit tensor-core GEMM of action and
 * literal bytes (exact integer accumulation: the same results), which keeps
 * a byte copy of the actions on the device (classes x clauses x 32 row
 * words bytes) until the automata change. */
int tm_predict(tm_machine *m, const uint8_t *problems, const int64_t *dim_offsets, uint64_t n,
               int64_t *out_classes, uint8_t *out_codes, int32_t on_device);

/* Per-class vote sums, out_scores[n * classes] (int64): the `sums` /
 * `votes` arrays of capi.c:924-933 and :968-981 before argmax / sign. */
int tm_predict_scores(tm_machine *m, const uint8_t *problems, const int64_t *dim_offsets,
                      uint64_t n, int64_t *out_scores, int32_t on_device);

/* machine:persist(path): capi.c:1538-1562.  Byte-identical file layout. */
int tm_persist(tm_machine *m, const char *path);
/* machine:persist() returning a string: *data is malloc'd; release with tm_free. */
int tm_persist_buf(tm_machine *m, uint8_t **data, uint64_t *len);
void tm_free(void *p);

/* tsetlin.load(data, from_string): capi.c:1751-1772.  from_string = 0:
 * `data` is a NUL-terminated path and `len` is ignored. */
int tm_load(const uint8_t *data, uint64_t len, int32_t from_string, int32_t device,
            tm_machine **out);

/* Versioned save with optional automaton state.  No counterpart in the
 * reference: its record (tm_persist) has no version field and drops the
 * count planes (capi.c:1509-1531, 1696), so a loaded machine cannot train
 * and files cannot evolve.  The container holds a magic "STMV", a format
 * version, `negative`, the default seed and the reusable flag, the
 * reference's record byte for byte, the count planes when flags has
 * TM_SAVE_STATE, and an FNV-1a 64 checksum.  tm_load reads both this
 * container and the reference's plain record; a machine loaded with state
 * trains, reconfigures and exports state like the one that was saved.
 * tm_save_buf returns a malloc'd buffer (release with tm_free). */
#define TM_SAVE_STATE 1u
int tm_save(tm_machine *m, const char *path, uint32_t flags);
int tm_save_buf(tm_machine *m, uint32_t flags, uint8_t **data, uint64_t *len);

/* machine:checkpoint(cvec) / machine:restore(cvec): capi.c:1564-1588.
 * The checkpoint is the reference's action bytes (action_chunks bytes).
 * With buf == NULL, *len receives the size. */
int tm_checkpoint(tm_machine *m, uint8_t *buf, uint64_t cap, uint64_t *len);
int tm_restore(tm_machine *m, const uint8_t *buf, uint64_t len);

/* machine:reconfigure(tbl): capi.c:1590-1673 */
int tm_reconfigure(tm_machine *m, const tm_reconfig *r);

/* machine:restrict(selected_dims): capi.c:752-901 */
int tm_restrict(tm_machine *m, const int64_t *dims, uint64_t n);

/* machine:type(): capi.c:1774-1788 -- TM_CLASSIFIER or TM_ENCODER */
int tm_type(const tm_machine *m);

/* machine:destroy() / __gc: capi.c:725-750 */
void tm_destroy(tm_machine *m);

const char *tm_last_error(void);

/* tsetlin.align: capi.c:1801-1802 */
uint32_t tm_align(void);

/* Derived parameters, the fields of the reference's machine struct
 * (capi.c:45-83): type, classes, features, clauses, clause_tolerance,
 * clause_maximum, target, state_bits, include_bits, input_bits,
 * input_chunks, clause_chunks, class_chunks, state_chunks, action_chunks,
 * tail_mask, individualized, reusable, has_state. */
#define TM_INFO_N 19
int tm_get_info(const tm_machine *m, uint64_t *out);

/* The machine's automata in the reference's byte layouts
 * (automata.h:17-31; individualized: capi.c:568-597): actions
 * [action_chunks] and count planes [state_chunks].  Either may be NULL. */
int tm_export_state(tm_machine *m, uint8_t *actions, uint8_t *state);
int tm_import_state(tm_machine *m, const uint8_t *actions, const uint8_t *state);

/* The slice of tm_export_state's two buffers that classes [class_begin,
 * class_end) occupy (their clause rows, in the same byte layout), copied
 * out of or into the machine.  `on_device` = 1: actions / state are device
 * pointers on the machine's device and the copies stay on the device.  The
 * unit of the multi-GPU exchange after a class-sharded training (each rank
 * trains a class range, then all ranks all-gather these slices device to
 * device).  No counterpart in the reference. */
int tm_export_classes(tm_machine *m, uint32_t class_begin, uint32_t class_end, uint8_t *actions,
                      uint8_t *state, int32_t on_device);
int tm_import_classes(tm_machine *m, uint32_t class_begin, uint32_t class_end,
                      const uint8_t *actions, const uint8_t *state, int32_t on_device);

/* ---- evaluator metrics and input packing (device) --------------------- */
/* evaluator.class_accuracy(predicted, expected, n_samples, n_classes):
 * evaluator/capi.c:119-202.  out[3 + 3 * n_classes] = macro precision,
 * recall, f1, then per class precision, recall, f1. */
int tm_class_accuracy(const int64_t *predicted, const int64_t *expected, uint64_t n,
                      uint32_t classes, int32_t on_device, int32_t device, double *out);
/* evaluator.encoding_accuracy(predicted, expected, n_samples, n_hidden):
 * evaluator/capi.c:497-574.  out[4 + n_hidden] = mean_hamming, ber_min,
 * ber_max, ber_std, then the per-bit error rates. */
int tm_encoding_accuracy(const uint8_t *predicted, const uint8_t *expected, uint64_t n,
                         uint32_t hidden, int32_t on_device, int32_t device, double *out);
/* santoku-matrix's bits_to_cvec(n, features, flip) on the set-bit list
 * `sample * features + feature` (as built by the reference's dataset
 * readers, dataset.lua:11-41): out[n * ceil((flip ? 2 : 1) * features / 8)];
 * with flip, bits features..2*features-1 are the complements
 * (doc/sth.md:70-78).  The input packing of the reference's tests. */
int tm_bits_to_cvec(const int64_t *set_bits, uint64_t n_set, uint64_t n, uint32_t features,
                    int32_t flip, int32_t on_device, int32_t device, uint8_t *out);

/* santoku-matrix's bits_to_cvec_ind(ind_offsets, feat_offsets, n, flip): the
 * individualized sample layout the reference reads at capi.c:1020-1023,
 * 1344-1354 and 1440-1451 (doc/sth.md:42-54).  Dimension h (a class, or a
 * code bit of an encoder) has k_h = feat_offsets[h+1] - feat_offsets[h]
 * features; its set bits are set_bits[ind_offsets[h] - ind_offsets[0] ..
 * ind_offsets[h+1] - ind_offsets[0]) as `sample * k_h + feature` (negative
 * entries and samples >= n are skipped).  Block h holds n rows of
 * ceil((flip ? 2 : 1) * k_h / 8) bytes (flip: bits k_h..2k_h-1 are the
 * complements) and starts at byte dim_offsets[h]; dim_offsets (host,
 * dims + 1 entries) ends with the total size.  ind_offsets and feat_offsets
 * are host arrays of dims + 1 entries; set_bits and out are device pointers
 * when on_device.  out == NULL only fills dim_offsets (a sizing call);
 * out_cap smaller than the total fails with TM_ERR_ARG. */
int tm_bits_to_cvec_ind(const int64_t *set_bits, const int64_t *ind_offsets,
                        const int64_t *feat_offsets, uint32_t dims, uint64_t n, int32_t flip,
                        int32_t on_device, int32_t device, uint8_t *out, uint64_t out_cap,
                        int64_t *dim_offsets);

/* Integer-pipe peaks of `device`, measured by microbenchmark kernels (16
 * independent inline-PTX chains per thread, 8 CTAs of 256 threads per SM,
 * timed with CUDA events): out[0] lop3.b32, out[1] popc.b32, out[2]
 * add.u32, in thread-operations per second.  The roofline denominators of
 * the bit-logic kernels.  No counterpart in the reference. */
int tm_int_peaks(int32_t device, double *out);

/* Predict without allocating.  No counterpart in the reference.  For
 * callers that must not call cudaMalloc / cudaFree while they run -- a
 * serving loop that cannot absorb the device-wide synchronisation those
 * calls cause, or an application whose own allocator already holds the GPU's
 * memory.  Works in one fixed 8 MiB scratch array compiled into the library
 * (held on every GPU that loads it until the process exits) instead of
 * buffers grown on demand.  Dense machines only; `problems` and the output
 * are device pointers; n * (row words * 4 + classes * 4) plus 256 bytes of
 * alignment must fit in 8 MiB, larger requests fail with TM_ERR_ARG.  The
 * first call on a device looks up the scratch array's device address (call
 * it once before any stream capture).  Calls share the array: calls whose
 * work overlaps on the GPU race.  Results equal tm_predict's. */
int tm_predict_noalloc(tm_machine *m, const uint8_t *problems, uint64_t n, int64_t *out_classes,
                       uint8_t *out_codes);

/* ---- instrumentation ------------------------------------------------------ */
/* Device-time accounting of the library's kernels for one machine, taken
 * with CUDA events on the machine's own stream.  The reference's analogue
 * is its perf build variant (make.perf.lua). */
typedef struct tm_stats {
  uint64_t train_launches;    /* fused train kernel launches */
  double train_kernel_ms;     /* their summed device time */
  uint64_t predict_launches;  /* predict (clause evaluation) kernel launches */
  double predict_kernel_ms;
  uint64_t kernel_launches;   /* every kernel the library launched */
  uint64_t train_unit_steps;  /* (unit, sample) steps examined by train kernels */
  int32_t train_mode;         /* last train kernel variant: 0 automata in shared memory,
                                 1 count planes in global memory, 2 split over a 2-CTA
                                 cluster, 3 one warp per unit (rows of at most 64 words),
                                 4 words owned by threads (automata in registers and
                                 shared memory) */
  int32_t train_autotuned;    /* 1 if the autotuner chose that variant */
  int32_t train_cpw;          /* modes 0-2: clauses per warp; mode 3: 1 = four units per
                                 CTA, 2 = one; mode 4: the configuration (1-7) */
  int32_t predict_gemm;       /* last predict: 0 bitwise kernels, 1 int8 GEMM, 2 e4m3 GEMM */
  uint64_t train_active_pairs; /* (unit, sample) steps trained after negative sampling */
  double search_epoch_ms;     /* device-resident search rounds: summed epoch graph time */
  uint64_t search_epochs;     /* epoch graph replays */
  double search_train_ms;     /* the train kernel's share of those replays */
  uint64_t train_resident;    /* units resident at once in the last train launch */
} tm_stats;
/* Train-kernel variant choice.  All variants end in the same automaton
 * state; they differ in speed.  mode 0: heuristic (resident CTAs per SM);
 * 1 (default, or TSETLIN_B200_AUTOTUNE at create): the first train call of
 * a launch shape times every feasible variant on a short trial (up to 2,048
 * samples of epoch 0 on up to 32 units per SM taken evenly from the launch's
 * work list, from the initial automata), then the three fastest on a longer
 * one (8,192 samples, 64 units per SM: positions 8,192-16,383 of epoch 0
 * from the automata as the first 8,192 leave them, or the first 8,192 from
 * the initial state for shorter launches) -- the automata are reset to the
 * initial state afterwards -- and caches the fastest for
 * the process; 2: tune on every train call.  No counterpart in the
 * reference (it has one CPU code path). */
int tm_set_autotune(tm_machine *m, int32_t mode);

/* Pins the train-kernel variant (train_mode values of tm_stats; cpw, the
 * clauses evaluated per warp in a single-CTA variant with 8 state bits: 1,
 * 2 or 4 -- 256 / cpw threads per unit; for mode 3, 1 or 2: four units or
 * one per CTA; for mode 4, the configuration); mode -1 returns to the automatic
 * choice.  A train call that the pinned variant cannot run fails with
 * TM_ERR_ARG.  The environment variable TSETLIN_B200_VARIANT=mode:cpw, read
 * when a machine is created, pins the same way.  For tests and
 * measurements; no counterpart in the reference. */
int tm_force_variant(tm_machine *m, int32_t mode, int32_t cpw);

/* Failure injection for tests of the error paths: after `after` more
 * successful device allocations, the next one the library makes fails as if
 * the GPU were out of memory (the call reports TM_ERR_OOM); then the
 * injection disarms itself.  after < 0 disarms it.  No counterpart in the
 * reference. */
int tm_debug_fail_alloc(int64_t after);

/* on != 0 starts timing (events around every train / predict kernel). */
int tm_stats_enable(tm_machine *m, int32_t on);
int tm_get_stats(const tm_machine *m, tm_stats *out);
int tm_reset_stats(tm_machine *m);

/* ---- serving: resident machines, continuous batching ------------------- */
/* No counterpart in the reference (its predict is one synchronous call per
 * batch, capi.c:1088-1110).  A server keeps machines resident, accepts
 * predict requests at any time, and packs queued requests -- for any of its
 * machines, in arrival order -- into shared device launches as launch slots
 * and its device-memory budget allow; each request completes with exactly
 * the result tm_predict gives for it alone.  Large requests of dense
 * machines run as the 8-bit GEMM tm_predict uses: the server holds each
 * dense machine's action bytes (outside hbm_budget_bytes) while open, and
 * the machines must not train meanwhile. */
typedef struct tm_server tm_server;

typedef struct tm_server_config {
  uint64_t hbm_budget_bytes;   /* memory of the launch slots (inputs, outputs, GEMM chunks) */
  uint32_t max_inflight;       /* launch slots on the device at once */
  uint32_t max_batch_samples;  /* samples packed into one launch slot */
  int32_t device;
  int32_t reserved;
  uint64_t max_queued_samples; /* samples waiting for a slot before submit refuses
                                  (TM_ERR_BUSY); 0: 64 x max_batch_samples */
} tm_server_config;

int tm_serve_open(const tm_server_config *cfg, tm_machine *const *machines, uint32_t count,
                  tm_server **out);
/* Queues a request; the input is copied before return (and dropped once it
 * is staged for the device).  Returns a request id in *id.  Fails with
 * TM_ERR_OOM if the request alone exceeds a launch slot, TM_ERR_BUSY if the
 * queue is full. */
int tm_serve_submit(tm_server *s, uint32_t machine, const uint8_t *problems, uint64_t n,
                    uint64_t *id);
/* Non-blocking: 1 when done (result copied to out_classes / out_codes; the
 * request is released and its id becomes unknown to later polls), 0 while
 * pending.  timeout_us > 0 waits up to that long. */
int tm_serve_poll(tm_server *s, uint64_t id, int64_t *out_classes, uint8_t *out_codes,
                  uint64_t timeout_us);
/* submit -> done latency of a completed request, microseconds (also after
 * it was polled, for the last 65,536 polled requests) */
int tm_serve_latency_us(tm_server *s, uint64_t id, double *us);
/* out[4], microseconds: the same request's latency in three phases --
 * out[0] the wait in the queue (submit -> taken by the worker), out[1] the
 * host's staging and launch calls for its launch slot, out[2] the device
 * work and the completion (launches queued -> done), which add up to the
 * latency -- and out[3] the device span of its launch, from the copy in to
 * the end of the copy out, measured with CUDA events */
int tm_serve_phases_us(tm_server *s, uint64_t id, double *out);
/* out[5]: queued requests, queued samples, requests not yet polled, busy
 * launch slots, launch slots */
int tm_serve_stats(tm_server *s, uint64_t *out);
int tm_serve_close(tm_server *s);

#ifdef __cplusplus
}
#endif
#endif
