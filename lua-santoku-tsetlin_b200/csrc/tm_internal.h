// Internal types shared by the host library (tm_api.cpp) and the kernels
// (tm_kernels.cu).  Not part of the C ABI.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace tmb {

// Device layout of one class's automata and samples.  Every clause row of
// the reference's byte layout (input_chunks bytes, automata.h:17-31) is held
// as little-endian 32-bit words, padded to Wp words (a multiple of 4, so
// each row starts on a 16-byte boundary for TMA bulk copies and 128-bit
// loads).  Count planes are [clause][plane][Wp] -- the reference's order.
struct ClassDev {
  uint64_t act_off;    // words: first clause row of this class in act[]
  uint64_t cnt_off;    // words: first clause's plane 0 in cnt[]
  uint64_t x_off;      // words: this class's sample block in x[]
  uint32_t W;          // words holding reference bytes
  uint32_t Wp;         // padded row stride (words)
  uint32_t input_bits; // 2 * features of this class
  uint32_t s_picks;    // Type Ib picks per event, (unsigned)((double)(2F)/specificity)
  uint32_t vmask;      // word W-1: bits of bytes that exist
  uint32_t emask;      // word W-1: evaluation mask (tail byte & tail_mask)
  uint32_t amask;      // word W-1: carry mask into the action plane
  uint32_t pad;
};

// One machine of a training launch.
struct TrainDev {
  uint32_t *act;
  uint32_t *cnt;
  const uint32_t *x;        // padded sample rows
  const int32_t *labels;    // classifier
  const uint8_t *codes;     // encoder
  const uint32_t *perm;     // [epochs][n] sample order
  const ClassDev *cls;      // [classes]
  uint64_t seed;
  uint64_t thr_neg;         // skip a non-target sample iff draw < thr_neg
  uint32_t n;
  uint32_t classes;
  uint32_t clause_chunks;   // chunks of 8 clauses per class
  uint32_t B;               // state bits
  uint32_t ib;              // include bits
  uint32_t tol;
  uint32_t maxlit;
  uint32_t T;               // target
  uint32_t type;            // 0 classifier, 1 encoder
  uint32_t code_bytes;
  uint32_t epochs;          // epochs this machine trains in this launch group
  uint32_t epoch_base;      // draw-contract epoch index of local epoch 0
  const uint32_t *gate;     // optional: the machine's units are skipped while *gate == 0
};

struct WorkItem {
  uint32_t m;   // machine index in the launch
  uint32_t h;   // class
  uint32_t k;   // chunk within the class
  uint32_t cost;
};

// Shared-memory plan of one training launch (byte offsets).
struct TrainSmem {
  uint32_t state_off, state_words;  // per-unit state copy (global-planes variant: actions only)
  uint32_t ring_off, ring_words;    // sample ring: TM_RING slots of ring_words
  uint32_t bar_off;                 // TM_RING mbarriers
  uint32_t list_off;                // active-sample list
  uint32_t votes_off;               // 2 x 8 x 2 clause partial sums
  uint32_t ib_off, ib_words;        // TM_IB_SLOTS slots: 2 levels x ib_words
  uint32_t ovf_off, ovf_cap;        // TM_IB_SLOTS slots: overflow entries
  uint32_t misc_off;
  uint32_t total;
  // try-wait iterations a thread spends on a sample row before it reports
  // the copy as lost (TM_ERR_DEVICE); the drain of copies still in flight
  // at exit always uses the full limit
  uint32_t wait_limit;
};

constexpr uint32_t TM_WAIT_LIMIT = 1u << 22;

constexpr int TM_TRAIN_THREADS = 256;  // 8 warps: warp j owns clause j of the unit
constexpr int TM_RING = 3;             // sample ring depth
constexpr int TM_IB_SLOTS = 2;         // Type Ib level-counter slots per CTA
constexpr int TM_BATCH = 256;          // samples examined per batch phase

// Draw-contract stream words (4th Philox counter word).
constexpr uint32_t ST_NEG = 0u;
constexpr uint32_t ST_CH0 = 1u;
constexpr uint32_t ST_CH1 = 2u;
constexpr uint32_t ST_IB = 0x01000000u;
constexpr uint32_t ST_PERM = 0xFFFFFFFFu;

// ---- launchers (tm_kernels.cu) -------------------------------------------
// Reference byte rows -> padded words; `zero` (optional) is cleared in the
// same launch (the vote sums of the predict that follows).
cudaError_t launch_repack(const uint8_t *src, uint64_t n, uint64_t row_bytes, uint64_t src_stride,
                          uint32_t *dst, uint32_t dst_words, cudaStream_t st,
                          uint32_t *zero = nullptr, uint64_t zero_words = 0);
cudaError_t launch_labels(const int64_t *src, int32_t *dst, uint64_t n, cudaStream_t st);
cudaError_t launch_setup(uint32_t *act, uint32_t *cnt, const ClassDev *cls, uint32_t classes,
                         uint32_t clauses, uint32_t B, uint64_t act_words, cudaStream_t st);
cudaError_t launch_perm(uint64_t seed, uint32_t epoch, uint32_t n, uint32_t *out,
                        void *scratch, size_t scratch_bytes, cudaStream_t st,
                        const uint32_t *epoch_dev = nullptr);
size_t perm_scratch_bytes(uint32_t n);
// k_train variants: automata in shared memory (one CTA per unit), in global
// memory (one CTA per unit), or split over a 2-CTA cluster in shared memory.
constexpr int TM_MODE_SMEM = 0;
constexpr int TM_MODE_GLOBAL = 1;
constexpr int TM_MODE_PAIR = 2;
cudaError_t launch_train(const TrainDev *machines, const WorkItem *work, uint32_t nwork,
                         uint32_t *counter, uint32_t e_begin, uint32_t e_end, const TrainSmem &lay,
                         int mode, uint32_t Bmin, uint32_t Bmax, int cpw, int grid,
                         uint32_t *err, cudaStream_t st);
int train_occupancy(const TrainSmem &lay, int mode, uint32_t Bmin, uint32_t Bmax, int cpw);
// threads per CTA of a train-kernel variant (cpw: clauses per warp)
int train_threads(int mode, int cpw);
// k_train_warp: one warp per unit for rows of at most 64 words and B <= 8,
// wpc (4 or 1) units per CTA
constexpr int TM_MODE_WARP = 3;
int train_warp_occupancy(uint32_t Wpmax, uint32_t Bmin, uint32_t Bmax, uint32_t smax, int wpc,
                         size_t *smem_bytes);
cudaError_t launch_train_warp(const TrainDev *machines, const WorkItem *work, uint32_t nwork,
                              uint32_t *counter, uint32_t e_begin, uint32_t e_end, uint32_t Wpmax,
                              uint32_t Bmin, uint32_t Bmax, uint32_t smax, int wpc, int grid,
                              cudaStream_t st, unsigned long long *pairs);
// Large-batch predict as an 8-bit GEMM (tm_gemm.cu)
constexpr int TM_GEMM_INT8 = 1;  // int8 operands, int32 accumulation
constexpr int TM_GEMM_FP8 = 2;   // e4m3 operands, fp32 accumulation
cudaError_t launch_expand_bits(const uint32_t *src, uint64_t rows, uint32_t stride, uint32_t W,
                               uint32_t last_mask, int kind, uint8_t *dst, cudaStream_t st);
// gate (optional, device): the kernel writes nothing while *gate == 0
cudaError_t launch_gemm_votes(const void *C, int kind, const int32_t *lits, uint32_t classes,
                              uint32_t clauses, uint32_t tol, uint32_t N, int32_t *sums,
                              cudaStream_t st, const uint32_t *gate = nullptr);
int gemm_clause_products(int dev, int kind, const uint8_t *A, const uint8_t *B, void *C,
                         uint64_t M, uint64_t N, uint64_t K, void *ws, size_t ws_bytes,
                         cudaStream_t st);
// The product width for k samples: the next power of two from 64, at most
// `cap` (the chunk size).  Products are asked for in these few widths (the
// columns past k are not read), so the library's choice and its kernels are
// set up once per width.
uint64_t gemm_bucket(uint64_t k, uint64_t cap);
// The fused train kernels report through err[0] (status bits) and
// err[2..3], a 64-bit count of active (unit, sample) steps -- the samples
// each unit actually trained on after negative sampling.
// k_train_wpt (tm_train_wpt.cu): one CTA per unit, every thread owning a
// few words of all eight clauses, the automata held in registers and shared
// memory; `cpw` of a plan with this mode is the configuration id (1-based).
constexpr int TM_MODE_WPT = 4;
int wpt_configs();
int train_wpt_occupancy(int id, uint32_t Wpmax, uint32_t smax, size_t *smem_bytes);
cudaError_t launch_train_wpt(int id, const TrainDev *machines, const WorkItem *work,
                             uint32_t nwork, uint32_t *counter, uint32_t e_begin, uint32_t e_end,
                             uint32_t Wpmax, uint32_t smax, uint32_t wait_limit, int grid,
                             uint32_t *err, cudaStream_t st);
cudaError_t launch_lits(const uint32_t *act, const ClassDev *cls, uint32_t classes,
                        uint32_t clauses, int32_t *lits, cudaStream_t st);
cudaError_t launch_predict(const uint32_t *act, const int32_t *lits, const ClassDev *cls,
                           const ClassDev *cls_host, uint32_t classes, uint32_t clauses,
                           uint32_t tol, const uint32_t *x, uint32_t n, int32_t *sums,
                           cudaStream_t st);
cudaError_t launch_finalize(const int32_t *sums, uint32_t n, uint32_t classes, int32_t type,
                            int64_t *out_classes, uint8_t *out_codes, int64_t *out_scores,
                            cudaStream_t st);


// One predict job of a multi-job launch (k_predict_multi): a machine's
// resident automata scored against n padded sample rows.  Its tiles are
// blocks tile0 .. tile0 + stiles * classes * tpc - 1 of the launch.
struct PredictJob {
  const uint32_t *act;
  const int32_t *lits;
  const ClassDev *cls;
  const uint32_t *x;
  int32_t *sums;          // n x classes, accumulated (zeroed by the caller)
  const uint32_t *gate;   // optional: the job runs only while *gate != 0
  uint32_t clauses, tpc, tol, n, classes;
  uint32_t tile0, stiles;
  uint32_t pad;
};
// tiles of one predict job (64 samples x 64 clauses each)
uint32_t predict_job_tiles(uint32_t n, uint32_t classes, uint32_t clauses, uint32_t *stiles,
                           uint32_t *tpc);
cudaError_t launch_predict_multi(const PredictJob *jobs_dev, uint32_t njobs, uint32_t total_tiles,
                                 cudaStream_t st);
// A small predict job (k_predict_small_multi): samples s0 .. s0 + ns - 1
// (ns <= 16) of x against a machine; blocks block0 .. block0 + classes *
// cblocks - 1 of the launch.
struct SmallJob {
  const uint32_t *act;
  const int32_t *lits;
  const ClassDev *cls;
  const uint32_t *x;
  int32_t *sums;
  uint32_t clauses, tol, classes, s0, ns, cblocks, block0, pad;
};
uint32_t small_job_blocks(uint32_t classes, uint32_t clauses, uint32_t *cblocks);
cudaError_t launch_predict_small_multi(const SmallJob *jobs_dev, uint32_t njobs,
                                       uint32_t total_blocks, cudaStream_t st);

// One request of a serving launch: its staged byte rows, padded rows, vote
// sums and output within the launch slot's buffers.
struct ServeJob {
  const uint8_t *raw;   // n rows of row_bytes
  uint32_t *x;          // n rows of Wp words
  int32_t *sums;        // n x classes
  uint8_t *out;         // n int64 classes or n x ceil(classes / 8) code bytes
  uint64_t row_bytes;
  uint32_t n, Wp, classes, type;
};
cudaError_t launch_serve_repack(const ServeJob *jobs_dev, uint32_t njobs, cudaStream_t st);
cudaError_t launch_serve_finalize(const ServeJob *jobs_dev, uint32_t njobs, cudaStream_t st);

// Predicts of at most this many samples read each clause row once with one
// warp per row (k_predict_small) instead of the 64 x 64 tiles.
constexpr uint32_t TM_SMALL_N_MAX = 32;
// k_lits with an optional gate (skipped while *gate == 0)
cudaError_t launch_lits_gated(const uint32_t *act, const ClassDev *cls, uint32_t classes,
                              uint32_t clauses, int32_t *lits, const uint32_t *gate,
                              cudaStream_t st);

// ---- device-resident search round (tm_train_batch_search) ----------------
// Per-machine state of the round, kept on the device and read by the host
// once per epoch.  The epoch logic of the reference's train_tm
// (optimize.lua:599-625): score, best + tolerance, patience, checkpoint.
struct SearchState {
  uint32_t live;        // still training: gates its units, its metric and its checkpoint
  uint32_t since;       // epochs since the best score improved
  uint32_t ckpt_now;    // the epoch just scored improved: checkpoint the actions
  uint32_t has_ckpt;    // a checkpoint exists: restored at the end
  uint32_t epochs_run;
  uint32_t best_epoch;  // 1-based epoch of the best score
  uint32_t patience;    // 0: no early stop and no checkpoint
  uint32_t iterations;
  double best;          // -inf before the first epoch
  double last;          // last score (after the final restore: the restored machine's)
  double tolerance;
};

// Scoring of one machine's vote sums against the truth.
struct ScoreJob {
  int32_t *sums;           // n x classes vote sums; zeroed once scored
  const int64_t *labels;   // classifier truth
  const uint8_t *codes;    // encoder truth codes, ceil(classes / 8) bytes per sample
  uint32_t n, classes, type, metric;
};

// Literal counts of one machine (k_lits), skipped while *gate == 0.
struct LitsJob {
  const uint32_t *act;
  const ClassDev *cls;
  int32_t *lits;
  const uint32_t *gate;
  uint32_t classes, clauses;
};

// A word copy run while *flag != 0 (checkpoint and restore of actions).
struct CopyJob {
  const uint32_t *src;
  uint32_t *dst;
  uint64_t words;  // a multiple of 4
  const uint32_t *flag;
};

constexpr uint32_t TM_SEARCH_MAX_CLASSES = 4000;  // counts of a score in shared memory
cudaError_t launch_lits_multi(const LitsJob *jobs, uint32_t njobs, uint32_t max_classes,
                              cudaStream_t st);
cudaError_t launch_search_score(const ScoreJob *jobs, SearchState *state, double *scores,
                                uint32_t max_epochs, uint32_t njobs, uint32_t max_classes,
                                int final_pass, cudaStream_t st);
cudaError_t launch_copy_multi(const CopyJob *jobs, uint32_t njobs, cudaStream_t st);
cudaError_t launch_tick(uint32_t *counter, cudaStream_t st);
// epoch_base += 1 of every machine of a launch's device table (a graph
// replayed once per epoch trains the next epoch on each replay)
cudaError_t launch_tick_machines(TrainDev *machines, uint32_t count, cudaStream_t st);

// Read-only view of a resident dense machine for the server (tm_serve.cpp).
struct MachineView {
  const uint32_t *act;
  const int32_t *lits;
  const ClassDev *cls;
  uint32_t classes, clauses, tol, type, input_chunks, Wp, class_chunks, W;
  int device;
  cudaStream_t st;  // the machine's own stream
  const uint8_t *act8;  // action bytes for the GEMM predict (tmb_machine_act8), or null
  int act8_kind;        // their TM_GEMM_* encoding
};

// Makes `d` the calling thread's current device for the guard's scope and
// gives the caller's device back at its end (an entry point leaves the
// caller's current device as it found it).  `err` is the result of
// switching.
struct DevGuard {
  int prev = -1;
  cudaError_t err = cudaSuccess;
  explicit DevGuard(int d) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != d) err = cudaSetDevice(d);
  }
  ~DevGuard() {
    int cur;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
  DevGuard(const DevGuard &) = delete;
  DevGuard &operator=(const DevGuard &) = delete;
};

}  // namespace tmb

struct tm_machine;
// Fills `v` (computing literal counts if needed).  Dense machines only;
// `who` names the caller in the error message.
int tmb_machine_view(tm_machine *m, tmb::MachineView *v, const char *who);
int tmb_fail(int code, const char *msg);
// Fills v->act8 / v->act8_kind with the machine's action bytes for the GEMM
// predict (built if stale, the machine's stream drained), or leaves them
// null when the device has no GEMM encoding or the machine is
// individualized.  The bytes stay valid until the automata change.
int tmb_machine_act8(tm_machine *m, tmb::MachineView *v);
// cudaMalloc behind the failure injection of tm_debug_fail_alloc
cudaError_t tmb_dev_malloc(void **p, size_t n);
