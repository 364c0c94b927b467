// Predict server: resident machines, continuous batching (tm_serve_* in
// include/tsetlin_b200.h).  No counterpart in the reference, whose predict
// is one synchronous call per batch (capi.c:1088-1110).
//
// A worker thread owns S launch slots (one CUDA stream, pinned host staging
// and device buffers each; S is bounded by max_inflight and by how many
// slots the HBM budget pays for).  Whenever a slot is free and requests are
// queued, it takes the queued requests in arrival order -- for any of the
// resident machines -- while they fit the slot (max_batch_samples, at most
// TM_SERVE_MAX_PACK requests), and outside the server lock stages their rows
// into the slot's pinned buffer (dropping each request's copy of its
// input), then launches on the slot's stream: one copy of the rows, one
// repack of every request's rows, the predict kernels of every request
// (requests of at most 32 samples as warp-per-clause jobs reading each
// clause row once, larger ones as 64 x 64 tiles; each kind for all requests
// and machines in one launch), the finalize of every request and one copy
// of the results.  Each slot has a completion thread: it sleeps on a CUDA
// event recorded behind the copy, then completes the slot's requests and
// frees the slot (the two events around the launch also give its device
// span).  Requests
// that arrive while slots are busy are admitted as slots free up, and the
// slots' streams overlap on the device.  Predict is independent per
// sample, so each request's result is the same alone or packed with
// others.  Small requests (at most TM_SERVE_SMALL samples) queue apart and
// launch on high-priority streams, so a small request does not wait behind
// the blocks of large requests already on the device.  The queues are
// bounded together (max_queued_samples): a request beyond the bound is
// refused with TM_ERR_BUSY rather than left to wait without limit.
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/tsetlin_b200.h"
#include "tm_internal.h"

using namespace tmb;
using clk = std::chrono::steady_clock;

namespace {

constexpr uint32_t TM_SERVE_MAX_PACK = 64;     // requests per launch slot
// Requests of at most this many samples are "small": they queue apart and
// launch on high-priority streams, so that the device's block scheduler
// starts their blocks ahead of those of large requests already queued
constexpr uint64_t TM_SERVE_SMALL = 256;
constexpr size_t TM_SERVE_LATENCY_KEEP = 1 << 16;  // polled requests whose latency is kept

struct Request {
  uint64_t id;
  uint32_t machine;
  uint64_t n;
  std::vector<uint8_t> input;   // dropped once staged
  std::vector<uint8_t> result;  // int64 classes or code bytes
  // submitted; taken by the worker; its slot's launches queued; completed
  clk::time_point t_submit, t_taken, t_launched, t_done;
  double gpu_us = 0;  // the device span of its launch (CUDA events)
  bool done = false;
};

// A request's phases, microseconds: submit -> done, the wait in the queue
// (submit -> taken), the host's staging and launch calls (taken ->
// launched), the device work and the completion (launched -> done).
struct Times {
  double total, queue, launch, device, gpu;
};

Times times_of(const Request &r) {
  auto us = [](clk::time_point a, clk::time_point b) {
    return std::chrono::duration<double, std::micro>(b - a).count();
  };
  return Times{us(r.t_submit, r.t_done), us(r.t_submit, r.t_taken), us(r.t_taken, r.t_launched),
               us(r.t_launched, r.t_done), r.gpu_us};
}

struct Slot {
  tm_server *srv = nullptr;
  cudaStream_t st = nullptr;
  uint8_t *h_in = nullptr, *h_out = nullptr, *h_jobs = nullptr;  // pinned
  uint8_t *d_raw = nullptr, *d_out = nullptr, *d_jobs = nullptr;
  uint32_t *d_x = nullptr;
  int32_t *d_sums = nullptr;
  // large requests through the GEMM: a chunk of sample bytes, the chunk's
  // clause x sample products, the library's workspace
  uint8_t *d_x8 = nullptr, *d_ws = nullptr;
  void *d_gc = nullptr;
  // recorded before the copy in and after the copy out (the completion
  // thread sleeps on ev1)
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::thread done_thread;
  std::vector<Request *> reqs;
  std::vector<uint64_t> out_off;  // each request's result offset in h_out
  bool busy = false;
  bool launched = false;  // queued launches wait for the completion thread
  bool high = false;      // a high-priority stream, kept for small requests
};

uint64_t round_up(uint64_t v, uint64_t a) { return (v + a - 1) / a * a; }

// The GEMM path of a slot: products of at most TM_SERVE_GEMM_C bytes per
// library call, its workspace.
constexpr uint64_t TM_SERVE_GEMM_C = 256ull << 20;
constexpr size_t TM_SERVE_GEMM_WS = 32u << 20;

// Samples per GEMM call for a machine of M clauses (a multiple of 64).
uint64_t gemm_chunk(uint64_t M) {
  return std::max<uint64_t>(64, TM_SERVE_GEMM_C / (4 * M) / 64 * 64);
}

// Whether a request goes through the GEMM (as the single-machine predict
// decides: past the small-batch sizes, at least 2^28 clause x sample x row
// word products).
bool gemm_request(const MachineView &v, uint64_t n) {
  return v.act8 && n > TM_SMALL_N_MAX &&
         (uint64_t)v.classes * v.clauses * n * v.W >= (1ull << 28);
}

}  // namespace

struct tm_server {
  tm_server_config cfg{};
  std::vector<MachineView> mv;
  std::vector<Slot> slots;
  uint64_t cap_in = 0, cap_out = 0, cap_x = 0, cap_sums = 0, cap_jobs = 0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done, cv_launched;
  std::deque<Request *> queue;    // large requests, arrival order
  std::deque<Request *> squeue;   // small requests, arrival order
  uint64_t queued_samples = 0;
  std::unordered_map<uint64_t, Request *> live;  // submitted, not yet polled done
  std::unordered_map<uint64_t, Times> latency;    // polled requests' phases
  std::deque<uint64_t> latency_order;
  uint64_t next_id = 1;
  bool stop = false;
  bool closing = false;  // the completion threads end once their slot is idle
  std::thread worker;
  int error = 0;
};

static uint64_t out_bytes(const MachineView &v, uint64_t n) {
  return v.type == TM_CLASSIFIER ? n * 8 : n * v.class_chunks;
}

// A slot's completion thread: for every launch of the slot, it waits (asleep)
// for the event recorded behind the result copy, then completes the
// launch's requests and frees the slot.  It ends when the server closes and
// the slot holds no launch.
static void slot_main(tm_server *s, Slot *sl) {
  cudaSetDevice(s->cfg.device);
  std::unique_lock<std::mutex> lk(s->mu);
  while (true) {
    s->cv_launched.wait(lk, [&] { return sl->launched || s->closing; });
    if (!sl->launched) break;
    lk.unlock();
    cudaError_t e = cudaEventSynchronize(sl->ev1);
    const clk::time_point now = clk::now();
    float ms = 0;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, sl->ev0, sl->ev1);
    lk.lock();
    if (e != cudaSuccess) {
      // the requests stay not done; polls report the failure
      s->error = TM_ERR_CUDA;
      s->stop = true;
    } else {
      for (size_t i = 0; i < sl->reqs.size(); i++) {
        Request *r = sl->reqs[i];
        const uint64_t b = out_bytes(s->mv[r->machine], r->n);
        r->result.assign(sl->h_out + sl->out_off[i], sl->h_out + sl->out_off[i] + b);
        r->t_done = now;
        r->gpu_us = 1e3 * ms;
        r->done = true;
      }
      sl->busy = false;
    }
    sl->reqs.clear();
    sl->launched = false;
    s->cv_done.notify_all();
    s->cv_work.notify_all();
  }
}

// Stages the slot's requests and queues its launches (called without the
// server lock: the slot and its requests belong to the worker until the
// slot's completion thread takes them).
static cudaError_t launch_slot(tm_server *s, Slot &sl) {
  const uint32_t R = (uint32_t)sl.reqs.size();
  const clk::time_point taken = clk::now();
  for (Request *r : sl.reqs) r->t_taken = taken;
  ServeJob *sj = (ServeJob *)sl.h_jobs;
  SmallJob *mj = (SmallJob *)(sl.h_jobs + round_up(TM_SERVE_MAX_PACK * sizeof(ServeJob), 256));
  PredictJob *pj = (PredictJob *)((uint8_t *)mj +
                                  round_up(2 * TM_SERVE_MAX_PACK * sizeof(SmallJob), 256));
  const size_t o_mj = (uint8_t *)mj - sl.h_jobs, o_pj = (uint8_t *)pj - sl.h_jobs;
  uint64_t in_off = 0, x_off = 0, s_off = 0, o_off = 0;
  uint32_t nsmall = 0, npred = 0, small_blocks = 0, tiles = 0;
  sl.out_off.assign(R, 0);
  for (uint32_t i = 0; i < R; i++) {
    Request *r = sl.reqs[i];
    const MachineView &v = s->mv[r->machine];
    memcpy(sl.h_in + in_off, r->input.data(), r->input.size());
    std::vector<uint8_t>().swap(r->input);
    ServeJob &J = sj[i];
    J.raw = sl.d_raw + in_off;
    J.x = sl.d_x + x_off;
    J.sums = sl.d_sums + s_off;
    J.out = sl.d_out + o_off;
    J.row_bytes = v.input_chunks;
    J.n = (uint32_t)r->n;
    J.Wp = v.Wp;
    J.classes = v.classes;
    J.type = v.type;
    if (gemm_request(v, r->n)) {
      // after the repack, below
    } else if (r->n <= TM_SMALL_N_MAX) {
      for (uint32_t s0 = 0; s0 < r->n; s0 += 16) {
        SmallJob &M = mj[nsmall++];
        M = SmallJob{v.act, v.lits, v.cls, J.x, J.sums, v.clauses, v.tol, v.classes, s0,
                     (uint32_t)std::min<uint64_t>(16, r->n - s0), 0, small_blocks, 0};
        small_blocks += small_job_blocks(v.classes, v.clauses, &M.cblocks);
      }
    } else {
      PredictJob &P = pj[npred++];
      P = PredictJob{};
      P.act = v.act;
      P.lits = v.lits;
      P.cls = v.cls;
      P.x = J.x;
      P.sums = J.sums;
      P.clauses = v.clauses;
      P.tol = v.tol;
      P.n = (uint32_t)r->n;
      P.classes = v.classes;
      P.tile0 = tiles;
      tiles += predict_job_tiles(P.n, v.classes, v.clauses, &P.stiles, &P.tpc);
    }
    sl.out_off[i] = o_off;
    in_off = round_up(in_off + r->n * v.input_chunks, 16);
    x_off = round_up(x_off + r->n * v.Wp, 4);
    s_off = round_up(s_off + r->n * v.classes, 4);
    o_off = round_up(o_off + out_bytes(v, r->n), 16);
  }
  cudaError_t e = cudaEventRecord(sl.ev0, sl.st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(sl.d_raw, sl.h_in, in_off, cudaMemcpyHostToDevice, sl.st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(sl.d_jobs, sl.h_jobs, o_pj + npred * sizeof(PredictJob),
                        cudaMemcpyHostToDevice, sl.st);
  if (e == cudaSuccess) e = cudaMemsetAsync(sl.d_sums, 0, s_off * 4, sl.st);
  if (e == cudaSuccess) e = launch_serve_repack((const ServeJob *)sl.d_jobs, R, sl.st);
  for (uint32_t i = 0; i < R && e == cudaSuccess; i++) {
    const Request *r = sl.reqs[i];
    const MachineView &v = s->mv[r->machine];
    if (!gemm_request(v, r->n)) continue;
    // the request's rows were repacked to sj[i].x; its sums go to sj[i].sums
    const uint64_t M = (uint64_t)v.classes * v.clauses, K = (uint64_t)v.W * 32;
    const uint64_t nc = gemm_chunk(M);
    for (uint64_t s0 = 0; s0 < r->n && e == cudaSuccess; s0 += nc) {
      const uint64_t k = std::min<uint64_t>(nc, r->n - s0);
      e = launch_expand_bits(sj[i].x + s0 * v.Wp, k, v.Wp, v.W, 0xFFFFFFFFu, v.act8_kind,
                             sl.d_x8, sl.st);
      if (e != cudaSuccess) break;
      const int g = gemm_clause_products(v.device, v.act8_kind, v.act8, sl.d_x8, sl.d_gc, M,
                                         gemm_bucket(k, std::min<uint64_t>(nc, s->cfg.max_batch_samples)),
                                         K, sl.d_ws, TM_SERVE_GEMM_WS, sl.st);
      if (g != 0) {
        e = cudaErrorUnknown;
        break;
      }
      e = launch_gemm_votes(sl.d_gc, v.act8_kind, v.lits, v.classes, v.clauses, v.tol,
                            (uint32_t)k, sj[i].sums + s0 * v.classes, sl.st);
    }
  }
  if (e == cudaSuccess)
    e = launch_predict_small_multi((const SmallJob *)(sl.d_jobs + o_mj), nsmall, small_blocks,
                                   sl.st);
  if (e == cudaSuccess)
    e = launch_predict_multi((const PredictJob *)(sl.d_jobs + o_pj), npred, tiles, sl.st);
  if (e == cudaSuccess) e = launch_serve_finalize((const ServeJob *)sl.d_jobs, R, sl.st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(sl.h_out, sl.d_out, o_off, cudaMemcpyDeviceToHost, sl.st);
  if (e == cudaSuccess) e = cudaEventRecord(sl.ev1, sl.st);
  const clk::time_point launched = clk::now();
  for (Request *r : sl.reqs) r->t_launched = launched;
  return e;
}

// The next launch: a free slot and the queue it serves.  High-priority
// slots take small requests only; normal slots take large ones, and small
// ones when no large request waits (or when every slot is normal).
static bool pick(tm_server *s, Slot *&slot, std::deque<Request *> *&q) {
  for (Slot &sl : s->slots) {
    if (sl.busy) continue;
    if (sl.high && !s->squeue.empty()) {
      slot = &sl, q = &s->squeue;
      return true;
    }
    if (!sl.high && !s->queue.empty()) {
      slot = &sl, q = &s->queue;
      return true;
    }
  }
  for (Slot &sl : s->slots)
    if (!sl.busy && !sl.high && !s->squeue.empty()) {
      slot = &sl, q = &s->squeue;
      return true;
    }
  return false;
}

static void worker_main(tm_server *s) {
  cudaSetDevice(s->cfg.device);
  std::unique_lock<std::mutex> lk(s->mu);
  while (true) {
    Slot *free_slot = nullptr;
    std::deque<Request *> *q = nullptr;
    s->cv_work.wait(lk, [&] { return s->stop || pick(s, free_slot, q); });
    if (s->stop) break;
    Slot &sl = *free_slot;
    // the oldest requests of that queue, any machine, while they fit the slot
    uint64_t n = 0;
    while (!q->empty() && sl.reqs.size() < TM_SERVE_MAX_PACK) {
      Request *r = q->front();
      if (!sl.reqs.empty() && n + r->n > s->cfg.max_batch_samples) break;
      q->pop_front();
      sl.reqs.push_back(r);
      n += r->n;
    }
    s->queued_samples -= n;
    sl.busy = true;
    lk.unlock();
    const cudaError_t e = launch_slot(s, sl);
    lk.lock();
    if (e != cudaSuccess) {
      s->error = TM_ERR_CUDA;
      s->stop = true;
      break;
    }
    sl.launched = true;  // to the slot's completion thread
    s->cv_launched.notify_all();
  }
  lk.unlock();
  // drain: every queued launch completes its requests through its slot's
  // completion thread
  for (Slot &sl : s->slots) cudaStreamSynchronize(sl.st);
  s->cv_done.notify_all();
}

// Ends the worker and the completion threads (queued launches complete
// first).
static void stop_threads(tm_server *s) {
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  if (s->worker.joinable()) s->worker.join();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->closing = true;
  }
  s->cv_launched.notify_all();
  for (Slot &sl : s->slots)
    if (sl.done_thread.joinable()) sl.done_thread.join();
}

static void free_server(tm_server *s) {
  stop_threads(s);
  DevGuard guard(s->cfg.device);
  for (Slot &sl : s->slots) {
    if (sl.ev0) cudaEventDestroy(sl.ev0);
    if (sl.ev1) cudaEventDestroy(sl.ev1);
    if (sl.st) cudaStreamDestroy(sl.st);
    if (sl.h_in) cudaFreeHost(sl.h_in);
    if (sl.h_out) cudaFreeHost(sl.h_out);
    if (sl.h_jobs) cudaFreeHost(sl.h_jobs);
    if (sl.d_raw) cudaFree(sl.d_raw);
    if (sl.d_out) cudaFree(sl.d_out);
    if (sl.d_jobs) cudaFree(sl.d_jobs);
    if (sl.d_x) cudaFree(sl.d_x);
    if (sl.d_sums) cudaFree(sl.d_sums);
    if (sl.d_x8) cudaFree(sl.d_x8);
    if (sl.d_gc) cudaFree(sl.d_gc);
    if (sl.d_ws) cudaFree(sl.d_ws);
  }
  for (auto *qq : {&s->queue, &s->squeue})
    for (Request *r : *qq) s->live.erase(r->id), delete r;
  for (auto &kv : s->live) delete kv.second;
  delete s;
}

extern "C" int tm_serve_open(const tm_server_config *cfg, tm_machine *const *machines,
                             uint32_t count, tm_server **out) {
  if (!cfg || !machines || !out || count == 0) return tmb_fail(TM_ERR_ARG, "serve_open: bad arguments");
  *out = nullptr;
  tm_server *s = new tm_server();
  s->cfg = *cfg;
  if (!s->cfg.max_batch_samples) s->cfg.max_batch_samples = 8192;
  if (!s->cfg.max_inflight) s->cfg.max_inflight = 4;
  if (!s->cfg.max_queued_samples) s->cfg.max_queued_samples = 64ull * s->cfg.max_batch_samples;
  DevGuard guard(s->cfg.device);
  for (uint32_t i = 0; i < count; i++) {
    MachineView v{};
    int rc = tmb_machine_view(machines[i], &v, "serving");
    if (rc) {
      delete s;
      return rc;
    }
    if (v.device != s->cfg.device) {
      delete s;
      return tmb_fail(TM_ERR_ARG, "serve_open: machine on another device");
    }
    rc = tmb_machine_act8(machines[i], &v);  // resident action bytes for large requests
    if (rc) {
      delete s;
      return rc;
    }
    s->mv.push_back(v);
  }
  // a slot holds up to max_batch_samples of the widest machine, plus the
  // alignment of up to TM_SERVE_MAX_PACK requests
  const uint64_t B = s->cfg.max_batch_samples, P = TM_SERVE_MAX_PACK;
  for (const MachineView &v : s->mv) {
    s->cap_in = std::max<uint64_t>(s->cap_in, B * v.input_chunks + 16 * P);
    s->cap_x = std::max<uint64_t>(s->cap_x, (B * v.Wp + 4 * P) * 4);
    s->cap_sums = std::max<uint64_t>(s->cap_sums, (B * v.classes + 4 * P) * 4);
    s->cap_out = std::max<uint64_t>(s->cap_out, out_bytes(v, B) + 16 * P);
  }
  s->cap_jobs = round_up(P * sizeof(ServeJob), 256) + round_up(2 * P * sizeof(SmallJob), 256) +
                P * sizeof(PredictJob);
  // the GEMM path: sample bytes of one chunk of the widest machine, the
  // products, the workspace
  // (only machines whose requests of up to max_batch_samples can reach it)
  uint64_t cap_x8 = 0, cap_gc = 0;
  for (MachineView &v : s->mv) {
    if (!gemm_request(v, B)) {
      v.act8 = nullptr;
      continue;
    }
    const uint64_t M = (uint64_t)v.classes * v.clauses;
    const uint64_t nc = std::min<uint64_t>(gemm_chunk(M), B);
    cap_x8 = std::max<uint64_t>(cap_x8, nc * (uint64_t)v.W * 32);
    cap_gc = std::max<uint64_t>(cap_gc, nc * M * 4);
  }
  const uint64_t cap_gemm = cap_x8 ? cap_x8 + cap_gc + TM_SERVE_GEMM_WS : 0;
  const uint64_t per_slot =
      s->cap_in + s->cap_x + s->cap_sums + s->cap_out + s->cap_jobs + cap_gemm;
  uint64_t nslots = s->cfg.hbm_budget_bytes ? s->cfg.hbm_budget_bytes / per_slot : s->cfg.max_inflight;
  nslots = std::min<uint64_t>(nslots, s->cfg.max_inflight);
  if (nslots == 0) {
    delete s;
    return tmb_fail(TM_ERR_OOM, "serve_open: the HBM budget does not cover one launch slot");
  }
  s->slots.resize(nslots);
  int prio_lo = 0, prio_hi = 0;
  cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi);
  // a third of the slots (at least one when there are two or more) on
  // high-priority streams for small requests
  const uint64_t nhigh = nslots >= 2 ? std::max<uint64_t>(1, nslots / 3) : 0;
  for (size_t i = 0; i < s->slots.size(); i++) {
    Slot &sl = s->slots[i];
    sl.srv = s;
    sl.high = i < nhigh;
    bool ok = cudaStreamCreateWithPriority(&sl.st, cudaStreamNonBlocking,
                                           sl.high ? prio_hi : prio_lo) == cudaSuccess &&
              cudaEventCreate(&sl.ev0) == cudaSuccess &&
              cudaEventCreateWithFlags(&sl.ev1, cudaEventBlockingSync) == cudaSuccess &&
              cudaHostAlloc(&sl.h_in, s->cap_in, cudaHostAllocDefault) == cudaSuccess &&
              cudaHostAlloc(&sl.h_out, s->cap_out, cudaHostAllocDefault) == cudaSuccess &&
              cudaHostAlloc(&sl.h_jobs, s->cap_jobs, cudaHostAllocDefault) == cudaSuccess &&
              tmb_dev_malloc((void **)&sl.d_raw, s->cap_in) == cudaSuccess &&
              tmb_dev_malloc((void **)&sl.d_out, s->cap_out) == cudaSuccess &&
              tmb_dev_malloc((void **)&sl.d_jobs, s->cap_jobs) == cudaSuccess &&
              tmb_dev_malloc((void **)&sl.d_x, s->cap_x) == cudaSuccess &&
              tmb_dev_malloc((void **)&sl.d_sums, s->cap_sums) == cudaSuccess;
    if (ok && cap_x8)
      ok = tmb_dev_malloc((void **)&sl.d_x8, cap_x8) == cudaSuccess &&
           tmb_dev_malloc(&sl.d_gc, cap_gc) == cudaSuccess &&
           tmb_dev_malloc((void **)&sl.d_ws, TM_SERVE_GEMM_WS) == cudaSuccess;
    if (!ok) {
      free_server(s);
      return tmb_fail(TM_ERR_OOM, "serve_open: device allocation failed");
    }
  }
  // every product width a machine's requests can use is run once on slot 0
  // (the library's choice and its kernels are set up before the first
  // request); a machine whose shape the library cannot take serves every
  // size with the bitwise kernels
  for (MachineView &v : s->mv) {
    if (!v.act8) continue;
    const uint64_t M = (uint64_t)v.classes * v.clauses;
    const uint64_t cap = std::min<uint64_t>(gemm_chunk(M), B);
    Slot &s0 = s->slots[0];
    for (uint64_t w = 64;; w = std::min<uint64_t>(2 * w, cap)) {
      const uint64_t N = gemm_bucket(w, cap);
      const int g = gemm_clause_products(v.device, v.act8_kind, v.act8, s0.d_x8, s0.d_gc, M, N,
                                         (uint64_t)v.W * 32, s0.d_ws, TM_SERVE_GEMM_WS, s0.st);
      if (g < 0) {
        v.act8 = nullptr;
        break;
      }
      if (g > 0 || cudaStreamSynchronize(s0.st) != cudaSuccess) {
        free_server(s);
        return tmb_fail(TM_ERR_CUDA, "serve_open: the GEMM library failed");
      }
      if (N >= cap) break;
    }
  }
  for (Slot &sl : s->slots) sl.done_thread = std::thread(slot_main, s, &sl);
  s->worker = std::thread(worker_main, s);
  *out = s;
  return TM_OK;
}

extern "C" int tm_serve_submit(tm_server *s, uint32_t machine, const uint8_t *problems, uint64_t n,
                               uint64_t *id) {
  if (!s || !id || (n && !problems)) return tmb_fail(TM_ERR_ARG, "serve_submit: bad arguments");
  if (machine >= s->mv.size()) return tmb_fail(TM_ERR_ARG, "serve_submit: no such machine");
  if (n == 0 || n > s->cfg.max_batch_samples)
    return tmb_fail(TM_ERR_OOM, "serve_submit: request larger than one launch slot");
  Request *r = new Request();
  r->machine = machine;
  r->n = n;
  r->input.assign(problems, problems + n * s->mv[machine].input_chunks);
  r->t_submit = clk::now();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) {
      delete r;
      return tmb_fail(s->error ? s->error : TM_ERR_STATE, "serve_submit: server stopped");
    }
    if (s->queued_samples + n > s->cfg.max_queued_samples) {
      char msg[96];
      snprintf(msg, sizeof msg, "serve_submit: queue full (%llu samples waiting)",
               (unsigned long long)s->queued_samples);
      delete r;
      return tmb_fail(TM_ERR_BUSY, msg);
    }
    r->id = s->next_id++;
    s->live[r->id] = r;
    (n <= TM_SERVE_SMALL ? s->squeue : s->queue).push_back(r);
    s->queued_samples += n;
    *id = r->id;
  }
  s->cv_work.notify_one();
  return TM_OK;
}

extern "C" int tm_serve_poll(tm_server *s, uint64_t id, int64_t *out_classes, uint8_t *out_codes,
                             uint64_t timeout_us) {
  if (!s) return tmb_fail(TM_ERR_ARG, "serve_poll: null server");
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->live.find(id);
  if (it == s->live.end()) return tmb_fail(TM_ERR_ARG, "serve_poll: unknown or already polled request");
  Request *r = it->second;
  if (!r->done && timeout_us)
    s->cv_done.wait_for(lk, std::chrono::microseconds(timeout_us),
                        [&] { return r->done || s->stop; });
  if (!r->done) return s->error ? tmb_fail(s->error, "serve_poll: server failed") : 0;
  const MachineView &v = s->mv[r->machine];
  if (v.type == TM_CLASSIFIER && out_classes) memcpy(out_classes, r->result.data(), r->result.size());
  if (v.type == TM_ENCODER && out_codes) memcpy(out_codes, r->result.data(), r->result.size());
  // the request is released; its latency stays queryable for a while
  s->latency[id] = times_of(*r);
  s->latency_order.push_back(id);
  while (s->latency_order.size() > TM_SERVE_LATENCY_KEEP) {
    s->latency.erase(s->latency_order.front());
    s->latency_order.pop_front();
  }
  s->live.erase(it);
  delete r;
  return 1;
}

static int find_times(tm_server *s, uint64_t id, Times *t, const char *who) {
  auto lt = s->latency.find(id);
  if (lt != s->latency.end()) {
    *t = lt->second;
    return TM_OK;
  }
  auto it = s->live.find(id);
  if (it == s->live.end() || !it->second->done) {
    char msg[64];
    snprintf(msg, sizeof msg, "%s: request not done", who);
    return tmb_fail(TM_ERR_ARG, msg);
  }
  *t = times_of(*it->second);
  return TM_OK;
}

extern "C" int tm_serve_latency_us(tm_server *s, uint64_t id, double *us) {
  if (!s || !us) return tmb_fail(TM_ERR_ARG, "serve_latency_us: bad arguments");
  std::lock_guard<std::mutex> lk(s->mu);
  Times t;
  const int rc = find_times(s, id, &t, "serve_latency_us");
  if (!rc) *us = t.total;
  return rc;
}

extern "C" int tm_serve_phases_us(tm_server *s, uint64_t id, double *out) {
  if (!s || !out) return tmb_fail(TM_ERR_ARG, "serve_phases_us: bad arguments");
  std::lock_guard<std::mutex> lk(s->mu);
  Times t;
  const int rc = find_times(s, id, &t, "serve_phases_us");
  if (!rc) out[0] = t.queue, out[1] = t.launch, out[2] = t.device, out[3] = t.gpu;
  return rc;
}

extern "C" int tm_serve_stats(tm_server *s, uint64_t *out) {
  if (!s || !out) return tmb_fail(TM_ERR_ARG, "serve_stats: bad arguments");
  std::lock_guard<std::mutex> lk(s->mu);
  uint32_t busy = 0;
  for (const Slot &sl : s->slots) busy += sl.busy ? 1 : 0;
  out[0] = s->queue.size() + s->squeue.size();
  out[1] = s->queued_samples;
  out[2] = s->live.size();
  out[3] = busy;
  out[4] = s->slots.size();
  return TM_OK;
}

extern "C" int tm_serve_close(tm_server *s) {
  if (!s) return TM_OK;
  stop_threads(s);
  const int err = s->error;
  free_server(s);
  return err ? tmb_fail(err, "serve: a launch failed") : TM_OK;
}
