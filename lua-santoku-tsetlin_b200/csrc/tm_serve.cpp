// Predict server: resident machines, continuous batching (tm_serve_* in
// include/tsetlin_b200.h).  No counterpart in the reference, whose predict
// is one synchronous call per batch (capi.c:1088-1110).
//
// A worker thread owns S launch slots (one CUDA stream, pinned host staging
// and device buffers each; S is bounded by max_inflight and by how many
// slots the HBM budget pays for).  It repeatedly
//   1. retires slots whose completion event has fired: results are copied
//      to their requests, which become visible to tm_serve_poll;
//   2. fills every free slot with the oldest queued request and every later
//      queued request for the same machine that still fits the slot
//      (max_batch_samples), then launches repack -> predict -> finalize and
//      the result copy on the slot's stream.
// Requests that arrive while slots are busy are admitted as soon as a slot
// frees up, and the slots' streams overlap on the device.  Predict is
// independent per sample, so each request's result is the same alone or
// packed with others.
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "../../include/tsetlin_b200.h"
#include "tm_internal.h"

using namespace tmb;
using clk = std::chrono::steady_clock;

namespace {

struct Request {
  uint64_t id;
  uint32_t machine;
  uint64_t n;
  std::vector<uint8_t> input;
  std::vector<uint8_t> result;  // int64 classes or code bytes
  clk::time_point t_submit, t_done;
  bool done = false;
};

struct Slot {
  cudaStream_t st = nullptr;
  cudaEvent_t ev = nullptr;
  uint8_t *h_in = nullptr, *h_out = nullptr;  // pinned
  uint8_t *d_raw = nullptr, *d_out = nullptr;
  uint32_t *d_x = nullptr;
  int32_t *d_sums = nullptr;
  std::vector<Request *> reqs;
  bool busy = false;
};

}  // namespace

struct tm_server {
  tm_server_config cfg{};
  std::vector<MachineView> mv;
  std::vector<Slot> slots;
  uint64_t cap_in = 0, cap_out = 0, cap_x = 0, cap_sums = 0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Request *> queue;
  std::map<uint64_t, Request *> all;
  uint64_t next_id = 1;
  bool stop = false;
  std::thread worker;
  int error = 0;
};

static uint64_t out_bytes(const MachineView &v, uint64_t n) {
  return v.type == TM_CLASSIFIER ? n * 8 : n * v.class_chunks;
}

static bool launch_slot(tm_server *s, Slot &sl) {
  const MachineView &v = s->mv[sl.reqs[0]->machine];
  uint64_t n = 0;
  for (Request *r : sl.reqs) {
    memcpy(sl.h_in + n * v.input_chunks, r->input.data(), r->n * v.input_chunks);
    n += r->n;
  }
  cudaError_t e = cudaMemcpyAsync(sl.d_raw, sl.h_in, n * v.input_chunks, cudaMemcpyHostToDevice, sl.st);
  if (e == cudaSuccess)
    e = launch_repack(sl.d_raw, n, v.input_chunks, v.input_chunks, sl.d_x, v.Wp, sl.st);
  if (e == cudaSuccess) e = cudaMemsetAsync(sl.d_sums, 0, n * v.classes * 4, sl.st);
  if (e == cudaSuccess)
    e = launch_predict(v.act, v.lits, v.cls, nullptr, v.classes, v.clauses, v.tol, sl.d_x,
                       (uint32_t)n, sl.d_sums, sl.st);
  if (e == cudaSuccess)
    e = launch_finalize(sl.d_sums, (uint32_t)n, v.classes, (int32_t)v.type,
                        v.type == TM_CLASSIFIER ? (int64_t *)sl.d_out : nullptr,
                        v.type == TM_ENCODER ? sl.d_out : nullptr, nullptr, sl.st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(sl.h_out, sl.d_out, out_bytes(v, n), cudaMemcpyDeviceToHost, sl.st);
  if (e == cudaSuccess) e = cudaEventRecord(sl.ev, sl.st);
  return e == cudaSuccess;
}

static void retire_slot(tm_server *s, Slot &sl) {
  const MachineView &v = s->mv[sl.reqs[0]->machine];
  uint64_t off = 0;
  const clk::time_point now = clk::now();
  for (Request *r : sl.reqs) {
    const uint64_t b = out_bytes(v, r->n);
    r->result.assign(sl.h_out + off, sl.h_out + off + b);
    off += b;
    r->t_done = now;
    r->done = true;
  }
  sl.reqs.clear();
  sl.busy = false;
}

static void worker_main(tm_server *s) {
  cudaSetDevice(s->cfg.device);
  std::unique_lock<std::mutex> lk(s->mu);
  while (true) {
    bool progressed = false;
    for (Slot &sl : s->slots) {
      if (sl.busy && cudaEventQuery(sl.ev) == cudaSuccess) {
        retire_slot(s, sl);
        progressed = true;
      }
    }
    if (progressed) s->cv_done.notify_all();
    for (Slot &sl : s->slots) {
      if (sl.busy || s->queue.empty()) continue;
      Request *head = s->queue.front();
      s->queue.pop_front();
      sl.reqs.push_back(head);
      uint64_t n = head->n;
      for (auto it = s->queue.begin(); it != s->queue.end();) {
        Request *r = *it;
        if (r->machine == head->machine && n + r->n <= s->cfg.max_batch_samples) {
          sl.reqs.push_back(r);
          n += r->n;
          it = s->queue.erase(it);
        } else {
          ++it;
        }
      }
      sl.busy = true;
      if (!launch_slot(s, sl)) {
        s->error = TM_ERR_CUDA;
        s->stop = true;
      }
      progressed = true;
    }
    if (s->stop) break;
    bool any_busy = false;
    for (Slot &sl : s->slots) any_busy |= sl.busy;
    if (!progressed) {
      if (any_busy) {
        lk.unlock();
        std::this_thread::sleep_for(std::chrono::microseconds(20));
        lk.lock();
      } else {
        s->cv_work.wait(lk, [&] { return s->stop || !s->queue.empty(); });
      }
    }
  }
  for (Slot &sl : s->slots)
    if (sl.busy) {
      cudaEventSynchronize(sl.ev);
      retire_slot(s, sl);
    }
  s->cv_done.notify_all();
}

static void free_server(tm_server *s) {
  for (Slot &sl : s->slots) {
    if (sl.st) cudaStreamDestroy(sl.st);
    if (sl.ev) cudaEventDestroy(sl.ev);
    if (sl.h_in) cudaFreeHost(sl.h_in);
    if (sl.h_out) cudaFreeHost(sl.h_out);
    if (sl.d_raw) cudaFree(sl.d_raw);
    if (sl.d_out) cudaFree(sl.d_out);
    if (sl.d_x) cudaFree(sl.d_x);
    if (sl.d_sums) cudaFree(sl.d_sums);
  }
  for (auto &kv : s->all) delete kv.second;
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
  cudaSetDevice(s->cfg.device);
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
    s->mv.push_back(v);
  }
  const uint64_t B = s->cfg.max_batch_samples;
  for (const MachineView &v : s->mv) {
    s->cap_in = std::max<uint64_t>(s->cap_in, B * v.input_chunks);
    s->cap_x = std::max<uint64_t>(s->cap_x, B * v.Wp * 4);
    s->cap_sums = std::max<uint64_t>(s->cap_sums, B * v.classes * 4);
    s->cap_out = std::max<uint64_t>(s->cap_out, out_bytes(v, B));
  }
  const uint64_t per_slot = s->cap_in + s->cap_x + s->cap_sums + s->cap_out;
  uint64_t nslots = s->cfg.hbm_budget_bytes ? s->cfg.hbm_budget_bytes / per_slot : s->cfg.max_inflight;
  nslots = std::min<uint64_t>(nslots, s->cfg.max_inflight);
  if (nslots == 0) {
    delete s;
    return tmb_fail(TM_ERR_OOM, "serve_open: the HBM budget does not cover one launch slot");
  }
  s->slots.resize(nslots);
  for (Slot &sl : s->slots) {
    bool ok = cudaStreamCreateWithFlags(&sl.st, cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreateWithFlags(&sl.ev, cudaEventDisableTiming) == cudaSuccess &&
              cudaHostAlloc(&sl.h_in, s->cap_in, cudaHostAllocDefault) == cudaSuccess &&
              cudaHostAlloc(&sl.h_out, s->cap_out, cudaHostAllocDefault) == cudaSuccess &&
              tmb_dev_malloc((void **)&sl.d_raw, s->cap_in) == cudaSuccess &&
              tmb_dev_malloc((void **)&sl.d_out, s->cap_out) == cudaSuccess &&
              tmb_dev_malloc((void **)&sl.d_x, s->cap_x) == cudaSuccess &&
              tmb_dev_malloc((void **)&sl.d_sums, s->cap_sums) == cudaSuccess;
    if (!ok) {
      free_server(s);
      return tmb_fail(TM_ERR_OOM, "serve_open: device allocation failed");
    }
  }
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
    r->id = s->next_id++;
    s->all[r->id] = r;
    s->queue.push_back(r);
    *id = r->id;
  }
  s->cv_work.notify_one();
  return TM_OK;
}

extern "C" int tm_serve_poll(tm_server *s, uint64_t id, int64_t *out_classes, uint8_t *out_codes,
                             uint64_t timeout_us) {
  if (!s) return tmb_fail(TM_ERR_ARG, "serve_poll: null server");
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->all.find(id);
  if (it == s->all.end()) return tmb_fail(TM_ERR_ARG, "serve_poll: unknown request");
  Request *r = it->second;
  if (!r->done && timeout_us)
    s->cv_done.wait_for(lk, std::chrono::microseconds(timeout_us),
                        [&] { return r->done || s->stop; });
  if (!r->done) return s->error ? tmb_fail(s->error, "serve_poll: server failed") : 0;
  const MachineView &v = s->mv[r->machine];
  if (v.type == TM_CLASSIFIER && out_classes) memcpy(out_classes, r->result.data(), r->result.size());
  if (v.type == TM_ENCODER && out_codes) memcpy(out_codes, r->result.data(), r->result.size());
  return 1;
}

extern "C" int tm_serve_latency_us(tm_server *s, uint64_t id, double *us) {
  if (!s || !us) return tmb_fail(TM_ERR_ARG, "serve_latency_us: bad arguments");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->all.find(id);
  if (it == s->all.end() || !it->second->done) return tmb_fail(TM_ERR_ARG, "serve_latency_us: request not done");
  *us = std::chrono::duration<double, std::micro>(it->second->t_done - it->second->t_submit).count();
  return TM_OK;
}

extern "C" int tm_serve_close(tm_server *s) {
  if (!s) return TM_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  if (s->worker.joinable()) s->worker.join();
  const int err = s->error;
  free_server(s);
  return err ? tmb_fail(err, "serve: a launch failed") : TM_OK;
}
