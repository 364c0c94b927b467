// tm_predict_noalloc: predict for callers that cannot allocate device memory.
//
// Some callers of this library must not call cudaMalloc or cudaFree while
// they run: a serving loop whose latency budget cannot absorb the implicit
// device-wide synchronisation those calls cause, or a host application whose
// own allocator has already reserved the GPU's memory, so that a raw
// cudaMalloc may fail at an arbitrary moment.  tm_predict stages its inputs
// and vote sums in buffers it grows on demand; this entry point instead
// works in one fixed scratch array compiled into the library.
//
// The scratch is a file-scope __device__ array of TM_NOALLOC_SCRATCH_BYTES
// (8 MiB).  Every GPU that loads the library holds it until the process
// exits.  Host code cannot use the array's name as a device address, so the
// first call on each device, with that device current, asks the runtime for
// the array's device address (cudaGetSymbolAddress) and keeps it; that first
// call should come before any stream capture.  All calls share the one
// array, which keeps whatever the last call left there: the vote sums are
// cleared at the start of every call, and calls whose work overlaps on the
// GPU (from different threads or machines at once) race on it.
#include <mutex>

#include "../../include/tsetlin_b200.h"
#include "tm_internal.h"

#define TM_NOALLOC_SCRATCH_BYTES (8u << 20)
#define TM_NOALLOC_MAX_DEVICES 64

static __device__ __align__(256) uint8_t g_noalloc_scratch[TM_NOALLOC_SCRATCH_BYTES];

static void *g_noalloc_ptr[TM_NOALLOC_MAX_DEVICES];
static std::mutex g_noalloc_mu;

// Device address of the scratch array on `dev` (which must be current).
static int noalloc_scratch(int dev, uint8_t **out) {
  if (dev < 0 || dev >= TM_NOALLOC_MAX_DEVICES)
    return tmb_fail(TM_ERR_ARG, "predict_noalloc: device ordinal out of range");
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return tmb_fail(TM_ERR_CUDA, "predict_noalloc: cudaGetSymbolAddress failed");
    g_noalloc_ptr[dev] = p;
  }
  *out = (uint8_t *)g_noalloc_ptr[dev];
  return TM_OK;
}

extern "C" int tm_predict_noalloc(tm_machine *m, const uint8_t *problems, uint64_t n,
                                  int64_t *out_classes, uint8_t *out_codes) {
  if (!m) return tmb_fail(TM_ERR_ARG, "predict_noalloc: null machine");
  if (n == 0) return TM_OK;
  if (!problems) return tmb_fail(TM_ERR_ARG, "predict_noalloc: problems missing");
  tmb::MachineView v{};
  int rc = tmb_machine_view(m, &v, "predict_noalloc");  // no allocation
  if (rc) return rc;
  if (v.type == TM_CLASSIFIER && !out_classes)
    return tmb_fail(TM_ERR_ARG, "predict_noalloc: out_classes missing");
  if (v.type == TM_ENCODER && !out_codes)
    return tmb_fail(TM_ERR_ARG, "predict_noalloc: out_codes missing");
  // Bound n before any size is multiplied out: a sample needs Wp words of
  // padded row and `classes` vote sums, plus up to 256 bytes of alignment
  // for the whole request.
  const uint64_t per_sample = (uint64_t)v.Wp * 4 + (uint64_t)v.classes * 4;
  if (n > (TM_NOALLOC_SCRATCH_BYTES - 256) / per_sample)
    return tmb_fail(TM_ERR_ARG,
                    "predict_noalloc: request needs more than the 8 MiB scratch; split it or use "
                    "tm_predict");
  int prev = -1;
  if (cudaGetDevice(&prev) != cudaSuccess)
    return tmb_fail(TM_ERR_CUDA, "predict_noalloc: cannot query the current device");
  if (prev != v.device && cudaSetDevice(v.device) != cudaSuccess)
    return tmb_fail(TM_ERR_CUDA, "predict_noalloc: cannot select the machine's device");
  // scratch: [padded rows, n * Wp words][vote sums, n * classes int32]
  const uint64_t xbytes = (n * v.Wp * 4 + 255) & ~255ull;
  const uint64_t sbytes = n * v.classes * 4;
  uint8_t *scratch = nullptr;
  rc = noalloc_scratch(v.device, &scratch);
  if (!rc) {
    uint32_t *x = (uint32_t *)scratch;
    int32_t *sums = (int32_t *)(scratch + xbytes);
    cudaError_t e = tmb::launch_repack(problems, n, v.input_chunks, v.input_chunks, x, v.Wp, v.st);
    if (e == cudaSuccess) e = cudaMemsetAsync(sums, 0, sbytes, v.st);
    if (e == cudaSuccess)
      e = tmb::launch_predict(v.act, v.lits, v.cls, nullptr, v.classes, v.clauses, v.tol, x,
                              (uint32_t)n, sums, v.st);
    if (e == cudaSuccess)
      e = tmb::launch_finalize(sums, (uint32_t)n, v.classes, (int32_t)v.type,
                               v.type == TM_CLASSIFIER ? out_classes : nullptr,
                               v.type == TM_ENCODER ? out_codes : nullptr, nullptr, v.st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(v.st);
    if (e != cudaSuccess) rc = tmb_fail(TM_ERR_CUDA, cudaGetErrorString(e));
  }
  if (prev != v.device) cudaSetDevice(prev);
  return rc;
}
