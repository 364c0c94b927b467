// Integer-pipe peaks of this GPU, measured: the roofline denominators of the
// bit-logic kernels (clause evaluation is AND-NOT + carry-save adders +
// POPC on 32-bit words; no tensor core or HBM peak bounds it).
//
//   tm_int_peaks(device, out[3]) -> thread-operations per second of
//     out[0]  LOP3 (lop3.b32, the ALU pipe's logic op)
//     out[1]  POPC (popc.b32)
//     out[2]  integer add (add.u32)
//
// Each thread runs 16 independent dependency chains of one instruction
// (inline PTX, so nothing is folded or hoisted) on a grid of 8 CTAs of 256
// threads per SM; CUDA events time the launch after a warm-up launch.  No
// counterpart in the reference.
#include <stdint.h>

#include "../../include/tsetlin_b200.h"
#include "tm_internal.h"

namespace {

constexpr int PK_CHAINS = 16, PK_THREADS = 256, PK_CTAS_PER_SM = 8;

__global__ void __launch_bounds__(PK_THREADS) k_peak_lop3(uint32_t iters, uint32_t *out) {
  uint32_t v[PK_CHAINS];
  const uint32_t b = blockIdx.x * 0x9E3779B9u, c = threadIdx.x * 0x85EBCA6Bu;
#pragma unroll
  for (int k = 0; k < PK_CHAINS; k++) v[k] = threadIdx.x + 0x1000193u * k;
  for (uint32_t it = 0; it < iters; it++) {
#pragma unroll
    for (int k = 0; k < PK_CHAINS; k++)
      asm volatile("lop3.b32 %0, %0, %1, %2, 0x96;" : "+r"(v[k]) : "r"(b), "r"(c));
  }
  uint32_t r = 0;
#pragma unroll
  for (int k = 0; k < PK_CHAINS; k++) r ^= v[k];
  if (r == 0x12345678u) out[0] = r;  // keeps the chains live
}

__global__ void __launch_bounds__(PK_THREADS) k_peak_popc(uint32_t iters, uint32_t *out) {
  uint32_t v[PK_CHAINS];
#pragma unroll
  for (int k = 0; k < PK_CHAINS; k++) v[k] = threadIdx.x * 0x01000193u + k;
  for (uint32_t it = 0; it < iters; it++) {
#pragma unroll
    for (int k = 0; k < PK_CHAINS; k++) asm volatile("popc.b32 %0, %0;" : "+r"(v[k]));
  }
  uint32_t r = 0;
#pragma unroll
  for (int k = 0; k < PK_CHAINS; k++) r += v[k];
  if (r == 0x12345678u) out[0] = r;
}

__global__ void __launch_bounds__(PK_THREADS) k_peak_iadd(uint32_t iters, uint32_t *out) {
  uint32_t v[PK_CHAINS];
  const uint32_t b = blockIdx.x | 1u;
#pragma unroll
  for (int k = 0; k < PK_CHAINS; k++) v[k] = threadIdx.x + k;
  for (uint32_t it = 0; it < iters; it++) {
#pragma unroll
    for (int k = 0; k < PK_CHAINS; k++) asm volatile("add.u32 %0, %0, %1;" : "+r"(v[k]) : "r"(b));
  }
  uint32_t r = 0;
#pragma unroll
  for (int k = 0; k < PK_CHAINS; k++) r ^= v[k];
  if (r == 0x12345678u) out[0] = r;
}

template <class K>
int time_peak(K kern, int sms, uint32_t iters, uint32_t *d_out, double *ops_per_s) {
  const int grid = sms * PK_CTAS_PER_SM;
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess) return -1;
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return -1;
  }
  kern<<<grid, PK_THREADS>>>(iters / 8, d_out);  // warm-up
  cudaEventRecord(e0);
  kern<<<grid, PK_THREADS>>>(iters, d_out);
  cudaEventRecord(e1);
  const cudaError_t err = cudaEventSynchronize(e1);
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (err != cudaSuccess || ms <= 0) return -1;
  *ops_per_s = (double)grid * PK_THREADS * PK_CHAINS * iters / (ms * 1e-3);
  return 0;
}

}  // namespace

extern "C" int tm_int_peaks(int32_t device, double *out) {
  if (!out) return tmb_fail(TM_ERR_ARG, "int_peaks: null output");
  tmb::DevGuard guard(device);
  if (guard.err != cudaSuccess) return tmb_fail(TM_ERR_CUDA, "int_peaks: bad device");
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  if (sms <= 0) return tmb_fail(TM_ERR_CUDA, "int_peaks: no multiprocessors");
  uint32_t *d_out = nullptr;
  if (cudaMalloc(&d_out, 64) != cudaSuccess) return tmb_fail(TM_ERR_OOM, "int_peaks: cudaMalloc");
  int rc = 0;
  // ~20-60 ms per launch at the B200's rates
  rc |= time_peak(k_peak_lop3, sms, 1u << 15, d_out, &out[0]);
  rc |= time_peak(k_peak_popc, sms, 1u << 13, d_out, &out[1]);
  rc |= time_peak(k_peak_iadd, sms, 1u << 15, d_out, &out[2]);
  cudaFree(d_out);
  if (rc) return tmb_fail(TM_ERR_CUDA, "int_peaks: launch failed");
  return TM_OK;
}
