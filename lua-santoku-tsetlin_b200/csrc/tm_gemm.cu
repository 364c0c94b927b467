// Large-batch predict as a GEMM.  For 0/1 operands the number of a clause's
// included literals that a sample satisfies is the dot product of the
// clause's action bits and the sample's literal bits, so the failed-literal
// counts of every (clause, sample) pair -- F = L - A.x, with L the clause's
// literal count (capi.c:97-122) -- come from one 8-bit tensor-core GEMM of
// the clauses' action bytes (M x K) and the samples' literal bytes (N x K)
// with exact integer accumulation (int8 with int32 accumulation, or e4m3
// with fp32 accumulation: every partial sum is an integer below 2^24).  The
// GEMM is the library's (cuBLASLt); the bytes are expanded here from the bit
// rows, and the epilogue turns C into the reference's votes (max(0,
// min(L, tol) - F), or tol for an empty clause; signed by clause parity,
// capi.c:110-118, 148-161) and class sums.  The same integer sums as the
// bitwise kernels, bit for bit.
#include <cublasLt.h>
#include <cuda_runtime.h>

#include <stdio.h>
#include <stdlib.h>

#include <map>
#include <mutex>

#include "tm_internal.h"

namespace tmb {

namespace {

// Four bits of `nib` (bit i -> byte i) as bytes 0 or `one`: the multiply
// places bit i at bit 8 i (the four shifted copies do not overlap).
__device__ __forceinline__ uint32_t spread4(uint32_t nib, uint32_t one) {
  return ((nib * 0x00204081u) & 0x01010101u) * one;
}

// rows x W words (stride `stride` words) -> rows x 32 W bytes; the last
// word of a row is ANDed with `last_mask`.
__global__ void k_expand_bits(const uint32_t *__restrict__ src, uint64_t rows, uint32_t stride,
                              uint32_t W, uint32_t last_mask, uint32_t one,
                              uint8_t *__restrict__ dst) {
  const uint64_t total = rows * W;
  for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t r = t / W;
    const uint32_t w = (uint32_t)(t - r * W);
    uint32_t v = src[r * stride + w];
    if (w == W - 1) v &= last_mask;
    uint4 lo, hi;
    lo.x = spread4(v & 15u, one);
    lo.y = spread4((v >> 4) & 15u, one);
    lo.z = spread4((v >> 8) & 15u, one);
    lo.w = spread4((v >> 12) & 15u, one);
    hi.x = spread4((v >> 16) & 15u, one);
    hi.y = spread4((v >> 20) & 15u, one);
    hi.z = spread4((v >> 24) & 15u, one);
    hi.w = spread4(v >> 28, one);
    uint4 *o = (uint4 *)(dst + (r * W + w) * 32);
    o[0] = lo;
    o[1] = hi;
  }
}

// C (M x N, column-major: sample n's M clause results contiguous) -> the
// vote sums of samples s0 .. s0 + N - 1: one warp per (sample, class).
template <typename T>
__global__ void k_gemm_votes(const T *__restrict__ C, const int32_t *__restrict__ lits,
                             uint32_t classes, uint32_t clauses, uint32_t tol, uint32_t N,
                             int32_t *__restrict__ sums, const uint32_t *__restrict__ gate) {
  if (gate && *gate == 0) return;  // a search machine that stopped training keeps its sums
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t M = (uint64_t)classes * clauses;
  const uint64_t items = (uint64_t)N * classes;
  for (uint64_t it = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; it < items;
       it += ((uint64_t)gridDim.x * blockDim.x) >> 5) {
    const uint32_t n = (uint32_t)(it / classes), h = (uint32_t)(it - (uint64_t)n * classes);
    const T *col = C + (uint64_t)n * M + (uint64_t)h * clauses;
    const int32_t *L = lits + (uint64_t)h * clauses;
    int32_t part = 0;
    for (uint32_t c = lane; c < clauses; c += 32) {
      const int32_t l = L[c];
      int32_t vote;
      if (l == 0) {
        vote = (int32_t)tol;
      } else {
        const int32_t f = l - (int32_t)col[c];  // failed literals
        vote = (l < (int32_t)tol ? l : (int32_t)tol) - f;
        vote = vote < 0 ? 0 : vote;
      }
      part += (c & 1) ? -vote : vote;
    }
    part = __reduce_add_sync(0xFFFFFFFFu, part);
    if (lane == 0) sums[(uint64_t)n * classes + h] = part;
  }
}

int grid_for(uint64_t items, int threads) {
  const uint64_t b = (items + threads - 1) / threads;
  return (int)(b < 148ull * 16 ? (b ? b : 1) : 148ull * 16);
}

std::mutex g_lt_mu;
cublasLtHandle_t g_lt[64];
int g_lt_state[64];  // 0 not created, 1 ready

// The library's choice per (device, encoding, M, N, K, workspace bytes):
// asked once per shape (products of few distinct widths are asked for:
// callers round N up to a bucket); the workspace limit is part of the key,
// so an algorithm chosen under a larger workspace is never run with a
// smaller one.  found == 0 records a shape without an algorithm.
struct AlgoKey {
  int dev, kind;
  uint64_t M, N, K, ws;
  bool operator<(const AlgoKey &o) const {
    if (dev != o.dev) return dev < o.dev;
    if (kind != o.kind) return kind < o.kind;
    if (M != o.M) return M < o.M;
    if (N != o.N) return N < o.N;
    if (K != o.K) return K < o.K;
    return ws < o.ws;
  }
};
struct AlgoVal {
  cublasLtMatmulAlgo_t algo;
  int found;
};
std::map<AlgoKey, AlgoVal> g_algos;

}  // namespace

uint32_t gemm_byte_one(int kind) { return kind == TM_GEMM_FP8 ? 0x38u : 0x01u; }

uint64_t gemm_bucket(uint64_t k, uint64_t cap) {
  uint64_t b = 64;
  while (b < k) b <<= 1;
  return b < cap ? b : cap;
}

cudaError_t launch_expand_bits(const uint32_t *src, uint64_t rows, uint32_t stride, uint32_t W,
                               uint32_t last_mask, int kind, uint8_t *dst, cudaStream_t st) {
  if (!rows || !W) return cudaSuccess;
  k_expand_bits<<<grid_for(rows * W, 256), 256, 0, st>>>(src, rows, stride, W, last_mask,
                                                          gemm_byte_one(kind), dst);
  return cudaGetLastError();
}

cudaError_t launch_gemm_votes(const void *C, int kind, const int32_t *lits, uint32_t classes,
                              uint32_t clauses, uint32_t tol, uint32_t N, int32_t *sums,
                              cudaStream_t st, const uint32_t *gate) {
  if (!N) return cudaSuccess;
  const int g = grid_for((uint64_t)N * classes * 32, 256);
  if (kind == TM_GEMM_FP8)
    k_gemm_votes<float><<<g, 256, 0, st>>>((const float *)C, lits, classes, clauses, tol, N, sums,
                                           gate);
  else
    k_gemm_votes<int32_t><<<g, 256, 0, st>>>((const int32_t *)C, lits, classes, clauses, tol, N,
                                             sums, gate);
  return cudaGetLastError();
}

// C = A B^T for A (M x K bytes, rows K-contiguous) and B (N x K): in
// cuBLASLt's column-major terms the "TN" product of A stored K x M and B
// stored K x N, with C M x N.  Returns 0, or -1 when the library has no
// algorithm for this kind and shape (the caller then uses the bitwise
// kernels), or a cuBLAS status > 0.
int gemm_clause_products(int dev, int kind, const uint8_t *A, const uint8_t *B, void *C,
                         uint64_t M, uint64_t N, uint64_t K, void *ws, size_t ws_bytes,
                         cudaStream_t st) {
  if (dev < 0 || dev >= 64) return -1;
  cublasLtHandle_t lt = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_lt_mu);
    // a failed creation is tried again at the next call
    if (g_lt_state[dev] == 0 && cublasLtCreate(&g_lt[dev]) == CUBLAS_STATUS_SUCCESS)
      g_lt_state[dev] = 1;
    if (g_lt_state[dev] != 1) return -1;
    lt = g_lt[dev];
  }
  const bool fp8 = kind == TM_GEMM_FP8;
  const cudaDataType_t ab = fp8 ? CUDA_R_8F_E4M3 : CUDA_R_8I;
  const cudaDataType_t ct = fp8 ? CUDA_R_32F : CUDA_R_32I;
  const cublasComputeType_t comp = fp8 ? CUBLAS_COMPUTE_32F : CUBLAS_COMPUTE_32I;
  cublasLtMatmulDesc_t op = nullptr;
  cublasLtMatrixLayout_t la = nullptr, lb = nullptr, lc = nullptr;
  cublasLtMatmulPreference_t pref = nullptr;
  int rc = 0;
  cublasStatus_t s = cublasLtMatmulDescCreate(&op, comp, ct);
  const cublasOperation_t ta = CUBLAS_OP_T, tb = CUBLAS_OP_N;
  if (s == CUBLAS_STATUS_SUCCESS)
    s = cublasLtMatmulDescSetAttribute(op, CUBLASLT_MATMUL_DESC_TRANSA, &ta, sizeof ta);
  if (s == CUBLAS_STATUS_SUCCESS)
    s = cublasLtMatmulDescSetAttribute(op, CUBLASLT_MATMUL_DESC_TRANSB, &tb, sizeof tb);
  if (s == CUBLAS_STATUS_SUCCESS && fp8) {
    const int8_t fast = 0;  // full fp32 accumulation: every partial sum stays exact
    s = cublasLtMatmulDescSetAttribute(op, CUBLASLT_MATMUL_DESC_FAST_ACCUM, &fast, sizeof fast);
  }
  if (s == CUBLAS_STATUS_SUCCESS) s = cublasLtMatrixLayoutCreate(&la, ab, K, M, K);
  if (s == CUBLAS_STATUS_SUCCESS) s = cublasLtMatrixLayoutCreate(&lb, ab, K, N, K);
  if (s == CUBLAS_STATUS_SUCCESS) s = cublasLtMatrixLayoutCreate(&lc, ct, M, N, M);
  if (s == CUBLAS_STATUS_SUCCESS) s = cublasLtMatmulPreferenceCreate(&pref);
  if (s == CUBLAS_STATUS_SUCCESS)
    s = cublasLtMatmulPreferenceSetAttribute(pref, CUBLASLT_MATMUL_PREF_MAX_WORKSPACE_BYTES,
                                             &ws_bytes, sizeof ws_bytes);
  cublasLtMatmulHeuristicResult_t h{};
  int found = 0;
  const AlgoKey key{dev, kind, M, N, K, (uint64_t)ws_bytes};
  bool cached = false;
  {
    std::lock_guard<std::mutex> lk(g_lt_mu);
    auto it = g_algos.find(key);
    if (it != g_algos.end()) {
      h.algo = it->second.algo;
      found = it->second.found;
      cached = true;
    }
  }
  if (!cached && s == CUBLAS_STATUS_SUCCESS) {
    s = cublasLtMatmulAlgoGetHeuristic(lt, op, la, lb, lc, lc, pref, 1, &h, &found);
    if (s == CUBLAS_STATUS_SUCCESS) {
      std::lock_guard<std::mutex> lk(g_lt_mu);
      g_algos[key] = AlgoVal{h.algo, found};
    }
  }
  {
    // TSETLIN_B200_GEMM_LOG=1: the library's answer for each shape on stderr
    const char *lg = getenv("TSETLIN_B200_GEMM_LOG");
    if (lg && lg[0] == '1' && !cached)
      fprintf(stderr, "tsetlin_b200 gemm: %s M=%llu N=%llu K=%llu status=%d algorithms=%d\n",
              fp8 ? "e4m3" : "int8", (unsigned long long)M, (unsigned long long)N,
              (unsigned long long)K, (int)s, found);
  }
  if (s != CUBLAS_STATUS_SUCCESS || found == 0) {
    rc = -1;
  } else {
    if (fp8) {
      const float one = 1.0f, zero = 0.0f;
      s = cublasLtMatmul(lt, op, &one, A, la, B, lb, &zero, C, lc, C, lc, &h.algo, ws, ws_bytes,
                         st);
    } else {
      const int32_t one = 1, zero = 0;
      s = cublasLtMatmul(lt, op, &one, A, la, B, lb, &zero, C, lc, C, lc, &h.algo, ws, ws_bytes,
                         st);
    }
    rc = s == CUBLAS_STATUS_SUCCESS ? 0 : (int)s;
  }
  if (pref) cublasLtMatmulPreferenceDestroy(pref);
  if (lc) cublasLtMatrixLayoutDestroy(lc);
  if (lb) cublasLtMatrixLayoutDestroy(lb);
  if (la) cublasLtMatrixLayoutDestroy(la);
  if (op) cublasLtMatmulDescDestroy(op);
  return rc;
}

}  // namespace tmb
