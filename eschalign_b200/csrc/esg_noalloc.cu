// esg_noalloc.cu -- a scoring entry point that allocates no memory.
//
// Some callers cannot call cudaMalloc: code running inside a CUDA graph
// being built by someone else, a host process whose allocator is owned by a
// framework that forbids side allocations, or a real-time loop that must not
// touch the driver's allocator after start-up.  esg_score_rows_noalloc
// serves them: the caller passes device buffers for the inputs and the
// output, and the only other memory the plain int32 kernel needs -- its
// stripe-boundary scratch (one int2 per reference column per thread) -- is
// the file-scope device array below, reserved when the library is loaded.
//
// That array is host-side a stand-in symbol, not a device address; host code
// gets its device address with cudaGetSymbolAddress, once per device, with
// that device current (see scratch_on_current_device).
#include "../../include/eschalign_b200.h"
#include "esg_kernels.cuh"

#include <algorithm>
#include <cstdlib>
#include <mutex>

using namespace esg;

extern "C" void esg_internal_set_error(esg_status st, const char* msg);

namespace {

// 2 Mi int2 = 16 MiB on every GPU that loads the library, held until exit.
constexpr size_t kScratchInt2 = (size_t)2 << 20;
static __device__ __align__(256) int2 g_noalloc_scratch[kScratchInt2];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
int2* g_ptr[kMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device, looked up once
// per device.
cudaError_t scratch_on_current_device(int2** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_ptr[dev] = static_cast<int2*>(p);
  }
  *out = g_ptr[dev];
  return cudaSuccess;
}

struct NoAllocParams {
  const uint8_t* codes;   // queries, scored as given (forward only)
  const uint64_t* off;
  const uint32_t* len;
  uint32_t n_queries;
  const uint8_t* rcodes;  // references in the caller's order
  const uint32_t* roff;
  const uint32_t* rlen;
  uint32_t n_refs;
  int32_t* rows;          // [q * n_refs + r]
  int2* scratch;
  uint32_t max_cols;      // the caller's max_ref_len: the scratch is sized for it
  int32_t ma, mi, o, e;
};

// k3_plain with the query list and reference order taken as the identity:
// one thread per (query, reference), int32 stripes, boundary in `scratch`.
template <bool kLocal>
__global__ void __launch_bounds__(kK3Threads) k3_noalloc(const NoAllocParams P) {
  const uint64_t total = (uint64_t)P.n_queries * P.n_refs;
  const size_t nthreads = (size_t)gridDim.x * blockDim.x;
  const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  int2* bnd = P.scratch + tid;
  for (uint64_t idx = tid; idx < total; idx += nthreads) {
    const uint32_t q = (uint32_t)(idx / P.n_refs);
    const uint32_t k = (uint32_t)(idx % P.n_refs);
    const int n = (int)P.len[q];
    const uint8_t* qc = P.codes + P.off[q];
    const int m = (int)P.rlen[k];
    if ((uint32_t)m > P.max_cols) {
      // longer than the caller said: the scratch has no room for its columns
      P.rows[(size_t)q * P.n_refs + k] = INT32_MIN;
      continue;
    }
    const uint8_t* rcodes = P.rcodes + P.roff[k];
    int best = kLocal ? 0 : kNeg32;
    for (int i0 = 0; i0 < n; i0 += kRows) {
      uint32_t qm[kRows];
#pragma unroll
      for (int r = 0; r < kRows; ++r) {
        const int i = i0 + r;
        qm[r] = i < n ? code_mask(qc[i] > 4 ? 4u : qc[i]) : 0u;
      }
      const int rows = min(kRows, n - i0);
      if (i0 + kRows >= n)
        k3_stripe<kLocal, true>(rcodes, m, qm, rows, i0 == 0, bnd, nthreads, P.ma, P.mi, P.o,
                                P.e, best);
      else
        k3_stripe<kLocal, false>(rcodes, m, qm, rows, i0 == 0, bnd, nthreads, P.ma, P.mi, P.o,
                                 P.e, best);
    }
    if (n == 0 || m == 0) best = 0;  // scalar.rs:123-125
    P.rows[(size_t)q * P.n_refs + k] = best;
  }
}

}  // namespace

extern "C" esg_status esg_score_rows_noalloc(const uint8_t* d_codes, const uint64_t* d_off,
                                             const uint32_t* d_len, uint32_t n_queries,
                                             const uint8_t* d_ref_codes, const uint32_t* d_ref_off,
                                             const uint32_t* d_ref_len, uint32_t n_refs,
                                             uint32_t max_ref_len, const esg_scoring* scoring,
                                             int32_t mode, int32_t* d_rows, void* stream) {
  if (!scoring || (n_queries && (!d_codes || !d_off || !d_len || !d_rows)) ||
      (n_refs && (!d_ref_codes || !d_ref_off || !d_ref_len))) {
    esg_internal_set_error(ESG_ERR_BAD_ARGUMENT, "esg_score_rows_noalloc: NULL argument");
    return ESG_ERR_BAD_ARGUMENT;
  }
  if (mode != ESG_MODE_LOCAL && mode != ESG_MODE_SEMIGLOBAL) {
    esg_internal_set_error(ESG_ERR_BAD_ARGUMENT, "esg_score_rows_noalloc: bad mode");
    return ESG_ERR_BAD_ARGUMENT;
  }
  const esg_scoring s = *scoring;
  if (s.match_score <= 0 || s.mismatch >= s.match_score || s.gap_open > 0 || s.gap_extend > 0 ||
      std::abs(s.match_score) > 1000 || std::abs(s.mismatch) > 1000 ||
      std::abs(s.gap_open) > 1000 || std::abs(s.gap_extend) > 1000) {
    esg_internal_set_error(ESG_ERR_SCORING_INVALID, "esg_score_rows_noalloc: invalid scoring");
    return ESG_ERR_SCORING_INVALID;
  }
  if (max_ref_len > ESG_NOALLOC_MAX_REF_LEN) {
    esg_internal_set_error(ESG_ERR_REFERENCE_TOO_LONG,
                           "esg_score_rows_noalloc: max_ref_len exceeds ESG_NOALLOC_MAX_REF_LEN "
                           "(8192); the static scratch holds 2^21 columns x threads");
    return ESG_ERR_REFERENCE_TOO_LONG;
  }
  if (n_queries == 0 || n_refs == 0) return ESG_OK;
  int2* scratch = nullptr;
  cudaError_t e = scratch_on_current_device(&scratch);
  if (e != cudaSuccess) {
    esg_internal_set_error(ESG_ERR_DRIVER, cudaGetErrorString(e));
    return ESG_ERR_DRIVER;
  }
  int dev = 0, sms = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  // threads x max_ref_len boundary cells must fit the static scratch
  const size_t cols = max_ref_len ? max_ref_len : 1;
  size_t threads = std::min<size_t>((size_t)sms * 4 * kK3Threads, kScratchInt2 / cols);
  threads = threads / kK3Threads * kK3Threads;
  if (threads == 0) threads = kK3Threads;  // max_ref_len <= 8192 keeps this in bounds
  NoAllocParams P{d_codes, d_off, d_len, n_queries, d_ref_codes, d_ref_off, d_ref_len, n_refs,
                  d_rows, scratch, (uint32_t)cols, s.match_score, s.mismatch, s.gap_open,
                  s.gap_extend};
  void* args[] = {&P};
  const void* fn = mode == ESG_MODE_LOCAL ? (const void*)k3_noalloc<true>
                                          : (const void*)k3_noalloc<false>;
  e = cudaLaunchKernel(fn, dim3((unsigned)(threads / kK3Threads)), dim3(kK3Threads), args, 0,
                       (cudaStream_t)stream);
  if (e != cudaSuccess) {
    esg_internal_set_error(ESG_ERR_DRIVER, cudaGetErrorString(e));
    return ESG_ERR_DRIVER;
  }
  return ESG_OK;
}
