// esg_noalloc.cu -- a scoring entry point that allocates no memory.
//
// Some callers cannot call cudaMalloc when they need scores: a process whose
// device memory belongs to a framework's caching allocator, which forbids
// allocations behind its back (they fragment its pool and escape its
// budget), or a real-time loop that must not enter the driver's allocator
// after start-up (cudaMalloc and cudaFree can block and synchronize the
// device).  esg_score_rows_noalloc serves them: the caller passes device
// buffers for the inputs and the output, and the one other buffer the int32
// kernel needs -- the column buffer that carries a reference's bottom row
// from one pass of a long query to the next (max_ref_len int2 per warp) --
// is the file-scope device array below.
//
// Under lazy module loading (the default since CUDA 12.2) that array is
// reserved on a device when the module is first loaded there, which the
// first call's cudaGetSymbolAddress triggers: that first call on a device
// can therefore fail for want of device memory.  On the host the array's
// name is a stand-in symbol, not a device address; the first call on each
// device, with that device current, looks the address up and keeps it for
// the life of the process (scratch_on_current_device).
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
                           "(8192); the static column buffer holds 2^21 columns");
    return ESG_ERR_REFERENCE_TOO_LONG;
  }
  if (n_queries == 0 || n_refs == 0) return ESG_OK;
  int2* scratch = nullptr;
  cudaError_t e = scratch_on_current_device(&scratch);
  if (e != cudaSuccess) {
    // the first call on a device loads the module and so reserves the array
    const esg_status st =
        e == cudaErrorMemoryAllocation ? ESG_ERR_OUT_OF_MEMORY : ESG_ERR_DRIVER;
    esg_internal_set_error(st, cudaGetErrorString(e));
    return st;
  }
  int dev = 0, sms = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  // one reference's bottom row (max_ref_len columns) per warp must fit the
  // static array: at most kScratchInt2 / max_ref_len warps
  const size_t cols = max_ref_len ? max_ref_len : 1;
  size_t blocks = std::min<size_t>((size_t)sms * 4, kScratchInt2 / (cols * kK3Warps));
  if (blocks == 0) blocks = 1;  // max_ref_len <= 8192 keeps 64 CTAs in bounds
  K3Params P{};
  P.codes = d_codes;
  P.off = d_off;
  P.len = d_len;
  P.n_reads = n_queries;
  P.list = nullptr;  // query p is read p, forward
  P.host_count = n_queries;
  P.rcodes = d_ref_codes;
  P.roff = d_ref_off;
  P.rlen = d_ref_len;
  P.ridx = nullptr;  // the caller's reference order
  P.n_refs = n_refs;
  P.max_cols = max_ref_len;
  P.out = nullptr;
  P.rows = d_rows;
  P.wmax = 32;
  P.refs_per_task = 32;
  P.task_counter = nullptr;  // units taken warp-strided: no counter to clear
  P.colbuf = scratch;
  P.ma = s.match_score;
  P.mi = s.mismatch;
  P.o = s.gap_open;
  P.e = s.gap_extend;
  P.one = 1;
  void* args[] = {&P};
  const void* fn = mode == ESG_MODE_LOCAL ? (const void*)k3_lanes<true>
                                          : (const void*)k3_lanes<false>;
  e = cudaLaunchKernel(fn, dim3((unsigned)blocks), dim3(kK3Threads), args, 0,
                       (cudaStream_t)stream);
  if (e != cudaSuccess) {
    esg_internal_set_error(ESG_ERR_DRIVER, cudaGetErrorString(e));
    return ESG_ERR_DRIVER;
  }
  return ESG_OK;
}
