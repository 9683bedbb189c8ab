// ref_gpu.cu -- launcher for the reference's own GPU kernels (comparison
// arms only).
//
// TEST INFRASTRUCTURE: used by bench.py's comparison arms and the tests,
// never by the product.  Loads oracle/_ref/ref_kernels.cubin -- the
// reference's align_score_kernel and align_score_kernel_h2
// (crates/eschalign/src/cuda/kernel.rs), compiled ahead of time for sm_100a
// from their source by oracle/Makefile -- and drives them the way
// eschalign's GpuScorer does:
//   * Layout::new (cuda/mod.rs:237-295): references longest first (stable),
//     one (int) or two (half2) per thread, grouped into blocks of at most 256
//     lanes that fit 48 KB of shared memory, 4-bit masks at 8 (int) or 4
//     (half2) columns per word, sp[word * lanes + lane]; grid
//     (ceil(SMs * blocks per SM / groups), groups);
//   * prepare (cuda/mod.rs:532-576): each query's 4-bit masks in whole
//     16-row stripes, the work list longest first;
//   * submit (cuda/mod.rs:581-699): the argument lists, per-group counters
//     zeroed, the scratch max_ref_len words (int) or uint2s (half2) per
//     launched thread, one int16 result per (query, reference).
#include <cuda.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

namespace {

constexpr int kMaxLanes = 256;
constexpr size_t kSmemBudget = 48 * 1024;
constexpr int kStripeRows = 16;

uint32_t mask_of(uint8_t c) { return c < 4 ? 1u << c : 0xFu; }

uint32_t half2_bits(int v) {
  const __half h = __float2half((float)v);  // exact for |v| <= 2048
  uint16_t b;
  memcpy(&b, &h, 2);
  return (uint32_t)b | ((uint32_t)b << 16);
}

struct Layout {
  bool ok = false;
  CUfunction fn = nullptr;
  int per_thread = 1, scratch_words = 1;
  int lanes = 0, n_groups = 0, grid_x = 0, words_per_lane = 0;
  size_t smem = 0;
  uint32_t* d_panel = nullptr;
  int* d_len = nullptr;
  int* d_idx = nullptr;
  size_t threads() const { return (size_t)grid_x * n_groups * lanes; }
};

struct RefGpu {
  int device = 0;
  CUmodule mod = nullptr;
  Layout lay[2];  // int, half2
  uint32_t n_refs = 0, max_len = 0;
  uint32_t* d_scratch = nullptr;
  std::string err;
};

#define RG_CU(call)                                                       \
  do {                                                                    \
    CUresult r_ = (call);                                                 \
    if (r_ != CUDA_SUCCESS) {                                             \
      const char* s_ = nullptr;                                           \
      cuGetErrorString(r_, &s_);                                          \
      g->err = std::string(#call) + ": " + (s_ ? s_ : "?");               \
      return 2;                                                           \
    }                                                                     \
  } while (0)
#define RG_RT(call)                                                       \
  do {                                                                    \
    cudaError_t e_ = (call);                                              \
    if (e_ != cudaSuccess) {                                              \
      g->err = std::string(#call) + ": " + cudaGetErrorString(e_);        \
      return 2;                                                           \
    }                                                                     \
  } while (0)

int build_layout(RefGpu* g, Layout& L, const char* name, int per_thread, int scratch_words,
                 const std::vector<uint32_t>& order, const uint8_t* codes, const uint64_t* off,
                 const uint32_t* len) {
  RG_CU(cuModuleGetFunction(&L.fn, g->mod, name));
  L.per_thread = per_thread;
  L.scratch_words = scratch_words;
  const int cols_per_word = 8 / per_thread;
  L.words_per_lane = (int)((g->max_len + cols_per_word - 1) / cols_per_word);
  int lanes = (int)((g->n_refs + per_thread - 1) / per_thread);
  lanes = std::min((lanes + 31) / 32 * 32, kMaxLanes);
  while (lanes > 32 && (size_t)L.words_per_lane * 4 * lanes > kSmemBudget) lanes -= 32;
  L.smem = (size_t)L.words_per_lane * 4 * lanes;
  if (L.smem > kSmemBudget) return 0;  // no layout (panel too long for this kernel)
  L.lanes = lanes;
  const int per_block = lanes * per_thread;
  L.n_groups = (int)((order.size() + per_block - 1) / per_block);
  std::vector<uint32_t> words((size_t)L.n_groups * L.words_per_lane * lanes, 0);
  std::vector<int> rlen((size_t)L.n_groups * per_block, 0), ridx((size_t)L.n_groups * per_block, -1);
  for (size_t i = 0; i < order.size(); ++i) {
    const size_t gi = i / per_block, slot = i % per_block;
    const size_t lane = slot / per_thread, h = slot % per_thread;
    const uint32_t r = order[i];
    rlen[gi * per_block + slot] = (int)len[r];
    ridx[gi * per_block + slot] = (int)r;
    const size_t base = gi * L.words_per_lane * lanes;
    for (uint32_t j = 0; j < len[r]; ++j) {
      const uint32_t shift = 4 * (j % cols_per_word) + 16 * h;
      words[base + (size_t)(j / cols_per_word) * lanes + lane] |= mask_of(codes[off[r] + j]) << shift;
    }
  }
  int per_sm = 0;
  RG_CU(cuOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, L.fn, lanes, L.smem));
  int sms = 0;
  RG_RT(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, g->device));
  L.grid_x = std::max(1, (std::max(sms, 1) * std::max(per_sm, 1) + L.n_groups - 1) / L.n_groups);
  RG_RT(cudaMalloc(&L.d_panel, words.size() * 4));
  RG_RT(cudaMemcpy(L.d_panel, words.data(), words.size() * 4, cudaMemcpyHostToDevice));
  RG_RT(cudaMalloc(&L.d_len, rlen.size() * 4));
  RG_RT(cudaMemcpy(L.d_len, rlen.data(), rlen.size() * 4, cudaMemcpyHostToDevice));
  RG_RT(cudaMalloc(&L.d_idx, ridx.size() * 4));
  RG_RT(cudaMemcpy(L.d_idx, ridx.data(), ridx.size() * 4, cudaMemcpyHostToDevice));
  L.ok = true;
  return 0;
}

}  // namespace

extern "C" {

const char* rg_error(void* h) { return h ? ((RefGpu*)h)->err.c_str() : "NULL handle"; }

void rg_free(void* h) {
  auto* g = (RefGpu*)h;
  if (!g) return;
  cudaSetDevice(g->device);
  for (auto& L : g->lay) {
    cudaFree(L.d_panel);
    cudaFree(L.d_len);
    cudaFree(L.d_idx);
  }
  cudaFree(g->d_scratch);
  if (g->mod) cuModuleUnload(g->mod);
  delete g;
}

// The panel on `device` with the reference's two layouts; `cubin` is the
// compiled oracle/_ref/ref_kernels.cubin.  Returns 0, or non-zero with
// rg_error(*out) set (*out must still be freed).
int rg_new(int device, const char* cubin, const uint8_t* codes, const uint64_t* off,
           const uint32_t* len, uint32_t n_refs, void** out) {
  auto* g = new RefGpu();
  *out = g;
  g->device = device;
  g->n_refs = n_refs;
  for (uint32_t r = 0; r < n_refs; ++r) g->max_len = std::max(g->max_len, len[r]);
  RG_RT(cudaSetDevice(device));
  RG_RT(cudaFree(nullptr));  // the primary context, current for the driver API
  RG_CU(cuModuleLoad(&g->mod, cubin));
  std::vector<uint32_t> order(n_refs);
  std::iota(order.begin(), order.end(), 0u);
  std::stable_sort(order.begin(), order.end(),
                   [&](uint32_t a, uint32_t b) { return len[a] > len[b]; });
  if (int rc = build_layout(g, g->lay[0], "align_score_kernel", 1, 1, order, codes, off, len))
    return rc;
  if (int rc = build_layout(g, g->lay[1], "align_score_kernel_h2", 2, 2, order, codes, off, len))
    return rc;
  size_t words = 0;
  for (auto& L : g->lay)
    if (L.ok) words = std::max(words, L.threads() * L.scratch_words);
  words *= std::max<uint32_t>(g->max_len, 1);
  RG_RT(cudaMalloc(&g->d_scratch, words * 4));
  RG_RT(cudaMemset(g->d_scratch, 0, words * 4));
  return 0;
}

// Geometry of layout `kernel` (0 int, 1 half2): lanes, groups, grid_x, smem;
// all 0 when the kernel has no layout for this panel.
void rg_geometry(void* h, int kernel, int* out4) {
  auto* g = (RefGpu*)h;
  const Layout& L = g->lay[kernel & 1];
  out4[0] = L.ok ? L.lanes : 0;
  out4[1] = L.ok ? L.n_groups : 0;
  out4[2] = L.ok ? L.grid_x : 0;
  out4[3] = L.ok ? (int)L.smem : 0;
}

// Score n_q queries (codes as for the product) with kernel 0 (int) or 1
// (half2) under one scoring and mode, `reps` launches after one untimed
// warm-up; *ms = mean device time of a launch (CUDA events); `out` (may be
// NULL) gets the int16 scores [q * n_refs + r].  The caller keeps every
// query within the reference's own routing bounds (fits_i16; fits_f16 for
// half2; 1..4096 nt).
int rg_score(void* h, int kernel, const uint8_t* codes, const uint64_t* off, const uint32_t* len,
             uint32_t n_q, int32_t ma, int32_t mi, int32_t o, int32_t e, int local, int reps,
             int16_t* out, float* ms) {
  auto* g = (RefGpu*)h;
  Layout& L = g->lay[kernel & 1];
  if (!L.ok) {
    g->err = "no layout for this kernel";
    return 1;
  }
  RG_RT(cudaSetDevice(g->device));
  // prepare: masks in whole 16-row stripes (2 words each), longest first
  std::vector<unsigned long long> qoff(n_q);
  std::vector<int> qlen(n_q);
  size_t total = 0;
  for (uint32_t k = 0; k < n_q; ++k) {
    qoff[k] = total;
    qlen[k] = (int)len[k];
    total += (size_t)(len[k] + kStripeRows - 1) / kStripeRows * (kStripeRows / 8);
  }
  std::vector<uint32_t> qwords(std::max<size_t>(total, 1), 0);
  for (uint32_t k = 0; k < n_q; ++k)
    for (uint32_t i = 0; i < len[k]; ++i)
      qwords[qoff[k] + i / 8] |= mask_of(codes[off[k] + i]) << (4 * (i % 8));
  std::vector<int> work(n_q);
  std::iota(work.begin(), work.end(), 0);
  std::stable_sort(work.begin(), work.end(), [&](int a, int b) { return len[a] > len[b]; });
  uint32_t *d_q = nullptr;
  unsigned long long* d_qoff = nullptr;
  int *d_qlen = nullptr, *d_work = nullptr, *d_cnt = nullptr;
  int16_t* d_out = nullptr;
  const size_t n_out = std::max<size_t>((size_t)n_q * g->n_refs, 1);
  RG_RT(cudaMalloc(&d_q, qwords.size() * 4));
  RG_RT(cudaMalloc(&d_qoff, std::max<size_t>(n_q, 1) * 8));
  RG_RT(cudaMalloc(&d_qlen, std::max<size_t>(n_q, 1) * 4));
  RG_RT(cudaMalloc(&d_work, std::max<size_t>(n_q, 1) * 4));
  RG_RT(cudaMalloc(&d_cnt, (size_t)L.n_groups * 4));
  RG_RT(cudaMalloc(&d_out, n_out * 2));
  RG_RT(cudaMemcpy(d_q, qwords.data(), qwords.size() * 4, cudaMemcpyHostToDevice));
  if (n_q) {
    RG_RT(cudaMemcpy(d_qoff, qoff.data(), n_q * 8, cudaMemcpyHostToDevice));
    RG_RT(cudaMemcpy(d_qlen, qlen.data(), n_q * 4, cudaMemcpyHostToDevice));
    RG_RT(cudaMemcpy(d_work, work.data(), n_q * 4, cudaMemcpyHostToDevice));
  }
  RG_RT(cudaMemset(d_out, 0, n_out * 2));
  int n_work = (int)n_q, n_refs = (int)g->n_refs, wpl = L.words_per_lane;
  uint32_t mi2 = half2_bits(mi), d2 = half2_bits(ma - mi), o2 = half2_bits(o), e2 = half2_bits(e);
  void* a_int[] = {&d_q, &d_qoff, &d_qlen, &d_work, &L.d_panel, &L.d_len, &L.d_idx, &d_out,
                   &g->d_scratch, &d_cnt, &n_work, &n_refs, &wpl, &ma, &mi, &o, &e, &local};
  void* a_h2[] = {&d_q, &d_qoff, &d_qlen, &d_work, &L.d_panel, &L.d_len, &L.d_idx, &d_out,
                  &g->d_scratch, &d_cnt, &n_work, &n_refs, &wpl, &mi2, &d2, &o2, &e2, &local};
  cudaEvent_t e0, e1;
  RG_RT(cudaEventCreate(&e0));
  RG_RT(cudaEventCreate(&e1));
  float total_ms = 0;
  for (int rep = -1; rep < std::max(reps, 1); ++rep) {
    RG_RT(cudaMemsetAsync(d_cnt, 0, (size_t)L.n_groups * 4, 0));
    RG_RT(cudaEventRecord(e0, 0));
    RG_CU(cuLaunchKernel(L.fn, L.grid_x, L.n_groups, 1, L.lanes, 1, 1, (unsigned)L.smem, 0,
                         kernel ? a_h2 : a_int, nullptr));
    RG_RT(cudaEventRecord(e1, 0));
    RG_RT(cudaEventSynchronize(e1));
    float t = 0;
    RG_RT(cudaEventElapsedTime(&t, e0, e1));
    if (rep >= 0) total_ms += t;
  }
  *ms = total_ms / std::max(reps, 1);
  if (out) RG_RT(cudaMemcpy(out, d_out, (size_t)n_q * g->n_refs * 2, cudaMemcpyDeviceToHost));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(d_q);
  cudaFree(d_qoff);
  cudaFree(d_qlen);
  cudaFree(d_work);
  cudaFree(d_cnt);
  cudaFree(d_out);
  return 0;
}

}  // extern "C"
