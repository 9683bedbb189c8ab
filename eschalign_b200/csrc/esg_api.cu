// esg_api.cu -- host side of the B200 panel scorer: the C ABI of
// include/eschalign_b200.h.
//
// Mirrors eschalign's GpuScorer (crates/eschalign/src/cuda/mod.rs:328-709):
// a panel laid out once on one device under one scoring and mode, batches
// prepared on the host (prepare), queued (submit) and collected (finish).
// What differs is what the device does with a batch (esg_kernels.cuh): every
// query is scored on the GPU -- nothing is left unscored for a CPU path --
// and the per-read best / XS / tie reduction runs there too.
#include "../../include/eschalign_b200.h"
#include "esg_internal.h"
#include "esg_kernels.cuh"

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

using namespace esg;

namespace {

thread_local std::string g_err;

esg_status fail(esg_status st, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
  return st;
}

esg_status cuda_fail(cudaError_t e, const char* what) {
  const esg_status st = (e == cudaErrorMemoryAllocation) ? ESG_ERR_OUT_OF_MEMORY
                        : (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver)
                            ? ESG_ERR_UNAVAILABLE
                            : ESG_ERR_DRIVER;
  return fail(st, "%s: %s", what, cudaGetErrorString(e));
}

#define ESG_CUDA(call)                                   \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call);  \
  } while (0)

constexpr uint32_t kMaxRefLen = 32768;
// device memory k3's column buffers may take (per scorer and arm)
constexpr size_t kColbufBudget = (size_t)1 << 30;
constexpr int kPad = 5;     // selector / table index of a padding column or row
constexpr int kWild = 4;

inline uint32_t code_of(uint8_t c) { return c > 4 ? 4u : c; }

// Pinned host memory, reused across batches of one scorer.
struct PinnedPool {
  std::mutex mu;
  std::vector<std::pair<void*, size_t>> free_;
  void* get(size_t bytes, size_t* got) {
    bytes = std::max<size_t>(bytes, 64);
    std::lock_guard<std::mutex> lk(mu);
    size_t best = (size_t)-1;
    for (size_t k = 0; k < free_.size(); ++k)
      if (free_[k].second >= bytes && (best == (size_t)-1 || free_[k].second < free_[best].second))
        best = k;
    if (best != (size_t)-1) {
      auto p = free_[best];
      free_.erase(free_.begin() + best);
      *got = p.second;
      return p.first;
    }
    void* p = nullptr;
    const size_t sz = bytes + bytes / 8;
    if (cudaHostAlloc(&p, sz, cudaHostAllocDefault) != cudaSuccess) return nullptr;
    *got = sz;
    return p;
  }
  void put(void* p, size_t sz) {
    if (!p) return;
    std::lock_guard<std::mutex> lk(mu);
    free_.push_back({p, sz});
  }
  ~PinnedPool() {
    for (auto& b : free_) cudaFreeHost(b.first);
  }
};

struct Pinned {
  void* p = nullptr;
  size_t cap = 0;
};

}  // namespace

struct esg_scorer {
  int device = 0;
  int sm_count = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  esg_scoring scoring{};
  int mode = ESG_MODE_LOCAL;
  int kernel = ESG_KERNEL_AUTO;
  uint32_t cap = 8;
  uint32_t n_refs = 0;
  uint32_t max_ref_len = 0;
  uint64_t panel_bases = 0;
  bool panel_w = false;
  bool batched_ok = false;
  // k2 panel
  uint32_t n_pairs = 0;
  uint32_t blob_bytes = 0;
  uint32_t sel_base = 0;
  bool smem_panel = false;
  void* d_blob = nullptr;
  std::vector<uint64_t> pair_cols;  // prefix sums of the pairs' column counts
  uint32_t tab_a[6]{}, tab_b[6]{};
  int sat = 0;
  size_t k2_smem = 0;
  uint2* d_lbuf = nullptr;   // long queries: one column buffer per k2 warp
  uint32_t lbuf_cols = 0;
  const void* k2_t16 = nullptr;   // tiles of 16-row stripes
  const void* k2_t32 = nullptr;   // tiles of 32-row stripes
  const void* k2_long = nullptr;  // one long query, 32-row stripes, in passes
  int blocks_t16 = 0, blocks_t32 = 0, blocks_long = 0;
  // semi-global: the same three with every cell's maximum checked against
  // the int16 lanes' upper limit, for batches holding queries past the
  // static bound (k2_checks)
  const void* k2c_t16 = nullptr;
  const void* k2c_t32 = nullptr;
  const void* k2c_long = nullptr;
  int blocksc_t16 = 0, blocksc_t32 = 0, blocksc_long = 0;
  // queries up to split_len bases take 16-row stripes, longer ones 32-row
  // stripes (esg_scorer_autotune measures where 32 rows start to win)
  uint32_t split_len = 256;
  bool tuned = false;
  // queries of this length and longer go to the int32 lanes instead of the
  // batched kernel (0: none; set by the autotuner where the batched kernel
  // would flag most of them)
  uint32_t int32_from = 0;
  // panel chunking aims for this many tasks per resident warp
  uint32_t chunk_target = 8;
  uint32_t max_chunks = 64;  // panel chunks per tile at most (1: never chunk)
  cudaStream_t aux = nullptr;          // second stream: the long-query kernel
  // batches' device memory: a pool of this scorer's own that keeps what
  // finished batches return, so the next batch maps no new memory
  cudaMemPool_t pool = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
  // k3 panel (longest first)
  uint8_t* d_rcodes = nullptr;
  uint32_t* d_roff = nullptr;
  uint32_t* d_rlen = nullptr;
  uint32_t* d_ridx = nullptr;
  std::vector<uint32_t> slot_of;   // reference -> slot of the k3 panel
  std::vector<uint32_t> len_of;    // reference lengths, panel order
  std::vector<uint8_t> h_codes;    // the panel's codes (0-4), panel order (host)
  std::vector<uint64_t> h_off;     // reference r at h_codes[h_off[r]]
  // k3's column buffers (a chain's bottom row between passes): per warp
  // max_ref_len int2 for the int32 lanes, 32x that for one thread per pair
  // (32 chains a warp), made when that arm is first chosen
  int2* d_colbuf = nullptr;
  int2* d_colbuf1 = nullptr;
  int k3_blocks = 0;   // CTAs of k3 (int32 lanes)
  int k3_blocks1 = 0;  // CTAs of k3 as one thread per pair (bounded by its buffer)
  const void* k3_fn = nullptr;
  PinnedPool pinned;
  esg_info info{};
  // CUDA graphs of batches' launch sequences: one instantiated graph per
  // sequence shape (which kernels a batch launches), updated in place with
  // each batch's parameters before it is launched
  bool use_graphs = true;
  std::vector<std::pair<uint32_t, cudaGraphExec_t>> graph_execs;
};

struct esg_batch {
  uint32_t n_reads = 0;
  uint32_t flags = 0;
  uint32_t n_q = 0;
  int kernel = ESG_KERNEL_AUTO;
  uint64_t total_bases = 0;
  // upload: reads packed at 2 bits a base, each read starting on a byte
  // (its offset a multiple of 4 bases); positions of bases that are not
  // A/C/G/T travel as a list and become the wildcard code on the device
  uint64_t padded_bases = 0;  // sum of lengths rounded up to 4
  uint64_t code_words = 0;    // 32-bit packed words (16 bases each) unpacked
  std::vector<uint64_t> exceptions;
  // host plan
  uint32_t n_tasks = 0;
  uint32_t n_long = 0;   // tasks are [n_long long | n_t32 tiles | n_t16 tiles]
  uint32_t n_t32 = 0;
  uint32_t n_t16 = 0;
  uint32_t n_order = 0;
  uint32_t host_list = 0;
  uint32_t redo_cap = 0;
  uint32_t n_chunks = 1;  // panel chunks per tile (k2 tasks = tiles x chunks)
  bool sg_check = false;  // semi-global: run the checked k2 variants
  // paired batches (esg_prepare_pairs): reads 2p, 2p + 1 are pair p's mates
  bool paired = false;
  bool pair_both = false;   // rank both template strands
  int32_t min_score = 0;
  uint32_t n_pairs = 0;
  std::vector<uint32_t> adapters;  // adapter bases removed, per mate
  // pinned staging (inputs, then outputs)
  Pinned in_buf, out_buf;
  uint8_t* h_packed = nullptr;
  uint64_t* h_off = nullptr;
  uint32_t* h_len = nullptr;
  uint32_t* h_order = nullptr;
  uint2* h_tasks = nullptr;
  uint32_t* h_list = nullptr;
  uint32_t* h_chunks = nullptr;
  size_t in_bytes = 0;
  int4* h_results = nullptr;
  uint32_t* h_ties = nullptr;
  int32_t* h_rows = nullptr;
  uint32_t* h_counters = nullptr;
  int4* h_pairs = nullptr;
  uint32_t* h_pties = nullptr;
  // device
  void* d_mem = nullptr;
  size_t d_bytes = 0;
  uint8_t* d_codes = nullptr;   // one byte a base, unpacked on the device
  uint8_t* d_packed = nullptr;  // the upload
  uint64_t* d_exc = nullptr;
  uint64_t* d_off = nullptr;
  uint32_t* d_len = nullptr;
  uint32_t* d_order = nullptr;
  uint2* d_tasks = nullptr;
  uint32_t* d_list = nullptr;
  uint32_t* d_chunks = nullptr;
  int4* d_part_head = nullptr;
  uint32_t* d_part_ties = nullptr;
  uint32_t* d_counters = nullptr;
  int4* d_qhead = nullptr;
  uint32_t* d_qties = nullptr;
  int32_t* d_k3out = nullptr;
  int4* d_results = nullptr;
  uint32_t* d_ties = nullptr;
  int32_t* d_rows = nullptr;
  int4* d_pairs = nullptr;
  uint32_t* d_pties = nullptr;
  cudaEvent_t done = nullptr;
  cudaGraph_t graph = nullptr;  // this batch's launch sequence, captured at submit
  uint32_t graph_key = 0;       // its shape
  bool submitted = false;
  esg_scorer* owner = nullptr;
  esg_batch_stats stats{};
};

extern "C" {
static esg_status launch_device_work(esg_scorer* sc, esg_batch* b, cudaStream_t st);
static esg_status launch_work(esg_scorer* sc, esg_batch* b, cudaStream_t st);
}

namespace {

// Static bound on every cell of a query of n rows (simd/mod.rs:59-69 argues
// the same bound for its i16 lanes): |H| <= min(n, L) * max(|ma|, |mi|).
int64_t value_bound(uint64_t n, uint32_t max_ref_len, const esg_scoring& s) {
  const int64_t k = (int64_t)std::min<uint64_t>(n, max_ref_len);
  const int64_t mm = std::max(std::abs(s.match_score), std::abs(s.mismatch));
  return k * mm + std::abs(s.gap_open) + std::abs(s.gap_extend);
}

// Semi-global cells go negative, and the biased lanes (H - 16384) must stay
// above the -infinity stand-in (-31500): every H is at least
// o + (min(i, j) - 1) e (a gap from the zero border), every E and F at least
// that + o, so 2 |o| + (min(n, L) - 1) |e| below 15000 keeps them there.
bool sg_floor_ok(const esg_scorer* sc, uint64_t n) {
  const int64_t k = (int64_t)std::min<uint64_t>(n, sc->max_ref_len);
  return 2 * (int64_t)std::abs(sc->scoring.gap_open) +
             (k - 1) * (int64_t)std::abs(sc->scoring.gap_extend) <
         15000;
}

// Semi-global queries inside this static bound never reach H = 12000 and run
// unchecked; past it the checked variant watches every cell's maximum and
// flags the query for the int32 re-score when one reaches 16384.
bool k2_checks(const esg_scorer* sc, uint64_t n) {
  if (sc->mode != ESG_MODE_SEMIGLOBAL) return false;
  const int64_t mm = std::max(std::abs(sc->scoring.match_score), std::abs(sc->scoring.mismatch));
  return value_bound(n, sc->max_ref_len, sc->scoring) + mm >= 12000;
}

bool k2_takes(const esg_scorer* sc, uint64_t n) {
  if (!sc->batched_ok || n == 0) return false;
  // queries over 32 stripes of 32 rows run in passes chained through the
  // column buffer
  if ((n + 31) / 32 > (uint64_t)kMaxStripes && !sc->d_lbuf) return false;
  if ((n + 31) / 32 > 0xffffu) return false;
  if (sc->mode == ESG_MODE_SEMIGLOBAL) return sg_floor_ok(sc, n);
  return true;  // local: a wrap is detected by the kernel (K2Params::sat)
}

// Queries whose k2 result may be flagged for the int32 re-score.
bool k2_may_flag(const esg_scorer* sc, uint64_t n) {
  if (sc->mode != ESG_MODE_LOCAL) return k2_checks(sc, n);
  const int64_t hmax = (int64_t)std::min<uint64_t>(n, sc->max_ref_len) * sc->scoring.match_score;
  return hmax >= sc->sat;
}

template <typename T>
T* carve(char*& at, size_t count) {
  T* p = reinterpret_cast<T*>(at);
  at += ((count * sizeof(T)) + 255) / 256 * 256;
  return p;
}

size_t carve_size(size_t count, size_t elem) { return (count * elem + 255) / 256 * 256; }

template <int R, bool kLong, bool kLocal, bool kCheck>
const void* pick_k2_ws(bool w, bool smem) {
  if (w)
    return smem ? (const void*)k2_batched<R, kLocal, true, true, kLong, kCheck>
                : (const void*)k2_batched<R, kLocal, true, false, kLong, kCheck>;
  return smem ? (const void*)k2_batched<R, kLocal, false, true, kLong, kCheck>
              : (const void*)k2_batched<R, kLocal, false, false, kLong, kCheck>;
}

template <int R, bool kLong>
const void* pick_k2(bool local, bool check, bool w, bool smem) {
  if (local) return pick_k2_ws<R, kLong, true, false>(w, smem);
  return check ? pick_k2_ws<R, kLong, false, true>(w, smem)
               : pick_k2_ws<R, kLong, false, false>(w, smem);
}

void set_k2_fn(esg_scorer* sc) {
  const bool local = sc->mode == ESG_MODE_LOCAL;
  sc->k2_t16 = pick_k2<16, false>(local, false, sc->panel_w, sc->smem_panel);
  sc->k2_t32 = pick_k2<32, false>(local, false, sc->panel_w, sc->smem_panel);
  sc->k2_long = pick_k2<32, true>(local, false, sc->panel_w, sc->smem_panel);
  sc->k2c_t16 = pick_k2<16, false>(local, !local, sc->panel_w, sc->smem_panel);
  sc->k2c_t32 = pick_k2<32, false>(local, !local, sc->panel_w, sc->smem_panel);
  sc->k2c_long = pick_k2<32, true>(local, !local, sc->panel_w, sc->smem_panel);
  sc->k3_fn = local ? (const void*)k3_lanes<true> : (const void*)k3_lanes<false>;
}

// 32-lane tiles of query stripes: best-fit decreasing.  `qs` holds
// (stripes, query) with stripes <= 32; the plan lists queries tile by tile
// and one task per tile {start, count | stripes of its largest query << 16}.
struct TilePlan {
  std::vector<uint32_t> order;
  std::vector<uint2> tasks;
  uint32_t lanes = 0;
};

void pack_tiles(std::vector<std::pair<uint32_t, uint32_t>>& qs, TilePlan& out) {
  const size_t nq = qs.size();
  if (!nq) return;
  std::vector<uint32_t> count(kMaxStripes + 2, 0);
  for (const auto& x : qs) ++count[x.first];
  std::vector<uint32_t> start(kMaxStripes + 2, 0);  // descending stripes
  for (int S = kMaxStripes; S >= 1; --S) start[S - 1] = start[S] + count[S];
  std::vector<uint32_t> sorted(nq), sorted_s(nq);
  for (const auto& x : qs) {
    const uint32_t at = start[x.first]++;
    sorted[at] = x.second;
    sorted_s[at] = x.first;
  }
  std::vector<uint32_t> bin_of(nq);
  std::vector<uint8_t> bin_free, bin_smax;
  std::vector<uint16_t> bin_count;
  std::vector<std::vector<uint32_t>> open(kMaxStripes);  // by free capacity 1..31
  uint32_t open_mask = 0;
  for (size_t i = 0; i < nq; ++i) {
    const uint32_t S = sorted_s[i];
    const uint32_t cand = open_mask & ~((1u << S) - 1u);
    uint32_t bin;
    if (cand) {
      const uint32_t f = __builtin_ctz(cand);
      bin = open[f].back();
      open[f].pop_back();
      if (open[f].empty()) open_mask &= ~(1u << f);
    } else {
      bin = (uint32_t)bin_free.size();
      bin_free.push_back(kMaxStripes);
      bin_smax.push_back((uint8_t)S);
      bin_count.push_back(0);
    }
    bin_of[i] = bin;
    bin_free[bin] = (uint8_t)(bin_free[bin] - S);
    bin_count[bin]++;
    const uint32_t f = bin_free[bin];
    if (f > 0) {
      open[f].push_back(bin);
      open_mask |= 1u << f;
    }
  }
  const uint32_t n_bins = (uint32_t)bin_free.size();
  std::vector<uint32_t> tstart(n_bins + 1, 0);
  for (uint32_t t = 0; t < n_bins; ++t) tstart[t + 1] = tstart[t] + bin_count[t];
  std::vector<uint32_t> fill(tstart.begin(), tstart.end() - 1);
  out.order.assign(nq, 0);
  for (size_t i = 0; i < nq; ++i) out.order[fill[bin_of[i]]++] = sorted[i];
  out.tasks.resize(n_bins);
  for (uint32_t t = 0; t < n_bins; ++t) {
    out.tasks[t] = make_uint2(tstart[t], (uint32_t)bin_count[t] | ((uint32_t)bin_smax[t] << 16));
    out.lanes += kMaxStripes - bin_free[t];
  }
}

}  // namespace

// The one-thread-per-pair arm's column buffers: 32 chains a warp, each a
// reference's bottom row per column; the grid shrinks to what kColbufBudget
// holds.  Made once, on first use.
static esg_status make_plain_buffers(esg_scorer* sc) {
  if (sc->d_colbuf1) return ESG_OK;
  const size_t per_block = (size_t)kK3Warps * 32 * sc->max_ref_len * sizeof(int2);
  const int blocks = (int)std::max<size_t>(
      1, std::min<size_t>((size_t)sc->k3_blocks, kColbufBudget / per_block));
  const cudaError_t e = cudaMalloc(&sc->d_colbuf1, (size_t)blocks * per_block);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(one-thread-per-pair column buffers)");
  sc->k3_blocks1 = blocks;
  return ESG_OK;
}

// ===================================================================== API

extern "C" {

int esg_abi_version(void) { return ESG_ABI_VERSION; }

const char* esg_status_string(esg_status st) {
  switch (st) {
    case ESG_OK: return "ok";
    case ESG_ERR_UNAVAILABLE: return "CUDA unavailable";
    case ESG_ERR_DRIVER: return "CUDA driver error";
    case ESG_ERR_REFERENCE_TOO_LONG: return "reference too long";
    case ESG_ERR_SCORING_INVALID: return "invalid scoring";
    case ESG_ERR_EMPTY_PANEL: return "empty panel";
    case ESG_ERR_EMPTY_REFERENCE: return "empty reference";
    case ESG_ERR_BAD_ARGUMENT: return "bad argument";
    case ESG_ERR_OUT_OF_MEMORY: return "out of memory";
    case ESG_ERR_TIMEOUT: return "device wait timed out";
    default: return "unknown status";
  }
}

const char* esg_last_error(void) { return g_err.c_str(); }

// Lets the other translation unit of the library (esg_noalloc.cu) report
// through esg_last_error.
void esg_internal_set_error(esg_status st, const char* msg) {
  (void)st;
  g_err = msg ? msg : "";
}

esg_status esg_device_count(int32_t* out) {
  if (!out) return fail(ESG_ERR_BAD_ARGUMENT, "out is NULL");
  int n = 0;
  const cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess) {
    cudaGetLastError();
    *out = 0;
    return ESG_OK;
  }
  *out = n;
  return ESG_OK;
}

int32_t esg_fits_i16(uint64_t len, uint64_t max_ref_len, const esg_scoring* s) {
  if (!s) return 0;
  const int64_t k = (int64_t)std::min(len, max_ref_len);
  const int64_t mm = std::max(std::abs(s->match_score), std::abs(s->mismatch));
  const int64_t bound = k * mm + std::abs(s->gap_open) + std::abs(s->gap_extend);
  return bound < 15000 && max_ref_len < 15000;
}

esg_status esg_scorer_new(int32_t device, const uint8_t* ref_codes, const uint64_t* ref_off,
                          const uint32_t* ref_len, uint32_t n_refs, const esg_scoring* scoring,
                          int32_t mode, const esg_options* options, esg_scorer** out) {
  g_err.clear();
  if (!out || !scoring) return fail(ESG_ERR_BAD_ARGUMENT, "out and scoring must not be NULL");
  *out = nullptr;
  if (mode != ESG_MODE_LOCAL && mode != ESG_MODE_SEMIGLOBAL)
    return fail(ESG_ERR_BAD_ARGUMENT, "mode %d is not local (0) or semiglobal (1)", mode);
  // scoring.rs:70-100
  const esg_scoring s = *scoring;
  if (s.match_score <= 0)
    return fail(ESG_ERR_SCORING_INVALID, "match must be positive, got %d", s.match_score);
  if (s.mismatch >= s.match_score)
    return fail(ESG_ERR_SCORING_INVALID, "mismatch (%d) must score below match (%d)", s.mismatch,
                s.match_score);
  if (s.gap_open > 0 || s.gap_extend > 0)
    return fail(ESG_ERR_SCORING_INVALID,
                "gap scores are penalties and must be zero or negative, got open %d extend %d",
                s.gap_open, s.gap_extend);
  for (int32_t v : {s.match_score, s.mismatch, s.gap_open, s.gap_extend})
    if (std::abs(v) > 1000)
      return fail(ESG_ERR_SCORING_INVALID, "|%d| exceeds the supported magnitude 1000", v);
  // panel.rs:34-55
  if (n_refs == 0) return fail(ESG_ERR_EMPTY_PANEL, "the reference panel is empty");
  if (!ref_codes || !ref_off || !ref_len)
    return fail(ESG_ERR_BAD_ARGUMENT, "reference arrays must not be NULL");
  uint32_t max_len = 0;
  uint64_t bases = 0;
  for (uint32_t r = 0; r < n_refs; ++r) {
    if (ref_len[r] == 0) return fail(ESG_ERR_EMPTY_REFERENCE, "reference %u has no bases", r);
    max_len = std::max(max_len, ref_len[r]);
    bases += ref_len[r];
  }
  if (max_len > kMaxRefLen)
    return fail(ESG_ERR_REFERENCE_TOO_LONG,
                "the panel's longest reference (%u nt) exceeds the GPU kernel's %u nt", max_len,
                kMaxRefLen);
  uint32_t cap = 8;
  int kernel = ESG_KERNEL_AUTO;
  void* ext_stream = nullptr;
  if (options) {
    if (options->tie_capacity) cap = options->tie_capacity;
    kernel = options->kernel;
    ext_stream = options->stream;
  }
  if (cap < 1 || cap > ESG_MAX_TIE_CAPACITY)
    return fail(ESG_ERR_BAD_ARGUMENT, "tie_capacity %u outside 1..%d", cap, ESG_MAX_TIE_CAPACITY);
  if (kernel != ESG_KERNEL_AUTO && kernel != ESG_KERNEL_PLAIN32 && kernel != ESG_KERNEL_INT32)
    return fail(ESG_ERR_BAD_ARGUMENT, "unknown kernel %d", kernel);

  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(ESG_ERR_UNAVAILABLE, "no CUDA device is visible");
  }
  if (device < 0 || device >= ndev)
    return fail(ESG_ERR_UNAVAILABLE, "device %d not present (%d visible)", device, ndev);
  ESG_CUDA(cudaSetDevice(device));

  auto* sc = new esg_scorer();
  sc->device = device;
  sc->scoring = s;
  sc->mode = mode;
  sc->kernel = kernel;
  sc->cap = cap;
  sc->n_refs = n_refs;
  sc->max_ref_len = max_len;
  sc->panel_bases = bases;
  cudaDeviceProp prop{};
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) {
    delete sc;
    return cuda_fail(cudaGetLastError(), "cudaGetDeviceProperties");
  }
  sc->sm_count = prop.multiProcessorCount;
  if (prop.major < 10) {
    delete sc;
    return fail(ESG_ERR_UNAVAILABLE,
                "device %d (%s, sm_%d%d) is not a Blackwell sm_100 part this library is built for",
                device, prop.name, prop.major, prop.minor);
  }
  if (ext_stream) {
    sc->stream = (cudaStream_t)ext_stream;
  } else {
    if (cudaStreamCreateWithFlags(&sc->stream, cudaStreamNonBlocking) != cudaSuccess) {
      delete sc;
      return cuda_fail(cudaGetLastError(), "cudaStreamCreate");
    }
    sc->own_stream = true;
  }

  // Longest first, stable (cuda/mod.rs:379-380; simd/mod.rs:294-296).
  std::vector<uint32_t> order(n_refs);
  for (uint32_t r = 0; r < n_refs; ++r) order[r] = r;
  std::stable_sort(order.begin(), order.end(),
                   [&](uint32_t a, uint32_t b) { return ref_len[a] > ref_len[b]; });
  for (uint32_t r = 0; r < n_refs; ++r)
    for (uint32_t j = 0; j < ref_len[r]; ++j)
      if (code_of(ref_codes[ref_off[r] + j]) == kWild) sc->panel_w = true;

  // --- scoring tables of the batched kernel: s - o as int8 per byte
  const int ma = s.match_score, mi = s.mismatch, o = s.gap_open;
  auto fits8 = [](int v) { return v >= -128 && v <= 127; };
  sc->batched_ok = fits8(ma - o) && fits8(mi - o) && fits8(-o);
  if (sc->batched_ok) {
    for (int c = 0; c < 6; ++c) {
      uint32_t a = 0, b = 0;
      for (int x = 0; x < 4; ++x) {
        int v;
        if (c == kPad) v = -o;
        else if (c == kWild) v = ma - o;
        else v = (c == x ? ma : mi) - o;
        a |= (uint32_t)(uint8_t)(int8_t)v << (8 * x);
      }
      const int w = (c == kPad) ? -o : ma - o;  // against a wildcard reference base
      b = (uint32_t)(uint8_t)(int8_t)w | (0x80u << 8);  // byte 5: a padding column, -128
      sc->tab_a[c] = a;
      sc->tab_b[c] = b;
    }
    // local: a best H at or above this may have left the int16 lanes (the
    // diagonal term reaches H + ma + bias); such queries are re-scored in int32
    sc->sat = 32767 - ma - kBiasLocal;
  }

  // --- reference pairs and their selectors
  sc->n_pairs = (n_refs + 1) / 2;
  std::vector<uint4> pairs(sc->n_pairs);
  std::vector<uint16_t> sels;
  for (uint32_t p = 0; p < sc->n_pairs; ++p) {
    const uint32_t ra = order[2 * p];
    const bool hasb = 2 * p + 1 < n_refs;
    const uint32_t rb = hasb ? order[2 * p + 1] : kNoRef;
    const uint32_t ma_ = ref_len[ra], mb_ = hasb ? ref_len[rb] : 0;
    const uint32_t m = std::max(ma_, mb_);
    pairs[p] = make_uint4((uint32_t)sels.size(), (ma_ & 0xffffu) | (mb_ << 16), ra, rb);
    for (uint32_t j = 0; j < m; ++j) {
      const uint32_t x = j < ma_ ? code_of(ref_codes[ref_off[ra] + j]) : kPad;
      const uint32_t y = (hasb && j < mb_) ? code_of(ref_codes[ref_off[rb] + j]) : kPad;
      sels.push_back((uint16_t)(x | ((x | 8u) << 4) | (y << 8) | ((y | 8u) << 12)));
    }
  }
  // m is stored in 16 bits: lengths up to kMaxRefLen (32768) fit.
  sc->pair_cols.assign(sc->n_pairs + 1, 0);
  for (uint32_t p = 0; p < sc->n_pairs; ++p)
    sc->pair_cols[p + 1] = sc->pair_cols[p] + (pairs[p].y & 0xffffu);
  sc->sel_base = sc->n_pairs * 8;  // uint16 units after the pair table
  const size_t raw = (size_t)sc->n_pairs * 16 + sels.size() * 2;
  // one spare selector past the last pair: a lane may load column m
  sc->blob_bytes = (uint32_t)((raw + 2 + 15) / 16 * 16);
  std::vector<unsigned char> blob(sc->blob_bytes, 0);
  memcpy(blob.data(), pairs.data(), pairs.size() * 16);
  memcpy(blob.data() + (size_t)sc->n_pairs * 16, sels.data(), sels.size() * 2);

  auto cleanup = [&](esg_status st) {
    esg_scorer_free(sc);
    return st;
  };
  cudaError_t e = cudaMalloc(&sc->d_blob, sc->blob_bytes);
  if (e != cudaSuccess) return cleanup(cuda_fail(e, "cudaMalloc(panel)"));
  e = cudaMemcpy(sc->d_blob, blob.data(), sc->blob_bytes, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cleanup(cuda_fail(e, "cudaMemcpy(panel)"));

  // --- k3 panel (longest first)
  {
    std::vector<uint8_t> rc;
    std::vector<uint32_t> roff(n_refs), rlen(n_refs);
    rc.reserve(bases);
    for (uint32_t k = 0; k < n_refs; ++k) {
      const uint32_t r = order[k];
      roff[k] = (uint32_t)rc.size();
      rlen[k] = ref_len[r];
      for (uint32_t j = 0; j < ref_len[r]; ++j) rc.push_back((uint8_t)code_of(ref_codes[ref_off[r] + j]));
    }
    if ((e = cudaMalloc(&sc->d_rcodes, rc.size())) != cudaSuccess ||
        (e = cudaMalloc(&sc->d_roff, n_refs * 4)) != cudaSuccess ||
        (e = cudaMalloc(&sc->d_rlen, n_refs * 4)) != cudaSuccess ||
        (e = cudaMalloc(&sc->d_ridx, n_refs * 4)) != cudaSuccess)
      return cleanup(cuda_fail(e, "cudaMalloc(k3 panel)"));
    if ((e = cudaMemcpy(sc->d_rcodes, rc.data(), rc.size(), cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(sc->d_roff, roff.data(), n_refs * 4, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(sc->d_rlen, rlen.data(), n_refs * 4, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(sc->d_ridx, order.data(), n_refs * 4, cudaMemcpyHostToDevice)) != cudaSuccess)
      return cleanup(cuda_fail(e, "cudaMemcpy(k3 panel)"));
    sc->slot_of.assign(n_refs, 0);
    sc->len_of.assign(ref_len, ref_len + n_refs);
    sc->h_off.resize(n_refs);
    sc->h_codes.reserve(bases);
    for (uint32_t r = 0; r < n_refs; ++r) {
      sc->h_off[r] = sc->h_codes.size();
      for (uint32_t j = 0; j < ref_len[r]; ++j)
        sc->h_codes.push_back((uint8_t)code_of(ref_codes[ref_off[r] + j]));
    }
    for (uint32_t k = 0; k < n_refs; ++k) sc->slot_of[order[k]] = k;
  }

  // --- launch geometry
  const size_t slots = (size_t)kK2Threads * (4 + cap + kScrWords) * 4;
  sc->smem_panel = (size_t)sc->blob_bytes + slots <= 100 * 1024;
  set_k2_fn(sc);
  sc->k2_smem = (sc->smem_panel ? sc->blob_bytes : 0) + slots;
  for (const void* fn : {sc->k2_t16, sc->k2_t32, sc->k2_long, sc->k2c_t16, sc->k2c_t32,
                         sc->k2c_long})
    if ((e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)sc->k2_smem)) != cudaSuccess)
      return cleanup(cuda_fail(e, "cudaFuncSetAttribute(k2)"));
  if ((e = cudaStreamCreateWithFlags(&sc->aux, cudaStreamNonBlocking)) != cudaSuccess ||
      (e = cudaEventCreateWithFlags(&sc->fork, cudaEventDisableTiming)) != cudaSuccess ||
      (e = cudaEventCreateWithFlags(&sc->join, cudaEventDisableTiming)) != cudaSuccess)
    return cleanup(cuda_fail(e, "cudaStreamCreate(aux)"));
  {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    if ((e = cudaMemPoolCreate(&sc->pool, &props)) != cudaSuccess)
      return cleanup(cuda_fail(e, "cudaMemPoolCreate"));
    uint64_t keep = UINT64_MAX;
    if ((e = cudaMemPoolSetAttribute(sc->pool, cudaMemPoolAttrReleaseThreshold, &keep)) !=
        cudaSuccess)
      return cleanup(cuda_fail(e, "cudaMemPoolSetAttribute"));
  }
  int occ16 = 0, occ32 = 0, occl = 0, occ3 = 0;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ16, sc->k2_t16, kK2Threads,
                                                         sc->k2_smem)) != cudaSuccess ||
      (e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ32, sc->k2_t32, kK2Threads,
                                                         sc->k2_smem)) != cudaSuccess ||
      (e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occl, sc->k2_long, kK2Threads,
                                                         sc->k2_smem)) != cudaSuccess ||
      (e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ3, sc->k3_fn, kK3Threads, 0)) !=
          cudaSuccess)
    return cleanup(cuda_fail(e, "cudaOccupancy"));
  sc->blocks_t16 = std::max(1, occ16) * sc->sm_count;
  sc->blocks_t32 = std::max(1, occ32) * sc->sm_count;
  sc->blocks_long = std::max(1, occl) * sc->sm_count;
  {
    int c16 = 0, c32 = 0, cl = 0;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c16, sc->k2c_t16, kK2Threads,
                                                           sc->k2_smem)) != cudaSuccess ||
        (e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c32, sc->k2c_t32, kK2Threads,
                                                           sc->k2_smem)) != cudaSuccess ||
        (e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&cl, sc->k2c_long, kK2Threads,
                                                           sc->k2_smem)) != cudaSuccess)
      return cleanup(cuda_fail(e, "cudaOccupancy"));
    sc->blocksc_t16 = std::max(1, c16) * sc->sm_count;
    sc->blocksc_t32 = std::max(1, c32) * sc->sm_count;
    // the long-query column buffer below is sized for blocks_long CTAs
    sc->blocksc_long = std::min(std::max(1, cl) * sc->sm_count, sc->blocks_long);
  }
  if (sc->batched_ok && max_len <= 8192) {
    sc->lbuf_cols = max_len;
    const size_t lb = (size_t)sc->blocks_long * kK2Warps * max_len * sizeof(uint2);
    if ((e = cudaMalloc(&sc->d_lbuf, lb)) != cudaSuccess)
      return cleanup(cuda_fail(e, "cudaMalloc(long-query buffer)"));
  }
  sc->k3_blocks = std::max(1, occ3) * sc->sm_count;
  // k3's column buffers: one reference's bottom row (G, F per column) per
  // warp, at most kColbufBudget
  {
    const size_t per_block = (size_t)kK3Warps * max_len * sizeof(int2);
    sc->k3_blocks = (int)std::max<size_t>(
        1, std::min<size_t>((size_t)sc->k3_blocks, kColbufBudget / per_block));
    if ((e = cudaMalloc(&sc->d_colbuf, (size_t)sc->k3_blocks * per_block)) != cudaSuccess)
      return cleanup(cuda_fail(e, "cudaMalloc(k3 column buffers)"));
  }
  if (kernel == ESG_KERNEL_PLAIN32) {
    const esg_status pst = make_plain_buffers(sc);
    if (pst != ESG_OK) {
      esg_scorer_free(sc);
      return pst;
    }
  }

  // --- info
  esg_info& inf = sc->info;
  snprintf(inf.device_name, sizeof inf.device_name, "%s", prop.name);
  inf.device = device;
  inf.sm_count = sc->sm_count;
  inf.n_refs = n_refs;
  inf.max_ref_len = max_len;
  inf.n_ref_pairs = sc->n_pairs;
  inf.panel_bytes = sc->smem_panel ? sc->blob_bytes : 0;
  inf.batched_ok = sc->batched_ok;
  cudaFuncAttributes fa{};
  if (cudaFuncGetAttributes(&fa, sc->k2_t16) == cudaSuccess) {
    inf.regs_batched = fa.numRegs;
    inf.local_bytes_batched = (int)fa.localSizeBytes;
  }
  if (cudaFuncGetAttributes(&fa, sc->k3_fn) == cudaSuccess) {
    inf.regs_plain = fa.numRegs;
    inf.local_bytes_plain = (int)fa.localSizeBytes;
  }
  inf.batched_blocks = sc->blocks_t16;
  inf.batched_threads = kK2Threads;
  inf.plain_blocks = sc->k3_blocks;
  inf.plain_threads = kK3Threads;
  inf.split_len = sc->split_len;
  inf.tuned = 0;
  *out = sc;
  return ESG_OK;
}

void esg_scorer_free(esg_scorer* sc) {
  if (!sc) return;
  cudaSetDevice(sc->device);
  if (sc->stream) cudaStreamSynchronize(sc->stream);
  cudaFree(sc->d_blob);
  cudaFree(sc->d_rcodes);
  cudaFree(sc->d_roff);
  cudaFree(sc->d_rlen);
  cudaFree(sc->d_ridx);
  cudaFree(sc->d_colbuf);
  cudaFree(sc->d_colbuf1);
  cudaFree(sc->d_lbuf);
  if (sc->aux) {
    cudaStreamSynchronize(sc->aux);
    cudaStreamDestroy(sc->aux);
  }
  if (sc->fork) cudaEventDestroy(sc->fork);
  if (sc->join) cudaEventDestroy(sc->join);
  for (auto& ge : sc->graph_execs) cudaGraphExecDestroy(ge.second);
  if (sc->pool) cudaMemPoolDestroy(sc->pool);
  if (sc->own_stream && sc->stream) cudaStreamDestroy(sc->stream);
  delete sc;
}

esg_status esg_scorer_info(const esg_scorer* sc, esg_info* out) {
  if (!sc || !out) return fail(ESG_ERR_BAD_ARGUMENT, "NULL argument");
  *out = sc->info;
  return ESG_OK;
}

esg_status esg_scorer_set_kernel(esg_scorer* sc, int32_t kernel) {
  g_err.clear();
  if (!sc) return fail(ESG_ERR_BAD_ARGUMENT, "NULL scorer");
  if (kernel != ESG_KERNEL_AUTO && kernel != ESG_KERNEL_PLAIN32 && kernel != ESG_KERNEL_INT32)
    return fail(ESG_ERR_BAD_ARGUMENT, "unknown kernel %d", kernel);
  if (kernel == ESG_KERNEL_PLAIN32) {
    ESG_CUDA(cudaSetDevice(sc->device));
    const esg_status st = make_plain_buffers(sc);
    if (st != ESG_OK) return st;
  }
  sc->kernel = kernel;
  return ESG_OK;
}

int32_t esg_scores_len(const esg_scorer* sc, uint64_t len) { return sc && len > 0; }

int32_t esg_batched_takes(const esg_scorer* sc, uint64_t len) {
  return sc && sc->kernel == ESG_KERNEL_AUTO && !(sc->int32_from && len >= sc->int32_from) &&
         k2_takes(sc, len);
}

esg_status esg_scorer_set_chunking(esg_scorer* sc, uint32_t max_chunks) {
  g_err.clear();
  if (!sc) return fail(ESG_ERR_BAD_ARGUMENT, "NULL scorer");
  if (max_chunks < 1 || max_chunks > 64)
    return fail(ESG_ERR_BAD_ARGUMENT, "max_chunks %u outside 1..64", max_chunks);
  sc->max_chunks = max_chunks;
  return ESG_OK;
}

esg_status esg_scorer_set_split(esg_scorer* sc, uint32_t split_len) {
  if (!sc) return fail(ESG_ERR_BAD_ARGUMENT, "NULL scorer");
  sc->split_len = split_len;
  sc->info.split_len = split_len;
  return ESG_OK;
}

}  // extern "C"

namespace {

// Calibration batch of the autotuner: n reads of L +- 25 % bases, nine in
// ten cut from the panel's references with 8 % substitutions (shorter
// references padded with random bases) and one in ten random, so the batch
// packs, scores and flags as reads of this panel do.
struct Calib {
  std::vector<uint8_t> codes;
  std::vector<uint64_t> off;
  std::vector<uint32_t> len;
  uint32_t n = 0;
};

// Read lengths: L +- 25 %, or (hist non-empty) drawn from the sample `hist`.
void calib_reads(const esg_scorer* sc, uint32_t L, uint32_t n, uint64_t& x, Calib& c,
                 const std::vector<uint32_t>& hist = {}) {
  auto next = [&x]() {  // xorshift64*
    x ^= x >> 12;
    x ^= x << 25;
    x ^= x >> 27;
    return x * 0x2545F4914F6CDD1Dull;
  };
  c.n = n;
  c.off.assign(n, 0);
  c.len.assign(n, 0);
  c.codes.clear();
  for (uint32_t k = 0; k < n; ++k) {
    const uint32_t len = hist.empty() ? L - L / 4 + (uint32_t)(next() % (L / 2 + 1))
                                      : std::max<uint32_t>(1, hist[next() % hist.size()]);
    c.off[k] = c.codes.size();
    c.len[k] = len;
    const bool derived = next() % 10 != 0;
    const uint32_t r = (uint32_t)(next() % sc->n_refs);
    const uint32_t m = sc->len_of[r];
    const uint32_t start = m > len ? (uint32_t)(next() % (m - len + 1)) : 0u;
    for (uint32_t i = 0; i < len; ++i) {
      uint8_t b = (uint8_t)(next() >> 62);
      if (derived && start + i < m && next() % 100 >= 8) b = sc->h_codes[sc->h_off[r] + start + i];
      c.codes.push_back(b);
    }
  }
}

}  // namespace

// Device time (ms) of a calibration batch's work under the scorer's current
// settings: prepared and submitted once, then launched twice more, timed.
static esg_status time_calib(esg_scorer* sc, const Calib& c, cudaEvent_t e0, cudaEvent_t e1,
                             float* ms) {
  esg_batch* b = nullptr;
  esg_status st =
      esg_prepare(sc, c.codes.data(), c.off.data(), c.len.data(), c.n, ESG_BOTH_STRANDS, &b);
  if (st == ESG_OK) st = esg_submit(sc, b);
  if (st == ESG_OK) st = esg_finish(sc, b, nullptr, nullptr, nullptr);
  if (st == ESG_OK) {
    cudaEventRecord(e0, sc->stream);
    for (int i = 0; i < 2 && st == ESG_OK; ++i) st = launch_work(sc, b, sc->stream);
    cudaEventRecord(e1, sc->stream);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(ms, e0, e1);
    *ms /= 2;
  }
  esg_batch_free(b);
  return st;
}

static esg_status autotune_impl(esg_scorer* sc, const std::vector<uint32_t>& hist,
                                esg_tune_report* out) {
  g_err.clear();
  if (!sc) return fail(ESG_ERR_BAD_ARGUMENT, "NULL scorer");
  esg_tune_report rep{};
  rep.chunk_target = sc->chunk_target;
  rep.ctas16 = sc->blocks_t16 / std::max(1, sc->sm_count);
  rep.ctas32 = sc->blocks_t32 / std::max(1, sc->sm_count);
  if (!sc->batched_ok || sc->kernel != ESG_KERNEL_AUTO) {
    rep.split_len = sc->split_len;
    rep.int32_from = sc->int32_from;
    if (out) *out = rep;
    return ESG_OK;
  }
  ESG_CUDA(cudaSetDevice(sc->device));
  static const uint32_t kLens[] = {48, 80, 112, 160, 224, 320, 448};
  const uint32_t n_lens = sizeof(kLens) / sizeof(kLens[0]);
  const uint32_t keep_split = sc->split_len, keep_from = sc->int32_from;
  const int keep16 = sc->blocks_t16, keep32 = sc->blocks_t32;
  const uint32_t keep_target = sc->chunk_target;
  auto restore = [&]() {
    sc->split_len = keep_split;
    sc->int32_from = keep_from;
    sc->kernel = ESG_KERNEL_AUTO;
    sc->blocks_t16 = keep16;
    sc->blocks_t32 = keep32;
    sc->chunk_target = keep_target;
  };
  uint64_t x = 0x9e3779b97f4a7c15ull;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  ESG_CUDA(cudaEventCreate(&e0));
  ESG_CUDA(cudaEventCreate(&e1));
  esg_status st = ESG_OK;
  Calib c;
  // about 2e11 cells per batch (~40 ms of device time), both strands: on a
  // small panel enough tiles to keep every resident warp busy without panel
  // chunks, the regime of a real batch (smaller batches measured the chunked
  // regime, where 16- and 32-row stripes time alike, and chose badly)
  auto reads_for = [&](uint32_t L) {
    const uint64_t want = (uint64_t)(2.0e11 / (2.0 * L * (double)sc->panel_bases));
    return (uint32_t)std::min<uint64_t>(std::max<uint64_t>(want, 64), 200000);
  };
  sc->int32_from = 0;
  // 1. per read length: 16-row stripes, 32-row stripes, the int32 lanes
  for (uint32_t li = 0; li < n_lens && st == ESG_OK; ++li) {
    const uint32_t L = kLens[li];
    calib_reads(sc, L, reads_for(L), x, c);
    float ms[3] = {0, 0, 0};
    for (int cfg = 0; cfg < 3 && st == ESG_OK; ++cfg) {
      sc->split_len = cfg == 0 ? 512u : 0u;
      sc->kernel = cfg == 2 ? ESG_KERNEL_INT32 : ESG_KERNEL_AUTO;
      st = time_calib(sc, c, e0, e1, &ms[cfg]);
    }
    sc->kernel = ESG_KERNEL_AUTO;
    rep.lengths[li] = L;
    rep.ms_rows16[li] = ms[0];
    rep.ms_rows32[li] = ms[1];
    rep.ms_int32[li] = ms[2];
    rep.n_lengths = li + 1;
  }
  if (st != ESG_OK) {
    restore();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return st;
  }
  // 16-row stripes up to the last length where they are as fast within 2 %
  // (timing noise), counting from the shortest; 32-row stripes from the
  // first length they win by more.  The int32 lanes from the length where
  // they win at it and every longer length (a scheme whose long queries
  // mostly flag, to be scored twice by the batched kernel), else never.
  uint32_t split = 0;
  for (uint32_t li = 0; li < rep.n_lengths; ++li) {
    if (rep.ms_rows16[li] <= 1.02f * rep.ms_rows32[li])
      split = rep.lengths[li];
    else
      break;
  }
  if (split == kLens[n_lens - 1]) split = 512;
  uint32_t from = 0;
  for (int li = (int)rep.n_lengths - 1; li >= 0; --li) {
    if (rep.ms_int32[li] < std::min(rep.ms_rows16[li], rep.ms_rows32[li]))
      from = rep.lengths[li];
    else
      break;
  }
  // 1b. with a sample of the workload's read lengths: every candidate split
  //     timed on one batch drawn from that histogram, the fastest kept (of
  //     equal times, within 1 %, the larger split: 16-row tiles carry less
  //     skew per pair)
  if (!hist.empty()) {
    uint64_t bases = 0;
    for (uint32_t v : hist) bases += v;
    const double mean = std::max(1.0, (double)bases / (double)hist.size());
    // about 1e12 cells (~0.2 s a launch): the splits differ by a percent or
    // two on a whole batch, less than the noise of a 40-ms one
    const uint64_t want = (uint64_t)(1.0e12 / (2.0 * mean * (double)sc->panel_bases));
    calib_reads(sc, 0, (uint32_t)std::min<uint64_t>(std::max<uint64_t>(want, 64), 500000), x, c,
                hist);
    static const uint32_t kSplits[] = {0, 48, 80, 112, 160, 224, 320, 512};
    float best = 0;
    for (uint32_t cand : kSplits) {
      if (st != ESG_OK) break;
      sc->split_len = cand;
      float ms = 0;
      st = time_calib(sc, c, e0, e1, &ms);
      rep.splits[rep.n_splits] = cand;
      rep.ms_splits[rep.n_splits] = ms;
      ++rep.n_splits;
      if (rep.n_splits == 1 || ms <= 1.01f * best) {
        if (rep.n_splits == 1 || ms < best) best = ms;
        split = cand;
      }
    }
  }
  // 2. resident CTAs per SM of the 16-row tiles (112-nt reads) and the
  //    32-row tiles (448-nt reads): the occupancy limit and one or two fewer
  for (int which = 0; which < 2 && st == ESG_OK; ++which) {
    const uint32_t L = which == 0 ? 112u : 448u;
    calib_reads(sc, L, reads_for(L), x, c);
    sc->split_len = which == 0 ? 512u : 0u;
    int& blocks = which == 0 ? sc->blocks_t16 : sc->blocks_t32;
    const int occ = (which == 0 ? keep16 : keep32) / std::max(1, sc->sm_count);
    uint32_t* cand = which == 0 ? rep.cand_ctas16 : rep.cand_ctas32;
    float* tms = which == 0 ? rep.ms_ctas16 : rep.ms_ctas32;
    uint32_t& n_c = which == 0 ? rep.n_ctas16 : rep.n_ctas32;
    float best = 0;
    int pick = occ;
    for (int k = occ; k >= std::max(1, occ - 2) && st == ESG_OK; --k) {
      blocks = k * sc->sm_count;
      float ms = 0;
      st = time_calib(sc, c, e0, e1, &ms);
      cand[n_c] = (uint32_t)k;
      tms[n_c] = ms;
      ++n_c;
      if (k == occ || ms < best) {
        best = ms;
        pick = k;
      }
    }
    blocks = pick * sc->sm_count;
    (which == 0 ? rep.ctas16 : rep.ctas32) = (uint32_t)pick;
  }
  sc->split_len = split;
  // 3. panel chunking: a batch of about one read per resident warp (too few
  //    tiles to fill the GPU), chunked to aim for 1-16 tasks per resident warp
  if (st == ESG_OK) {
    calib_reads(sc, 112, (uint32_t)std::max(64, sc->blocks_t16 * kK2Warps), x, c);
    static const uint32_t kTargets[] = {1, 2, 4, 8, 16};
    float best = 0;
    uint32_t pick = keep_target;
    for (uint32_t t : kTargets) {
      if (st != ESG_OK) break;
      sc->chunk_target = t;
      float ms = 0;
      st = time_calib(sc, c, e0, e1, &ms);
      rep.chunk_targets[rep.n_chunk_targets] = t;
      rep.ms_chunks[rep.n_chunk_targets] = ms;
      ++rep.n_chunk_targets;
      if (rep.n_chunk_targets == 1 || ms < best) {
        best = ms;
        pick = t;
      }
    }
    sc->chunk_target = pick;
    rep.chunk_target = pick;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st != ESG_OK) {
    restore();
    return st;
  }
  sc->split_len = split;
  sc->int32_from = from;
  sc->tuned = true;
  sc->info.split_len = split;
  sc->info.tuned = 1;
  sc->info.batched_blocks = sc->blocks_t16;
  rep.split_len = split;
  rep.int32_from = from;
  if (out) *out = rep;
  return ESG_OK;
}

extern "C" {

esg_status esg_scorer_autotune(esg_scorer* sc, esg_tune_report* out) {
  return autotune_impl(sc, {}, out);
}

esg_status esg_scorer_autotune_lengths(esg_scorer* sc, const uint32_t* lens, uint32_t n,
                                       esg_tune_report* out) {
  g_err.clear();
  if (!sc || (n && !lens)) return fail(ESG_ERR_BAD_ARGUMENT, "NULL argument");
  std::vector<uint32_t> hist;
  hist.reserve(n);
  for (uint32_t k = 0; k < n; ++k)
    if (lens[k]) hist.push_back(lens[k]);
  return autotune_impl(sc, hist, out);
}

// ---------------------------------------------------------------- prepare
}  // extern "C"

// Read codes packed at 2 bits a base into `out` (base i of a byte in bits
// 2i..2i+1); a code above 3 (the wildcard, or any other byte) packs as 0 and
// its stream position base + i goes to `exc`.  Eight bases at a time: the
// shifts gather the low two bits of eight bytes into 16 bits.
static void pack_read(const uint8_t* src, uint32_t n, uint8_t* out, uint64_t base,
                      std::vector<uint64_t>& exc) {
  uint32_t i = 0;
  for (; i + 8 <= n; i += 8) {
    uint64_t v;
    memcpy(&v, src + i, 8);
    if (v & 0xFCFCFCFCFCFCFCFCull) {
      for (uint32_t j = 0; j < 8; ++j)
        if (src[i + j] > 3) exc.push_back(base + i + j);
      v &= 0x0303030303030303ull;
      for (uint32_t j = 0; j < 8; ++j)
        if (src[i + j] > 3) v &= ~(0xffull << (8 * j));
    }
    uint64_t x = (v | (v >> 6)) & 0x000F000F000F000Full;
    x = (x | (x >> 12)) & 0x000000FF000000FFull;
    x = x | (x >> 24);
    out[i / 4] = (uint8_t)x;
    out[i / 4 + 1] = (uint8_t)(x >> 8);
  }
  for (; i < n; i += 4) {
    uint8_t byte = 0;
    for (uint32_t j = 0; j < 4 && i + j < n; ++j) {
      uint8_t c = src[i + j];
      if (c > 3) {
        exc.push_back(base + i + j);
        c = 0;
      }
      byte |= (uint8_t)(c << (2 * j));
    }
    out[i / 4] = byte;
  }
}

// The packing esg_prepare does, for the host-side tests: reads k at
// out + pos_k / 4 with pos_k the sum of the earlier lengths rounded up to 4;
// returns the packed bytes, exceptions to `exc` (up to exc_cap), their count
// to *n_exc.
extern "C" uint64_t esg_internal_pack_reads(const uint8_t* codes, const uint64_t* off,
                                            const uint32_t* len, uint32_t n, uint8_t* out,
                                            uint64_t* exc, uint64_t exc_cap, uint64_t* n_exc) {
  std::vector<uint64_t> e;
  uint64_t pos = 0;
  for (uint32_t k = 0; k < n; ++k) {
    if (len[k]) pack_read(codes + off[k], len[k], out + pos / 4, pos, e);
    pos += ((uint64_t)len[k] + 3) & ~(uint64_t)3;
  }
  for (uint64_t i = 0; i < e.size() && i < exc_cap; ++i) exc[i] = e[i];
  *n_exc = e.size();
  return pos / 4;
}

// The planning half of esg_prepare.  Read k is `ptrs[k]` when `ptrs` is
// given (reads gathered from several requests), else codes + off[k].
static esg_status prepare_impl(esg_scorer* sc, const uint8_t* const* ptrs, const uint8_t* codes,
                               const uint64_t* off, const uint32_t* len, uint32_t n_reads,
                               uint32_t flags, esg_batch** out) {
  g_err.clear();
  if (!sc || !out) return fail(ESG_ERR_BAD_ARGUMENT, "NULL scorer or out");
  *out = nullptr;
  if (flags & ~(ESG_BOTH_STRANDS | ESG_FULL_ROWS))
    return fail(ESG_ERR_BAD_ARGUMENT, "unknown flags 0x%x", flags);
  if (n_reads && (!(off || ptrs) || !len))
    return fail(ESG_ERR_BAD_ARGUMENT, "off/len must not be NULL");
  if (n_reads >= (1u << 30)) return fail(ESG_ERR_BAD_ARGUMENT, "too many reads (%u)", n_reads);
  uint64_t total = 0;
  for (uint32_t k = 0; k < n_reads; ++k) total += len[k];
  if (total && !codes && !ptrs) return fail(ESG_ERR_BAD_ARGUMENT, "codes must not be NULL");

  auto* b = new esg_batch();
  b->owner = sc;
  b->n_reads = n_reads;
  b->flags = flags;
  b->kernel = sc->kernel;
  const bool both = flags & ESG_BOTH_STRANDS;
  b->n_q = n_reads * (both ? 2u : 1u);
  b->total_bases = total;

  // --- plan: which queries go where.  Short queries take 16-row stripes,
  // longer ones 32-row stripes (from sc->split_len, set by the autotuner),
  // queries over 32 stripes of 32 rows run alone in passes; what the
  // batched kernel cannot take goes to the int32 kernel.
  std::vector<std::pair<uint32_t, uint32_t>> q16, q32, qlong;  // (stripes, query)
  std::vector<uint8_t> route(b->n_q, 0);  // 0 empty or k2, 2 k3
  uint32_t n_k3 = 0, n_empty = 0, redo_cap = 0;
  uint64_t cells = 0;
  const uint32_t split = std::min<uint32_t>(sc->split_len, 16 * kMaxStripes);
  for (uint32_t q = 0; q < b->n_q; ++q) {
    const uint32_t n = len[q < n_reads ? q : q - n_reads];
    if (n == 0) {
      ++n_empty;
      continue;
    }
    cells += (uint64_t)n * sc->panel_bases;
    const bool lanes32 = sc->int32_from && n >= sc->int32_from;
    if (b->kernel == ESG_KERNEL_AUTO && !lanes32 && k2_takes(sc, n)) {
      if (n <= split)
        q16.push_back({(n + 15) / 16, q});
      else if (n <= 32 * kMaxStripes)
        q32.push_back({(n + 31) / 32, q});
      else
        qlong.push_back({(n + 31) / 32, q});
      if (k2_may_flag(sc, n)) ++redo_cap;
      if (k2_checks(sc, n)) b->sg_check = true;
    } else {
      route[q] = 2;
      ++n_k3;
    }
  }
  b->host_list = n_k3;
  b->redo_cap = redo_cap;
  std::stable_sort(qlong.begin(), qlong.end(),
                   [](const std::pair<uint32_t, uint32_t>& a,
                      const std::pair<uint32_t, uint32_t>& c) { return a.first > c.first; });
  TilePlan p32, p16;
  pack_tiles(q32, p32);
  pack_tiles(q16, p16);
  const uint32_t n_long = (uint32_t)qlong.size();
  b->n_long = n_long;
  b->n_t32 = (uint32_t)p32.tasks.size();
  b->n_t16 = (uint32_t)p16.tasks.size();
  b->n_tasks = b->n_long + b->n_t32 + b->n_t16;
  b->n_order = n_long + (uint32_t)(q32.size() + q16.size());
  // --- panel chunks: when the tiles are too few to keep every resident warp
  // busy to the end (few reads, or a large panel), each tile's reference
  // pairs are cut into chunks of about equal columns, one task each, and
  // the per-chunk query states are merged afterwards
  {
    const uint64_t tiles = b->n_tasks;
    const uint64_t target =
        (uint64_t)sc->chunk_target * (uint64_t)std::max(sc->blocks_t16, 1) * kK2Warps;
    uint32_t nc = 1;
    if (tiles && tiles < target) nc = (uint32_t)((target + tiles - 1) / tiles);
    nc = std::min<uint32_t>(nc, std::max<uint32_t>(1, sc->n_pairs / 4));
    nc = std::min<uint32_t>(nc, sc->max_chunks);
    b->n_chunks = std::max<uint32_t>(nc, 1);
  }

  // --- pinned staging for the inputs (reads packed at 2 bits a base)
  uint64_t padded = 0;
  for (uint32_t k = 0; k < n_reads; ++k) padded += ((uint64_t)len[k] + 3) & ~(uint64_t)3;
  b->padded_bases = padded;
  b->code_words = (padded + 15) / 16;
  const size_t sz_codes = carve_size(b->code_words ? b->code_words * 4 : 1, 1);
  const size_t sz_off = carve_size(n_reads ? n_reads : 1, 8);
  const size_t sz_len = carve_size(n_reads ? n_reads : 1, 4);
  const size_t sz_order = carve_size(b->n_order ? b->n_order : 1, 4);
  const size_t sz_tasks = carve_size(b->n_tasks ? b->n_tasks : 1, 8);
  const size_t sz_list = carve_size(n_k3 + redo_cap ? n_k3 + redo_cap : 1, 4);
  const size_t sz_chunks = carve_size(b->n_chunks + 1, 4);
  b->in_bytes = sz_codes + sz_off + sz_len + sz_order + sz_tasks + sz_list + sz_chunks;
  b->in_buf.p = sc->pinned.get(b->in_bytes, &b->in_buf.cap);
  if (!b->in_buf.p) {
    const size_t want = b->in_bytes;
    delete b;
    return fail(ESG_ERR_OUT_OF_MEMORY, "pinned host memory (%zu bytes)", want);
  }
  char* at = (char*)b->in_buf.p;
  b->h_packed = carve<uint8_t>(at, b->code_words ? b->code_words * 4 : 1);
  b->h_off = carve<uint64_t>(at, n_reads ? n_reads : 1);
  b->h_len = carve<uint32_t>(at, n_reads ? n_reads : 1);
  b->h_order = carve<uint32_t>(at, b->n_order ? b->n_order : 1);
  b->h_tasks = carve<uint2>(at, b->n_tasks ? b->n_tasks : 1);
  b->h_list = carve<uint32_t>(at, n_k3 + redo_cap ? n_k3 + redo_cap : 1);
  b->h_chunks = carve<uint32_t>(at, b->n_chunks + 1);
  {
    // chunk c covers pairs [h_chunks[c], h_chunks[c + 1]) of about equal columns
    const uint32_t nc = b->n_chunks, np = sc->n_pairs;
    const uint64_t total_cols = sc->pair_cols.empty() ? 0 : sc->pair_cols[np];
    b->h_chunks[0] = 0;
    uint32_t p = 0;
    for (uint32_t c = 1; c < nc; ++c) {
      const uint64_t want = total_cols * c / nc;
      while (p < np && sc->pair_cols[p] < want) ++p;
      // every chunk keeps at least one pair
      p = std::max(p, b->h_chunks[c - 1] + 1);
      p = std::min(p, np - (nc - c));
      b->h_chunks[c] = p;
    }
    b->h_chunks[nc] = np;
  }
  uint64_t pos = 0;
  for (uint32_t k = 0; k < n_reads; ++k) {
    b->h_off[k] = pos;
    b->h_len[k] = len[k];
    if (len[k]) pack_read(ptrs ? ptrs[k] : codes + off[k], len[k], b->h_packed + pos / 4, pos,
                          b->exceptions);
    pos += ((uint64_t)len[k] + 3) & ~(uint64_t)3;
  }
  // the packed tail up to the last whole word unpacks to padding
  memset(b->h_packed + pos / 4, 0, b->code_words * 4 - pos / 4);
  // order[] and tasks[] laid out [long | 32-row tiles | 16-row tiles];
  // tasks[t] = {start in order[], count | stripes << 16}
  {
    uint32_t lanes = 0, o = 0, t = 0;
    for (const auto& lq : qlong) {
      b->h_order[o] = lq.second;
      b->h_tasks[t++] = make_uint2(o++, 1u | (lq.first << 16));
      lanes += lq.first;
    }
    for (const TilePlan* tp : {&p32, &p16}) {
      const uint32_t base = o;
      for (uint32_t q : tp->order) b->h_order[o++] = q;
      for (const uint2& tk : tp->tasks) b->h_tasks[t++] = make_uint2(base + tk.x, tk.y);
      lanes += tp->lanes;
    }
    b->stats.lanes_used = lanes;
  }
  {
    uint32_t w = 0;
    for (uint32_t q = 0; q < b->n_q; ++q)
      if (route[q] == 2) b->h_list[w++] = q;
  }
  b->stats.n_reads = n_reads;
  b->stats.n_queries = b->n_q;
  b->stats.n_empty = n_empty;
  b->stats.queries_batched = n_long + (uint32_t)(q32.size() + q16.size());
  b->stats.queries_plain = n_k3;
  b->stats.tasks = b->n_tasks;
  b->stats.panel_chunks = b->n_chunks;
  b->stats.cells = cells;
  *out = b;
  return ESG_OK;
}

esg_status esg_internal_prepare_ptrs(esg_scorer* sc, const uint8_t* const* reads,
                                     const uint32_t* len, uint32_t n_reads, uint32_t flags,
                                     esg_batch** out) {
  return prepare_impl(sc, reads, nullptr, nullptr, len, n_reads, flags, out);
}

size_t esg_internal_pool_spare(esg_scorer* sc) {
  if (!sc || !sc->pool) return 0;
  cudaSetDevice(sc->device);
  uint64_t reserved = 0, used = 0;
  if (cudaMemPoolGetAttribute(sc->pool, cudaMemPoolAttrReservedMemCurrent, &reserved) !=
          cudaSuccess ||
      cudaMemPoolGetAttribute(sc->pool, cudaMemPoolAttrUsedMemCurrent, &used) != cudaSuccess)
    return 0;
  return reserved > used ? (size_t)(reserved - used) : 0;
}

int esg_internal_device(const esg_scorer* sc) { return sc ? sc->device : 0; }

uint32_t esg_internal_tie_capacity(const esg_scorer* sc) { return sc ? sc->cap : 0; }

uint64_t esg_internal_panel_bases(const esg_scorer* sc) { return sc ? sc->panel_bases : 0; }

void esg_internal_panel_of(esg_scorer* sc, esg_internal_panel* p) {
  p->rcodes = sc->d_rcodes;
  p->roff = sc->d_roff;
  p->rlen = sc->d_rlen;
  p->slot_of = sc->slot_of.data();
  p->len_of = sc->len_of.data();
  p->h_codes = sc->h_codes.data();
  p->h_off = sc->h_off.data();
  p->n_refs = sc->n_refs;
  p->max_ref_len = sc->max_ref_len;
  p->device = sc->device;
  p->sm_count = sc->sm_count;
  p->mode = sc->mode;
  p->scoring = sc->scoring;
  p->stream = sc->stream;
  p->pool = sc->pool;
}

void esg_internal_batch_reads(const esg_batch* b, const uint8_t** codes, const uint64_t** off,
                              const uint32_t** len, uint32_t* n_reads, const uint32_t** host_len) {
  *codes = b->submitted ? b->d_codes : nullptr;
  *off = b->d_off;
  *len = b->d_len;
  *n_reads = b->n_reads;
  *host_len = b->h_len;
}

extern "C" {

esg_status esg_prepare(esg_scorer* sc, const uint8_t* codes, const uint64_t* off,
                       const uint32_t* len, uint32_t n_reads, uint32_t flags, esg_batch** out) {
  return prepare_impl(sc, nullptr, codes, off, len, n_reads, flags, out);
}

// Device bytes of a batch: the one allocation esg_submit carves (and the
// figure admission control weighs).
static size_t batch_device_bytes(const esg_scorer* sc, const esg_batch* b) {
  const bool dev_rows = (b->flags & ESG_FULL_ROWS) || b->paired;
  const size_t np = b->paired ? std::max<uint32_t>(b->n_pairs, 1) : 0;
  const uint32_t nlist = b->host_list + b->redo_cap;
  const size_t nr = b->n_reads ? b->n_reads : 1, nq = b->n_q ? b->n_q : 1;
  const size_t sizes[] = {
      carve_size(b->code_words ? b->code_words * 16 : 1, 1),
      carve_size(b->code_words ? b->code_words * 4 : 1, 1),
      carve_size(b->exceptions.empty() ? 1 : b->exceptions.size(), 8),
      carve_size(nr, 8),
      carve_size(nr, 4),
      carve_size(b->n_order ? b->n_order : 1, 4),
      carve_size(b->n_tasks ? b->n_tasks : 1, 8),
      carve_size(nlist ? nlist : 1, 4),
      carve_size(b->n_chunks + 1, 4),
      carve_size(8, 4),
      carve_size(nq, 16),
      carve_size(nq * sc->cap, 4),
      carve_size(nlist ? (size_t)nlist * sc->n_refs : 1, 4),
      carve_size(nr, 16),
      carve_size(nr * sc->cap, 4),
      dev_rows ? carve_size(nq * sc->n_refs, 4) : 0,
      carve_size(2 * np, 16),
      carve_size(np * sc->cap, 4),
      b->n_chunks > 1 ? carve_size(nq * b->n_chunks, 16) : 0,
      b->n_chunks > 1 ? carve_size(nq * b->n_chunks * sc->cap, 4) : 0,
  };
  size_t total = 0;
  for (size_t v : sizes) total += v;
  return total;
}

// ---------------------------------------------------------------- device work
static esg_status launch_device_work(esg_scorer* sc, esg_batch* b, cudaStream_t st) {
  const bool both = b->flags & ESG_BOTH_STRANDS;
  uint32_t kernels = 0;
  const bool rows = b->d_rows != nullptr;
  ESG_CUDA(cudaMemsetAsync(b->d_counters, 0, 8 * sizeof(uint32_t), st));
  if (b->n_tasks) {
    K2Params P{};
    P.blob = (const uint4*)sc->d_blob;
    P.blob_bytes = sc->blob_bytes;
    P.n_pairs = sc->n_pairs;
    P.sel_base = sc->sel_base;
    P.codes = b->d_codes;
    P.off = b->d_off;
    P.len = b->d_len;
    P.n_reads = b->n_reads;
    P.order = b->d_order;
    P.tasks = b->d_tasks;
    P.n_tasks = b->n_tasks;
    P.counters = b->d_counters;
    P.qhead = b->d_qhead;
    P.qties = b->d_qties;
    P.rows = rows ? b->d_rows : nullptr;
    P.n_refs = sc->n_refs;
    P.redo_list = b->d_list;
    P.redo_base = b->host_list;
    P.redo_cap = b->redo_cap;
    P.n_chunks = b->n_chunks;
    P.chunk_lo = b->d_chunks;
    P.part_head = b->d_part_head;
    P.part_ties = b->d_part_ties;
    memcpy(P.tab_a, sc->tab_a, sizeof P.tab_a);
    memcpy(P.tab_b, sc->tab_b, sizeof P.tab_b);
    P.e2 = pack16x2(sc->scoring.gap_extend, sc->scoring.gap_extend);
    P.o = sc->scoring.gap_open;
    P.e = sc->scoring.gap_extend;
    P.bias = sc->mode == ESG_MODE_LOCAL ? kBiasLocal : kBiasSemiGlobal;
    P.one = 1;
    P.lbuf = sc->d_lbuf;
    P.lbuf_cols = sc->lbuf_cols;
    P.sat = sc->sat;
    P.cap = sc->cap;
    // The three task groups: long queries, then 32-row tiles, on the aux
    // stream; 16-row tiles on the batch's stream.  Launched first, the aux
    // kernels' CTAs share the SMs with the persistent 16-row kernel and
    // fill its tail, instead of queueing behind it.
    // tasks of a group: its tiles x the panel chunks
    const uint32_t nc = b->n_chunks;
    const uint32_t n_long = b->n_long * nc, n_t32 = b->n_t32 * nc, n_t16 = b->n_t16 * nc;
    auto grid = [](int cap, uint32_t tasks) {
      return (int)std::max<uint64_t>(
          1, std::min<uint64_t>((uint64_t)cap, (tasks + kK2Warps - 1) / kK2Warps));
    };
    const bool aux = n_long || n_t32;
    const bool chk = b->sg_check;
    if (aux) {
      ESG_CUDA(cudaEventRecord(sc->fork, st));
      ESG_CUDA(cudaStreamWaitEvent(sc->aux, sc->fork, 0));
    }
    if (n_long) {
      K2Params L = P;
      L.n_tasks = n_long;
      L.task_counter = b->d_counters + 3;
      void* largs[] = {&L};
      ESG_CUDA(cudaLaunchKernel(chk ? sc->k2c_long : sc->k2_long,
                                dim3(grid(chk ? sc->blocksc_long : sc->blocks_long, n_long)),
                                dim3(kK2Threads), largs, sc->k2_smem, sc->aux));
      ++kernels;
    }
    if (n_t32) {
      K2Params T = P;
      T.tasks = P.tasks + b->n_long;
      T.n_tasks = n_t32;
      T.task_counter = b->d_counters + 4;
      void* targs[] = {&T};
      ESG_CUDA(cudaLaunchKernel(chk ? sc->k2c_t32 : sc->k2_t32,
                                dim3(grid(chk ? sc->blocksc_t32 : sc->blocks_t32, n_t32)),
                                dim3(kK2Threads),
                                targs, sc->k2_smem, sc->aux));
      ++kernels;
    }
    if (n_t16) {
      K2Params T = P;
      T.tasks = P.tasks + b->n_long + b->n_t32;
      T.n_tasks = n_t16;
      T.task_counter = b->d_counters + 0;
      void* targs[] = {&T};
      ESG_CUDA(cudaLaunchKernel(chk ? sc->k2c_t16 : sc->k2_t16,
                                dim3(grid(chk ? sc->blocksc_t16 : sc->blocks_t16, n_t16)),
                                dim3(kK2Threads),
                                targs, sc->k2_smem, st));
      ++kernels;
    }
    if (aux) {
      ESG_CUDA(cudaEventRecord(sc->join, sc->aux));
      ESG_CUDA(cudaStreamWaitEvent(st, sc->join, 0));
    }
    if (nc > 1) {
      KMParams M{};
      M.order = b->d_order;
      M.n_order = b->n_order;
      M.n_chunks = nc;
      M.part_head = b->d_part_head;
      M.part_ties = b->d_part_ties;
      M.qhead = b->d_qhead;
      M.qties = b->d_qties;
      M.cap = sc->cap;
      M.counters = b->d_counters;
      M.redo_list = b->d_list;
      M.redo_base = b->host_list;
      M.redo_cap = b->redo_cap;
      const int blocks =
          (int)std::max<uint64_t>(1, std::min<uint64_t>(4096, (b->n_order + 127) / 128));
      void* margs[] = {&M};
      ESG_CUDA(cudaLaunchKernel((const void*)k2_merge_chunks, dim3(blocks), dim3(128), margs, 0,
                                st));
      ++kernels;
    }
  }
  const bool k3 = b->host_list + b->redo_cap > 0;
  if (k3) {
    const bool plain = b->kernel == ESG_KERNEL_PLAIN32;
    K3Params P{};
    P.codes = b->d_codes;
    P.off = b->d_off;
    P.len = b->d_len;
    P.n_reads = b->n_reads;
    P.list = b->d_list;
    P.host_count = b->host_list;
    P.redo_count = b->redo_cap ? b->d_counters + 1 : nullptr;
    P.redo_cap = b->redo_cap;
    P.rcodes = sc->d_rcodes;
    P.roff = sc->d_roff;
    P.rlen = sc->d_rlen;
    P.ridx = sc->d_ridx;
    P.n_refs = sc->n_refs;
    P.max_cols = sc->max_ref_len;
    P.out = b->d_k3out;
    P.rows = rows ? b->d_rows : nullptr;
    P.wmax = plain ? 1u : 32u;
    P.refs_per_task = 32;
    // counters[6..7]: the units' 64-bit counter (8-byte aligned, reset with
    // the rest each launch)
    P.task_counter = reinterpret_cast<unsigned long long*>(b->d_counters + 6);
    P.colbuf = plain ? sc->d_colbuf1 : sc->d_colbuf;
    P.ma = sc->scoring.match_score;
    P.mi = sc->scoring.mismatch;
    P.o = sc->scoring.gap_open;
    P.e = sc->scoring.gap_extend;
    P.one = 1;
    void* args[] = {&P};
    ESG_CUDA(cudaLaunchKernel(sc->k3_fn, dim3(plain ? sc->k3_blocks1 : sc->k3_blocks),
                              dim3(kK3Threads), args, 0, st));
    ++kernels;
    K4Params Q{};
    Q.list = b->d_list;
    Q.host_count = b->host_list;
    Q.redo_count = P.redo_count;
    Q.redo_cap = b->redo_cap;
    Q.rows = b->d_k3out;
    Q.n_refs = sc->n_refs;
    Q.n_reads = b->n_reads;
    Q.qhead = b->d_qhead;
    Q.qties = b->d_qties;
    Q.cap = sc->cap;
    const uint32_t need = b->host_list + b->redo_cap;
    const int blocks = (int)std::max<uint64_t>(
        1, std::min<uint64_t>((uint64_t)sc->sm_count * 8, (need + 7) / 8));
    void* qargs[] = {&Q};
    ESG_CUDA(cudaLaunchKernel((const void*)k4_rows, dim3(blocks), dim3(256), qargs, 0, st));
    ++kernels;
  }
  if (b->n_reads) {
    K5Params M{};
    M.len = b->d_len;
    M.n_reads = b->n_reads;
    M.both = both;
    M.qhead = b->d_qhead;
    M.qties = b->d_qties;
    M.cap = sc->cap;
    M.results = b->d_results;
    M.ties = b->d_ties;
    M.rows = b->d_rows;
    M.n_refs = sc->n_refs;
    const int blocks = (int)std::min<uint64_t>(4096, (b->n_reads + 255) / 256);
    void* margs[] = {&M};
    ESG_CUDA(cudaLaunchKernel((const void*)k5_merge, dim3(blocks), dim3(256), margs, 0, st));
    ++kernels;
  }
  if (b->paired && b->n_pairs) {
    K6Params X{};
    X.rows = b->d_rows;
    X.len = b->d_len;
    X.mates = b->d_results;
    X.n_pairs = b->n_pairs;
    X.n_reads = b->n_reads;
    X.n_refs = sc->n_refs;
    X.cap = sc->cap;
    X.min_score = b->min_score;
    X.both = b->pair_both;
    X.out = b->d_pairs;
    X.ties = b->d_pties;
    const int blocks = (int)std::min<uint64_t>((uint64_t)sc->sm_count * 16, (b->n_pairs + 7) / 8);
    void* xargs[] = {&X};
    ESG_CUDA(cudaLaunchKernel((const void*)k6_pairs, dim3(blocks), dim3(256), xargs, 0, st));
    ++kernels;
  }
  b->stats.kernels = kernels;
  return ESG_OK;
}

// The shape of a batch's launch sequence: which of its kernels run.  Batches
// of one shape differ only in kernel parameters and sizes, which an
// instantiated graph takes by update.
static uint32_t work_key(const esg_scorer* sc, const esg_batch* b) {
  const uint32_t nc = b->n_chunks;
  const bool k3 = b->host_list + b->redo_cap > 0;
  return (b->n_long ? 1u : 0u) | (b->n_t32 ? 2u : 0u) | (b->n_t16 ? 4u : 0u) |
         ((b->n_tasks && nc > 1) ? 8u : 0u) | (k3 ? 16u : 0u) | (b->n_reads ? 32u : 0u) |
         ((b->paired && b->n_pairs) ? 64u : 0u) | (b->sg_check ? 128u : 0u) |
         (b->kernel == ESG_KERNEL_PLAIN32 ? 256u : 0u) | (sc->mode == ESG_MODE_LOCAL ? 512u : 0u);
}

// The batch's device work as one CUDA graph launch on `st`: the launch
// sequence (counter reset, the three k2 groups on two streams joined by
// events, chunk merge, k3 / k4, k5, k6) is captured from the scorer's
// stream once per batch, and the scorer's instantiated graph of that shape
// is updated with the batch's parameters and launched.  Work already in
// flight from an earlier launch of the same graph keeps its own parameters.
// A stream that is itself being captured by the caller, or the legacy
// default stream (which cannot be captured), gets the launches directly.
static esg_status launch_work(esg_scorer* sc, esg_batch* b, cudaStream_t st) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (!sc->use_graphs || !sc->stream || cudaStreamIsCapturing(st, &cs) != cudaSuccess ||
      cs != cudaStreamCaptureStatusNone ||
      cudaStreamIsCapturing(sc->stream, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone)
    return launch_device_work(sc, b, st);
  if (!b->graph) {
    ESG_CUDA(cudaStreamBeginCapture(sc->stream, cudaStreamCaptureModeThreadLocal));
    const esg_status ls = launch_device_work(sc, b, sc->stream);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(sc->stream, &g);
    if (ls != ESG_OK || e != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();
      if (ls != ESG_OK) return ls;
      // the capture was refused: this scorer launches one by one from now on
      sc->use_graphs = false;
      return launch_device_work(sc, b, st);
    }
    b->graph = g;
    b->graph_key = work_key(sc, b);
  }
  cudaGraphExec_t exec = nullptr;
  for (auto& ge : sc->graph_execs) {
    if (ge.first != b->graph_key) continue;
    cudaGraphExecUpdateResultInfo info{};
    if (cudaGraphExecUpdate(ge.second, b->graph, &info) == cudaSuccess) {
      exec = ge.second;
    } else {
      cudaGetLastError();
      cudaGraphExecDestroy(ge.second);
      ge.second = nullptr;
      ESG_CUDA(cudaGraphInstantiate(&ge.second, b->graph, 0));
      exec = ge.second;
    }
    break;
  }
  if (!exec) {
    ESG_CUDA(cudaGraphInstantiate(&exec, b->graph, 0));
    sc->graph_execs.emplace_back(b->graph_key, exec);
  }
  ESG_CUDA(cudaGraphLaunch(exec, st));
  return ESG_OK;
}

esg_status esg_submit(esg_scorer* sc, esg_batch* b) {
  g_err.clear();
  if (!sc || !b || b->owner != sc) return fail(ESG_ERR_BAD_ARGUMENT, "batch/scorer mismatch");
  if (b->submitted) return fail(ESG_ERR_BAD_ARGUMENT, "batch already submitted");
  ESG_CUDA(cudaSetDevice(sc->device));
  cudaStream_t st = sc->stream;
  const bool rows = b->flags & ESG_FULL_ROWS;
  const bool dev_rows = rows || b->paired;  // the pair ranking reads the rows
  const size_t np = b->paired ? std::max<uint32_t>(b->n_pairs, 1) : 0;
  const uint32_t nlist = b->host_list + b->redo_cap;
  const size_t nr = b->n_reads ? b->n_reads : 1, nq = b->n_q ? b->n_q : 1;
  // device buffers, one stream-ordered allocation
  const size_t total = batch_device_bytes(sc, b);
  ESG_CUDA(cudaMallocFromPoolAsync(&b->d_mem, total, sc->pool, st));
  b->d_bytes = total;
  char* at = (char*)b->d_mem;
  b->d_codes = carve<uint8_t>(at, b->code_words ? b->code_words * 16 : 1);
  b->d_exc = carve<uint64_t>(at, b->exceptions.empty() ? 1 : b->exceptions.size());
  b->d_packed = carve<uint8_t>(at, b->code_words ? b->code_words * 4 : 1);
  b->d_off = carve<uint64_t>(at, nr);
  b->d_len = carve<uint32_t>(at, nr);
  b->d_order = carve<uint32_t>(at, b->n_order ? b->n_order : 1);
  b->d_tasks = carve<uint2>(at, b->n_tasks ? b->n_tasks : 1);
  b->d_list = carve<uint32_t>(at, nlist ? nlist : 1);
  b->d_chunks = carve<uint32_t>(at, b->n_chunks + 1);
  b->d_counters = carve<uint32_t>(at, 8);
  b->d_qhead = carve<int4>(at, nq);
  b->d_qties = carve<uint32_t>(at, nq * sc->cap);
  b->d_k3out = carve<int32_t>(at, nlist ? (size_t)nlist * sc->n_refs : 1);
  b->d_results = carve<int4>(at, nr);
  b->d_ties = carve<uint32_t>(at, nr * sc->cap);
  b->d_rows = dev_rows ? carve<int32_t>(at, nq * sc->n_refs) : nullptr;
  b->d_pairs = np ? carve<int4>(at, 2 * np) : nullptr;
  b->d_pties = np ? carve<uint32_t>(at, np * sc->cap) : nullptr;
  if (b->n_chunks > 1) {
    b->d_part_head = carve<int4>(at, nq * b->n_chunks);
    b->d_part_ties = carve<uint32_t>(at, nq * b->n_chunks * sc->cap);
  }
  // uploads: the pinned staging is one contiguous block laid out the same way
  // as the device buffers from d_packed on (packed reads, offsets, lengths,
  // the plan); then the reads are unpacked to a byte a base
  ESG_CUDA(cudaMemcpyAsync(b->d_packed, b->in_buf.p, b->in_bytes, cudaMemcpyHostToDevice, st));
  b->stats.h2d_bytes = b->in_bytes;
  if (!b->exceptions.empty()) {
    ESG_CUDA(cudaMemcpyAsync(b->d_exc, b->exceptions.data(), b->exceptions.size() * 8,
                             cudaMemcpyHostToDevice, st));
    b->stats.h2d_bytes += b->exceptions.size() * 8;
  }
  if (b->code_words) {
    const int ublocks = (int)std::min<uint64_t>(
        (uint64_t)sc->sm_count * 8, (b->code_words + 255) / 256);
    k0_unpack<<<ublocks, 256, 0, st>>>(reinterpret_cast<const uint32_t*>(b->d_packed),
                                       b->code_words, reinterpret_cast<uint4*>(b->d_codes));
    ESG_CUDA(cudaGetLastError());
    if (!b->exceptions.empty()) {
      const int eblocks = (int)std::min<uint64_t>(
          (uint64_t)sc->sm_count * 4, (b->exceptions.size() + 255) / 256);
      k0_exceptions<<<eblocks, 256, 0, st>>>(b->d_exc, b->exceptions.size(), b->d_codes);
      ESG_CUDA(cudaGetLastError());
    }
  }
  esg_status s = launch_work(sc, b, st);
  if (s != ESG_OK) return s;
  // downloads into pinned staging
  const size_t out_bytes = carve_size(nr, 16) + carve_size(nr * sc->cap, 4) +
                           (rows ? carve_size(nq * sc->n_refs, 4) : 0) + carve_size(4, 4) +
                           carve_size(2 * np, 16) + carve_size(np * sc->cap, 4);
  b->out_buf.p = sc->pinned.get(out_bytes, &b->out_buf.cap);
  if (!b->out_buf.p) return fail(ESG_ERR_OUT_OF_MEMORY, "pinned host memory (%zu bytes)", out_bytes);
  char* o = (char*)b->out_buf.p;
  b->h_results = carve<int4>(o, nr);
  b->h_ties = carve<uint32_t>(o, nr * sc->cap);
  b->h_counters = carve<uint32_t>(o, 4);
  b->h_rows = rows ? carve<int32_t>(o, nq * sc->n_refs) : nullptr;
  b->h_pairs = np ? carve<int4>(o, 2 * np) : nullptr;
  b->h_pties = np ? carve<uint32_t>(o, np * sc->cap) : nullptr;
  // d_results and d_ties are adjacent in device memory, as in the staging
  ESG_CUDA(cudaMemcpyAsync(b->h_results, b->d_results,
                           carve_size(nr, 16) + carve_size(nr * sc->cap, 4),
                           cudaMemcpyDeviceToHost, st));
  ESG_CUDA(cudaMemcpyAsync(b->h_counters, b->d_counters, 16, cudaMemcpyDeviceToHost, st));
  if (rows)
    ESG_CUDA(cudaMemcpyAsync(b->h_rows, b->d_rows, (size_t)b->n_q * sc->n_refs * 4,
                             cudaMemcpyDeviceToHost, st));
  if (np)  // d_pairs and d_pties are adjacent too
    ESG_CUDA(cudaMemcpyAsync(b->h_pairs, b->d_pairs, carve_size(2 * np, 16) + np * sc->cap * 4,
                             cudaMemcpyDeviceToHost, st));
  b->stats.d2h_bytes = carve_size(nr, 16) + carve_size(nr * sc->cap, 4) + 16 +
                       (rows ? (size_t)b->n_q * sc->n_refs * 4 : 0) +
                       (np ? carve_size(2 * np, 16) + np * sc->cap * 4 : 0);
  ESG_CUDA(cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming));
  ESG_CUDA(cudaEventRecord(b->done, st));
  b->submitted = true;
  return ESG_OK;
}

esg_status esg_relaunch(esg_scorer* sc, esg_batch* b, void* stream) {
  g_err.clear();
  if (!sc || !b || b->owner != sc || !b->submitted)
    return fail(ESG_ERR_BAD_ARGUMENT, "relaunch needs a submitted batch of this scorer");
  ESG_CUDA(cudaSetDevice(sc->device));
  cudaStream_t st = stream ? (cudaStream_t)stream : sc->stream;
  return launch_work(sc, b, st);
}

esg_status esg_scorer_set_graphs(esg_scorer* sc, int32_t enabled) {
  g_err.clear();
  if (!sc) return fail(ESG_ERR_BAD_ARGUMENT, "NULL scorer");
  sc->use_graphs = enabled != 0;
  return ESG_OK;
}

esg_status esg_batch_read_results(esg_scorer* sc, esg_batch* b, esg_read_result* results,
                                  uint32_t* ties) {
  g_err.clear();
  if (!sc || !b || b->owner != sc || !b->submitted || !results)
    return fail(ESG_ERR_BAD_ARGUMENT, "read_results needs a submitted batch of this scorer");
  ESG_CUDA(cudaSetDevice(sc->device));
  ESG_CUDA(cudaDeviceSynchronize());
  if (b->n_reads) {
    ESG_CUDA(cudaMemcpy(results, b->d_results, (size_t)b->n_reads * 16, cudaMemcpyDeviceToHost));
    if (ties)
      ESG_CUDA(cudaMemcpy(ties, b->d_ties, (size_t)b->n_reads * sc->cap * 4,
                          cudaMemcpyDeviceToHost));
  }
  return ESG_OK;
}

esg_status esg_finish(esg_scorer* sc, esg_batch* b, esg_read_result* results, uint32_t* ties,
                      int32_t* rows) {
  g_err.clear();
  if (!sc || !b || b->owner != sc || !b->submitted)
    return fail(ESG_ERR_BAD_ARGUMENT, "finish needs a submitted batch of this scorer");
  ESG_CUDA(cudaSetDevice(sc->device));
  ESG_CUDA(cudaEventSynchronize(b->done));
  ESG_CUDA(cudaGetLastError());
  const uint32_t errbits = b->h_counters[2];
  b->stats.queries_rescored = std::min(b->h_counters[1], b->redo_cap);
  if (errbits & kErrPanelWait)
    return fail(ESG_ERR_TIMEOUT, "the panel's shared-memory staging did not complete");
  if (errbits & kErrRedoOverflow)
    return fail(ESG_ERR_DRIVER, "re-score list overflow (internal error)");
  if (results && b->n_reads) memcpy(results, b->h_results, (size_t)b->n_reads * 16);
  if (ties && b->n_reads) memcpy(ties, b->h_ties, (size_t)b->n_reads * sc->cap * 4);
  if (rows) {
    if (!(b->flags & ESG_FULL_ROWS)) return fail(ESG_ERR_BAD_ARGUMENT, "batch has no rows");
    memcpy(rows, b->h_rows, (size_t)b->n_q * sc->n_refs * 4);
  }
  return ESG_OK;
}

void esg_batch_free(esg_batch* b) {
  if (!b) return;
  esg_scorer* sc = b->owner;
  if (sc) {
    cudaSetDevice(sc->device);
    if (b->done) {
      cudaEventSynchronize(b->done);
      cudaEventDestroy(b->done);
    }
    if (b->d_mem) cudaFreeAsync(b->d_mem, sc->stream);
    if (b->graph) cudaGraphDestroy(b->graph);
    sc->pinned.put(b->in_buf.p, b->in_buf.cap);
    sc->pinned.put(b->out_buf.p, b->out_buf.cap);
  }
  delete b;
}

esg_status esg_merge_read_results(const esg_read_result* a, const uint32_t* ta,
                                  const esg_read_result* b, const uint32_t* tb, uint32_t n,
                                  uint32_t cap, esg_read_result* out, uint32_t* tout) {
  g_err.clear();
  if (n && (!a || !b || !out || !ta || !tb || !tout))
    return fail(ESG_ERR_BAD_ARGUMENT, "NULL argument");
  if (cap < 1 || cap > ESG_MAX_TIE_CAPACITY)
    return fail(ESG_ERR_BAD_ARGUMENT, "tie_capacity %u outside 1..%d", cap, ESG_MAX_TIE_CAPACITY);
  std::vector<uint32_t> buf(cap);
  for (uint32_t k = 0; k < n; ++k) {
    const esg_read_result x = a[k], y = b[k];
    const uint32_t* tx = ta + (size_t)k * cap;
    const uint32_t* ty = tb + (size_t)k * cap;
    esg_read_result r{};
    const uint32_t keep = (x.flags | y.flags) & ESG_RESULT_RESCORED32;
    if ((x.flags & ESG_RESULT_EMPTY) && (y.flags & ESG_RESULT_EMPTY)) {
      r = x;
      r.flags = ESG_RESULT_EMPTY;
      for (uint32_t w = 0; w < cap; ++w) buf[w] = ESG_NO_TIE;
    } else if (x.flags & ESG_RESULT_EMPTY || y.flags & ESG_RESULT_EMPTY) {
      const bool use_x = !(x.flags & ESG_RESULT_EMPTY);
      r = use_x ? x : y;
      const uint32_t* t = use_x ? tx : ty;
      for (uint32_t w = 0; w < cap; ++w) buf[w] = t[w];
    } else {
      const uint32_t nx = std::min(x.n_tied, cap), ny = std::min(y.n_tied, cap);
      uint32_t w = 0;
      if (x.best > y.best) {
        r.best = x.best;
        r.n_tied = x.n_tied;
        r.suboptimal = std::max(std::max(x.suboptimal, y.suboptimal), y.best);
        for (; w < nx; ++w) buf[w] = tx[w];
      } else if (y.best > x.best) {
        r.best = y.best;
        r.n_tied = y.n_tied;
        r.suboptimal = std::max(std::max(x.suboptimal, y.suboptimal), x.best);
        for (; w < ny; ++w) buf[w] = ty[w];
      } else {
        r.best = x.best;
        r.n_tied = x.n_tied + y.n_tied;
        r.suboptimal = std::max(x.suboptimal, y.suboptimal);
        uint32_t i = 0, j = 0;
        while (w < cap && (i < nx || j < ny)) {
          if (j >= ny || (i < nx && tx[i] < ty[j]))
            buf[w++] = tx[i++];
          else
            buf[w++] = ty[j++];
        }
      }
      for (; w < cap; ++w) buf[w] = ESG_NO_TIE;
      r.flags = keep | (r.n_tied > cap ? ESG_RESULT_TIES_TRUNCATED : 0u);
    }
    out[k] = r;
    memcpy(tout + (size_t)k * cap, buf.data(), (size_t)cap * 4);
  }
  return ESG_OK;
}

esg_status esg_batch_stats_get(const esg_batch* b, esg_batch_stats* out) {
  if (!b || !out) return fail(ESG_ERR_BAD_ARGUMENT, "NULL argument");
  *out = b->stats;
  if (b->owner) out->device_bytes = batch_device_bytes(b->owner, b);
  return ESG_OK;
}

esg_status esg_score_batch(esg_scorer* sc, const uint8_t* codes, const uint64_t* off,
                           const uint32_t* len, uint32_t n_reads, uint32_t flags,
                           esg_read_result* results, uint32_t* ties, int32_t* rows) {
  esg_batch* b = nullptr;
  esg_status s = esg_prepare(sc, codes, off, len, n_reads, flags, &b);
  if (s != ESG_OK) return s;
  s = esg_submit(sc, b);
  if (s == ESG_OK) s = esg_finish(sc, b, results, ties, rows);
  const std::string keep = g_err;
  esg_batch_free(b);
  g_err = keep;
  return s;
}

}  // extern "C"

// ---------------------------------------------------------------- pairs
namespace {

// Adapter bases at the 3' end of `read` (crates/eschalign/src/adapter.rs:68-91):
// the leftmost start whose overlap with the adapter's prefix has at most one
// mismatch per ten bases (the wildcard matching anything) marks everything
// from there as adapter.  A start is given up at its first mismatch past
// the allowance, which gives the same answer as counting them all.
uint32_t adapter_at(const uint8_t* read, uint32_t n, const uint8_t* ad, uint32_t a,
                    uint32_t min_overlap) {
  if (n < min_overlap || a == 0) return 0;
  for (uint32_t p = 0; p + min_overlap <= n; ++p) {
    const uint32_t overlap = std::min(a, n - p);
    if (overlap < min_overlap) break;
    const uint32_t allow = overlap / 10;
    uint32_t mism = 0, k = 0;
    for (; k < overlap; ++k) {
      const uint8_t x = read[p + k], y = ad[k];
      if (x != y && x != 4 && y != 4 && ++mism > allow) break;
    }
    if (k == overlap) return n - p;
  }
  return 0;
}

// pair_adapters (crates/eschalign-cli/src/align.rs:934-949) and detect_pair
// (adapter.rs:95-110): a mate over max_read_len is neither aligned nor
// searched; otherwise both are searched and, where their insert ends
// disagree, the weaker detection (shorter overlap) is dropped, both on a tie.
void pair_adapters(const uint8_t* m1, uint32_t l1, const uint8_t* m2, uint32_t l2,
                   const esg_adapter_config& c, uint32_t out[2]) {
  const uint32_t mo = std::max<uint32_t>(c.min_overlap, 1);
  const bool o1 = c.max_read_len && l1 > c.max_read_len;
  const bool o2 = c.max_read_len && l2 > c.max_read_len;
  out[0] = o1 ? 0 : adapter_at(m1, l1, c.r1, c.r1_len, mo);
  out[1] = o2 ? 0 : adapter_at(m2, l2, c.r2, c.r2_len, mo);
  if (!o1 && !o2 && out[0] && out[1] && l1 - out[0] != l2 - out[1]) {
    const uint32_t e1 = std::min(out[0], c.r1_len), e2 = std::min(out[1], c.r2_len);
    if (e1 > e2)
      out[1] = 0;
    else if (e1 < e2)
      out[0] = 0;
    else
      out[0] = out[1] = 0;
  }
}

// Adapters and aligned lengths of every mate of a batch (align.rs:2844-2863:
// the mate less its 3' adapter; nothing for a mate over max_read_len), on up
// to 32 host threads.
void trim_batch(const uint8_t* codes, const uint64_t* off, const uint32_t* len, uint32_t n_pairs,
                const esg_adapter_config& cfg, uint32_t* ads, uint32_t* tl) {
  const bool trim = cfg.r1_len || cfg.r2_len;
  auto work = [&](uint32_t p0, uint32_t p1) {
    for (uint32_t p = p0; p < p1; ++p) {
      const uint32_t a = 2 * p, b = a + 1;
      uint32_t ad[2] = {0, 0};
      if (trim) pair_adapters(codes + off[a], len[a], codes + off[b], len[b], cfg, ad);
      for (uint32_t m = 0; m < 2; ++m) {
        const uint32_t k = a + m;
        ads[k] = ad[m];
        tl[k] = (cfg.max_read_len && len[k] > cfg.max_read_len) ? 0 : len[k] - ad[m];
      }
    }
  };
  const uint32_t hw = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
  const uint32_t nt = std::max(1u, std::min(hw, n_pairs / 8192));
  if (nt == 1) {
    work(0, n_pairs);
    return;
  }
  std::vector<std::thread> th;
  const uint32_t per = (n_pairs + nt - 1) / nt;
  for (uint32_t t = 0; t < nt; ++t)
    th.emplace_back(work, std::min(n_pairs, t * per), std::min(n_pairs, (t + 1) * per));
  for (auto& x : th) x.join();
}

esg_status check_adapters(const esg_adapter_config* adapters, esg_adapter_config* cfg) {
  *cfg = esg_adapter_config{};
  if (!adapters) return ESG_OK;
  *cfg = *adapters;
  if ((cfg->r1_len && !cfg->r1) || (cfg->r2_len && !cfg->r2))
    return fail(ESG_ERR_BAD_ARGUMENT, "adapter codes must not be NULL");
  return ESG_OK;
}

}  // namespace

extern "C" {

esg_status esg_pair_adapters(const uint8_t* codes, const uint64_t* off, const uint32_t* len,
                             uint32_t n_pairs, const esg_adapter_config* adapters,
                             uint32_t* adapter_bases, uint32_t* aligned_len) {
  g_err.clear();
  if (n_pairs && (!off || !len || !adapter_bases || !aligned_len))
    return fail(ESG_ERR_BAD_ARGUMENT, "off/len/outputs must not be NULL");
  esg_adapter_config cfg{};
  if (esg_status s = check_adapters(adapters, &cfg); s != ESG_OK) return s;
  if (n_pairs && !codes && (cfg.r1_len || cfg.r2_len)) {
    uint64_t total = 0;
    for (uint64_t k = 0; k < 2ull * n_pairs; ++k) total += len[k];
    if (total) return fail(ESG_ERR_BAD_ARGUMENT, "codes must not be NULL");
  }
  trim_batch(codes, off, len, n_pairs, cfg, adapter_bases, aligned_len);
  return ESG_OK;
}

esg_status esg_prepare_pairs(esg_scorer* sc, const uint8_t* codes, const uint64_t* off,
                             const uint32_t* len, uint32_t n_pairs,
                             const esg_adapter_config* adapters, int32_t min_score,
                             uint32_t flags, esg_batch** out) {
  g_err.clear();
  if (!sc || !out) return fail(ESG_ERR_BAD_ARGUMENT, "NULL scorer or out");
  *out = nullptr;
  if (flags & ~(ESG_BOTH_STRANDS | ESG_FULL_ROWS))
    return fail(ESG_ERR_BAD_ARGUMENT, "unknown flags 0x%x", flags);
  if (n_pairs >= (1u << 29)) return fail(ESG_ERR_BAD_ARGUMENT, "too many pairs (%u)", n_pairs);
  if (n_pairs && (!off || !len)) return fail(ESG_ERR_BAD_ARGUMENT, "off/len must not be NULL");
  const uint32_t n_reads = 2 * n_pairs;
  std::vector<uint32_t> tl(n_reads), ads(n_reads, 0);
  esg_adapter_config cfg{};
  if (esg_status s = check_adapters(adapters, &cfg); s != ESG_OK) return s;
  if (n_reads && !codes) {
    uint64_t total = 0;
    for (uint32_t k = 0; k < n_reads; ++k) total += len[k];
    if (total) return fail(ESG_ERR_BAD_ARGUMENT, "codes must not be NULL");
  }
  trim_batch(codes, off, len, n_pairs, cfg, ads.data(), tl.data());
  esg_batch* b = nullptr;
  // every mate on both strands: the template strands need mate 1 forward and
  // mate 2 reverse-complemented (and the opposite), the Separate fallback
  // ranks each mate on both strands (pair.rs:366-387)
  esg_status s = esg_prepare(sc, codes, off, tl.data(), n_reads,
                             ESG_BOTH_STRANDS | (flags & ESG_FULL_ROWS), &b);
  if (s != ESG_OK) return s;
  b->paired = true;
  b->pair_both = flags & ESG_BOTH_STRANDS;
  b->min_score = min_score;
  b->n_pairs = n_pairs;
  uint32_t mt = 0;
  uint64_t bt = 0;
  for (uint32_t v : ads) {
    mt += v != 0;
    bt += v;
  }
  b->adapters = std::move(ads);
  b->stats.n_pairs = n_pairs;
  b->stats.mates_trimmed = mt;
  b->stats.bases_trimmed = bt;
  *out = b;
  return ESG_OK;
}

esg_status esg_finish_pairs(esg_scorer* sc, esg_batch* b, esg_pair_result* pairs,
                            uint32_t* pair_ties, esg_read_result* mates, uint32_t* mate_ties,
                            uint32_t* adapter_bases, int32_t* rows) {
  if (b && !b->paired) {
    g_err.clear();
    return fail(ESG_ERR_BAD_ARGUMENT, "not a paired batch");
  }
  esg_status s = esg_finish(sc, b, mates, mate_ties, rows);
  if (s != ESG_OK) return s;
  if (pairs && b->n_pairs) {
    static_assert(sizeof(esg_pair_result) == 32, "esg_pair_result is two int4");
    memcpy(pairs, b->h_pairs, (size_t)b->n_pairs * 32);
  }
  if (pair_ties && b->n_pairs) memcpy(pair_ties, b->h_pties, (size_t)b->n_pairs * sc->cap * 4);
  if (adapter_bases && b->n_pairs)
    memcpy(adapter_bases, b->adapters.data(), (size_t)b->n_pairs * 2 * 4);
  return ESG_OK;
}

esg_status esg_score_pairs(esg_scorer* sc, const uint8_t* codes, const uint64_t* off,
                           const uint32_t* len, uint32_t n_pairs,
                           const esg_adapter_config* adapters, int32_t min_score, uint32_t flags,
                           esg_pair_result* pairs, uint32_t* pair_ties, esg_read_result* mates,
                           uint32_t* mate_ties, uint32_t* adapter_bases, int32_t* rows) {
  esg_batch* b = nullptr;
  esg_status s = esg_prepare_pairs(sc, codes, off, len, n_pairs, adapters, min_score, flags, &b);
  if (s != ESG_OK) return s;
  s = esg_submit(sc, b);
  if (s == ESG_OK)
    s = esg_finish_pairs(sc, b, pairs, pair_ties, mates, mate_ties, adapter_bases, rows);
  const std::string keep = g_err;
  esg_batch_free(b);
  g_err = keep;
  return s;
}

}  // extern "C"
