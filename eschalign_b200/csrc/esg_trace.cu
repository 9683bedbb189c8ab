// esg_trace.cu -- traceback of winners on the device: the alignment
// (coordinates and CIGAR) of chosen (read, reference, strand) jobs, as
// crates/eschalign/src/scalar.rs:182-364 computes it.
//
// k7_trace: one warp per task.  A task is a tile of jobs whose 16-row
// stripes fill the warp's lanes (a job of n rows takes ceil(n / 16) lanes;
// each job has its own reference), or one long job (over 32 stripes) run in
// passes of 32 stripes chained through a per-warp column buffer.  Lanes
// walk their job's reference columns as a systolic array (lane l one step
// behind lane l - 1, the stripe's bottom row passed down by shuffle) in
// int32 -- the recurrence of scalar.rs:213-289 exactly, no saturation --
// and write one 4-bit trace code per cell (source: stop / diagonal /
// insertion / deletion, plus the E- and F-extended bits) to a per-warp
// scratch: 8 bytes per lane per column, lane-contiguous, so a warp writes
// 256 coalesced bytes a column and the scratch of the resident warps stays
// in L2.  Reads are top-padded so the last row sits at row 15 of the last
// stripe; pad rows hold H = 0, the zero border.  Each lane keeps its first
// maximum in column-major order (local: every cell; semi-global: the last
// row and the last column); a segmented shuffle reduction gives the job's
// end cell, and the job's last lane follows the trace codes back
// (scalar.rs:292-364), writing run-length CIGAR words.  k7_compact packs
// the jobs' words into the caller's layout.
#include "../../include/eschalign_b200.h"
#include "esg_internal.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

extern "C" void esg_internal_set_error(esg_status st, const char* msg);

namespace {

constexpr int kTR = 16;                 // rows per lane stripe
constexpr int kTWarps = 4;              // warps per CTA
constexpr int kTThreads = kTWarps * 32;
constexpr int kNegT = INT32_MIN / 4;    // scalar.rs's NEG
constexpr uint32_t kFullT = 0xffffffffu;
// trace codes (scalar.rs:167-175)
constexpr uint32_t kStop = 0, kDiag = 1, kIns = 2, kDel = 3, kEExt = 4, kFExt = 8;
// cigar ops (BAM)
constexpr uint32_t kOpM = 0, kOpI = 1, kOpD = 2;

struct K7Params {
  const uint8_t* codes;       // reads, 1 B codes
  const uint64_t* off;
  const uint32_t* len;
  const uint8_t* rcodes;      // panel, longest first (slot order)
  const uint32_t* roff;
  const uint32_t* rlen;
  const uint32_t* job_q;      // read | reverse << 31
  const uint32_t* job_slot;   // panel slot of the job's reference
  const uint64_t* job_at;     // the job's first word in the ops staging
  const uint32_t* order;      // jobs in task order
  const uint2* tasks;         // {start in order, count | stripes << 16}; stripes > 32: one long job
  uint32_t n_tasks;
  uint32_t* task_counter;
  uint2* trace;               // per warp: trace_words uint2
  size_t trace_words;
  uint32_t mcols;             // columns of one pass in the trace scratch
  uint2* colbuf;              // per warp: mcols (H, F), long jobs
  int ma, mi, o, e;
  int4* res;                  // per job {score, query_start, query_end, ref_start}
  int4* res2;                 // per job {ref_end, n_ops, 0, 0}
  uint32_t* ops;              // staging
};

__device__ __forceinline__ uint32_t mask4(uint32_t c) { return c < 4 ? 1u << c : 0xfu; }

// (b1, j1, i1) better than (b0, j0, i0): higher score, then smaller column,
// then smaller row -- the first maximum of a column-major scan.
__device__ __forceinline__ bool better(int b1, int j1, int i1, int b0, int j0, int i0) {
  return b1 > b0 || (b1 == b0 && (j1 < j0 || (j1 == j0 && i1 < i0)));
}

template <bool kLocal>
__global__ void __launch_bounds__(kTThreads) k7_trace(const K7Params P) {
  const int lane = threadIdx.x & 31;
  const size_t warp = (size_t)blockIdx.x * kTWarps + (threadIdx.x >> 5);
  uint2* trace = P.trace + warp * P.trace_words;
  uint2* colbuf = P.colbuf + warp * P.mcols;
  for (;;) {
    uint32_t task = 0;
    if (lane == 0) task = atomicAdd(P.task_counter, 1u);
    task = __shfl_sync(kFullT, task, 0);
    if (task >= P.n_tasks) break;
    const uint2 tk = P.tasks[task];
    const uint32_t count = tk.y & 0xffffu;
    const int smax = (int)(tk.y >> 16);
    const bool long_job = smax > 32;

    // --- lane -> (job, first lane of the job, stripes)
    uint32_t job = 0, n = 0;
    int S = 0, s0 = 0;
    bool has_job = false;
    if (long_job) {
      job = P.order[tk.x];
      n = P.len[P.job_q[job] & 0x7fffffffu];
      S = smax;
      has_job = true;
    } else {
      uint32_t kj = 0, kn = 0, kS = 0;
      if ((uint32_t)lane < count) {
        kj = P.order[tk.x + lane];
        kn = P.len[P.job_q[kj] & 0x7fffffffu];
        kS = (kn + kTR - 1) / kTR;
      }
      uint32_t incl = kS;
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const uint32_t v = __shfl_up_sync(kFullT, incl, d);
        if (lane >= d) incl += v;
      }
      for (uint32_t k = 0; k < count; ++k) {
        const uint32_t ek = __shfl_sync(kFullT, incl, k);
        const uint32_t sk = __shfl_sync(kFullT, kS, k);
        const uint32_t jk = __shfl_sync(kFullT, kj, k);
        const uint32_t nk = __shfl_sync(kFullT, kn, k);
        if ((uint32_t)lane >= ek - sk && (uint32_t)lane < ek) {
          job = jk;
          n = nk;
          S = (int)sk;
          s0 = (int)(ek - sk);
          has_job = true;
        }
      }
    }
    const uint32_t jq = has_job ? P.job_q[job] : 0u;
    const uint32_t rd = jq & 0x7fffffffu;
    const bool rc = (jq >> 31) != 0;
    const uint32_t slot = has_job ? P.job_slot[job] : 0u;
    const int m = has_job ? (int)P.rlen[slot] : 0;
    const uint8_t* rp = P.rcodes + (has_job ? P.roff[slot] : 0u);
    const uint8_t* q = P.codes + (has_job ? P.off[rd] : 0ull);
    const int pad = S * kTR - (int)n;
    const int passes = long_job ? (S + 31) / 32 : 1;

    int best = kLocal ? 0 : kNegT, bj = 0, bi = 0;  // 1-based end cell, 0: none
    for (int pass = 0; pass < passes; ++pass) {
      const int s = long_job ? pass * 32 + lane : lane - s0;  // stripe of the job
      const bool valid = has_job && s >= 0 && s < S;
      const bool first = valid && s == 0;
      const bool from_buf = long_job && pass > 0 && lane == 0;
      const bool to_buf = long_job && pass + 1 < passes && lane == 31;
      const int padrows = (valid && s == 0) ? pad : 0;
      uint32_t qm[kTR];
#pragma unroll
      for (int r = 0; r < kTR; ++r) {
        const int i = s * kTR + r - pad;  // 0-based read row
        uint32_t c = 4;
        if (valid && i >= 0) {
          uint32_t x = rc ? q[n - 1 - i] : q[i];
          x = x > 4 ? 4 : x;
          c = (rc && x < 4) ? 3 - x : x;
        }
        qm[r] = mask4(c);
      }
      int H[kTR], E[kTR];
#pragma unroll
      for (int r = 0; r < kTR; ++r) {
        H[r] = 0;
        E[r] = kNegT;
      }
      int hbot = 0, fbot = kNegT, hdg = 0;
      const int skew = long_job ? lane : s;
      int steps = valid ? m + skew : 0;
#pragma unroll
      for (int d = 16; d; d >>= 1) steps = max(steps, __shfl_xor_sync(kFullT, steps, d));
#pragma unroll 1
      for (int t = 0; t < steps; ++t) {
        const int j = t - skew;
        int ht = __shfl_up_sync(kFullT, hbot, 1);
        int ft = __shfl_up_sync(kFullT, fbot, 1);
        if (first) {
          ht = 0;
          ft = kNegT;
        }
        if (valid && (unsigned)j < (unsigned)m) {
          if (from_buf) {
            const uint2 b = colbuf[j];
            ht = (int)b.x;
            ft = (int)b.y;
          }
          const uint32_t rm = mask4(rp[j]);
          int hup = ht, f = ft, hdiag = hdg;
          hdg = ht;
          uint32_t w0 = 0, w1 = 0;
#pragma unroll
          for (int r = 0; r < kTR; ++r) {
            const int hleft = H[r];
            const int e_ext = E[r] + P.e, e_open = hleft + P.o;
            const int ev = max(e_open, e_ext);
            const int f_ext = f + P.e, f_open = hup + P.o;
            f = max(f_open, f_ext);
            const int hd = hdiag + ((qm[r] & rm) ? P.ma : P.mi);
            int h = max(max(hd, ev), f);
            if (kLocal) h = max(h, 0);
            if (r < padrows) h = 0;  // the zero border above the read
            uint32_t t4 = h == f ? kIns : kDel;
            if (h == hd) t4 = kDiag;
            if (kLocal && h == 0) t4 = kStop;
            t4 |= (ev == e_ext ? kEExt : 0u) | (f == f_ext ? kFExt : 0u);
            if (r < 8)
              w0 |= t4 << (4 * r);
            else
              w1 |= t4 << (4 * (r - 8));
            E[r] = ev;
            hdiag = hleft;
            H[r] = h;
            hup = h;
            if (kLocal && h > best) {  // pad rows hold 0: never above best
              best = h;
              bi = s * kTR + r - pad + 1;
              bj = j + 1;
            }
          }
          trace[((size_t)pass * P.mcols + j) * 32 + lane] = make_uint2(w0, w1);
          hbot = H[kTR - 1];
          fbot = f;
          if (to_buf) colbuf[j] = make_uint2((uint32_t)hbot, (uint32_t)fbot);
          if (!kLocal) {
            if (j < m - 1) {
              if (s == S - 1 && hbot > best) {  // the last row
                best = hbot;
                bi = (int)n;
                bj = j + 1;
              }
            } else {
#pragma unroll
              for (int r = 0; r < kTR; ++r) {  // the last column, rows in order
                const int i = s * kTR + r - pad + 1;
                if (i >= 1 && H[r] > best) {
                  best = H[r];
                  bi = i;
                  bj = m;
                }
              }
            }
          }
        }
      }
      __syncwarp();  // trace and column buffer writes visible to the warp
    }

    // --- the job's end cell: first maximum over its lanes
    {
      const int sj = long_job ? lane : lane - s0;
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const int b2 = __shfl_up_sync(kFullT, best, d);
        const int j2 = __shfl_up_sync(kFullT, bj, d);
        const int i2 = __shfl_up_sync(kFullT, bi, d);
        if (has_job && sj >= d && better(b2, j2, i2, best, bj, bi)) {
          best = b2;
          bj = j2;
          bi = i2;
        }
      }
    }
    // --- the walk, by the job's last lane
    const bool walker = has_job && (long_job ? lane == 31 : lane - s0 == S - 1);
    if (walker) {
      int i = bi, j = bj;
      uint32_t* out = P.ops + P.job_at[job];
      uint32_t runs = 0, cur = 4, cnt = 0;
      int state = 0;  // 0 H, 1 E (deletion), 2 F (insertion)
      while (i > 0 && j > 0) {
        const int ip = i - 1 + pad;
        const int st = ip >> 4, r = ip & 15;
        const int ln = long_job ? (st & 31) : s0 + st;
        const int ps = long_job ? (st >> 5) : 0;
        const uint2 w = trace[((size_t)ps * P.mcols + (j - 1)) * 32 + ln];
        const uint32_t t4 = ((r < 8 ? w.x : w.y) >> (4 * (r & 7))) & 0xfu;
        uint32_t op = 4;
        if (state == 0) {
          const uint32_t src = t4 & 3u;
          if (src == kStop) break;
          if (src == kDiag) {
            op = kOpM;
            --i;
            --j;
          } else if (src == kIns) {
            state = 2;
          } else {
            state = 1;
          }
        } else if (state == 2) {
          op = kOpI;
          if (!(t4 & kFExt)) state = 0;
          --i;
        } else {
          op = kOpD;
          if (!(t4 & kEExt)) state = 0;
          --j;
        }
        if (op != 4) {
          if (op == cur) {
            ++cnt;
          } else {
            if (cnt) out[runs++] = (cnt << 4) | cur;
            cur = op;
            cnt = 1;
          }
        }
      }
      if (cnt) out[runs++] = (cnt << 4) | cur;
      for (uint32_t a = 0, b = runs ? runs - 1 : 0; a < b; ++a, --b) {  // first to last
        const uint32_t x = out[a];
        out[a] = out[b];
        out[b] = x;
      }
      const bool none = bi == 0 || bj == 0;
      P.res[job] = none ? make_int4(0, 0, 0, 0) : make_int4(best, i, bi, j);
      P.res2[job] = make_int4(none ? 0 : bj, (int)runs, 0, 0);
    }
    __syncwarp();  // the walk is done before the scratch is reused
  }
}

// Pack each job's CIGAR words from the staging into the caller's layout.
__global__ void __launch_bounds__(256) k7_compact(const uint32_t* staging, const uint64_t* at,
                                                  const uint64_t* dst, const int4* res2,
                                                  uint32_t n_jobs, uint32_t* out) {
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n_jobs;
       k += gridDim.x * blockDim.x) {
    const uint32_t nr = (uint32_t)res2[k].y;
    for (uint32_t w = 0; w < nr; ++w) out[dst[k] + w] = staging[at[k] + w];
  }
}

esg_status terr(esg_status st, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  esg_internal_set_error(st, buf);
  return st;
}

#define TCUDA(call)                                                          \
  do {                                                                       \
    cudaError_t e_ = (call);                                                 \
    if (e_ != cudaSuccess) {                                                 \
      if (mem) cudaFreeAsync(mem, st);                                       \
      return terr(ESG_ERR_DRIVER, "%s: %s", #call, cudaGetErrorString(e_));  \
    }                                                                        \
  } while (0)

size_t align256(size_t v) { return (v + 255) / 256 * 256; }

// Align the jobs against reads already on the device.
esg_status align_impl(esg_scorer* sc, const uint8_t* d_codes, const uint64_t* d_off,
                      const uint32_t* d_len, uint32_t n_reads, const uint32_t* h_len,
                      const esg_align_job* jobs, uint32_t n_jobs, esg_alignment* out,
                      uint32_t* ops, uint64_t ops_capacity, uint64_t* ops_needed,
                      std::vector<uint32_t>* grow = nullptr, cudaStream_t stream = nullptr) {
  esg_internal_panel P{};
  esg_internal_panel_of(sc, &P);
  if (n_jobs && (!jobs || !out)) return terr(ESG_ERR_BAD_ARGUMENT, "jobs/out must not be NULL");
  // --- plan on the host
  std::vector<uint32_t> job_q(n_jobs), job_slot(n_jobs), S(n_jobs), M(n_jobs);
  std::vector<uint64_t> job_at(n_jobs);
  uint64_t staging = 0;
  uint32_t mcols = 1, passes_max = 1;
  std::vector<uint32_t> live;
  for (uint32_t k = 0; k < n_jobs; ++k) {
    const esg_align_job& jb = jobs[k];
    if (jb.read >= n_reads) return terr(ESG_ERR_BAD_ARGUMENT, "job %u: no read %u", k, jb.read);
    if (jb.ref >= P.n_refs) return terr(ESG_ERR_BAD_ARGUMENT, "job %u: no reference %u", k, jb.ref);
    if (jb.reverse > 1) return terr(ESG_ERR_BAD_ARGUMENT, "job %u: reverse must be 0 or 1", k);
    const uint32_t n = h_len[jb.read], m = P.len_of[jb.ref];
    job_q[k] = jb.read | (jb.reverse << 31);
    job_slot[k] = P.slot_of[jb.ref];
    job_at[k] = staging;
    staging += (uint64_t)n + m + 1;
    S[k] = (n + kTR - 1) / kTR;
    M[k] = m;
    if (n && m) {
      live.push_back(k);
      mcols = std::max(mcols, m);
      if (S[k] > 32) passes_max = std::max(passes_max, (S[k] + 31) / 32);
    }
    if (S[k] > 0xffffu) return terr(ESG_ERR_BAD_ARGUMENT, "job %u: read too long", k);
  }
  // tiles of jobs up to 32 stripes (next fit, longest first); longer jobs alone
  {
    // longest first, stable: a counting sort on the stripes (long jobs, over
    // 32 stripes, are few and sorted apart)
    std::vector<uint32_t> longs, cnt(34, 0), sorted(live.size());
    for (uint32_t k : live) ++cnt[std::min<uint32_t>(S[k], 33)];
    uint32_t at = 0;
    std::vector<uint32_t> start(34, 0);
    for (int v = 33; v >= 1; --v) {
      start[v] = at;
      at += cnt[v];
    }
    for (uint32_t k : live) sorted[start[std::min<uint32_t>(S[k], 33)]++] = k;
    const uint32_t n_long = cnt[33];
    std::stable_sort(sorted.begin(), sorted.begin() + n_long,
                     [&](uint32_t a, uint32_t b) { return S[a] > S[b]; });
    live.swap(sorted);
  }
  std::vector<uint32_t> order;
  std::vector<uint2> tasks;
  order.reserve(live.size());
  uint32_t open_start = 0, open_count = 0, open_free = 0, open_smax = 0;
  auto close_tile = [&]() {
    if (open_count) tasks.push_back(make_uint2(open_start, open_count | (open_smax << 16)));
    open_count = 0;
  };
  for (uint32_t k : live) {
    if (S[k] > 32) {
      tasks.push_back(make_uint2((uint32_t)order.size(), 1u | (S[k] << 16)));
      order.push_back(k);
      continue;
    }
    if (!open_count || S[k] > open_free) {
      close_tile();
      open_start = (uint32_t)order.size();
      open_free = 32;
      open_smax = S[k];
    }
    order.push_back(k);
    open_free -= S[k];
    ++open_count;
  }
  close_tile();
  const uint32_t n_tasks = (uint32_t)tasks.size();

  // --- geometry and scratch: per warp passes x columns x 32 lanes of 8 B,
  // capped at 4 GiB in all
  const size_t trace_words = (size_t)passes_max * mcols * 32;
  if (trace_words * 8 > (1ull << 30))
    return terr(ESG_ERR_BAD_ARGUMENT,
                "a job of %u stripes x %u columns needs over 1 GiB of trace per warp", passes_max * 32,
                mcols);
  int per_sm = 0;
  cudaSetDevice(P.device);
  const void* fn = P.mode == ESG_MODE_LOCAL ? (const void*)k7_trace<true>
                                            : (const void*)k7_trace<false>;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kTThreads, 0) != cudaSuccess)
    per_sm = 1;
  uint64_t warps = std::min<uint64_t>((uint64_t)std::max(per_sm, 1) * P.sm_count * kTWarps,
                                      std::max<uint32_t>(n_tasks, 1));
  warps = std::min<uint64_t>(warps, std::max<uint64_t>(kTWarps, (4ull << 30) / (trace_words * 8)));
  const uint64_t blocks = std::max<uint64_t>(1, (warps + kTWarps - 1) / kTWarps);
  warps = blocks * kTWarps;

  const size_t nj = std::max<uint32_t>(n_jobs, 1);
  const size_t sizes[] = {
      align256(nj * 4),                          // job_q
      align256(nj * 4),                          // job_slot
      align256(nj * 8),                          // job_at
      align256(std::max<size_t>(order.size(), 1) * 4),
      align256(std::max<uint32_t>(n_tasks, 1) * 8),
      align256(4),                               // task counter
      align256(nj * 16),                         // res
      align256(nj * 16),                         // res2
      align256(std::max<uint64_t>(staging, 1) * 4),
      align256(warps * trace_words * 8),
      align256(warps * (size_t)mcols * 8),
      align256(nj * 8),                          // dst
  };
  size_t total = 0;
  for (size_t v : sizes) total += v;
  cudaStream_t st = stream ? stream : P.stream;
  void* mem = nullptr;
  TCUDA(cudaMallocFromPoolAsync(&mem, total, P.pool, st));
  char* at = (char*)mem;
  auto take = [&](size_t i) {
    char* p = at;
    at += sizes[i];
    return p;
  };
  uint32_t* d_job_q = (uint32_t*)take(0);
  uint32_t* d_job_slot = (uint32_t*)take(1);
  uint64_t* d_job_at = (uint64_t*)take(2);
  uint32_t* d_order = (uint32_t*)take(3);
  uint2* d_tasks = (uint2*)take(4);
  uint32_t* d_counter = (uint32_t*)take(5);
  int4* d_res = (int4*)take(6);
  int4* d_res2 = (int4*)take(7);
  uint32_t* d_staging = (uint32_t*)take(8);
  uint2* d_trace = (uint2*)take(9);
  uint2* d_colbuf = (uint2*)take(10);
  uint64_t* d_dst = (uint64_t*)take(11);
  if (n_jobs) {
    TCUDA(cudaMemcpyAsync(d_job_q, job_q.data(), n_jobs * 4, cudaMemcpyHostToDevice, st));
    TCUDA(cudaMemcpyAsync(d_job_slot, job_slot.data(), n_jobs * 4, cudaMemcpyHostToDevice, st));
    TCUDA(cudaMemcpyAsync(d_job_at, job_at.data(), n_jobs * 8, cudaMemcpyHostToDevice, st));
  }
  if (!order.empty())
    TCUDA(cudaMemcpyAsync(d_order, order.data(), order.size() * 4, cudaMemcpyHostToDevice, st));
  if (n_tasks)
    TCUDA(cudaMemcpyAsync(d_tasks, tasks.data(), n_tasks * 8, cudaMemcpyHostToDevice, st));
  TCUDA(cudaMemsetAsync(d_counter, 0, 4, st));
  TCUDA(cudaMemsetAsync(d_res, 0, nj * 16, st));   // empty jobs stay all zero
  TCUDA(cudaMemsetAsync(d_res2, 0, nj * 16, st));
  if (n_tasks) {
    K7Params K{};
    K.codes = d_codes;
    K.off = d_off;
    K.len = d_len;
    K.rcodes = P.rcodes;
    K.roff = P.roff;
    K.rlen = P.rlen;
    K.job_q = d_job_q;
    K.job_slot = d_job_slot;
    K.job_at = d_job_at;
    K.order = d_order;
    K.tasks = d_tasks;
    K.n_tasks = n_tasks;
    K.task_counter = d_counter;
    K.trace = d_trace;
    K.trace_words = trace_words;
    K.mcols = mcols;
    K.colbuf = d_colbuf;
    K.ma = P.scoring.match_score;
    K.mi = P.scoring.mismatch;
    K.o = P.scoring.gap_open;
    K.e = P.scoring.gap_extend;
    K.res = d_res;
    K.res2 = d_res2;
    K.ops = d_staging;
    void* args[] = {&K};
    TCUDA(cudaLaunchKernel(fn, dim3((unsigned)blocks), dim3(kTThreads), args, 0, st));
  }
  // --- results, then the words packed into the caller's layout
  std::vector<int4> res(nj), res2(nj);
  TCUDA(cudaMemcpyAsync(res.data(), d_res, nj * 16, cudaMemcpyDeviceToHost, st));
  TCUDA(cudaMemcpyAsync(res2.data(), d_res2, nj * 16, cudaMemcpyDeviceToHost, st));
  TCUDA(cudaStreamSynchronize(st));
  std::vector<uint64_t> dst(nj, 0);
  uint64_t need = 0;
  for (uint32_t k = 0; k < n_jobs; ++k) {
    dst[k] = need;
    need += (uint32_t)res2[k].y;
  }
  if (ops_needed) *ops_needed = need;
  if (grow) {
    grow->resize(need);
    ops = grow->data();
    ops_capacity = need;
  }
  if (need > ops_capacity || (need && !ops)) {
    cudaFreeAsync(mem, st);
    return terr(ESG_ERR_BAD_ARGUMENT, "the alignments need %llu CIGAR words, room for %llu",
                (unsigned long long)need, (unsigned long long)ops_capacity);
  }
  if (need) {
    uint32_t* d_out = nullptr;
    TCUDA(cudaMemcpyAsync(d_dst, dst.data(), n_jobs * 8, cudaMemcpyHostToDevice, st));
    // the packed words go where the trace scratch was (it is no longer needed)
    if (need * 4 <= sizes[9]) {
      d_out = (uint32_t*)d_trace;
    } else {
      TCUDA(cudaMallocFromPoolAsync((void**)&d_out, need * 4, P.pool, st));
    }
    const int cb = (int)std::min<uint64_t>(4096, (n_jobs + 255) / 256);
    k7_compact<<<cb, 256, 0, st>>>(d_staging, d_job_at, d_dst, d_res2, n_jobs, d_out);
    TCUDA(cudaGetLastError());
    TCUDA(cudaMemcpyAsync(ops, d_out, need * 4, cudaMemcpyDeviceToHost, st));
    TCUDA(cudaStreamSynchronize(st));
    if ((void*)d_out != (void*)d_trace) cudaFreeAsync(d_out, st);
  }
  for (uint32_t k = 0; k < n_jobs; ++k) {
    out[k].score = res[k].x;
    out[k].query_start = (uint32_t)res[k].y;
    out[k].query_end = (uint32_t)res[k].z;
    out[k].ref_start = (uint32_t)res[k].w;
    out[k].ref_end = (uint32_t)res2[k].x;
    out[k].n_ops = (uint32_t)res2[k].y;
    out[k].ops_offset = dst[k];
  }
  cudaFreeAsync(mem, st);
  esg_internal_set_error(ESG_OK, "");
  return ESG_OK;
}

}  // namespace

esg_status esg_internal_align_batch(esg_scorer* sc, esg_batch* b, const esg_align_job* jobs,
                                    uint32_t n_jobs, esg_alignment* out,
                                    std::vector<uint32_t>* ops, cudaStream_t stream) {
  const uint8_t* codes = nullptr;
  const uint64_t* off = nullptr;
  const uint32_t* len = nullptr;
  const uint32_t* h_len = nullptr;
  uint32_t n_reads = 0;
  esg_internal_batch_reads(b, &codes, &off, &len, &n_reads, &h_len);
  if (!codes) return terr(ESG_ERR_BAD_ARGUMENT, "the batch is not submitted");
  return align_impl(sc, codes, off, len, n_reads, h_len, jobs, n_jobs, out, nullptr, 0, nullptr,
                    ops, stream);
}

extern "C" {

esg_status esg_align_batch(esg_scorer* sc, esg_batch* b, const esg_align_job* jobs,
                           uint32_t n_jobs, esg_alignment* out, uint32_t* ops,
                           uint64_t ops_capacity, uint64_t* ops_needed) {
  if (!sc || !b) return terr(ESG_ERR_BAD_ARGUMENT, "NULL scorer or batch");
  const uint8_t* codes = nullptr;
  const uint64_t* off = nullptr;
  const uint32_t* len = nullptr;
  const uint32_t* h_len = nullptr;
  uint32_t n_reads = 0;
  esg_internal_batch_reads(b, &codes, &off, &len, &n_reads, &h_len);
  if (!codes) return terr(ESG_ERR_BAD_ARGUMENT, "the batch is not submitted");
  return align_impl(sc, codes, off, len, n_reads, h_len, jobs, n_jobs, out, ops, ops_capacity,
                    ops_needed);
}

esg_status esg_align_reads(esg_scorer* sc, const uint8_t* codes, const uint64_t* off,
                           const uint32_t* len, uint32_t n_reads, const esg_align_job* jobs,
                           uint32_t n_jobs, esg_alignment* out, uint32_t* ops,
                           uint64_t ops_capacity, uint64_t* ops_needed) {
  if (!sc) return terr(ESG_ERR_BAD_ARGUMENT, "NULL scorer");
  if (n_reads && (!off || !len)) return terr(ESG_ERR_BAD_ARGUMENT, "off/len must not be NULL");
  esg_internal_panel P{};
  esg_internal_panel_of(sc, &P);
  // the reads, packed, to the device (no scoring)
  std::vector<uint64_t> poff(std::max<uint32_t>(n_reads, 1), 0);
  uint64_t total = 0;
  for (uint32_t k = 0; k < n_reads; ++k) {
    poff[k] = total;
    total += len[k];
  }
  if (total && !codes) return terr(ESG_ERR_BAD_ARGUMENT, "codes must not be NULL");
  std::vector<uint8_t> pc(std::max<uint64_t>(total, 1));
  for (uint32_t k = 0; k < n_reads; ++k)
    if (len[k]) memcpy(pc.data() + poff[k], codes + off[k], len[k]);
  cudaSetDevice(P.device);
  cudaStream_t st = P.stream;
  const size_t b0 = align256(pc.size()), b1 = align256(poff.size() * 8),
               b2 = align256(std::max<uint32_t>(n_reads, 1) * 4);
  void* mem = nullptr;
  TCUDA(cudaMallocFromPoolAsync(&mem, b0 + b1 + b2, P.pool, st));
  uint8_t* d_codes = (uint8_t*)mem;
  uint64_t* d_off = (uint64_t*)((char*)mem + b0);
  uint32_t* d_len = (uint32_t*)((char*)mem + b0 + b1);
  TCUDA(cudaMemcpyAsync(d_codes, pc.data(), pc.size(), cudaMemcpyHostToDevice, st));
  TCUDA(cudaMemcpyAsync(d_off, poff.data(), poff.size() * 8, cudaMemcpyHostToDevice, st));
  if (n_reads) TCUDA(cudaMemcpyAsync(d_len, len, n_reads * 4, cudaMemcpyHostToDevice, st));
  const esg_status s = align_impl(sc, d_codes, d_off, d_len, n_reads, len, jobs, n_jobs, out,
                                  ops, ops_capacity, ops_needed);
  cudaFreeAsync(mem, st);
  cudaStreamSynchronize(st);
  return s;
}

}  // extern "C"
