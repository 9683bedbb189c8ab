// esg_kernels.cuh -- device code of the B200 panel scorer (sm_100a).
//
// Four kernels, launched in this order on one stream per batch:
//
//   k2_batched   the product: every (query, reference pair) of the panel in
//                int16x2 lanes.  One warp is a 32-lane systolic array: each
//                lane holds a 16- or 32-row stripe of one query (G, E and
//                the row's substitution table or score-record address in
//                registers) and walks the columns of a reference pair; the
//                stripe's bottom row goes to the next lane by shuffle, so no
//                DP state ever leaves the register file.  The two 16-bit
//                halves of every register are two references (a
//                length-sorted pair).  Substitution is one PRMT per cell
//                pair, or (local mode, and semi-global 32-row stripes) one
//                shared-memory load from the lane's per-column score record;
//                the recurrence is three VIADDMNMX and one VIMNMX (DPX) plus
//                one IMAD.  The argmax / tie / XS reduction is folded in per
//                query, online, in shared memory.
//                Pairs that may have left int16 are flagged and their query
//                is re-scored by the int32 kernel.
//   k3_lanes     the exact int32 path: the recurrence of
//                crates/eschalign/src/scalar.rs:120-163 on chains of lanes
//                (16-row stripes, bottom rows passed by shuffle, several
//                references a warp for short queries); what k2 cannot take
//                or flags.  With one lane a chain it is the one-thread-per-
//                pair comparison arm.
//   k4_rows      per-query reduction of k3's rows (mapper.rs:444-472).
//   k5_merge     per read: forward and reverse-complement query states
//                merged into the read's result.
//   k6_pairs     paired batches: per pair, the (reference, template strand)
//                candidates of crates/eschalign/src/mapper/pair.rs:195-234
//                ranked from the four mate rows (one warp per pair).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace esg {

constexpr int kRows = 16;             // rows per lane stripe (k2)
constexpr int kMaxStripes = 32;       // a query spans at most one warp (k2)
constexpr int kNeg16 = -31500;        // int16 stand-in for -infinity (biased domain)
constexpr int kBiasLocal = 2048;      // local: H + B >= B >= |o|, |e|
constexpr int kBiasSemiGlobal = -16384;  // semi-global: H + B < 0 while |H| < 12000
constexpr int kNeg32 = -(1 << 29);    // int32 stand-in for -infinity, i32::MIN / 4 (scalar.rs:42)
// k2 CTA shape: 4 warps, 4 resident CTAs per SM (16 warps, <= 128
// registers; 3 for 32-row stripes).  Tuning knobs, each measured on B200 on
// the C2 workload (1 M reads of ~110 nt x 164 references, both strands):
//   ESG_K2_WARPS / ESG_K2_MIN_BLOCKS  CTA shape (4 x 4 beat 4 x 5 at 96
//       registers once local mode reads its scores from shared memory, and
//       8 warps x 2 CTAs)
//   ESG_SC_LDS  modes whose per-cell scores come from a per-thread record in
//       shared memory (bit 0 local, bit 1 semi-global) instead of one PRMT
//       per cell: local +5.0 %; semi-global on 32-row stripes
//       (ESG_SC_LDS_SG_MINR 32) +1.9 % on C4 pairs and C2 semi-global once
//       its last-column snapshot stopped spilling (-1.0 % before), 16-row
//       stripes as well -0.4 %
//   ESG_SEL_PREFETCH  modes that load a lane's next column selector a column
//       ahead (bit 0 local, bit 1 semi-global): +2 % in both with the above
//   ESG_STEADY_UNROLL  unroll of local mode's unchecked column loop, 16-row
//       stripes (8: +0.9 % over 4)
//   ESG_STEADY_UNROLL32  the same for 32-row stripes reading the panel from
//       L2 (C3: 4 +3.9 % over 1, 8 -1.1 % against 4); with the panel in
//       shared memory they stay at 1 (unrolled, they spill)
//   ESG_K2_R32_BLOCKS  resident CTAs of 32-row stripes (3; 2 lets
//       semi-global keep its state without spilling but measured -4.6 % on
//       C2 semi-global, local and C3 unchanged)
#ifndef ESG_K2_WARPS
#define ESG_K2_WARPS 4
#endif
#ifndef ESG_K2_MIN_BLOCKS
#define ESG_K2_MIN_BLOCKS 4
#endif
#ifndef ESG_K2_R32_BLOCKS
#define ESG_K2_R32_BLOCKS 3
#endif
#ifndef ESG_SC_LDS
#define ESG_SC_LDS 3
#endif
#ifndef ESG_SEL_PREFETCH
#define ESG_SEL_PREFETCH 3
#endif
#ifndef ESG_STEADY_UNROLL
#define ESG_STEADY_UNROLL 8
#endif
#ifndef ESG_STEADY_UNROLL32
#define ESG_STEADY_UNROLL32 4
#endif
constexpr int kK2Warps = ESG_K2_WARPS;  // warps per k2 CTA
constexpr int kK2Threads = kK2Warps * 32;
constexpr uint32_t kFull = 0xffffffffu;
constexpr uint32_t kNoRef = 0xffffffffu;
constexpr uint32_t kMaxCap = 32;       // largest tie capacity (ESG_MAX_TIE_CAPACITY)
// per-thread shared words of the column score record (one per row code
// 0-5), word c of thread t at c * kK2Threads + t: every thread in its own bank
constexpr int kScrWords = ESG_SC_LDS ? 6 : 0;
constexpr uint32_t kScrStride = (uint32_t)kK2Threads * 4;  // bytes between code words
#ifndef ESG_SC_LDS_SG_MINR
#define ESG_SC_LDS_SG_MINR 32
#endif
template <bool kLocal, int R>
__host__ __device__ constexpr bool sc_lds() {
  return (ESG_SC_LDS & (kLocal ? 1 : 2)) != 0 && (kLocal || R >= ESG_SC_LDS_SG_MINR);
}
template <bool kLocal>
__host__ __device__ constexpr bool sel_prefetch() {
  return (ESG_SEL_PREFETCH & (kLocal ? 1 : 2)) != 0;
}

// error bits in counters[2]
constexpr uint32_t kErrPanelWait = 1u;
constexpr uint32_t kErrRedoOverflow = 2u;

// query-state flags (device side, mirrored into esg_read_result.flags)
constexpr int kQRedo = 8;       // k2 flagged a pair; the query is re-scored by k3
constexpr int kQRescored = 4;   // == ESG_RESULT_RESCORED32

// ---------------------------------------------------------------- helpers
__device__ __forceinline__ uint32_t prmt(uint32_t a, uint32_t b, uint32_t sel) {
  uint32_t d;
  asm("prmt.b32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(sel));
  return d;
}
__device__ __forceinline__ void st_shared_u32(uint32_t addr, uint32_t v) {
  asm volatile("st.shared.u32 [%0], %1;" ::"r"(addr), "r"(v));
}
__device__ __forceinline__ uint32_t ld_shared_u32(uint32_t addr) {
  uint32_t v;
  asm volatile("ld.shared.u32 %0, [%1];" : "=r"(v) : "r"(addr));
  return v;
}
__device__ __forceinline__ uint32_t add16x2(uint32_t a, uint32_t b) {
  uint32_t d;
  asm("add.s16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
  return d;
}
// a * b + c as a 32-bit IMAD, which issues to the FMA pipe and so keeps the
// integer ALU free for the DPX ops
__device__ __forceinline__ uint32_t mad_lo(uint32_t a, uint32_t b, uint32_t c) {
  uint32_t d;
  asm("mad.lo.u32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
  return d;
}
__device__ __forceinline__ uint32_t max16x2(uint32_t a, uint32_t b) {
  uint32_t d;
  asm("max.s16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
  return d;
}
__device__ __forceinline__ int lo16(uint32_t v) { return (int)(int16_t)(v & 0xffffu); }
__device__ __forceinline__ int hi16(uint32_t v) { return ((int)v) >> 16; }
__host__ __device__ __forceinline__ uint32_t pack16x2(int lo, int hi) {
  return (uint32_t)(uint16_t)(int16_t)lo | ((uint32_t)(uint16_t)(int16_t)hi << 16);
}

// Online reduction of one query's candidates (mapper.rs:444-472): best, XS,
// n_tied counted in full, and the `cap` smallest tie candidates in order.
// Candidates may arrive in any order; the result does not depend on it.
// slot = {best, suboptimal, n_tied, flags}; ties = cap entries.
__device__ __forceinline__ void slot_add(int* slot, uint32_t* ties, uint32_t cap, uint32_t idx,
                                         int score) {
  const int best = slot[0];
  if (score > best) {
    if (slot[2] > 0) slot[1] = max(slot[1], best);
    slot[0] = score;
    slot[2] = 1;
    ties[0] = idx;
  } else if (score == best) {
    const uint32_t n = (uint32_t)slot[2];
    slot[2] = (int)(n + 1);
    const uint32_t listed = n < cap ? n : cap;
    if (listed < cap || idx < ties[cap - 1]) {
      uint32_t pos = listed < cap ? listed : cap - 1;
      while (pos > 0 && ties[pos - 1] > idx) {
        ties[pos] = ties[pos - 1];
        --pos;
      }
      ties[pos] = idx;
    }
  } else {
    slot[1] = max(slot[1], score);
  }
}

// ---------------------------------------------------------------- k2
struct K2Params {
  // panel blob: n_pairs uint4 {sel offset, mA | mB << 16, refA, refB} then the
  // 16-bit PRMT selectors of every pair's columns
  const uint4* blob;
  uint32_t blob_bytes;   // multiple of 16
  uint32_t n_pairs;
  uint32_t sel_base;     // uint16 index of the first selector in the blob
  // reads (codes 0..4); query q < n_reads is read q forward, else the
  // reverse complement of read q - n_reads
  const uint8_t* codes;
  const uint64_t* off;
  const uint32_t* len;
  uint32_t n_reads;
  // work tiles: tasks[t] = {start in order[], count | smax << 16}
  const uint32_t* order;
  const uint2* tasks;
  uint32_t n_tasks;
  uint32_t* counters;    // [1] redo count, [2] error bits (and the task counters)
  uint32_t* task_counter;  // this launch's task counter
  // outputs
  int4* qhead;           // per query {best, suboptimal, n_tied, flags}
  uint32_t* qties;       // per query cap candidates
  int32_t* rows;         // optional [q * n_refs + r]
  uint32_t n_refs;
  uint32_t* redo_list;   // k3 list; redo entries go after redo_base
  uint32_t redo_base;
  uint32_t redo_cap;
  // panel chunks: with n_chunks > 1 a task is (tile, chunk), the chunk's
  // reference pairs are chunk_lo[c] .. chunk_lo[c + 1], and each query's
  // partial state goes to part_head / part_ties [q * n_chunks + c] for
  // k2_merge_chunks; with n_chunks == 1 a task is a tile over every pair
  uint32_t n_chunks;
  const uint32_t* chunk_lo;
  int4* part_head;
  uint32_t* part_ties;
  // scoring, pre-shifted by the gap open (see k2_batched)
  uint32_t tab_a[6];
  uint32_t tab_b[6];
  uint32_t e2;           // e in both halves
  int32_t o, e;
  int32_t bias;          // value bias of the int16 lanes
  uint32_t one;          // the constant 1 (a multiplier the compiler cannot fold)
  uint2* lbuf;           // long queries: per-warp column buffer (G, F), lbuf_cols each
  uint32_t lbuf_cols;
  int32_t sat;           // local: a best (unbiased) at or above this may have wrapped
  uint32_t cap;
};

// Bounded wait on an mbarrier phase (a TMA bulk copy's completion).  Gives
// up after 2^26 polls, setting an error bit the host reads.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase, uint32_t* err) {
  const uint32_t addr = (uint32_t)__cvta_generic_to_shared(bar);
  // 2^26 polls; past them the thread that issued the copies (thread 0)
  // keeps polling up to 2^24 more so that its copies in flight land before
  // the CTA's shared memory is released
  const uint32_t limit = (1u << 26) + (threadIdx.x == 0 ? (1u << 24) : 0u);
  for (uint32_t it = 0; it < limit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(addr), "r"(phase)
        : "memory");
    if (done) {
      if (it < (1u << 26)) return true;
      break;  // landed only in thread 0's extra polls: still a timeout
    }
  }
  atomicOr(err, kErrPanelWait);
  return false;
}

// Stage the panel blob into shared memory with TMA bulk copies, each CTA
// its own: one thread arms an mbarrier with the byte count and issues
// cp.async.bulk in chunks; every thread waits on the phase.
__device__ __forceinline__ bool stage_panel(void* smem, const void* gsrc, uint32_t bytes,
                                            uint64_t* bar, uint32_t* err) {
  const uint32_t bar_a = (uint32_t)__cvta_generic_to_shared(bar);
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_a) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar_a), "r"(bytes)
                 : "memory");
    const uint32_t dst = (uint32_t)__cvta_generic_to_shared(smem);
    const char* src = (const char*)gsrc;
    constexpr uint32_t kChunk = 32768;
    for (uint32_t at = 0; at < bytes; at += kChunk) {
      const uint32_t n = (bytes - at) < kChunk ? (bytes - at) : kChunk;
      asm volatile(
          "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
              dst + at),
          "l"(src + at), "r"(n), "r"(bar_a)
          : "memory");
    }
  }
  const bool ok = mbar_wait(bar, 0, err);
  // One decision for the whole CTA: a thread that gave up and one that saw
  // the phase flip must not part ways (the survivors' warp-wide shuffles
  // would then run with exited lanes).
  return __syncthreads_and(ok) != 0;
}

// One systolic pass of a warp over the columns of one reference pair.
//
// Values are held biased: every H, E, F of the recurrence is stored as
// value + B (B = bias: +2048 in local mode, -16384 in semi-global), in signed
// 16-bit halves, two references per register (low half: the longer
// reference of the pair, high half: the shorter one).
//
// Lane state (rows r = 0..15 of the lane's stripe):
//   ta[r], tb[r]  PRMT tables of the row's read code c (or, with score
//                 records, the shared address of code c's word): byte x of {tb, ta} is
//                 s(c, x) - o for reference code x = 0..3, 4 (wildcard), and
//                 a padding column's score at x = 5.  Both halves use the
//                 same table; the column's selector picks a byte per half
//                 and sign-extends it to 16 bits.
//   g[r]          G = H + o + B of the row at the previous column
//   ev[r]         E + B of the row at the previous column
// Every integer ALU instruction (PRMT, the DPX VIADDMNMX / VIMNMX3, plain
// MAX) takes the same ALU issue slot, so the loop is written for the fewest
// of them: G feeds E of the next column and F of the next row (one
// VIADDMNMX each: max(X + e, G)); the diagonal term is G_diag + (s - o), which
// is why the tables hold s - o (one VIADDMNMX); H + B = max(h1, F, B) is one
// VIMNMX3 in local mode (B, the zero floor), one MAX in semi-global; the
// running best takes one VIMNMX3 per two rows.  G = H + B + o is a 32-bit
// IMAD (H * 1 + o * 65537, on the FMA pipe): exact in both halves because
// the low half's value is never in [0, |o|) -- local H + B >= B >= |o|,
// semi-global H + B < 0 -- so its borrow cancels the constant's, and the
// high half's carry-out is discarded.  Padding columns (garbage that may
// wrap) are only ever in the high half.  5.5 ALU instructions per cell pair
// in local mode, 5 in semi-global, plus one IMAD.
//
// Score records (kLds, local mode): the PRMT moves from every cell to every
// column.  At each column the lane writes the column's score word for each
// read code (PRMT of that code's tables, codes 0-3, and the wildcard code 4
// when the warp holds a wildcard row) to its own record in shared memory,
// then each row loads its code's word: ta[r] holds that word's shared
// address instead of a table.  The padding code's word is a constant written
// once per pass (local: -128 in both halves, H stays 0 under the floor).
// The record's words of one code are kK2Threads words apart, so every lane
// reads and writes its own bank.  4.5 ALU instructions per cell pair plus
// four PRMTs per column, one shared load per cell pair, one IMAD; the
// loads go to the otherwise idle load/store pipe (C2 local: +5 %).
//
// The lane with skew k works on column j = t - k at step t; its top input
// (G and F of the row above) is the previous lane's bottom output of step
// t-1, fetched by shuffle.  A query's first lane takes the border instead.
// In a long pass (kLong), lane 0 takes its top input from `buf` (the bottom
// row of the previous pass) when `from_buf`, and lane 31 writes its bottom
// row to `buf` when `to_buf`: lane 0 reads column j at step j, lane 31
// overwrites it at step j + 31, so one buffer serves every pass.
//
// Returns, per lane, the pass's local best (H + B) or semi-global last-column
// maximum (G, the short half's taken at its own end) in `v`, and the
// semi-global maximum of row 15 over the lane's columns (H + B) in `lr`.
struct PassConst {
  uint32_t g0, neg2, e2, o32, one, bias2;
};

// A column's 16-bit PRMT selector: an explicit shared-memory load when the
// panel is staged in shared memory, a read-only global load otherwise.
template <bool kSmem>
__device__ __forceinline__ uint32_t load_sel(const uint16_t* sp, int j) {
  if constexpr (kSmem) {
    uint16_t v;
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(sp + j);
    asm volatile("ld.shared.u16 %0, [%1];" : "=h"(v) : "r"(a));
    return v;
  } else {
    return __ldg(sp + j);
  }
}

template <int R, bool kLocal, bool kPanelW, bool kLong, bool kSmem, bool kCheck>
__device__ __forceinline__ void pair_pass(const K2Params& P, uint32_t scr, bool wild,
                                          const uint32_t (&ta)[R],
                                          const uint32_t (&tb)[kPanelW ? R : 1], int skew,
                                          bool active_lane, bool first, uint32_t padmask, int m,
                                          int jshort, const uint16_t* __restrict__ sp, int steps,
                                          const PassConst& K, uint2* buf, bool from_buf,
                                          bool to_buf, uint32_t& v, uint32_t& lr, uint32_t& am) {
  const int lane = threadIdx.x & 31;
  constexpr bool kLds = sc_lds<kLocal, R>() && !kLong;
  constexpr bool kPre = sel_prefetch<kLocal>();
  if constexpr (kLds) {
    // padding rows: local, -128 against every column (H stays 0 under the
    // floor); semi-global, s = 0 (H = 0 exactly against real columns; the
    // short half's columns past its end are never read)
    st_shared_u32(scr + 5 * kScrStride, kLocal ? 0xff80ff80u : pack16x2(-P.o, -P.o));
  }
  uint32_t g[R], ev[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    g[r] = K.g0;
    ev[r] = K.neg2;
  }
  uint32_t gdc = K.g0;  // G of the row above, previous column
  uint32_t gbot = K.g0, fbot = K.neg2;
  // local: max H + B over this lane's cells; checked semi-global: the same
  // without the floor (the short half's taken at its own end)
  uint32_t best = kLocal ? K.bias2 : K.neg2, s_best = K.neg2;
  uint32_t lastrow = K.neg2;               // semi-global: max H + B of row 15
  uint32_t s_col = K.neg2, s_last = K.neg2;  // semi-global short-half snapshot
  // inactive lanes of a tile sit at a skew no step reaches; only the long
  // path needs the per-lane bound (its lanes past the query's last stripe)
  const int mlim = (kLong && !active_lane) ? 0 : m;
  uint32_t seln = kPre ? load_sel<kSmem>(sp, 0) : 0u;

  // One column of the lane's stripe, given the top input (G, F of the row
  // above at this column).
  auto column = [&](int j, uint32_t gt, uint32_t ft) {
    if constexpr (kLong) {
      if (from_buf && lane == 0) {
        const uint2 b = buf[j];
        gt = b.x;
        ft = b.y;
      }
    }
    uint32_t sel;
    if constexpr (kPre) {
      // columns of a lane come in order: the next one's selector is loaded
      // a column ahead (the blob holds one spare selector past the last pair)
      sel = seln;
      seln = load_sel<kSmem>(sp, j + 1);
    } else {
      sel = load_sel<kSmem>(sp, j);
    }
    if constexpr (kLds) {
      // the column's score record: one word per read code, in this thread's
      // own bank, read back per row below (wildcard rows only when the warp
      // has some)
#pragma unroll
      for (int c = 0; c < 4; ++c) st_shared_u32(scr + c * kScrStride, prmt(P.tab_a[c], P.tab_b[c], sel));
      if (wild) st_shared_u32(scr + 4 * kScrStride, prmt(P.tab_a[4], P.tab_b[4], sel));
    }
    uint32_t gd = gdc;
    gdc = gt;
    uint32_t gup = gt, f = ft, h15 = 0, hprev = 0;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      uint32_t sc;
      if constexpr (kLds)
        sc = ld_shared_u32(ta[r]);
      else
        sc = prmt(ta[r], tb[kPanelW ? r : 0], sel);
      ev[r] = __viaddmax_s16x2(ev[r], K.e2, g[r]);
      f = __viaddmax_s16x2(f, K.e2, gup);
      const uint32_t h1 = __viaddmax_s16x2(gd, sc, ev[r]);
      uint32_t h;
      if constexpr (kLocal) {
        h = __vimax3_s16x2(h1, f, K.bias2);
        if (r & 1)
          best = __vimax3_s16x2(best, hprev, h);
        else
          hprev = h;
      } else {
        h = max16x2(h1, f);
        if constexpr (kCheck) {
          if (r & 1)
            best = __vimax3_s16x2(best, hprev, h);
          else
            hprev = h;
        }
      }
      gd = g[r];
      g[r] = mad_lo(h, K.one, K.o32);
      gup = g[r];
      if (r == R - 1) h15 = h;
    }
    gbot = g[R - 1];
    fbot = f;
    if constexpr (kLong) {
      if (to_buf && lane == 31) buf[j] = make_uint2(gbot, fbot);
    }
    if constexpr (!kLocal) {
      lastrow = max16x2(lastrow, h15);
      if (j == jshort) {
        // the short half's last column, padding rows left out.  Padding
        // rows hold G = o + B exactly (H = 0), so a maximum above that is a
        // read row's and the unmasked maximum stands; only a maximum equal
        // to it takes the masked one.  (Masking every time kept the pad
        // mask's selects live across the column loop: 40-52 bytes of spill
        // in the 32-row kernel.)
        uint32_t cm = K.neg2;
#pragma unroll
        for (int r = 0; r < R; ++r) cm = max16x2(cm, g[r]);
        if (padmask && (cm >> 16) == (K.g0 >> 16)) {
          cm = K.neg2;
#pragma unroll
          for (int r = 0; r < R; ++r) cm = max16x2(cm, ((padmask >> r) & 1u) ? K.neg2 : g[r]);
        }
        s_col = cm;
        s_last = lastrow;
        if constexpr (kCheck) s_best = best;
      }
    }
  };
  // The top input: the previous lane's bottom row of the previous step, or
  // the border for a query's first lane.
  auto top = [&](uint32_t& gt, uint32_t& ft) {
    gt = __shfl_up_sync(kFull, gbot, 1);
    ft = __shfl_up_sync(kFull, fbot, 1);
    if (first) {
      gt = K.g0;
      ft = K.neg2;
    }
  };

  int t = 0;
  // (local mode only: semi-global measured slower with a second copy of the
  // column body, whose last-row and short-reference state cost it registers:
  // again at 4 CTAs and 128 registers, -0.7 % to -1.6 % for unrolls 1-8 on
  // C2 semi-global, its 32-row stripes spilling more; and once the snapshot
  // stopped spilling, on 32-row stripes alone, -2.0 % on C4 pairs)
  if constexpr (kLocal && !kLong) {
    // Steps fill .. m - 1, where fill = steps - m is the tile's largest skew,
    // have every lane of the tile's queries inside the pair's columns: they
    // run without the column check.  Lanes past the tile's queries take
    // skew 0 there (columns in range, values nobody reads: only later lanes,
    // also past the queries, see them, and a pass's results are taken from
    // the queries' own lanes).
    const int fill = steps - m;
    if (fill < m) {
#pragma unroll 1
      for (; t < fill; ++t) {
        uint32_t gt, ft;
        top(gt, ft);
        const int j = t - skew;
        if ((unsigned)j < (unsigned)mlim) column(j, gt, ft);
      }
      const int sk = active_lane ? skew : 0;
      // unrolled (ESG_STEADY_UNROLL, ESG_STEADY_UNROLL32); 32-row stripes
      // with the panel in shared memory have no registers to spare
      constexpr int kUnroll = R <= 16 ? ESG_STEADY_UNROLL : (kSmem ? 1 : ESG_STEADY_UNROLL32);
#pragma unroll kUnroll
      for (; t < m; ++t) {
        uint32_t gt, ft;
        top(gt, ft);
        column(t - sk, gt, ft);
      }
    }
  }
#pragma unroll 1
  for (; t < steps; ++t) {
    uint32_t gt, ft;
    top(gt, ft);
    const int j = t - skew;
    if ((unsigned)j < (unsigned)mlim) column(j, gt, ft);
  }
  am = K.neg2;
  if constexpr (kLocal) {
    v = best;
    lr = 0;
  } else {
    if constexpr (kCheck)
      am = active_lane ? (jshort >= 0 ? (best & 0xffffu) | (s_best & 0xffff0000u) : best) : K.neg2;
    uint32_t cm = K.neg2;
#pragma unroll
    for (int r = 0; r < R; ++r) cm = max16x2(cm, ((padmask >> r) & 1u) ? K.neg2 : g[r]);
    if (jshort >= 0) {
      // the short (high) half's last column and last row, taken at its end
      cm = (cm & 0xffffu) | (s_col & 0xffff0000u);
      lastrow = (lastrow & 0xffffu) | (s_last & 0xffff0000u);
    }
    v = active_lane ? cm : K.neg2;
    lr = lastrow;
  }
}

// Row tables of stripe `s` of a query (n codes at q, reverse complement if
// rc): row r is read row i = 16 s + r - pad; rows before the read are padding.
template <int R, bool kPanelW, bool kLds>
__device__ __forceinline__ bool row_tables(const K2Params& P, const uint8_t* q, uint32_t n,
                                           bool rc, bool valid, int s, int pad,
                                           uint32_t (&ta)[R],
                                           uint32_t (&tb)[kPanelW ? R : 1], uint32_t scr = 0) {
  bool wild = false;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int i = s * R + r - pad;
    uint32_t c = 5;  // padding row
    if (valid && i >= 0) {
      uint32_t x = rc ? q[n - 1 - i] : q[i];
      x = x > 4 ? 4 : x;
      c = (rc && x < 4) ? 3 - x : x;
    }
    wild |= c == 4;
    if constexpr (kLds) {
      ta[r] = scr + c * kScrStride;  // the row code's word in the column record
    } else {
      ta[r] = P.tab_a[c];
      if constexpr (kPanelW) tb[r] = P.tab_b[c];
    }
  }
  if constexpr (!kPanelW) tb[0] = P.tab_b[0];
  return __any_sync(kFull, wild);
}

// The last lane of a query folds one reference pair's two scores into the
// query's slot (and its rows, when asked for).  A pair that may have left
// the int16 lanes flags its query for the int32 re-score: in local mode a
// best at or above P.sat; in checked semi-global mode any cell with
// H + B >= 0 (H >= 16384), where G's IMAD may borrow wrongly (see
// pair_pass) -- the first such cell is itself exact, its inputs being below
// the mark, so the maximum over every cell, `am`, catches it.
template <bool kLocal, bool kCheck>
__device__ __forceinline__ void fold_pair(const K2Params& P, int* slot, uint32_t* sties,
                                          uint32_t cap, uint4 pm, int mB, bool rc, uint32_t qid,
                                          uint32_t v, uint32_t lr, uint32_t am, int bias) {
  int scA, scB;
  if constexpr (kLocal) {
    scA = lo16(v) - bias;
    scB = hi16(v) - bias;
    if (scA >= P.sat || (mB > 0 && scB >= P.sat)) slot[3] |= kQRedo;
  } else {
    scA = max(lo16(v) - P.o, lo16(lr)) - bias;
    scB = max(hi16(v) - P.o, hi16(lr)) - bias;
    if constexpr (kCheck)
      if (lo16(am) >= 0 || (mB > 0 && hi16(am) >= 0)) slot[3] |= kQRedo;
  }
  const uint32_t rbit = rc ? 1u : 0u;
  slot_add(slot, sties, cap, (pm.z << 1) | rbit, scA);
  if (P.rows) P.rows[(size_t)qid * P.n_refs + pm.z] = scA;
  if (pm.w != kNoRef) {
    slot_add(slot, sties, cap, (pm.w << 1) | rbit, scB);
    if (P.rows) P.rows[(size_t)qid * P.n_refs + pm.w] = scB;
  }
}

// A query's state at the end of a task: its final state (and a re-score
// request if it may have wrapped), or with panel chunks its partial state
// for k2_merge_chunks.
__device__ __forceinline__ void flush_query(const K2Params& P, uint32_t qid, uint32_t chunk,
                                            const int* slot, const uint32_t* sties,
                                            uint32_t cap) {
  const int fl = slot[3];
  const uint32_t nl = min((uint32_t)slot[2], cap);
  if (P.n_chunks > 1) {
    const size_t at = (size_t)qid * P.n_chunks + chunk;
    P.part_head[at] = make_int4(slot[0], slot[1], slot[2], fl);
    for (uint32_t k = 0; k < nl; ++k) P.part_ties[at * cap + k] = sties[k];
    return;
  }
  P.qhead[qid] = make_int4(slot[0], slot[1], slot[2], fl);
  for (uint32_t k = 0; k < nl; ++k) P.qties[(size_t)qid * cap + k] = sties[k];
  if (fl & kQRedo) {
    const uint32_t at = atomicAdd(&P.counters[1], 1u);
    if (at < P.redo_cap)
      P.redo_list[P.redo_base + at] = qid;
    else
      atomicOr(&P.counters[2], kErrRedoOverflow);
  }
}

// One warp, one task at a time, tasks pulled from an atomic counter.  The
// kernel is instantiated twice: kLong = false takes tiles of up to 32
// queries whose stripes fill the warp's lanes (a query of n rows takes
// S = ceil(n / 16) lanes), scored in one pass per reference pair; kLong =
// true takes one long query (S > 32) per task, scored in ceil(S / 32) passes
// per pair chained through a per-warp column buffer in global memory.  Two
// instantiations keep the register allocation of the short-read path free of
// the long path's state; the host runs them concurrently.
// Stripes are aligned so the read's last row is row 15 of its last stripe;
// the 16 S - n rows before the read's first row score 0 against every real
// column and hold H = 0 exactly, the top border the first real row needs.
template <int R, bool kLocal, bool kPanelW, bool kSmemPanel, bool kLong, bool kCheck>
__global__ void __launch_bounds__(kK2Threads, R > 16 ? ESG_K2_R32_BLOCKS : (kPanelW ? 4 : ESG_K2_MIN_BLOCKS))
    k2_batched(const K2Params P) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ uint64_t panel_bar;
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const uint32_t cap = P.cap;

  const uint4* pairs;
  const uint16_t* sels;
  int* slots;
  if constexpr (kSmemPanel) {
    if (!stage_panel(smem_raw, P.blob, P.blob_bytes, &panel_bar, &P.counters[2])) return;
    pairs = reinterpret_cast<const uint4*>(smem_raw);
    sels = reinterpret_cast<const uint16_t*>(smem_raw) + P.sel_base;
    slots = reinterpret_cast<int*>(smem_raw + P.blob_bytes);
  } else {
    pairs = P.blob;
    sels = reinterpret_cast<const uint16_t*>(P.blob) + P.sel_base;
    slots = reinterpret_cast<int*>(smem_raw);
  }
  // this lane's query slot: {best, suboptimal, n_tied, flags, ties[cap]}
  int* slot = slots + (size_t)(wib * 32 + lane) * (4 + cap);
  uint32_t* sties = reinterpret_cast<uint32_t*>(slot + 4);
  // column score records: word c * kK2Threads + thread (bank = lane)
  const uint32_t scr = (uint32_t)__cvta_generic_to_shared(slots + (size_t)kK2Threads * (4 + cap)) +
                       threadIdx.x * 4u;
  uint2* lbuf = P.lbuf ? P.lbuf + ((size_t)blockIdx.x * kK2Warps + wib) * P.lbuf_cols : nullptr;

  const int bias = P.bias;
  PassConst K;
  K.g0 = pack16x2(bias + P.o, bias + P.o);  // G of a zero border cell
  K.bias2 = pack16x2(bias, bias);           // H = 0 (the local floor)
  K.o32 = (uint32_t)(P.o * 65537);           // + o in both halves, one 32-bit add
  K.e2 = P.e2;
  K.one = P.one;  // 1, opaque to the compiler: keeps G's add an IMAD
  K.neg2 = pack16x2(kNeg16, kNeg16);

  for (;;) {
    uint32_t task = 0;
    if (lane == 0) task = atomicAdd(P.task_counter, 1u);
    task = __shfl_sync(kFull, task, 0);
    if (task >= P.n_tasks) break;
    const uint32_t tile = P.n_chunks > 1 ? task / P.n_chunks : task;
    const uint32_t chunk = task - tile * P.n_chunks;
    const uint32_t p_lo = P.n_chunks > 1 ? P.chunk_lo[chunk] : 0u;
    const uint32_t p_hi = P.n_chunks > 1 ? P.chunk_lo[chunk + 1] : P.n_pairs;
    const uint2 tk = P.tasks[tile];
    const uint32_t count = tk.y & 0xffffu;
    const int smax = (int)(tk.y >> 16);

    if constexpr (kLong) {
      // ---------------- one long query, ceil(S / 32) passes per pair
      const uint32_t qid = P.order[tk.x];
      const bool rc = qid >= P.n_reads;
      const uint32_t rd = rc ? qid - P.n_reads : qid;
      const uint32_t n = P.len[rd];
      const int S = smax;
      const int pad = S * R - (int)n;
      const int passes = (S + 31) / 32;
      const int owner = (S - 1) & 31;  // lane holding the last stripe
      const uint8_t* q = P.codes + P.off[rd];
      if (lane == owner) {
        slot[0] = INT32_MIN;
        slot[1] = INT32_MIN;
        slot[2] = 0;
        slot[3] = 0;
      }
      for (uint32_t p = p_lo; p < p_hi; ++p) {
        const uint4 pm = pairs[p];
        const int mA = (int)(pm.y & 0xffffu), mB = (int)(pm.y >> 16);  // mA >= mB
        const int jshort = (mB > 0 && mB < mA) ? mB - 1 : -1;
        const uint16_t* sp = sels + pm.x;
        uint32_t acc = kLocal ? K.bias2 : K.neg2, lr_last = K.neg2, amacc = K.neg2;
        for (int pass = 0; pass < passes; ++pass) {
          const int s = pass * 32 + lane;
          const bool valid = s < S;
          uint32_t ta[R];
          uint32_t tb[kPanelW ? R : 1];
          row_tables<R, kPanelW, false>(P, q, n, rc, valid, s, pad, ta, tb);
          const uint32_t padmask = (s == 0) ? ((1u << pad) - 1u) : 0u;
          uint32_t v, lr, am;
          pair_pass<R, kLocal, kPanelW, true, kSmemPanel, kCheck>(
              P, 0u, false, ta, tb, lane, valid, s == 0, padmask, mA, jshort, sp, mA + 31, K,
              lbuf, pass > 0, pass + 1 < passes, v, lr, am);
          acc = max16x2(acc, v);
          if constexpr (kCheck) amacc = max16x2(amacc, am);
          if (pass + 1 == passes) lr_last = lr;
          __syncwarp();  // the buffer's writes are visible to the next pass
        }
#pragma unroll
        for (int d = 16; d; d >>= 1) acc = max16x2(acc, __shfl_xor_sync(kFull, acc, d));
        if constexpr (kCheck) {
#pragma unroll
          for (int d = 16; d; d >>= 1) amacc = max16x2(amacc, __shfl_xor_sync(kFull, amacc, d));
        }
        if (lane == owner)
          fold_pair<kLocal, kCheck>(P, slot, sties, cap, pm, mB, rc, qid, acc, lr_last, amacc,
                                    bias);
      }
      if (lane == owner) flush_query(P, qid, chunk, slot, sties, cap);
      __syncwarp();
      continue;
    } else {
    // ---------------- up to 32 queries, one pass per pair
    uint32_t kq = 0, kn = 0, kS = 0;
    if ((uint32_t)lane < count) {
      kq = P.order[tk.x + lane];
      const uint32_t rd = kq < P.n_reads ? kq : kq - P.n_reads;
      kn = P.len[rd];
      kS = (kn + R - 1) / R;
    }
    uint32_t incl = kS;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t v = __shfl_up_sync(kFull, incl, d);
      if (lane >= d) incl += v;
    }
    uint32_t qid = 0, n = 0;
    int s = 1 << 20, S = 0;  // lanes past the task's queries never become active
    bool valid = false;
    for (uint32_t k = 0; k < count; ++k) {
      const uint32_t ek = __shfl_sync(kFull, incl, k);
      const uint32_t sk = __shfl_sync(kFull, kS, k);
      const uint32_t qk = __shfl_sync(kFull, kq, k);
      const uint32_t nk = __shfl_sync(kFull, kn, k);
      if ((uint32_t)lane >= ek - sk && (uint32_t)lane < ek) {
        qid = qk;
        n = nk;
        s = lane - (int)(ek - sk);
        S = (int)sk;
        valid = true;
      }
    }
    const bool first = valid ? (s == 0) : true;
    const bool last = valid && (s == S - 1);
    const int pad = valid ? S * R - (int)n : 0;
    const bool rc = qid >= P.n_reads;
    const uint32_t rd = rc ? qid - P.n_reads : qid;

    uint32_t ta[R];
    uint32_t tb[kPanelW ? R : 1];
    const bool wild = row_tables<R, kPanelW, sc_lds<kLocal, R>()>(
        P, valid ? P.codes + P.off[rd] : P.codes, n, rc, valid, s, pad, ta, tb, scr);
    // rows of the read's top padding (first lane only): excluded from the
    // semi-global last-column maximum
    const uint32_t padmask = (valid && first) ? ((1u << pad) - 1u) : 0u;

    if (last) {
      slot[0] = INT32_MIN;
      slot[1] = INT32_MIN;
      slot[2] = 0;
      slot[3] = 0;
    }

    for (uint32_t p = p_lo; p < p_hi; ++p) {
      const uint4 pm = pairs[p];
      const int mA = (int)(pm.y & 0xffffu), mB = (int)(pm.y >> 16);  // mA >= mB
      const int jshort = (mB > 0 && mB < mA) ? mB - 1 : -1;
      uint32_t v, lr, am;
      pair_pass<R, kLocal, kPanelW, false, kSmemPanel, kCheck>(
          P, scr, wild, ta, tb, s, valid, first, padmask, mA, jshort, sels + pm.x, mA + smax - 1,
          K, nullptr, false, false, v, lr, am);
      // per-query maximum, to the query's last lane
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const uint32_t w = __shfl_up_sync(kFull, v, d);
        if (s >= d) v = max16x2(v, w);
        if constexpr (kCheck) {
          const uint32_t wa = __shfl_up_sync(kFull, am, d);
          if (s >= d) am = max16x2(am, wa);
        }
      }
      if (last) fold_pair<kLocal, kCheck>(P, slot, sties, cap, pm, mB, rc, qid, v, lr, am, bias);
    }

    // --- flush the query states of this task
    if (last) flush_query(P, qid, chunk, slot, sties, cap);
    __syncwarp();
    }
  }
}

// ---------------------------------------------------------------- chunk merge
// Two query states over disjoint candidate sets, each with its first
// min(n_tied, cap) ties in candidate order, into one (mapper.rs:444-472
// over the union): the higher best wins, equal bests add their tie counts
// and merge their lists in candidate order.  `out` must not alias ta / tb.
__device__ __forceinline__ int4 merge_state(int4 a, const uint32_t* ta, int4 b,
                                            const uint32_t* tb, uint32_t cap, uint32_t* out) {
  const uint32_t na = min((uint32_t)a.z, cap), nb = min((uint32_t)b.z, cap);
  if (a.x > b.x) {
    for (uint32_t k = 0; k < na; ++k) out[k] = ta[k];
    return make_int4(a.x, max(max(a.y, b.y), b.x), a.z, a.w | b.w);
  }
  if (b.x > a.x) {
    for (uint32_t k = 0; k < nb; ++k) out[k] = tb[k];
    return make_int4(b.x, max(max(a.y, b.y), a.x), b.z, a.w | b.w);
  }
  uint32_t i = 0, j = 0, w = 0;
  while (w < cap && (i < na || j < nb)) {
    if (j >= nb || (i < na && ta[i] < tb[j]))
      out[w++] = ta[i++];
    else
      out[w++] = tb[j++];
  }
  return make_int4(a.x, max(a.y, b.y), a.z + b.z, a.w | b.w);
}

struct KMParams {
  const uint32_t* order;   // the queries k2 scored
  uint32_t n_order;
  uint32_t n_chunks;
  const int4* part_head;   // [q * n_chunks + c]
  const uint32_t* part_ties;
  int4* qhead;
  uint32_t* qties;
  uint32_t cap;
  uint32_t* counters;      // [1] redo count, [2] error bits
  uint32_t* redo_list;
  uint32_t redo_base;
  uint32_t redo_cap;
};

// One thread per query: its panel chunks' partial states merged in chunk
// order, and a re-score request where any chunk may have wrapped.
static __global__ void __launch_bounds__(128) k2_merge_chunks(const KMParams P) {
  uint32_t buf[2][kMaxCap];
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < P.n_order;
       i += gridDim.x * blockDim.x) {
    const uint32_t q = P.order[i];
    const size_t base = (size_t)q * P.n_chunks;
    const uint32_t cap = P.cap;
    int4 acc = P.part_head[base];
    const uint32_t n0 = min((uint32_t)acc.z, cap);
    for (uint32_t k = 0; k < n0; ++k) buf[0][k] = P.part_ties[base * cap + k];
    int cur = 0;
    for (uint32_t c = 1; c < P.n_chunks; ++c) {
      const int4 b = P.part_head[base + c];
      acc = merge_state(acc, buf[cur], b, P.part_ties + (base + c) * cap, cap, buf[cur ^ 1]);
      cur ^= 1;
    }
    P.qhead[q] = acc;
    const uint32_t nl = min((uint32_t)acc.z, cap);
    for (uint32_t k = 0; k < nl; ++k) P.qties[(size_t)q * cap + k] = buf[cur][k];
    if (acc.w & kQRedo) {
      const uint32_t at = atomicAdd(&P.counters[1], 1u);
      if (at < P.redo_cap)
        P.redo_list[P.redo_base + at] = q;
      else
        atomicOr(&P.counters[2], kErrRedoOverflow);
    }
  }
}

// ---------------------------------------------------------------- k3
// k3_lanes: the exact int32 path.  It scores a list of queries against every
// reference of the panel and writes the rows (k4 reduces them).  The work
// unit is (query, a run of references); one warp takes one unit at a time.
//
// Lanes hold 16-row stripes of the query.  A query of S stripes is scored
// against a reference by a chain of W = min(S, wmax) lanes: the lane at
// position w of the chain holds stripes w, W + w, 2W + w, ... in successive
// passes, walks the reference's columns one per step, lagging the lane
// before it by one step, and takes its top input (G and F of the row above)
// from that lane by shuffle.  The chain's first lane takes the zero border
// in the first pass and, in later passes, the bottom row the chain's last
// lane left in the warp's column buffer (global memory) in the pass before.
// A warp runs 32 / W chains side by side, one reference each, so short
// queries fill the warp with references instead of idle lanes.  wmax = 32 is
// the product setting; wmax = 1 makes every lane a chain of its own -- one
// thread per (query, reference) pair, the stripes' bottom row through the
// buffer -- the plain comparison arm.
//
// Per cell: G = H + o is kept instead of H, so E, F and the diagonal term
// are one VIADDMNMX each (max(X + e, G) and max(G_diag + (s - o), E)), H one
// VIMNMX3 (with the zero floor in local mode), G one IMAD on the FMA pipe;
// the substitution s - o comes from the lane's per-column record in shared
// memory (word c = the score of read code c against this column, one
// 16-byte table load and four stores per column), one load per cell.  The
// query is padded at the top to whole stripes with rows that score 0, which
// hold H = 0 exactly -- the top border -- and are left out of the
// semi-global last-column maximum.
constexpr int kK3Rows = 16;
constexpr int kK3Warps = 4;
constexpr int kK3Threads = kK3Warps * 32;
constexpr uint32_t kK3Stride = (uint32_t)kK3Threads * 4;  // bytes between record words

struct K3Params {
  // queries: list entry p is query list[p] (q < n_reads: read q forward,
  // else the reverse complement of read q - n_reads); without a list, entry
  // p is read p forward
  const uint8_t* codes;
  const uint64_t* off;
  const uint32_t* len;
  uint32_t n_reads;
  const uint32_t* list;
  uint32_t host_count;         // entries listed by the host
  const uint32_t* redo_count;  // device count of entries after them (may be null)
  uint32_t redo_cap;           // capacity after host_count
  // references: slot k is panel reference ridx[k] (identity without ridx)
  const uint8_t* rcodes;
  const uint32_t* roff;
  const uint32_t* rlen;
  const uint32_t* ridx;
  uint32_t n_refs;
  uint32_t max_cols;           // longer references score kNoScore (no room in colbuf)
  int32_t* out;                // [p * n_refs + ref] (may be null)
  int32_t* rows;               // [q * n_refs + ref] (may be null)
  uint32_t wmax;               // lanes per chain at most: 32, or 1 (one thread per pair)
  uint32_t refs_per_task;
  unsigned long long* task_counter;  // null: units taken warp-strided
  int2* colbuf;                // per warp (32 / wmax) * max_cols int2
  int32_t ma, mi, o, e;
  int32_t one;                 // 1, opaque to the compiler (keeps G's add an IMAD)
};

constexpr int32_t kNoScore = INT32_MIN;

template <bool kLocal>
__global__ void __launch_bounds__(kK3Threads, 4) k3_lanes(const K3Params P) {
  constexpr int R = kK3Rows;
  __shared__ int4 tab[5];                      // words of read codes 0-3 against reference code x
  __shared__ uint32_t rec[6 * kK3Threads];     // word c of thread t at c * kK3Threads + t
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const int o = P.o, e = P.e;
  const int mao = P.ma - o, mio = P.mi - o;
  if (threadIdx.x < 5) {
    const int x = threadIdx.x;  // 4: a wildcard reference base matches every read code
    tab[x] = make_int4((x == 0 || x == 4) ? mao : mio, (x == 1 || x == 4) ? mao : mio,
                       (x == 2 || x == 4) ? mao : mio, (x == 3 || x == 4) ? mao : mio);
  }
  const uint32_t my = (uint32_t)__cvta_generic_to_shared(rec) + threadIdx.x * 4u;
  st_shared_u32(my + 4 * kK3Stride, (uint32_t)mao);  // read wildcard: a match everywhere
  st_shared_u32(my + 5 * kK3Stride, (uint32_t)-o);   // padding row: s = 0
  __syncthreads();

  const uint32_t n_list =
      P.host_count + (P.redo_count ? min(*P.redo_count, P.redo_cap) : 0u);
  const uint32_t tpq = (P.n_refs + P.refs_per_task - 1) / P.refs_per_task;
  const unsigned long long n_units = (unsigned long long)n_list * tpq;
  const size_t warp_id = (size_t)blockIdx.x * kK3Warps + wib;
  const size_t n_warps = (size_t)gridDim.x * kK3Warps;
  const int cmax = 32 / (int)P.wmax;
  int2* const buf = P.colbuf ? P.colbuf + warp_id * (size_t)cmax * P.max_cols : nullptr;

  unsigned long long unit = warp_id;
  for (;; unit += P.task_counter ? 0ull : n_warps) {
    if (P.task_counter) {
      unsigned long long u = 0;
      if (lane == 0) u = atomicAdd(P.task_counter, 1ull);
      unit = __shfl_sync(kFull, u, 0);
    }
    if (unit >= n_units) break;
    const uint32_t pos = (uint32_t)(unit / tpq);
    const uint32_t u = (uint32_t)(unit - (unsigned long long)pos * tpq);
    const uint32_t q = P.list ? P.list[pos] : pos;
    const bool rc = q >= P.n_reads;
    const uint32_t rd = rc ? q - P.n_reads : q;
    const int n = (int)P.len[rd];
    const uint8_t* qc = P.codes + P.off[rd];

    const int S = n > 0 ? (n + R - 1) / R : 1;
    const int W = min(S, (int)P.wmax);
    const int C = 32 / W;                // chains in the warp
    const int passes = (S + W - 1) / W;
    const int c = lane / W, w = lane - c * W;
    const int pad = S * R - n;
    // this unit's references: its share of the query's groups of C (whole
    // groups, so only the query's very last group can be short)
    const uint32_t groups = (P.n_refs + (uint32_t)C - 1) / (uint32_t)C;
    const uint32_t k_lo = (uint32_t)((uint64_t)u * groups / tpq) * (uint32_t)C;
    const uint32_t k_hi = min((uint32_t)((uint64_t)(u + 1) * groups / tpq) * (uint32_t)C, P.n_refs);

    for (uint32_t k0 = k_lo; k0 < k_hi; k0 += (uint32_t)C) {
      const uint32_t k = k0 + (uint32_t)c;
      const bool has = c < C && k < k_hi;
      const uint32_t mref = has ? P.rlen[k] : 0u;
      // (a reference longer than the column buffer's rows, or a query that
      // needs passes without a buffer, is not scored)
      const bool fits = mref <= P.max_cols && (passes == 1 || buf != nullptr);
      const int m = (fits && n > 0) ? (int)mref : 0;
      const int M = (int)__reduce_max_sync(kFull, (unsigned)m);
      const uint8_t* rcs = has ? P.rcodes + P.roff[k] : P.rcodes;
      // local: the best H over the chain's cells; semi-global: the best of
      // the last column and (on the lane of the last stripe) the last row
      int acc = kLocal ? 0 : kNeg32;
      for (int pass = 0; pass < passes; ++pass) {
        const int s = pass * W + w;
        const bool valid = m > 0 && s < S;
        uint32_t addr[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int i = s * R + r - pad;
          uint32_t code = 5;  // padding row
          if (valid && i >= 0) {
            uint32_t x = rc ? qc[n - 1 - i] : qc[i];
            x = x > 4 ? 4 : x;
            code = (rc && x < 4) ? 3 - x : x;
          }
          addr[r] = my + code * kK3Stride;
        }
        const uint32_t padmask = (valid && s == 0) ? ((1u << pad) - 1u) : 0u;
        const bool from_buf = pass > 0 && w == 0;
        const bool to_buf = pass + 1 < passes && w == W - 1;
        int g[R], ev[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
          g[r] = o;  // G of a zero border cell
          ev[r] = kNeg32;
        }
        int gdc = o, gbot = o, fbot = kNeg32;
        int best = kLocal ? 0 : kNeg32;
        int lastrow = kNeg32, lastcol = kNeg32;
        const int steps = M + W - 1;
#pragma unroll 1
        for (int t = 0; t < steps; ++t) {
          int gt = __shfl_up_sync(kFull, gbot, 1);
          int ft = __shfl_up_sync(kFull, fbot, 1);
          if (w == 0) {
            gt = o;
            ft = kNeg32;
          }
          const int j = t - w;
          if (valid && (unsigned)j < (unsigned)m) {
            if (from_buf) {
              const int2 b = buf[(size_t)j * C + c];
              gt = b.x;
              ft = b.y;
            }
            // this column's record: the score (s - o) of read codes 0-3
            const int x = min((int)rcs[j], 4);
            const int4 tw = tab[x];
            st_shared_u32(my, (uint32_t)tw.x);
            st_shared_u32(my + kK3Stride, (uint32_t)tw.y);
            st_shared_u32(my + 2 * kK3Stride, (uint32_t)tw.z);
            st_shared_u32(my + 3 * kK3Stride, (uint32_t)tw.w);
            int gd = gdc;
            gdc = gt;
            int gup = gt, f = ft, hprev = 0, hlast = 0;
#pragma unroll
            for (int r = 0; r < R; ++r) {
              const int sc = (int)ld_shared_u32(addr[r]);
              ev[r] = __viaddmax_s32(ev[r], e, g[r]);
              f = __viaddmax_s32(f, e, gup);
              const int h1 = __viaddmax_s32(gd, sc, ev[r]);
              int h;
              if constexpr (kLocal) {
                h = __vimax3_s32(h1, f, 0);
                if (r & 1)
                  best = __vimax3_s32(best, hprev, h);
                else
                  hprev = h;
              } else {
                h = max(h1, f);
              }
              gd = g[r];
              g[r] = (int)mad_lo((uint32_t)h, (uint32_t)P.one, (uint32_t)o);
              gup = g[r];
              if (r == R - 1) hlast = h;
            }
            gbot = g[R - 1];
            fbot = f;
            if (to_buf) buf[(size_t)j * C + c] = make_int2(gbot, fbot);
            if constexpr (!kLocal) {
              lastrow = max(lastrow, hlast);
              if (j == m - 1) {
                int cm = kNeg32;
#pragma unroll
                for (int r = 0; r < R; ++r) cm = max(cm, ((padmask >> r) & 1u) ? kNeg32 : g[r]);
                lastcol = cm - o;
              }
            }
          }
        }
        __syncwarp();  // the buffer's writes are seen by the next pass
        if constexpr (kLocal) {
          acc = max(acc, best);
        } else {
          acc = max(acc, lastcol);
          if (valid && s == S - 1) acc = max(acc, lastrow);
        }
      }
      // the chain's maximum, to its first lane
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const int v = __shfl_down_sync(kFull, acc, d);
        if (w + d < W) acc = max(acc, v);
      }
      if (has && w == 0) {
        // scalar.rs:123-125: an empty query or reference scores 0
        const int score = !fits ? kNoScore : (m == 0 ? 0 : acc);
        const uint32_t ref = P.ridx ? P.ridx[k] : k;
        if (P.out) P.out[(size_t)pos * P.n_refs + ref] = score;
        if (P.rows) P.rows[(size_t)q * P.n_refs + ref] = score;
      }
    }
  }
}

// ---------------------------------------------------------------- k4
struct K4Params {
  const uint32_t* list;
  uint32_t host_count;
  const uint32_t* redo_count;
  uint32_t redo_cap;
  const int32_t* rows;  // k3 output, [pos * n_refs + r]
  uint32_t n_refs;
  uint32_t n_reads;
  int4* qhead;
  uint32_t* qties;
  uint32_t cap;
};

// One warp per listed query: mapper.rs:444-472 over its row.
static __global__ void __launch_bounds__(256) k4_rows(const K4Params P) {
  const uint32_t n_list = P.host_count + (P.redo_count ? min(*P.redo_count, P.redo_cap) : 0u);
  const int lane = threadIdx.x & 31;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t pos = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; pos < n_list; pos += warps) {
    const uint32_t q = P.list[pos];
    const uint32_t rbit = q >= P.n_reads ? 1u : 0u;
    const int32_t* row = P.rows + (size_t)pos * P.n_refs;
    int best = INT32_MIN;
    for (uint32_t r = lane; r < P.n_refs; r += 32) best = max(best, row[r]);
#pragma unroll
    for (int d = 16; d; d >>= 1) best = max(best, __shfl_xor_sync(kFull, best, d));
    int sub = INT32_MIN;
    uint32_t n_tied = 0, listed = 0;
    for (uint32_t base = 0; base < P.n_refs; base += 32) {
      const uint32_t r = base + lane;
      const int v = r < P.n_refs ? row[r] : INT32_MIN;
      const bool tie = r < P.n_refs && v == best;
      if (r < P.n_refs && !tie) sub = max(sub, v);
      const uint32_t bal = __ballot_sync(kFull, tie);
      if (tie) {
        const uint32_t rank = listed + __popc(bal & ((1u << lane) - 1u));
        if (rank < P.cap) P.qties[(size_t)q * P.cap + rank] = (r << 1) | rbit;
      }
      listed += __popc(bal);
      n_tied += __popc(bal);
    }
#pragma unroll
    for (int d = 16; d; d >>= 1) sub = max(sub, __shfl_xor_sync(kFull, sub, d));
    if (lane == 0) P.qhead[q] = make_int4(best, sub, (int)n_tied, kQRescored);
  }
}

// ---------------------------------------------------------------- k0
// Reads travel host to device packed at 2 bits a base (base i of a byte in
// bits 2i..2i+1, each read starting on a byte); these two kernels run once
// after the upload.  k0_unpack writes one byte a base: each thread takes a
// 32-bit word (16 bases) and stores 16 bytes.  k0_exceptions then sets the
// listed positions -- read bases that were not A/C/G/T -- to the wildcard
// code 4.
__device__ __forceinline__ uint32_t spread4(uint32_t b) {
  return (b & 3u) | ((b >> 2) & 3u) << 8 | ((b >> 4) & 3u) << 16 | ((b >> 6) & 3u) << 24;
}

static __global__ void __launch_bounds__(256) k0_unpack(const uint32_t* __restrict__ packed,
                                                        uint64_t n_words, uint4* __restrict__ codes) {
  for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < n_words;
       w += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t p = packed[w];
    codes[w] = make_uint4(spread4(p & 0xffu), spread4((p >> 8) & 0xffu), spread4((p >> 16) & 0xffu),
                          spread4(p >> 24));
  }
}

static __global__ void __launch_bounds__(256) k0_exceptions(const uint64_t* __restrict__ at,
                                                            uint64_t n, uint8_t* __restrict__ codes) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    codes[at[i]] = 4;
}

// ---------------------------------------------------------------- k5
struct K5Params {
  const uint32_t* len;
  uint32_t n_reads;
  int both;
  const int4* qhead;
  const uint32_t* qties;
  uint32_t cap;
  int4* results;       // esg_read_result layout
  uint32_t* ties;      // [read * cap + k]
  int32_t* rows;       // optional rows: an empty read's rows score 0 (no cell)
  uint32_t n_refs;
};

static __global__ void __launch_bounds__(256) k5_merge(const K5Params P) {
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < P.n_reads;
       r += gridDim.x * blockDim.x) {
    const uint32_t cap = P.cap;
    uint32_t* out_t = P.ties + (size_t)r * cap;
    if (P.len[r] == 0) {
      P.results[r] = make_int4(INT32_MIN, INT32_MIN, 0, 1 /* ESG_RESULT_EMPTY */);
      for (uint32_t k = 0; k < cap; ++k) out_t[k] = kNoRef;
      if (P.rows) {
        for (uint32_t j = 0; j < P.n_refs; ++j) P.rows[(size_t)r * P.n_refs + j] = 0;
        if (P.both)
          for (uint32_t j = 0; j < P.n_refs; ++j)
            P.rows[((size_t)P.n_reads + r) * P.n_refs + j] = 0;
      }
      continue;
    }
    const int4 a = P.qhead[r];
    const uint32_t* ta = P.qties + (size_t)r * cap;
    int best = a.x, sub = a.y, flags = a.w & kQRescored;
    uint32_t n_tied = (uint32_t)a.z;
    if (!P.both) {
      const uint32_t nl = min(n_tied, cap);
      for (uint32_t k = 0; k < nl; ++k) out_t[k] = ta[k];
    } else {
      const uint32_t qb = P.n_reads + r;
      const int4 b = P.qhead[qb];
      const uint32_t* tb = P.qties + (size_t)qb * cap;
      flags |= b.w & kQRescored;
      const uint32_t na = min((uint32_t)a.z, cap), nb = min((uint32_t)b.z, cap);
      if (a.x > b.x) {
        sub = max(max(a.y, b.y), b.x);
        for (uint32_t k = 0; k < na; ++k) out_t[k] = ta[k];
      } else if (b.x > a.x) {
        best = b.x;
        n_tied = (uint32_t)b.z;
        sub = max(max(a.y, b.y), a.x);
        for (uint32_t k = 0; k < nb; ++k) out_t[k] = tb[k];
      } else {
        n_tied = (uint32_t)a.z + (uint32_t)b.z;
        sub = max(a.y, b.y);
        uint32_t i = 0, k2 = 0, w = 0;
        while (w < cap && (i < na || k2 < nb)) {
          if (k2 >= nb || (i < na && ta[i] < tb[k2]))
            out_t[w++] = ta[i++];
          else
            out_t[w++] = tb[k2++];
        }
      }
    }
    for (uint32_t k = min(n_tied, cap); k < cap; ++k) out_t[k] = kNoRef;  // ESG_NO_TIE
    if (n_tied > cap) flags |= 2;  // ESG_RESULT_TIES_TRUNCATED
    P.results[r] = make_int4(best, sub, (int)n_tied, flags);
  }
}

// ---------------------------------------------------------------- k6_pairs
// One warp per read pair.  Rows: mate m of pair p is read 2p + m; its
// forward row is query 2p + m, its reverse-complement row n_reads + 2p + m.
// Candidate (r, t): t = 0 pairs mate 1 forward with mate 2 reverse-
// complemented, t = 1 mate 1 reverse-complemented with mate 2 forward
// (pair.rs:135-137); eligible when both mate scores are >= min_score.
// Pass 1 takes the best eligible sum; pass 2 walks the references in
// 32-wide chunks and, in (r, t) order, lists the first tier (ballots give
// each tie its rank), and takes the next tier's sum and the per-mate best
// over candidates outside the tier (pair.rs:297-314).
struct K6Params {
  const int32_t* rows;   // [q * n_refs + r], q < 2 n_reads
  const uint32_t* len;   // trimmed mate lengths [n_reads]
  const int4* mates;     // k5's per-mate results (for RESCORED32)
  uint32_t n_pairs;
  uint32_t n_reads;
  uint32_t n_refs;
  uint32_t cap;
  int32_t min_score;
  int both;              // both template strands
  int4* out;             // [2 p]: best, next, n_tied, flags; [2 p + 1]: xs[2], primary[2]
  uint32_t* ties;        // [p * cap + k]
};

static __global__ void __launch_bounds__(256) k6_pairs(const K6Params P) {
  const int lane = threadIdx.x & 31;
  const uint32_t lt = (1u << lane) - 1u;
  const uint32_t wpb = blockDim.x >> 5;
  const int32_t ms = P.min_score;
  for (uint32_t p = blockIdx.x * wpb + (threadIdx.x >> 5); p < P.n_pairs; p += gridDim.x * wpb) {
    uint32_t* out_t = P.ties + (size_t)p * P.cap;
    const size_t nr = P.n_refs;
    const int32_t* f0 = P.rows + (size_t)(2 * p) * nr;
    const int32_t* f1 = f0 + nr;
    const int32_t* r0 = P.rows + (size_t)(P.n_reads + 2 * p) * nr;
    const int32_t* r1 = r0 + nr;
    const bool empty = P.len[2 * p] == 0 || P.len[2 * p + 1] == 0;
    int32_t best = INT32_MIN;
    if (!empty) {
      for (uint32_t r = lane; r < P.n_refs; r += 32) {
        const int32_t a = f0[r], b = r1[r];
        if (a >= ms && b >= ms) best = max(best, a + b);
        if (P.both) {
          const int32_t c = r0[r], d = f1[r];
          if (c >= ms && d >= ms) best = max(best, c + d);
        }
      }
    }
    best = __reduce_max_sync(kFull, best);
    const bool any = best != INT32_MIN;
    int32_t next = INT32_MIN, xs0 = INT32_MIN, xs1 = INT32_MIN, pa = INT32_MIN, pb = INT32_MIN;
    uint32_t n = 0;
    if (!empty) {
      for (uint32_t c0 = 0; c0 < P.n_refs; c0 += 32) {
        const uint32_t r = c0 + lane;
        const bool valid = r < P.n_refs;
        int32_t a = 0, b = 0, c = 0, d = 0;
        bool tie0 = false, tie1 = false;
        if (valid) {
          a = f0[r];
          b = r1[r];
          const bool e0 = a >= ms && b >= ms;
          tie0 = e0 && a + b == best;
          if (!tie0) {
            if (e0) next = max(next, a + b);
            xs0 = max(xs0, a);
            xs1 = max(xs1, b);
          }
          if (P.both) {
            c = r0[r];
            d = f1[r];
            const bool e1 = c >= ms && d >= ms;
            tie1 = e1 && c + d == best;
            if (!tie1) {
              if (e1) next = max(next, c + d);
              xs0 = max(xs0, c);
              xs1 = max(xs1, d);
            }
          }
        }
        const uint32_t b0 = __ballot_sync(kFull, tie0), b1 = __ballot_sync(kFull, tie1);
        if ((b0 | b1) == 0) continue;
        if (n == 0) {  // the primary: the first tie in (r, t) order
          const int src = __ffs(b0 | b1) - 1;
          const bool t0 = (b0 >> src) & 1u;
          pa = __shfl_sync(kFull, t0 ? a : c, src);
          pb = __shfl_sync(kFull, t0 ? b : d, src);
        }
        const uint32_t pre = n + __popc(b0 & lt) + __popc(b1 & lt);
        if (tie0 && pre < P.cap) out_t[pre] = r << 1;
        if (tie1 && pre + tie0 < P.cap) out_t[pre + tie0] = (r << 1) | 1u;
        n += __popc(b0) + __popc(b1);
      }
    }
    next = __reduce_max_sync(kFull, next);
    xs0 = __reduce_max_sync(kFull, xs0);
    xs1 = __reduce_max_sync(kFull, xs1);
    for (uint32_t k = min(n, P.cap) + lane; k < P.cap; k += 32) out_t[k] = kNoRef;  // ESG_NO_TIE
    if (lane == 0) {
      int flags = (any ? 0 : 1) | (n > P.cap ? 2 : 0);  // ESG_RESULT_EMPTY / _TIES_TRUNCATED
      if (!empty) flags |= (P.mates[2 * p].w | P.mates[2 * p + 1].w) & kQRescored;
      P.out[2 * p] = make_int4(best, next, (int)n, flags);
      P.out[2 * p + 1] = make_int4(xs0, xs1, pa, pb);
    }
  }
}

}  // namespace esg
