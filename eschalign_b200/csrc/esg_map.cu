// esg_map.cu -- Aligner::map_reads_scored (crates/eschalign/src/mapper.rs:
// 400-552) over the fused reduction: score the reads (the batched kernels,
// best / XS / tie count / first ties per read on the device), take each
// read's tie set in candidate order (mapper.rs:444-472), trace the taken
// members on the device (esg_trace.cu), and write each hit's MD and NM as
// samtools calmd does (crates/eschalign/src/sam.rs:55-121).  Host code only:
// the device work is the scorer's and the traceback's.
#include "../../include/eschalign_b200.h"
#include "esg_internal.h"

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <functional>
#include <memory>
#include <string>
#include <thread>
#include <utility>
#include <vector>

extern "C" void esg_internal_set_error(esg_status st, const char* msg);

struct esg_mapping {
  std::vector<esg_read_mapping> reads;
  std::vector<esg_hit> hits;
  std::vector<uint32_t> ops;
  std::vector<char> md;
  std::vector<esg_pair_mapping> pairs;  // esg_map_pairs only
  std::vector<esg_pair_hit> pair_hits;
};

namespace {

esg_status merr(esg_status st, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  esg_internal_set_error(st, buf);
  return st;
}

struct BatchGuard {
  esg_batch* b = nullptr;
  ~BatchGuard() {
    if (b) esg_batch_free(b);
  }
};

constexpr uint32_t kOpM = 0, kOpI = 1, kOpD = 2;
const char kLetter[5] = {'A', 'C', 'G', 'T', 'N'};

inline uint32_t code_at(const uint8_t* q, uint32_t n, bool reverse, uint32_t i) {
  if (!reverse) return q[i] > 4 ? 4u : q[i];
  const uint32_t c = q[n - 1 - i] > 4 ? 4u : q[n - 1 - i];
  return c == 4 ? 4u : 3u - c;  // alphabet.rs:58-64
}

inline char upper(uint8_t c) { return (c >= 'a' && c <= 'z') ? (char)(c - 32) : (char)c; }

// md_nm (sam.rs:76-121) on codes: calmd_match (sam.rs:63-69) holds when both
// letters are A/C/G/T (U as T) and equal, which on codes is "equal and < 4"
// (alphabet.rs:29-50 folds case and U); reference letters go into MD
// upper-cased, from the caller's letters when given.
void md_nm(const uint8_t* q, uint32_t n, bool reverse, const uint8_t* r, const uint8_t* rl,
           const esg_alignment& a, const uint32_t* ops, std::string& md, uint32_t& nm) {
  md.clear();
  nm = 0;
  uint32_t run = 0, i = a.query_start, j = a.ref_start;
  auto letter = [&](uint32_t jj) { return rl ? upper(rl[jj]) : kLetter[r[jj] > 4 ? 4 : r[jj]]; };
  auto flush = [&]() {  // the run of matches in decimal
    char digits[10];
    int w = 0;
    do {
      digits[w++] = (char)('0' + run % 10);
      run /= 10;
    } while (run);
    while (w) md.push_back(digits[--w]);
  };
  for (uint32_t k = 0; k < a.n_ops; ++k) {
    const uint32_t op = ops[k] & 0xfu, len = ops[k] >> 4;
    if (op == kOpM) {
      for (uint32_t t = 0; t < len; ++t, ++i, ++j) {
        const uint32_t x = code_at(q, n, reverse, i), y = r[j] > 4 ? 4u : r[j];
        if (x == y && y < 4) {
          ++run;
        } else {
          flush();
          md.push_back(letter(j));
          ++nm;
        }
      }
    } else if (op == kOpI) {
      i += len;
      nm += len;
    } else if (op == kOpD) {
      flush();
      md.push_back('^');
      for (uint32_t t = 0; t < len; ++t) md.push_back(letter(j + t));
      j += len;
      nm += len;
    }
  }
  flush();
}

bool has_match(const esg_alignment& a, const uint32_t* ops) {
  for (uint32_t k = 0; k < a.n_ops; ++k)
    if ((ops[k] & 0xfu) == kOpM) return true;
  return false;
}

}  // namespace

// The mapping of reads whose batch `b` is submitted: wait for it, take the
// tie sets, trace them on the scorer's stream, call `after_trace` (the
// caller queues its next batch there, so the device scores it while this
// batch is assembled), assemble.
static esg_status map_scored(esg_scorer* sc, esg_batch* b, const uint8_t* codes,
                             const uint64_t* off, const uint32_t* len, uint32_t n_reads,
                             const esg_map_options* o, const uint8_t* ref_letters,
                             const uint64_t* ref_letter_off,
                             const std::function<esg_status()>& after_trace,
                             std::unique_ptr<esg_mapping>& result) {
  esg_internal_panel P{};
  esg_internal_panel_of(sc, &P);
  const uint32_t cap = esg_internal_tie_capacity(sc);
  const uint32_t flags = o->both_strands ? ESG_BOTH_STRANDS : 0u;
  esg_status st;
  std::vector<esg_read_result> res(std::max<uint32_t>(n_reads, 1));
  std::vector<uint32_t> ties(std::max<size_t>((size_t)n_reads * cap, 1));
  if ((st = esg_finish(sc, b, res.data(), ties.data(), nullptr)) != ESG_OK) return st;

  // --- the taken ties (mapper.rs:458-465): reads whose list the tie
  // capacity cut short get it from full rows
  std::vector<uint32_t> take(n_reads, 0);
  std::vector<uint32_t> redo;
  for (uint32_t k = 0; k < n_reads; ++k) {
    if (res[k].flags & ESG_RESULT_EMPTY) continue;
    if (res[k].best < o->min_score) continue;
    const uint32_t nt = res[k].n_tied;
    take[k] = (o->max_ties == ESG_ALL_TIES || o->max_ties >= nt) ? nt : o->max_ties + 1;
    if (take[k] > std::min(nt, cap)) redo.push_back(k);
  }
  std::vector<std::vector<uint32_t>> full(redo.size());
  if (!redo.empty()) {
    const uint32_t m = (uint32_t)redo.size(), nr = P.n_refs, strands = o->both_strands ? 2 : 1;
    std::vector<uint64_t> roff(m);
    std::vector<uint32_t> rlen(m);
    for (uint32_t i = 0; i < m; ++i) {
      roff[i] = off[redo[i]];
      rlen[i] = len[redo[i]];
    }
    std::vector<esg_read_result> r2(m);
    std::vector<int32_t> rows((size_t)strands * m * nr);
    if ((st = esg_score_batch(sc, codes, roff.data(), rlen.data(), m, flags | ESG_FULL_ROWS,
                              r2.data(), nullptr, rows.data())) != ESG_OK)
      return st;
    for (uint32_t i = 0; i < m; ++i) {
      const int32_t best = res[redo[i]].best;
      for (uint32_t r = 0; r < nr; ++r) {
        if (rows[(size_t)i * nr + r] == best) full[i].push_back(r << 1);
        if (strands == 2 && rows[((size_t)m + i) * nr + r] == best) full[i].push_back((r << 1) | 1u);
      }
      if (full[i].size() != res[redo[i]].n_tied || r2[i].best != best)
        return merr(ESG_ERR_DRIVER, "read %u: rows disagree with the reduction", redo[i]);
    }
  }

  // --- trace every taken tie of every read in one batch
  std::vector<esg_align_job> jobs;
  std::vector<uint64_t> first_job(n_reads + 1, 0);
  {
    size_t ri = 0;
    for (uint32_t k = 0; k < n_reads; ++k) {
      first_job[k] = jobs.size();
      const uint32_t* list = ties.data() + (size_t)k * cap;
      if (ri < redo.size() && redo[ri] == k) list = full[ri++].data();
      for (uint32_t t = 0; t < take[k]; ++t)
        jobs.push_back(esg_align_job{k, list[t] >> 1, list[t] & 1u});
    }
    first_job[n_reads] = jobs.size();
  }
  std::vector<esg_alignment> al(jobs.size());
  std::vector<uint32_t> ops;
  if (!jobs.empty() &&
      (st = esg_internal_align_batch(sc, b, jobs.data(), (uint32_t)jobs.size(), al.data(),
                                     &ops)) != ESG_OK)
    return st;
  if (after_trace && (st = after_trace()) != ESG_OK) return st;

  // --- the mappings (mapper.rs:497-552), reads split over host threads,
  // each part's hits / words / MD concatenated in read order
  std::unique_ptr<esg_mapping> m(new esg_mapping);
  m->reads.resize(n_reads);
  struct Part {
    std::vector<esg_hit> hits;
    std::vector<uint32_t> ops;
    std::vector<char> md;
  };
  auto assemble = [&](uint32_t k0, uint32_t k1, Part& p) {
    std::string md;
    for (uint32_t k = k0; k < k1; ++k) {
      esg_read_mapping& rm = m->reads[k];
      rm = esg_read_mapping{};
      rm.first_hit = p.hits.size();
      if (res[k].flags & ESG_RESULT_EMPTY) continue;
      rm.best_score = res[k].best;
      rm.n_tied = res[k].n_tied;
      rm.flags = ESG_MAPPING_HAS_BEST;
      if (res[k].suboptimal != ESG_NO_SCORE) {
        rm.suboptimal = res[k].suboptimal;
        rm.flags |= ESG_MAPPING_HAS_SUBOPTIMAL;
      }
      const uint64_t j0 = first_job[k], j1 = first_job[k + 1];
      if (j0 == j1 || !has_match(al[j0], ops.data() + al[j0].ops_offset)) continue;
      const uint8_t* q = codes + off[k];
      for (uint64_t jb = j0; jb < j1; ++jb) {
        const esg_align_job& J = jobs[jb];
        esg_alignment a = al[jb];
        const uint32_t* w = ops.data() + a.ops_offset;
        esg_hit h{};
        h.reference = J.ref;
        h.reverse = J.reverse;
        md_nm(q, len[k], J.reverse != 0, P.h_codes + P.h_off[J.ref],
              ref_letters ? ref_letters + ref_letter_off[J.ref] : nullptr, a, w, md, h.nm);
        h.md_offset = p.md.size();
        h.md_len = (uint32_t)md.size();
        p.md.insert(p.md.end(), md.begin(), md.end());
        a.ops_offset = p.ops.size();
        p.ops.insert(p.ops.end(), w, w + a.n_ops);
        h.alignment = a;
        p.hits.push_back(h);
      }
      rm.n_hits = (uint32_t)(j1 - j0);
    }
  };
  const uint32_t hw = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
  const uint32_t n_parts = std::max(1u, std::min(hw, n_reads / 4096));
  std::vector<Part> parts(n_parts);
  std::vector<uint32_t> cut(n_parts + 1);
  for (uint32_t t = 0; t <= n_parts; ++t) cut[t] = (uint32_t)((uint64_t)n_reads * t / n_parts);
  if (n_parts == 1) {
    assemble(0, n_reads, parts[0]);
  } else {
    std::vector<std::thread> th;
    for (uint32_t t = 0; t < n_parts; ++t)
      th.emplace_back(assemble, cut[t], cut[t + 1], std::ref(parts[t]));
    for (auto& x : th) x.join();
  }
  size_t nh = 0, no = 0, nm = 0;
  for (const Part& p : parts) {
    nh += p.hits.size();
    no += p.ops.size();
    nm += p.md.size();
  }
  m->hits.reserve(nh);
  m->ops.reserve(no);
  m->md.reserve(nm);
  for (uint32_t t = 0; t < n_parts; ++t) {
    const uint64_t hb = m->hits.size(), ob = m->ops.size(), mb = m->md.size();
    for (uint32_t k = cut[t]; k < cut[t + 1]; ++k) m->reads[k].first_hit += hb;
    for (esg_hit h : parts[t].hits) {
      h.alignment.ops_offset += ob;
      h.md_offset += mb;
      m->hits.push_back(h);
    }
    m->ops.insert(m->ops.end(), parts[t].ops.begin(), parts[t].ops.end());
    m->md.insert(m->md.end(), parts[t].md.begin(), parts[t].md.end());
  }
  result = std::move(m);
  return ESG_OK;
}

// Reads per batch of a large mapping call.  The scoring kernel holds every
// SM until it ends, so a batch's traceback cannot run beside the next
// batch's scoring: each batch is traced as soon as it is scored, the next
// one (prepared meanwhile) is queued, and the traced batch is assembled on
// the host while the device scores the next.
constexpr uint32_t kMapChunk = 131072;

static esg_status map_reads_impl(esg_scorer* sc, const uint8_t* codes, const uint64_t* off,
                                 const uint32_t* len, uint32_t n_reads, const esg_map_options* o,
                                 const uint8_t* ref_letters, const uint64_t* ref_letter_off,
                                 std::unique_ptr<esg_mapping>& result) {
  if (n_reads && (!off || !len)) return merr(ESG_ERR_BAD_ARGUMENT, "off/len must not be NULL");
  if (o->both_strands > 1 || o->reserved)
    return merr(ESG_ERR_BAD_ARGUMENT, "both_strands must be 0 or 1, reserved 0");
  if (ref_letters && !ref_letter_off)
    return merr(ESG_ERR_BAD_ARGUMENT, "ref_letters needs ref_letter_off");
  uint64_t total = 0;
  for (uint32_t k = 0; k < n_reads; ++k) total += len[k];
  if (total && !codes) return merr(ESG_ERR_BAD_ARGUMENT, "codes must not be NULL");
  const uint32_t flags = o->both_strands ? ESG_BOTH_STRANDS : 0u;
  esg_status st;
  if (n_reads <= kMapChunk + kMapChunk / 2) {
    BatchGuard g;
    if ((st = esg_prepare(sc, codes, off, len, n_reads, flags, &g.b)) != ESG_OK ||
        (st = esg_submit(sc, g.b)) != ESG_OK)
      return st;
    return map_scored(sc, g.b, codes, off, len, n_reads, o, ref_letters, ref_letter_off, {},
                      result);
  }
  std::vector<uint32_t> cut;
  for (uint32_t k = 0; k < n_reads; k += kMapChunk) cut.push_back(k);
  cut.push_back(n_reads);
  std::unique_ptr<esg_mapping> all(new esg_mapping);
  all->reads.reserve(n_reads);
  BatchGuard cur, nxt;
  auto prepare = [&](size_t c, BatchGuard& into) {
    return esg_prepare(sc, codes, off + cut[c], len + cut[c], cut[c + 1] - cut[c], flags,
                       &into.b);
  };
  if ((st = prepare(0, cur)) != ESG_OK || (st = esg_submit(sc, cur.b)) != ESG_OK ||
      (st = prepare(1, nxt)) != ESG_OK)
    return st;
  for (size_t c = 0; c + 1 < cut.size(); ++c) {
    const uint32_t k0 = cut[c], nk = cut[c + 1] - cut[c];
    const bool more = c + 2 < cut.size();
    std::unique_ptr<esg_mapping> part;
    if ((st = map_scored(sc, cur.b, codes, off + k0, len + k0, nk, o, ref_letters,
                         ref_letter_off,
                         [&]() { return more ? esg_submit(sc, nxt.b) : ESG_OK; }, part)) != ESG_OK)
      return st;
    const uint64_t hb = all->hits.size(), ob = all->ops.size(), mb = all->md.size();
    for (esg_read_mapping rm : part->reads) {
      rm.first_hit += hb;
      all->reads.push_back(rm);
    }
    for (esg_hit h : part->hits) {
      h.alignment.ops_offset += ob;
      h.md_offset += mb;
      all->hits.push_back(h);
    }
    all->ops.insert(all->ops.end(), part->ops.begin(), part->ops.end());
    all->md.insert(all->md.end(), part->md.begin(), part->md.end());
    esg_batch_free(cur.b);
    cur.b = nxt.b;
    nxt.b = nullptr;
    if (c + 3 < cut.size() && (st = prepare(c + 2, nxt)) != ESG_OK) return st;
  }
  result = std::move(all);
  return ESG_OK;
}

namespace {

// Aligner::pair_ok (pair.rs:392-410): both mates align a base, the mate
// read as sequenced on the template strand starts before the other ends,
// the insert (leftmost to rightmost aligned base) within max_insert.
bool pair_ok(const esg_alignment& a0, const uint32_t* w0, const esg_alignment& a1,
             const uint32_t* w1, bool template_reverse, uint32_t max_insert) {
  if (!has_match(a0, w0) || !has_match(a1, w1)) return false;
  const esg_alignment& fwd = template_reverse ? a1 : a0;
  const esg_alignment& rev = template_reverse ? a0 : a1;
  if (fwd.ref_start >= rev.ref_end) return false;
  const uint32_t lo = std::min(a0.ref_start, a1.ref_start);
  const uint32_t hi = std::max(a0.ref_end, a1.ref_end);
  return hi - lo <= max_insert;
}

// PairState::mate_reverse (pair.rs:135-137)
inline uint32_t mate_reverse(uint32_t m, uint32_t t) { return t ^ (m == 1 ? 1u : 0u); }

struct PairCand {
  int32_t sum;
  uint32_t ref, t;
  int32_t a, b;
};

}  // namespace

// Aligner::map_pairs_scored (pair.rs:157-390) over the device ranking.
// Phase 1 is the device's (k6_pairs): each pair's first tier -- its sum,
// size, first members and the per-mate XS outside it.  Phase 2 traces the
// first tier of every pair at once; a pair whose first tier holds members
// that fail pair_ok keeps the ones that pass and adds the failed members'
// mate scores to its XS (the device XS excludes the whole tier).  Pairs
// whose first tier all fails, or is longer than the tie capacity, are
// scored again with full rows and walked tier by tier on the host as
// pair.rs:246-292 does, every open pair's next tier traced together.
// Phase 3 builds the Proper mappings; the rest map each mate on its own,
// both strands (pair.rs:362-387).
static esg_status map_pairs_impl(esg_scorer* sc, const uint8_t* codes, const uint64_t* off,
                                 const uint32_t* len, uint32_t n_pairs,
                                 const esg_pair_map_options* o, const uint8_t* ref_letters,
                                 const uint64_t* ref_letter_off,
                                 std::unique_ptr<esg_mapping>& result) {
  esg_internal_panel P{};
  esg_internal_panel_of(sc, &P);
  const uint32_t cap = esg_internal_tie_capacity(sc), nr = P.n_refs;
  const uint32_t pflags = o->both_strands ? ESG_BOTH_STRANDS : 0u;
  const uint32_t n_mates = 2 * n_pairs;

  BatchGuard g;
  esg_status st = esg_prepare_pairs(sc, codes, off, len, n_pairs, nullptr, o->min_score, pflags,
                                    &g.b);
  if (st != ESG_OK) return st;
  if ((st = esg_submit(sc, g.b)) != ESG_OK) return st;
  std::vector<esg_pair_result> pr(std::max<uint32_t>(n_pairs, 1));
  std::vector<uint32_t> pties(std::max<size_t>((size_t)n_pairs * cap, 1));
  if ((st = esg_finish_pairs(sc, g.b, pr.data(), pties.data(), nullptr, nullptr, nullptr,
                             nullptr)) != ESG_OK)
    return st;

  // per pair: the found set (candidates with their two traced jobs)
  struct Found {
    PairCand c;
    esg_alignment al[2];
    const uint32_t* w[2];
  };
  std::vector<std::vector<Found>> found(n_pairs);
  std::vector<int32_t> xs(2 * (size_t)n_pairs, ESG_NO_SCORE);
  std::vector<uint8_t> kind(n_pairs, 0);  // 0 separate, 1 proper
  std::vector<uint32_t> deep;             // pairs for the rows path
  std::vector<uint8_t> deep_from0;        // ... starting at the first tier
  std::vector<uint32_t> ops1, ops2;       // CIGAR words: first-tier round, deep rounds' found

  // --- phase 2a: every pair's first tier from the device ranking
  {
    std::vector<esg_align_job> jobs;
    std::vector<uint32_t> tp;  // pair of each candidate
    for (uint32_t p = 0; p < n_pairs; ++p) {
      if (pr[p].flags & ESG_RESULT_EMPTY) continue;
      if (pr[p].n_tied > cap) {
        deep.push_back(p);
        deep_from0.push_back(1);
        continue;
      }
      for (uint32_t i = 0; i < pr[p].n_tied; ++i) {
        const uint32_t c = pties[(size_t)p * cap + i];
        for (uint32_t m = 0; m < 2; ++m)
          jobs.push_back(esg_align_job{2 * p + m, c >> 1, mate_reverse(m, c & 1u)});
        tp.push_back(p);
      }
    }
    std::vector<esg_alignment> al(jobs.size());
    if (!jobs.empty() &&
        (st = esg_internal_align_batch(sc, g.b, jobs.data(), (uint32_t)jobs.size(), al.data(),
                                       &ops1)) != ESG_OK)
      return st;
    size_t k = 0;
    while (k < tp.size()) {
      const uint32_t p = tp[k];
      int32_t x0 = pr[p].xs[0], x1 = pr[p].xs[1];
      for (; k < tp.size() && tp[k] == p; ++k) {
        const esg_alignment &a0 = al[2 * k], &a1 = al[2 * k + 1];
        const uint32_t* w0 = ops1.data() + a0.ops_offset;
        const uint32_t* w1 = ops1.data() + a1.ops_offset;
        const uint32_t t = jobs[2 * k].reverse;  // mate 1 follows the template
        if (pair_ok(a0, w0, a1, w1, t != 0, o->max_insert)) {
          found[p].push_back(Found{PairCand{a0.score + a1.score, jobs[2 * k].ref, t, a0.score,
                                            a1.score},
                                   {a0, a1},
                                   {w0, w1}});
        } else {
          x0 = std::max(x0, a0.score);
          x1 = std::max(x1, a1.score);
        }
      }
      if (found[p].empty()) {
        deep.push_back(p);
        deep_from0.push_back(0);
      } else {
        kind[p] = 1;
        xs[2 * (size_t)p] = x0;
        xs[2 * (size_t)p + 1] = x1;
      }
    }
  }

  // --- phase 2b: full rows, tier by tier on the host
  if (!deep.empty()) {
    std::vector<uint32_t> order(deep.size());
    for (uint32_t i = 0; i < order.size(); ++i) order[i] = i;
    std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return deep[a] < deep[b]; });
    std::vector<uint32_t> dp(deep.size());
    std::vector<uint8_t> d0(deep.size());
    for (uint32_t i = 0; i < order.size(); ++i) {
      dp[i] = deep[order[i]];
      d0[i] = deep_from0[order[i]];
    }
    const uint32_t m = (uint32_t)dp.size();
    std::vector<uint64_t> soff(2 * (size_t)m);
    std::vector<uint32_t> slen(2 * (size_t)m);
    for (uint32_t i = 0; i < m; ++i)
      for (uint32_t q = 0; q < 2; ++q) {
        soff[2 * i + q] = off[2 * dp[i] + q];
        slen[2 * i + q] = len[2 * dp[i] + q];
      }
    BatchGuard g2;
    if ((st = esg_prepare_pairs(sc, codes, soff.data(), slen.data(), m, nullptr, o->min_score,
                                pflags | ESG_FULL_ROWS, &g2.b)) != ESG_OK ||
        (st = esg_submit(sc, g2.b)) != ESG_OK)
      return st;
    std::vector<int32_t> rows((size_t)4 * m * nr);
    std::vector<esg_pair_result> pr2(m);
    if ((st = esg_finish_pairs(sc, g2.b, pr2.data(), nullptr, nullptr, nullptr, nullptr,
                               rows.data())) != ESG_OK)
      return st;
    auto row = [&](uint32_t mate, uint32_t rev) {
      return rows.data() + ((size_t)(rev ? 2 * m : 0) + mate) * nr;
    };
    // phase 1 on the host (pair.rs:175-231)
    std::vector<std::vector<PairCand>> cands(m);
    std::vector<std::vector<std::pair<size_t, size_t>>> tiers(m);
    std::vector<size_t> next(m, 0);
    const uint32_t n_strands = o->both_strands ? 2 : 1;
    for (uint32_t i = 0; i < m; ++i) {
      auto& cs = cands[i];
      for (uint32_t t = 0; t < n_strands; ++t) {
        const int32_t* r0 = row(2 * i, mate_reverse(0, t));
        const int32_t* r1 = row(2 * i + 1, mate_reverse(1, t));
        for (uint32_t r = 0; r < nr; ++r)
          if (r0[r] >= o->min_score && r1[r] >= o->min_score)
            cs.push_back(PairCand{r0[r] + r1[r], r, t, r0[r], r1[r]});
      }
      std::stable_sort(cs.begin(), cs.end(), [](const PairCand& a, const PairCand& b) {
        if (a.sum != b.sum) return a.sum > b.sum;
        if (a.ref != b.ref) return a.ref < b.ref;
        return a.t < b.t;
      });
      size_t start = 0;
      for (size_t k = 1; k <= cs.size(); ++k)
        if (k == cs.size() || cs[k].sum != cs[start].sum) {
          tiers[i].push_back({start, k});
          start = k;
        }
      next[i] = d0[i] ? 0 : 1;  // the first tier already failed on the device path
    }
    // phase 2 (pair.rs:246-292): trace every open pair's next tier together
    std::vector<std::vector<esg_alignment>> kept_al;
    std::vector<std::vector<uint32_t>> kept_ops;
    for (;;) {
      std::vector<esg_align_job> jobs;
      std::vector<std::pair<uint32_t, size_t>> who;  // (deep pair, candidate)
      for (uint32_t i = 0; i < m; ++i) {
        if (!found[dp[i]].empty() || next[i] >= tiers[i].size()) continue;
        const auto [a, b] = tiers[i][next[i]];
        for (size_t k = a; k < b; ++k) {
          for (uint32_t q = 0; q < 2; ++q)
            jobs.push_back(esg_align_job{2 * i + q, cands[i][k].ref,
                                         mate_reverse(q, cands[i][k].t)});
          who.push_back({i, k});
        }
      }
      if (jobs.empty()) break;
      kept_al.emplace_back(jobs.size());
      kept_ops.emplace_back();
      if ((st = esg_internal_align_batch(sc, g2.b, jobs.data(), (uint32_t)jobs.size(),
                                         kept_al.back().data(), &kept_ops.back())) != ESG_OK)
        return st;
      const auto& al = kept_al.back();
      const auto& w = kept_ops.back();
      for (size_t k = 0; k < who.size(); ++k) {
        const auto [i, ci] = who[k];
        const PairCand& c = cands[i][ci];
        const uint32_t* w0 = w.data() + al[2 * k].ops_offset;
        const uint32_t* w1 = w.data() + al[2 * k + 1].ops_offset;
        if (pair_ok(al[2 * k], w0, al[2 * k + 1], w1, c.t != 0, o->max_insert))
          found[dp[i]].push_back(Found{c, {al[2 * k], al[2 * k + 1]}, {w0, w1}});
      }
      for (uint32_t i = 0; i < m; ++i)
        if (found[dp[i]].empty() && next[i] < tiers[i].size()) ++next[i];
    }
    // XS outside the found set, from the rows (pair.rs:297-314)
    std::vector<uint8_t> in_set(2 * (size_t)nr);
    for (uint32_t i = 0; i < m; ++i) {
      const uint32_t p = dp[i];
      if (found[p].empty()) continue;
      kind[p] = 1;
      std::fill(in_set.begin(), in_set.end(), 0);
      for (const Found& f : found[p]) in_set[2 * (size_t)f.c.ref + f.c.t] = 1;
      for (uint32_t t = 0; t < n_strands; ++t)
        for (uint32_t r = 0; r < nr; ++r) {
          if (in_set[2 * (size_t)r + t]) continue;
          for (uint32_t q = 0; q < 2; ++q)
            xs[2 * (size_t)p + q] = std::max(xs[2 * (size_t)p + q], row(2 * i + q, mate_reverse(q, t))[r]);
        }
    }
    // the found sets' words live in this block's trace rounds: copy them
    // out for phase 3
    for (uint32_t i = 0; i < m; ++i)
      for (Found& f : found[dp[i]])
        for (uint32_t q = 0; q < 2; ++q) {
          const size_t at = ops2.size();
          ops2.insert(ops2.end(), f.w[q], f.w[q] + f.al[q].n_ops);
          f.al[q].ops_offset = at;
          f.w[q] = nullptr;  // resolved against ops2 below
        }
  }

  // --- phase 3: Proper mappings (pair.rs:294-360), pairs split over host
  // threads, each part's pair hits / words / MD concatenated in pair order
  std::unique_ptr<esg_mapping> out(new esg_mapping);
  out->pairs.resize(n_pairs);
  out->reads.resize(n_mates);
  struct Part {
    std::vector<esg_pair_hit> hits;
    std::vector<uint32_t> ops;
    std::vector<char> md;
  };
  auto assemble = [&](uint32_t p0, uint32_t p1, Part& part) {
    std::string md;
    for (uint32_t p = p0; p < p1; ++p) {
      esg_pair_mapping& pm = out->pairs[p];
      pm = esg_pair_mapping{};
      pm.first_hit = part.hits.size();
      pm.suboptimal[0] = pm.suboptimal[1] = ESG_NO_SCORE;
      if (!kind[p]) continue;
      const auto& fs = found[p];
      pm.flags = ESG_PAIR_PROPER;
      pm.score = fs[0].c.sum;
      pm.n_tied = (uint32_t)fs.size();
      for (uint32_t q = 0; q < 2; ++q)
        if (xs[2 * (size_t)p + q] != ESG_NO_SCORE) {
          pm.suboptimal[q] = xs[2 * (size_t)p + q];
          pm.flags |= q ? ESG_PAIR_HAS_XS2 : ESG_PAIR_HAS_XS1;
        }
      const uint32_t keep = (o->max_ties == ESG_ALL_TIES || o->max_ties >= pm.n_tied)
                                ? pm.n_tied
                                : o->max_ties + 1;
      for (uint32_t k = 0; k < keep; ++k) {
        const Found& f = fs[k];
        esg_pair_hit ph{};
        ph.reference = f.c.ref;
        ph.reverse = f.c.t;
        for (uint32_t q = 0; q < 2; ++q) {
          const uint32_t* w = f.w[q] ? f.w[q] : ops2.data() + f.al[q].ops_offset;
          esg_alignment a = f.al[q];
          esg_hit& h = ph.mates[q];
          h.reference = f.c.ref;
          h.reverse = mate_reverse(q, f.c.t);
          md_nm(codes + off[2 * p + q], len[2 * p + q], h.reverse != 0,
                P.h_codes + P.h_off[f.c.ref],
                ref_letters ? ref_letters + ref_letter_off[f.c.ref] : nullptr, a, w, md, h.nm);
          h.md_offset = part.md.size();
          h.md_len = (uint32_t)md.size();
          part.md.insert(part.md.end(), md.begin(), md.end());
          a.ops_offset = part.ops.size();
          part.ops.insert(part.ops.end(), w, w + a.n_ops);
          h.alignment = a;
        }
        ph.insert = std::max(ph.mates[0].alignment.ref_end, ph.mates[1].alignment.ref_end) -
                    std::min(ph.mates[0].alignment.ref_start, ph.mates[1].alignment.ref_start);
        part.hits.push_back(ph);
      }
      pm.n_hits = keep;
    }
  };
  {
    const uint32_t hw = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    const uint32_t n_parts = std::max(1u, std::min(hw, n_pairs / 2048));
    std::vector<Part> parts(n_parts);
    std::vector<uint32_t> cut(n_parts + 1);
    for (uint32_t t = 0; t <= n_parts; ++t) cut[t] = (uint32_t)((uint64_t)n_pairs * t / n_parts);
    if (n_parts == 1) {
      assemble(0, n_pairs, parts[0]);
    } else {
      std::vector<std::thread> th;
      for (uint32_t t = 0; t < n_parts; ++t)
        th.emplace_back(assemble, cut[t], cut[t + 1], std::ref(parts[t]));
      for (auto& x : th) x.join();
    }
    for (uint32_t t = 0; t < n_parts; ++t) {
      const uint64_t hb = out->pair_hits.size(), ob = out->ops.size(), mb = out->md.size();
      for (uint32_t p = cut[t]; p < cut[t + 1]; ++p) out->pairs[p].first_hit += hb;
      for (esg_pair_hit ph : parts[t].hits) {
        for (uint32_t q = 0; q < 2; ++q) {
          ph.mates[q].alignment.ops_offset += ob;
          ph.mates[q].md_offset += mb;
        }
        out->pair_hits.push_back(ph);
      }
      out->ops.insert(out->ops.end(), parts[t].ops.begin(), parts[t].ops.end());
      out->md.insert(out->md.end(), parts[t].md.begin(), parts[t].md.end());
    }
  }

  // --- the rest: each mate on its own, both strands (pair.rs:362-387)
  std::vector<uint32_t> sep;
  for (uint32_t p = 0; p < n_pairs; ++p)
    if (!kind[p]) sep.push_back(p);
  if (!sep.empty()) {
    std::vector<uint64_t> soff(2 * sep.size());
    std::vector<uint32_t> slen(2 * sep.size());
    for (size_t i = 0; i < sep.size(); ++i)
      for (uint32_t q = 0; q < 2; ++q) {
        soff[2 * i + q] = off[2 * sep[i] + q];
        slen[2 * i + q] = len[2 * sep[i] + q];
      }
    esg_map_options mo{o->min_score, o->max_ties, 1u, 0u};
    std::unique_ptr<esg_mapping> each;
    if ((st = map_reads_impl(sc, codes, soff.data(), slen.data(), (uint32_t)(2 * sep.size()), &mo,
                             ref_letters, ref_letter_off, each)) != ESG_OK)
      return st;
    const uint64_t hb = out->hits.size(), ob = out->ops.size(), mb = out->md.size();
    for (esg_hit h : each->hits) {
      h.alignment.ops_offset += ob;
      h.md_offset += mb;
      out->hits.push_back(h);
    }
    out->ops.insert(out->ops.end(), each->ops.begin(), each->ops.end());
    out->md.insert(out->md.end(), each->md.begin(), each->md.end());
    for (size_t i = 0; i < sep.size(); ++i)
      for (uint32_t q = 0; q < 2; ++q) {
        esg_read_mapping rm = each->reads[2 * i + q];
        rm.first_hit += hb;
        out->reads[2 * sep[i] + q] = rm;
      }
  }
  for (uint32_t k = 0; k < n_mates; ++k)
    if (kind[k / 2]) out->reads[k].first_hit = out->hits.size();
  result = std::move(out);
  return ESG_OK;
}

extern "C" {

esg_status esg_map_reads(esg_scorer* sc, const uint8_t* codes, const uint64_t* off,
                         const uint32_t* len, uint32_t n_reads, const esg_map_options* o,
                         const uint8_t* ref_letters, const uint64_t* ref_letter_off,
                         esg_mapping** out) {
  if (out) *out = nullptr;
  if (!sc || !o || !out) return merr(ESG_ERR_BAD_ARGUMENT, "NULL scorer, options or out");
  std::unique_ptr<esg_mapping> m;
  const esg_status st =
      map_reads_impl(sc, codes, off, len, n_reads, o, ref_letters, ref_letter_off, m);
  if (st != ESG_OK) return st;
  *out = m.release();
  esg_internal_set_error(ESG_OK, "");
  return ESG_OK;
}

esg_status esg_map_pairs(esg_scorer* sc, const uint8_t* codes, const uint64_t* off,
                         const uint32_t* len, uint32_t n_pairs, const esg_pair_map_options* o,
                         const uint8_t* ref_letters, const uint64_t* ref_letter_off,
                         esg_mapping** out) {
  if (out) *out = nullptr;
  if (!sc || !o || !out) return merr(ESG_ERR_BAD_ARGUMENT, "NULL scorer, options or out");
  if (n_pairs && (!off || !len)) return merr(ESG_ERR_BAD_ARGUMENT, "off/len must not be NULL");
  if (o->both_strands > 1) return merr(ESG_ERR_BAD_ARGUMENT, "both_strands must be 0 or 1");
  if (ref_letters && !ref_letter_off)
    return merr(ESG_ERR_BAD_ARGUMENT, "ref_letters needs ref_letter_off");
  uint64_t total = 0;
  for (uint64_t k = 0; k < 2 * (uint64_t)n_pairs; ++k) total += len[k];
  if (total && !codes) return merr(ESG_ERR_BAD_ARGUMENT, "codes must not be NULL");
  std::unique_ptr<esg_mapping> m;
  const esg_status st =
      map_pairs_impl(sc, codes, off, len, n_pairs, o, ref_letters, ref_letter_off, m);
  if (st != ESG_OK) return st;
  *out = m.release();
  esg_internal_set_error(ESG_OK, "");
  return ESG_OK;
}

const esg_pair_mapping* esg_mapping_pairs(const esg_mapping* m, uint32_t* n) {
  if (n) *n = m ? (uint32_t)m->pairs.size() : 0u;
  return m ? m->pairs.data() : nullptr;
}

const esg_pair_hit* esg_mapping_pair_hits(const esg_mapping* m, uint64_t* n) {
  if (n) *n = m ? m->pair_hits.size() : 0u;
  return m ? m->pair_hits.data() : nullptr;
}

// What is wrong with a caller's hit, or NULL: the strand is 0 or 1, each
// start is at most its end, and the CIGAR words (BAM ops M..X) consume
// exactly [query_start, query_end) of the read and [ref_start, ref_end) of
// the reference, as every traced hit does.  Its ops must already be known
// to lie inside `ops`.
static const char* hit_inconsistency(const esg_hit& h, const uint32_t* ops) {
  const esg_alignment& a = h.alignment;
  if (h.reverse > 1) return "its strand is not 0 or 1";
  if (a.query_start > a.query_end || a.ref_start > a.ref_end) return "a start is past its end";
  uint64_t q = 0, r = 0;
  for (uint32_t k = 0; k < a.n_ops; ++k) {
    const uint32_t w = ops[a.ops_offset + k], op = w & 0xfu, n = w >> 4;
    if (op > 8) return "a CIGAR op is past X";
    if (op == 0 || op == 1 || op == 4 || op == 7 || op == 8) q += n;  // M I S = X
    if (op == 0 || op == 2 || op == 3 || op == 7 || op == 8) r += n;  // M D N = X
  }
  if (q != (uint64_t)(a.query_end - a.query_start) || r != (uint64_t)(a.ref_end - a.ref_start))
    return "its CIGAR does not span its coordinates";
  return nullptr;
}

esg_status esg_mapping_from_arrays(const esg_read_mapping* reads, uint32_t n_reads,
                                   const esg_hit* hits, uint64_t n_hits, const uint32_t* ops,
                                   uint64_t n_ops, const char* md, uint64_t n_md,
                                   esg_mapping** out) {
  if (!out || (n_reads && !reads) || (n_hits && !hits) || (n_ops && !ops) || (n_md && !md))
    return merr(ESG_ERR_BAD_ARGUMENT, "NULL argument");
  *out = nullptr;
  for (uint32_t k = 0; k < n_reads; ++k)
    if (reads[k].first_hit > n_hits || reads[k].n_hits > n_hits - reads[k].first_hit)
      return merr(ESG_ERR_BAD_ARGUMENT, "read %u's hits run past the hit array", k);
  for (uint64_t h = 0; h < n_hits; ++h)
    if (hits[h].alignment.ops_offset > n_ops ||
        hits[h].alignment.n_ops > n_ops - hits[h].alignment.ops_offset ||
        hits[h].md_offset > n_md || hits[h].md_len > n_md - hits[h].md_offset)
      return merr(ESG_ERR_BAD_ARGUMENT, "hit %llu's ops or MD run past their arrays",
                  (unsigned long long)h);
  for (uint64_t h = 0; h < n_hits; ++h)
    if (const char* why = hit_inconsistency(hits[h], ops))
      return merr(ESG_ERR_BAD_ARGUMENT, "hit %llu: %s", (unsigned long long)h, why);
  auto* m = new esg_mapping();
  m->reads.assign(reads, reads + n_reads);
  m->hits.assign(hits, hits + n_hits);
  m->ops.assign(ops, ops + n_ops);
  m->md.assign(md, md + n_md);
  *out = m;
  return ESG_OK;
}

esg_status esg_mapping_set_pairs(esg_mapping* m, const esg_pair_mapping* pairs, uint32_t n_pairs,
                                 const esg_pair_hit* pair_hits, uint64_t n_pair_hits) {
  if (!m || (n_pairs && !pairs) || (n_pair_hits && !pair_hits))
    return merr(ESG_ERR_BAD_ARGUMENT, "NULL argument");
  if (m->reads.size() != 2 * (size_t)n_pairs)
    return merr(ESG_ERR_BAD_ARGUMENT, "a paired mapping holds two read entries per pair");
  for (uint32_t p = 0; p < n_pairs; ++p)
    if (pairs[p].first_hit > n_pair_hits || pairs[p].n_hits > n_pair_hits - pairs[p].first_hit)
      return merr(ESG_ERR_BAD_ARGUMENT, "pair %u's hits run past the pair-hit array", p);
  for (uint32_t p = 0; p < n_pairs; ++p)
    if ((pairs[p].flags & ESG_PAIR_PROPER) && pairs[p].n_hits == 0)
      return merr(ESG_ERR_BAD_ARGUMENT, "pair %u is proper but has no pair hit", p);
  const uint64_t n_ops = m->ops.size(), n_md = m->md.size();
  for (uint64_t h = 0; h < n_pair_hits; ++h)
    for (const esg_hit& e : pair_hits[h].mates)
      if (e.alignment.ops_offset > n_ops || e.alignment.n_ops > n_ops - e.alignment.ops_offset ||
          e.md_offset > n_md || e.md_len > n_md - e.md_offset)
        return merr(ESG_ERR_BAD_ARGUMENT, "pair hit %llu's ops or MD run past their arrays",
                    (unsigned long long)h);
  for (uint64_t h = 0; h < n_pair_hits; ++h)
    for (const esg_hit& e : pair_hits[h].mates)
      if (const char* why = hit_inconsistency(e, m->ops.data()))
        return merr(ESG_ERR_BAD_ARGUMENT, "pair hit %llu, a mate: %s", (unsigned long long)h,
                    why);
  m->pairs.assign(pairs, pairs + n_pairs);
  m->pair_hits.assign(pair_hits, pair_hits + n_pair_hits);
  return ESG_OK;
}

const esg_read_mapping* esg_mapping_reads(const esg_mapping* m, uint32_t* n) {
  if (n) *n = m ? (uint32_t)m->reads.size() : 0u;
  return m ? m->reads.data() : nullptr;
}

const esg_hit* esg_mapping_hits(const esg_mapping* m, uint64_t* n) {
  if (n) *n = m ? m->hits.size() : 0u;
  return m ? m->hits.data() : nullptr;
}

const uint32_t* esg_mapping_ops(const esg_mapping* m, uint64_t* n) {
  if (n) *n = m ? m->ops.size() : 0u;
  return m ? m->ops.data() : nullptr;
}

const char* esg_mapping_md(const esg_mapping* m, uint64_t* n) {
  if (n) *n = m ? m->md.size() : 0u;
  return m ? m->md.data() : nullptr;
}

void esg_mapping_free(esg_mapping* m) { delete m; }

}  // extern "C"
