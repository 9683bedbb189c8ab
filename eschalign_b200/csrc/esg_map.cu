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
#include <memory>
#include <string>
#include <thread>
#include <vector>

extern "C" void esg_internal_set_error(esg_status st, const char* msg);

struct esg_mapping {
  std::vector<esg_read_mapping> reads;
  std::vector<esg_hit> hits;
  std::vector<uint32_t> ops;
  std::vector<char> md;
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
  char num[16];
  auto letter = [&](uint32_t jj) { return rl ? upper(rl[jj]) : kLetter[r[jj] > 4 ? 4 : r[jj]]; };
  auto flush = [&]() {
    const int w = snprintf(num, sizeof num, "%u", run);
    md.append(num, (size_t)w);
    run = 0;
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

extern "C" {

esg_status esg_map_reads(esg_scorer* sc, const uint8_t* codes, const uint64_t* off,
                         const uint32_t* len, uint32_t n_reads, const esg_map_options* o,
                         const uint8_t* ref_letters, const uint64_t* ref_letter_off,
                         esg_mapping** out) {
  if (!sc || !o || !out) return merr(ESG_ERR_BAD_ARGUMENT, "NULL scorer, options or out");
  *out = nullptr;
  if (n_reads && (!off || !len)) return merr(ESG_ERR_BAD_ARGUMENT, "off/len must not be NULL");
  if (o->both_strands > 1 || o->reserved)
    return merr(ESG_ERR_BAD_ARGUMENT, "both_strands must be 0 or 1, reserved 0");
  if (ref_letters && !ref_letter_off)
    return merr(ESG_ERR_BAD_ARGUMENT, "ref_letters needs ref_letter_off");
  uint64_t total = 0;
  for (uint32_t k = 0; k < n_reads; ++k) total += len[k];
  if (total && !codes) return merr(ESG_ERR_BAD_ARGUMENT, "codes must not be NULL");

  esg_internal_panel P{};
  esg_internal_panel_of(sc, &P);
  const uint32_t cap = esg_internal_tie_capacity(sc);
  const uint32_t flags = o->both_strands ? ESG_BOTH_STRANDS : 0u;

  // --- score: the fused reduction
  BatchGuard g;
  esg_status st = esg_prepare(sc, codes, off, len, n_reads, flags, &g.b);
  if (st != ESG_OK) return st;
  if ((st = esg_submit(sc, g.b)) != ESG_OK) return st;
  std::vector<esg_read_result> res(std::max<uint32_t>(n_reads, 1));
  std::vector<uint32_t> ties(std::max<size_t>((size_t)n_reads * cap, 1));
  if ((st = esg_finish(sc, g.b, res.data(), ties.data(), nullptr)) != ESG_OK) return st;

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
      (st = esg_internal_align_batch(sc, g.b, jobs.data(), (uint32_t)jobs.size(), al.data(),
                                     &ops)) != ESG_OK)
    return st;

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
  *out = m.release();
  esg_internal_set_error(ESG_OK, "");
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
