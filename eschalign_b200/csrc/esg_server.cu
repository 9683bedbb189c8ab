// esg_server.cu -- request queue over resident scorers (host only).
//
// Each scorer slot has a worker thread that owns every call on its scorer.
// The worker takes the slot's waiting requests with one strand flag, up to
// max_batch_reads reads, as one batch (continuous batching: whatever has
// arrived while earlier batches ran), plans it straight from the requests'
// copies (no staging copy), admits it against device memory, submits it and
// keeps up to max_inflight batches queued on the scorer's stream; finishing
// the oldest scatters its per-read results back to the requests.
//
// Admission: under the server lock, a batch of B device bytes is admitted
// when B fits the free device memory (cudaMemGetInfo) plus the spare memory
// of the scorer's pool, less the headroom, and, with a budget, the bytes of
// admitted batches plus B stay within it.  Otherwise the worker first
// finishes its own oldest batch, or with none in flight waits for other
// slots to release memory.  A batch that could not fit even on an idle
// device (B above the budget, or above total memory less the headroom) is
// refused: its requests end with ESG_ERR_OUT_OF_MEMORY.  All of this is
// host logic; nothing waits on the device except esg_finish.
#include "../../include/eschalign_b200.h"
#include "esg_internal.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdarg>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

extern "C" void esg_internal_set_error(esg_status st, const char* msg);

namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

struct Request {
  uint64_t id = 0;
  uint32_t slot = 0;
  uint32_t flags = 0;
  uint32_t n_reads = 0;
  std::vector<uint8_t> codes;
  std::vector<uint64_t> off;
  std::vector<uint32_t> len;
  // results, filled piece by piece
  std::vector<esg_read_result> results;
  std::vector<uint32_t> ties;
  uint32_t pieces_left = 0;
  std::vector<std::pair<uint32_t, uint64_t>> cuts;  // piece ends (k1) and cells
  uint32_t next_piece = 0;                          // the next piece to queue
  esg_status status = ESG_OK;
  std::string error;
  bool done = false;
  bool started = false;
  Clock::time_point t_submit, t_device, t_done;
  uint32_t batch_reads = 0, batch_requests = 0;
};

using RequestP = std::shared_ptr<Request>;

// A request's reads k0 .. k1 - 1: the unit of batching.  A request whose
// cells exceed max_batch_cells is cut into several pieces, so no batch runs
// much longer than that.  Only a request's next piece waits in the queue,
// and the one after it joins the back when it is taken: requests share the
// scorer round-robin, and a small one is not stuck behind a giant.
struct Piece {
  RequestP r;
  uint32_t k0 = 0, k1 = 0;
  uint64_t cells = 0;
  uint32_t reads() const { return k1 - k0; }
};

struct InFlight {
  esg_batch* batch = nullptr;
  std::vector<Piece> pieces;
  uint64_t bytes = 0;
  uint32_t n_reads = 0;
};

struct Slot {
  esg_scorer* scorer = nullptr;
  uint32_t cap = 8;
  int device = 0;
  uint64_t panel_bases = 0;
  std::deque<Piece> pending;
  std::deque<Piece> solo;  // go next, one at a time (their batch with others did not fit)
  std::deque<InFlight> inflight;
  std::condition_variable cv;
  std::thread worker;
};

}  // namespace

struct esg_server {
  esg_server_options opt{};
  std::mutex mu;
  std::condition_variable done_cv;   // a request finished, or memory was released
  std::vector<std::unique_ptr<Slot>> slots;
  std::unordered_map<uint64_t, RequestP> requests;
  uint64_t next_id = 1;
  bool stop = false;
  esg_server_stats stats{};
};

namespace {

esg_status set_err(esg_status st, const char* fmt, ...) __attribute__((format(printf, 2, 3)));
esg_status set_err(esg_status st, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  esg_internal_set_error(st, buf);
  return st;
}

// The request's next piece, if any, to the back of the slot's queue (lock
// held by the caller).
void queue_next(Slot& s, const RequestP& r) {
  if (r->next_piece >= r->cuts.size()) return;
  Piece p;
  p.r = r;
  p.k0 = r->next_piece ? r->cuts[r->next_piece - 1].first : 0;
  p.k1 = r->cuts[r->next_piece].first;
  p.cells = r->cuts[r->next_piece].second;
  r->next_piece++;
  s.pending.push_back(p);
}

// A piece failed: its request fails (once).  Lock held by the caller.
void fail_pieces(esg_server* sv, std::vector<Piece>& ps, esg_status st, const std::string& msg) {
  const auto now = Clock::now();
  for (auto& p : ps) {
    Request& r = *p.r;
    if (r.done) continue;
    r.status = st;
    r.error = msg;
    r.done = true;
    r.t_done = now;
    if (!r.started) r.t_device = now;
    sv->stats.completed++;
    if (st == ESG_ERR_OUT_OF_MEMORY) sv->stats.refused++;
  }
}

// Finish the slot's oldest batch and scatter its results (lock not held).
void finish_oldest(esg_server* sv, Slot& s) {
  InFlight f;
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    if (s.inflight.empty()) return;  // (woken for pieces that turned out dead)
    f = std::move(s.inflight.front());
    s.inflight.pop_front();
  }
  std::vector<esg_read_result> res(f.n_reads ? f.n_reads : 1);
  std::vector<uint32_t> ties((size_t)(f.n_reads ? f.n_reads : 1) * s.cap);
  const esg_status st = esg_finish(s.scorer, f.batch, res.data(), ties.data(), nullptr);
  const std::string msg = st == ESG_OK ? std::string() : std::string(esg_last_error());
  esg_batch_free(f.batch);
  std::lock_guard<std::mutex> lk(sv->mu);
  if (st != ESG_OK) {
    fail_pieces(sv, f.pieces, st, msg);
  } else {
    const auto now = Clock::now();
    size_t at = 0;
    for (auto& p : f.pieces) {
      Request& r = *p.r;
      const uint32_t n = p.reads();
      if (!r.done) {
        std::copy(res.begin() + at, res.begin() + at + n, r.results.begin() + p.k0);
        std::copy(ties.begin() + at * s.cap, ties.begin() + (at + n) * s.cap,
                  r.ties.begin() + (size_t)p.k0 * s.cap);
        if (--r.pieces_left == 0) {
          r.status = ESG_OK;
          r.done = true;
          r.t_done = now;
          r.codes.clear();
          r.codes.shrink_to_fit();
          sv->stats.completed++;
        }
      }
      at += n;
    }
  }
  sv->stats.bytes_in_flight -= f.bytes;
  sv->done_cv.notify_all();
  for (auto& other : sv->slots) other->cv.notify_all();
}

void worker(esg_server* sv, Slot* sp) {
  Slot& s = *sp;
  cudaSetDevice(s.device);
  const uint32_t max_reads = sv->opt.max_batch_reads;
  const uint64_t max_cells = sv->opt.max_batch_cells;
  const uint32_t max_inflight = sv->opt.max_inflight;
  for (;;) {
    std::vector<Piece> group;
    uint32_t flags = 0, n_reads = 0;
    {
      std::unique_lock<std::mutex> lk(sv->mu);
      s.cv.wait(lk, [&] {
        return sv->stop ||
               ((!s.pending.empty() || !s.solo.empty()) && s.inflight.size() < max_inflight) ||
               !s.inflight.empty();
      });
      if (sv->stop && s.inflight.empty()) {
        std::vector<Piece> left(s.pending.begin(), s.pending.end());
        left.insert(left.end(), s.solo.begin(), s.solo.end());
        s.pending.clear();
        s.solo.clear();
        fail_pieces(sv, left, ESG_ERR_BAD_ARGUMENT, "server stopped");
        sv->done_cv.notify_all();
        return;
      }
      // pieces of a request that already failed do not run
      auto dead = [](const Piece& p) { return p.r->done; };
      s.pending.erase(std::remove_if(s.pending.begin(), s.pending.end(), dead), s.pending.end());
      s.solo.erase(std::remove_if(s.solo.begin(), s.solo.end(), dead), s.solo.end());
      if (!sv->stop && !s.solo.empty() && s.inflight.size() < max_inflight) {
        // a piece whose batch with others did not fit: alone this time
        group.push_back(s.solo.front());
        s.solo.pop_front();
        flags = group[0].r->flags;
        n_reads = group[0].reads();
      } else if (!sv->stop && !s.pending.empty() && s.inflight.size() < max_inflight) {
        // the waiting pieces with the first one's strand flag, in order, up
        // to the batch's read and cell caps
        flags = s.pending.front().r->flags;
        uint64_t cells = 0;
        for (auto it = s.pending.begin(); it != s.pending.end();) {
          if (it->r->flags != flags) {
            ++it;
            continue;
          }
          if (!group.empty() &&
              (n_reads + it->reads() > max_reads || cells + it->cells > max_cells))
            break;
          n_reads += it->reads();
          cells += it->cells;
          group.push_back(*it);
          const RequestP r = it->r;
          it = s.pending.erase(it);
          const size_t at = it - s.pending.begin();
          queue_next(s, r);  // at the back: behind what already waits
          it = s.pending.begin() + at;
        }
      }
    }
    if (group.empty()) {  // nothing to start: finish the oldest batch
      finish_oldest(sv, s);
      continue;
    }
    // plan the batch straight from the requests' copies
    std::vector<const uint8_t*> ptrs;
    std::vector<uint32_t> lens;
    ptrs.reserve(n_reads);
    lens.reserve(n_reads);
    for (auto& p : group)
      for (uint32_t k = p.k0; k < p.k1; ++k) {
        ptrs.push_back(p.r->codes.data() + p.r->off[k]);
        lens.push_back(p.r->len[k]);
      }
    esg_batch* b = nullptr;
    esg_status st = esg_internal_prepare_ptrs(s.scorer, ptrs.data(), lens.data(), n_reads, flags, &b);
    if (st != ESG_OK) {
      const std::string msg = esg_last_error();
      std::lock_guard<std::mutex> lk(sv->mu);
      fail_pieces(sv, group, st, msg);
      sv->done_cv.notify_all();
      continue;
    }
    esg_batch_stats bst{};
    esg_batch_stats_get(b, &bst);
    const uint64_t need = bst.device_bytes;
    // admission
    bool refused = false;
    // with nothing of the server's in flight, memory held outside the server
    // may never come back: give up after this long
    const auto give_up = Clock::now() + std::chrono::seconds(5);
    for (;;) {
      size_t free_b = 0, total_b = 0;
      cudaMemGetInfo(&free_b, &total_b);
      const uint64_t spare = esg_internal_pool_spare(s.scorer);
      std::unique_lock<std::mutex> lk(sv->mu);
      const uint64_t head = sv->opt.memory_headroom;
      const uint64_t budget = sv->opt.memory_budget;
      const uint64_t ceiling = budget ? budget : (total_b > head ? total_b - head : 0);
      if (need > ceiling) {
        refused = true;
        break;
      }
      const bool mem_ok = (uint64_t)free_b + spare >= need + head;
      const bool budget_ok = !budget || sv->stats.bytes_in_flight + need <= budget;
      if (mem_ok && budget_ok) {
        sv->stats.bytes_in_flight += need;
        sv->stats.peak_bytes_in_flight =
            std::max(sv->stats.peak_bytes_in_flight, sv->stats.bytes_in_flight);
        break;
      }
      sv->stats.admission_waits++;
      if (!s.inflight.empty()) {  // release our own memory first
        lk.unlock();
        finish_oldest(sv, s);
        continue;
      }
      if (sv->stats.bytes_in_flight == 0 && Clock::now() > give_up) {
        refused = true;  // memory held outside the server did not come back
        break;
      }
      // other slots' batches hold the memory (or, with none, something
      // outside the server): wait for a release and look again
      sv->done_cv.wait_for(lk, std::chrono::milliseconds(2));
    }
    if (refused && group.size() > 1) {
      // too big together: one at a time, in order (only a piece that cannot
      // fit by itself is refused)
      esg_batch_free(b);
      std::lock_guard<std::mutex> lk(sv->mu);
      for (size_t k = group.size(); k-- > 0;) s.solo.push_front(group[k]);
      continue;
    }
    if (refused) {
      esg_batch_free(b);
      std::lock_guard<std::mutex> lk(sv->mu);
      char msg[256];
      snprintf(msg, sizeof msg,
               "batch of %u reads needs %llu device bytes, above what admission allows",
               n_reads, (unsigned long long)need);
      fail_pieces(sv, group, ESG_ERR_OUT_OF_MEMORY, msg);
      sv->done_cv.notify_all();
      continue;
    }
    st = esg_submit(s.scorer, b);
    std::lock_guard<std::mutex> lk(sv->mu);
    if (st != ESG_OK) {
      const std::string msg = esg_last_error();
      esg_batch_free(b);
      sv->stats.bytes_in_flight -= need;
      fail_pieces(sv, group, st, msg);
      sv->done_cv.notify_all();
      continue;
    }
    const auto now = Clock::now();
    for (auto& p : group) {
      Request& r = *p.r;
      if (!r.started) {
        r.started = true;
        r.t_device = now;
        r.batch_reads = n_reads;
        r.batch_requests = (uint32_t)group.size();
      }
    }
    esg_batch_stats_get(b, &bst);  // the kernel count is known once submitted
    sv->stats.batches++;
    sv->stats.cells += bst.cells;
    sv->stats.kernels += bst.kernels;
    InFlight f;
    f.batch = b;
    f.pieces = std::move(group);
    f.bytes = need;
    f.n_reads = n_reads;
    s.inflight.push_back(std::move(f));
  }
}

}  // namespace

extern "C" {

esg_status esg_server_new(const esg_server_options* options, esg_server** out) {
  if (!out) return set_err(ESG_ERR_BAD_ARGUMENT, "out is NULL");
  *out = nullptr;
  auto* sv = new esg_server();
  if (options) sv->opt = *options;
  if (!sv->opt.max_batch_reads) sv->opt.max_batch_reads = 262144;
  if (!sv->opt.max_batch_cells) sv->opt.max_batch_cells = 150000000000ull;
  if (!sv->opt.max_inflight) sv->opt.max_inflight = 2;
  if (!sv->opt.memory_headroom) sv->opt.memory_headroom = 256ull << 20;
  *out = sv;
  return ESG_OK;
}

esg_status esg_server_add_scorer(esg_server* sv, esg_scorer* sc, uint32_t* slot) {
  if (!sv || !sc || !slot) return set_err(ESG_ERR_BAD_ARGUMENT, "NULL argument");
  esg_info info{};
  esg_status st = esg_scorer_info(sc, &info);
  if (st != ESG_OK) return st;
  std::lock_guard<std::mutex> lk(sv->mu);
  for (auto& s : sv->slots)
    if (s->scorer == sc) return set_err(ESG_ERR_BAD_ARGUMENT, "scorer already added");
  auto s = std::make_unique<Slot>();
  s->scorer = sc;
  s->cap = esg_internal_tie_capacity(sc);
  s->panel_bases = esg_internal_panel_bases(sc);
  s->device = esg_internal_device(sc);
  *slot = (uint32_t)sv->slots.size();
  Slot* raw = s.get();
  sv->slots.push_back(std::move(s));
  raw->worker = std::thread(worker, sv, raw);
  return ESG_OK;
}

esg_status esg_server_submit(esg_server* sv, uint32_t slot, const uint8_t* codes,
                             const uint64_t* off, const uint32_t* len, uint32_t n_reads,
                             uint32_t flags, uint64_t* ticket) {
  if (!sv || !ticket) return set_err(ESG_ERR_BAD_ARGUMENT, "NULL argument");
  if (flags & ~ESG_BOTH_STRANDS)
    return set_err(ESG_ERR_BAD_ARGUMENT, "server requests take 0 or ESG_BOTH_STRANDS, got 0x%x",
                   flags);
  if (n_reads && (!off || !len)) return set_err(ESG_ERR_BAD_ARGUMENT, "off/len must not be NULL");
  if (n_reads >= (1u << 29)) return set_err(ESG_ERR_BAD_ARGUMENT, "too many reads (%u)", n_reads);
  auto r = std::make_shared<Request>();
  r->flags = flags;
  r->n_reads = n_reads;
  uint64_t total = 0;
  for (uint32_t k = 0; k < n_reads; ++k) total += len[k];
  if (total && !codes) return set_err(ESG_ERR_BAD_ARGUMENT, "codes must not be NULL");
  r->codes.resize(total ? total : 1);
  r->off.resize(n_reads);
  r->len.assign(len, len + n_reads);
  uint64_t pos = 0;
  for (uint32_t k = 0; k < n_reads; ++k) {
    r->off[k] = pos;
    if (len[k]) memcpy(r->codes.data() + pos, codes + off[k], len[k]);
    pos += len[k];
  }
  std::lock_guard<std::mutex> lk(sv->mu);
  if (slot >= sv->slots.size()) return set_err(ESG_ERR_BAD_ARGUMENT, "no scorer slot %u", slot);
  if (sv->stop) return set_err(ESG_ERR_BAD_ARGUMENT, "server stopped");
  Slot& sl = *sv->slots[slot];
  r->id = sv->next_id++;
  r->slot = slot;
  r->results.resize(n_reads);
  r->ties.resize((size_t)n_reads * sl.cap);
  // pieces of at most max_batch_cells cells (at least one read each)
  const uint64_t per_base = sl.panel_bases * ((flags & ESG_BOTH_STRANDS) ? 2 : 1);
  uint32_t k0 = 0;
  uint64_t cells = 0;
  for (uint32_t k = 0; k < n_reads; ++k) {
    const uint64_t c = (uint64_t)len[k] * per_base;
    if (k > k0 && cells + c > sv->opt.max_batch_cells) {
      r->cuts.push_back({k, cells});
      k0 = k;
      cells = 0;
    }
    cells += c;
  }
  r->cuts.push_back({n_reads, cells});  // the last (for an empty request, the only) piece
  r->pieces_left = (uint32_t)r->cuts.size();
  r->t_submit = Clock::now();
  sv->requests[r->id] = r;
  queue_next(sl, r);
  sv->stats.requests++;
  sv->slots[slot]->cv.notify_all();
  *ticket = r->id;
  return ESG_OK;
}

esg_status esg_server_wait(esg_server* sv, uint64_t ticket, int32_t timeout_ms,
                           esg_read_result* results, uint32_t* ties, esg_request_timing* timing) {
  if (!sv) return set_err(ESG_ERR_BAD_ARGUMENT, "NULL server");
  std::unique_lock<std::mutex> lk(sv->mu);
  auto it = sv->requests.find(ticket);
  if (it == sv->requests.end()) return set_err(ESG_ERR_BAD_ARGUMENT, "unknown ticket %llu",
                                               (unsigned long long)ticket);
  RequestP r = it->second;
  auto ready = [&] { return r->done; };
  if (timeout_ms < 0) {
    sv->done_cv.wait(lk, ready);
  } else if (!sv->done_cv.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready)) {
    return set_err(ESG_ERR_TIMEOUT, "request %llu not done after %d ms",
                   (unsigned long long)ticket, timeout_ms);
  }
  sv->requests.erase(it);
  const uint32_t cap = sv->slots[r->slot]->cap;
  lk.unlock();
  if (timing) {
    timing->queued_ms = ms_between(r->t_submit, r->t_device);
    timing->total_ms = ms_between(r->t_submit, r->t_done);
    timing->batch_reads = r->batch_reads;
    timing->batch_requests = r->batch_requests;
  }
  if (r->status != ESG_OK) return set_err(r->status, "%s", r->error.c_str());
  if (results && r->n_reads) memcpy(results, r->results.data(), (size_t)r->n_reads * 16);
  if (ties && r->n_reads) memcpy(ties, r->ties.data(), (size_t)r->n_reads * cap * 4);
  esg_internal_set_error(ESG_OK, "");
  return ESG_OK;
}

esg_status esg_server_stats_get(esg_server* sv, esg_server_stats* out) {
  if (!sv || !out) return set_err(ESG_ERR_BAD_ARGUMENT, "NULL argument");
  std::lock_guard<std::mutex> lk(sv->mu);
  *out = sv->stats;
  return ESG_OK;
}

void esg_server_free(esg_server* sv) {
  if (!sv) return;
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->stop = true;
    for (auto& s : sv->slots) s->cv.notify_all();
  }
  // a stopping worker finishes its batches on the device, fails what is
  // still queued, and returns
  for (auto& s : sv->slots)
    if (s->worker.joinable()) s->worker.join();
  delete sv;
}

}  // extern "C"
