// z80b_serve.cpp -- serving loop over the C ABI: optimisation queries (a
// target plus its dead flags / dead registers) arrive one by one and are
// answered with the shortest equivalent, as z80opt target / SearchSingle
// would answer them, while other queries are on the device.
//
// Continuous batching at batch granularity: `workers` threads each own a
// context (its own stream and device buffers; the length-2 pair pool is
// shared per device).  A free worker takes every waiting query of one class
// up to max_batch and runs them as one first-found job, so new arrivals are
// admitted by the next free worker while earlier batches are still in
// flight and their work overlaps on the GPU.  A class is the candidate
// length cap (1 or 2 instructions) and whether the target alone already
// reads enough registers for an ExhaustiveCheck sweep of 2^32 states or
// more (a "giant": e.g. SET 1, D : SBC HL, BC : XOR (HL) : OR 0C0h sweeps
// 2^39 states, several seconds of the whole GPU).  With two or more
// workers, worker 0 serves giants first, one query per batch, on a
// low-priority stream, and the others serve every other query on
// high-priority streams; since the sweep kernel's blocks retire every few
// chunks, the block scheduler hands SMs to their kernels while a giant sweep
// runs.  Admission charges each query the device memory its batch holds for
// it (z80b::target_frontier_bytes: its lanes, survivor records at their
// bound for its target size and passes, pair slots, length-2 slots, rule
// records) against the budget, and a query waits while the in-flight total
// would exceed it.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <vector>

#include "../../include/z80b200.h"
#include "z80_tables.h"
#include "z80b_engine.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Pending {
  z80b_query q;
  Clock::time_point t_submit;
  uint32_t cand;    // candidate length cap of this query
  uint32_t klass;   // batch class: cand | giant << 2
  uint32_t flags;   // Z80B_ANSWER_* bits of its answer
  uint64_t bytes;   // device frontier its batch holds for it (admission charge)
};

// Rule records of one query in the batch's output (full and masked rule).
constexpr uint64_t kRuleBytes = 2 * sizeof(z80b_rule);

constexpr uint64_t kGiantStates = 1ull << 32;

}  // namespace

struct z80b_server {
  z80b_server_config cfg{};
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Pending> pending;
  std::deque<z80b_answer> done;
  uint64_t inflight_bytes = 0;
  bool stopping = false;
  std::vector<std::thread> workers;
  std::vector<z80b_ctx*> ctxs;
  z80b_server_stats stats{};
};

namespace {

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

// One running batch: answers leave as soon as z80b_search_cb reports a
// target final, so a slow target does not hold the others of its batch.
struct BatchRun {
  z80b_server* S;
  const std::vector<Pending>* batch;
  Clock::time_point t_start;
  std::vector<uint8_t> answered;
};

void on_target(void* user, uint32_t t, const z80b_rule* rules, uint32_t n) {
  BatchRun* b = static_cast<BatchRun*>(user);
  const Pending& p = (*b->batch)[t];
  const auto now = Clock::now();
  z80b_answer a;
  std::memset(&a, 0, sizeof a);
  a.id = p.q.id;
  a.status = Z80B_OK;
  a.batch_size = uint32_t(b->batch->size());
  a.queued_ms = ms_between(p.t_submit, b->t_start);
  a.service_ms = ms_between(b->t_start, now);
  a.latency_ms = ms_between(p.t_submit, now);
  a.flags = p.flags;
  for (uint32_t k = 0; k < n && k < 2; k++) a.rules[a.n_rules++] = rules[k];
  b->answered[t] = 1;
  {
    std::lock_guard<std::mutex> lk(b->S->mu);
    b->S->done.push_back(a);
    b->S->stats.answered++;
  }
  b->S->cv_done.notify_all();
}

// role: 0 any class (single worker), 1 giants first, 2 everything but giants
void worker_loop(z80b_server* S, z80b_ctx* ctx, int role) {
  std::vector<Pending> batch;
  std::vector<uint32_t> tg;
  std::vector<uint8_t> lens, dead, dregs;
  std::vector<z80b_rule> rules;
  for (;;) {
    batch.clear();
    uint32_t cand = 1;
    {
      std::unique_lock<std::mutex> lk(S->mu);
      // the oldest query this worker may take: its class is the batch's
      auto pick = [&]() -> const Pending* {
        const Pending* first_any = nullptr;
        for (const Pending& p : S->pending) {
          const bool giant = (p.klass & 4u) != 0;
          if (role == 2 && giant) continue;
          if (role == 1 && giant) return &p;
          if (!first_any) first_any = &p;
          if (role != 1) return first_any;
        }
        return first_any;
      };
      S->cv_work.wait(lk, [&] {
        const Pending* h = pick();
        return S->stopping || (h && S->inflight_bytes + h->bytes <= S->cfg.memory_budget);
      });
      const Pending* head = pick();
      if (!head) {
        if (S->stopping) return;  // stopping and nothing left for this worker
        continue;
      }
      cand = head->cand;
      const uint32_t klass = head->klass;
      const uint32_t cap = (klass & 4u) ? 1u : S->cfg.max_batch;  // giants run alone
      for (auto it = S->pending.begin(); it != S->pending.end() && batch.size() < cap;) {
        if (it->klass == klass && S->inflight_bytes + it->bytes <= S->cfg.memory_budget) {
          batch.push_back(*it);
          S->inflight_bytes += it->bytes;
          S->stats.peak_inflight_bytes = std::max(S->stats.peak_inflight_bytes, S->inflight_bytes);
          it = S->pending.erase(it);
        } else {
          ++it;
        }
      }
      if (!batch.empty()) {
        S->stats.batches++;
        S->stats.max_batch_seen = std::max<uint64_t>(S->stats.max_batch_seen, batch.size());
      }
    }
    if (batch.empty()) {  // nothing of this class fits the budget yet
      std::this_thread::sleep_for(std::chrono::milliseconds(1));
      continue;
    }
    const auto t_start = Clock::now();
    const uint32_t n = uint32_t(batch.size());
    tg.assign(size_t(n) * 4, 0);
    lens.resize(n);
    dead.resize(n);
    dregs.resize(n);
    for (uint32_t i = 0; i < n; i++) {
      std::memcpy(&tg[size_t(i) * 4], batch[i].q.target, sizeof batch[i].q.target);
      lens[i] = batch[i].q.len;
      dead[i] = batch[i].q.dead_flags;
      dregs[i] = batch[i].q.dead_regs;
    }
    z80b_job job{};
    job.targets = tg.data();
    job.target_lens = lens.data();
    job.dead_flags = dead.data();
    job.dead_regs = dregs.data();
    job.n_targets = n;
    job.target_stride = 4;
    job.max_cand_len = cand;
    job.mode = Z80B_MODE_FIRST;
    job.path = Z80B_PATH_BATCHED;
    rules.resize(size_t(n) * 2 + 16);
    uint64_t nr = 0;
    z80b_stats st{};
    BatchRun run{S, &batch, t_start, std::vector<uint8_t>(n, 0)};
    const int status = z80b_search_cb(ctx, &job, rules.data(), rules.size(), &nr, &st, on_target, &run);
    const auto t_end = Clock::now();
    // targets the callback did not answer (the batch failed)
    std::vector<z80b_answer> ans;
    for (uint32_t i = 0; i < n; i++) {
      if (run.answered[i]) continue;
      z80b_answer a;
      std::memset(&a, 0, sizeof a);
      a.id = batch[i].q.id;
      a.status = status == Z80B_OK ? Z80B_ESTATE : status;
      a.batch_size = n;
      a.queued_ms = ms_between(batch[i].t_submit, t_start);
      a.service_ms = ms_between(t_start, t_end);
      a.latency_ms = ms_between(batch[i].t_submit, t_end);
      a.flags = batch[i].flags;
      ans.push_back(a);
    }
    uint64_t held = 0;
    for (const Pending& p : batch) held += p.bytes;
    {
      std::lock_guard<std::mutex> lk(S->mu);
      S->inflight_bytes -= held;
      for (auto& a : ans) S->done.push_back(a);
      S->stats.answered += ans.size();
      S->stats.device_ms += st.device_ms;
      S->stats.errors += ans.size();
    }
    S->cv_done.notify_all();
    S->cv_work.notify_all();
  }
}

}  // namespace

extern "C" {

int z80b_server_start(const z80b_server_config* cfg, z80b_server** out) {
  if (!out) return Z80B_EINVAL;
  *out = nullptr;
  z80b_server_config c{};
  if (cfg) c = *cfg;
  if (c.workers <= 0) c.workers = 4;
  if (c.workers > 16) return Z80B_EINVAL;
  if (c.max_batch == 0) c.max_batch = 512;
  if (c.memory_budget == 0) c.memory_budget = 64ull << 30;
  if (c.max_cand_len == 0) c.max_cand_len = 2;
  if (c.max_cand_len > 2) return Z80B_EINVAL;
  z80b_server* S = new z80b_server();
  S->cfg = c;
  for (int w = 0; w < c.workers; w++) {
    z80b_ctx* ctx = nullptr;
    int st = z80b_init(c.device, &ctx);
    if (st != Z80B_OK) {
      for (auto* x : S->ctxs) z80b_destroy(x);
      delete S;
      return st;
    }
    S->ctxs.push_back(ctx);
  }
  for (size_t w = 0; w < S->ctxs.size(); w++) {
    const int role = S->ctxs.size() < 2 ? 0 : (w == 0 ? 1 : 2);
    z80b_set_option(S->ctxs[w], Z80B_OPT_STREAM_PRIORITY, role == 1 ? 1 : (role == 2 ? -1 : 0));
    S->workers.emplace_back(worker_loop, S, S->ctxs[w], role);
  }
  *out = S;
  return Z80B_OK;
}

int z80b_server_submit(z80b_server* S, const z80b_query* q, uint32_t n) {
  if (!S || (n && !q)) return Z80B_EINVAL;
  for (uint32_t i = 0; i < n; i++) {
    if (q[i].len < 1 || q[i].len > 4 || (q[i].dead_regs & ~0x3Fu)) return Z80B_EINVAL;
    for (uint32_t k = 0; k < q[i].len; k++)
      if ((q[i].target[k] & 0xFFFFu) >= Z80B_NUM_OPS) return Z80B_EINVAL;
    // a query whose frontier alone exceeds the budget could never be admitted
    const uint32_t cap = std::min<uint32_t>(uint32_t(q[i].len) - 1, S->cfg.max_cand_len);
    if (cap && z80b::target_frontier_bytes(q[i].target, int(q[i].len), int(cap), q[i].dead_flags || q[i].dead_regs) +
                       kRuleBytes > S->cfg.memory_budget)
      return Z80B_ECAPACITY;
  }
  const auto now = Clock::now();
  {
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->stopping) return Z80B_ESTATE;
    for (uint32_t i = 0; i < n; i++) {
      S->stats.submitted++;
      // SearchSingle's MaxCandLen is the target length - 1 (pkg/search/search.go:27-29);
      // the server searches at most max_cand_len (<= 2) and says so when it cut
      const uint32_t want = uint32_t(q[i].len) - 1;
      const uint32_t cap = std::min<uint32_t>(want, S->cfg.max_cand_len);
      const uint32_t flags = cap < want ? Z80B_ANSWER_TRUNCATED : 0u;
      if (cap == 0) {
        // a single instruction has no shorter equivalent (MaxCandLen = 0)
        z80b_answer a;
        std::memset(&a, 0, sizeof a);
        a.id = q[i].id;
        a.status = Z80B_OK;
        S->done.push_back(a);
        S->stats.answered++;
        continue;
      }
      const bool giant =
          z80b::sweep_for(z80b::seq_reads(q[i].target, int(q[i].len))).states >= kGiantStates;
      const uint64_t bytes =
          z80b::target_frontier_bytes(q[i].target, int(q[i].len), int(cap), q[i].dead_flags || q[i].dead_regs) +
          kRuleBytes;
      S->pending.push_back(Pending{q[i], now, cap, cap | (giant ? 4u : 0u), flags, bytes});
    }
  }
  S->cv_work.notify_all();
  S->cv_done.notify_all();
  return Z80B_OK;
}

int z80b_server_poll(z80b_server* S, z80b_answer* out, uint32_t cap, uint32_t* n, int timeout_ms) {
  if (!S || !n || (cap && !out)) return Z80B_EINVAL;
  std::unique_lock<std::mutex> lk(S->mu);
  if (S->done.empty() && timeout_ms > 0)
    S->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), [&] { return !S->done.empty(); });
  uint32_t k = 0;
  while (k < cap && !S->done.empty()) {
    out[k++] = S->done.front();
    S->done.pop_front();
  }
  *n = k;
  return Z80B_OK;
}

int z80b_server_get_stats(z80b_server* S, z80b_server_stats* out) {
  if (!S || !out) return Z80B_EINVAL;
  std::lock_guard<std::mutex> lk(S->mu);
  *out = S->stats;
  out->pending = S->pending.size();
  out->inflight_bytes = S->inflight_bytes;
  return Z80B_OK;
}

int z80b_server_stop(z80b_server* S) {
  if (!S) return Z80B_EINVAL;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stopping = true;
  }
  S->cv_work.notify_all();
  for (auto& t : S->workers) t.join();
  for (auto* c : S->ctxs) z80b_destroy(c);
  delete S;
  return Z80B_OK;
}

}  // extern "C"
