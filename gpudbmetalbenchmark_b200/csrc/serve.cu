// Serving loop: lanes of (context, worker thread) over a shared FIFO with admission by
// predicted device footprint. See gpudb_serve_* in include/gpudb_capi.h.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "engine.h"

namespace {

double now_ms() {
  using namespace std::chrono;
  return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

uint64_t pow2_at_least(uint64_t v, uint64_t lo) {
  uint64_t p = lo;
  while (p < v) p <<= 1;
  return p;
}

struct Ticket {
  gpudb_request* req = nullptr;
  double t_submit = 0, t_done = 0;
  uint64_t footprint = 0;
  bool done = false;
  bool heavy = false;   // a scan of a large table (the heavy lanes' class)
};

// A Q6/Q1 request over more than 2^24 rows: the scans that end a batch (about 0.3 ms for a
// Q1 and a Q6 over 60M rows). With heavy lanes configured, only those lanes take them.
constexpr uint64_t kHeavyRows = 1ull << 24;
bool heavy_request(const gpudb_request* r) {
  if ((r->pipeline != GPUDB_PIPE_Q6 && r->pipeline != GPUDB_PIPE_Q1) || !r->li) return false;
  const uint64_t end = r->row_end ? std::min<uint64_t>(r->row_end, r->li->n_rows) : r->li->n_rows;
  return end - std::min<uint64_t>(r->row_begin, end) > kHeavyRows;
}

}  // namespace

extern "C" uint64_t gpudb_request_footprint(const gpudb_request* r) {
  if (!r) return 0;
  switch (r->pipeline) {
    case GPUDB_PIPE_Q6: return 256;
    case GPUDB_PIPE_Q1: return 2048;
    case GPUDB_PIPE_Q3: {
      if (!r->q3) return 0;
      const uint64_t n_or = r->q3->od.n_rows, cap = pow2_at_least(2 * n_or, 2048);
      // bitmap + orders staging + hash table (16 B) + hit counters + top-k candidates
      return (uint64_t)(r->q3->cu.key_max / 8 + 64) + n_or * 8 + cap * 20 + (cap / 4096 + 1) * 64 * 16 * 2;
    }
    case GPUDB_PIPE_Q9: {
      if (!r->q9) return 0;
      const uint64_t ps = r->q9->ps.n_rows, cap = pow2_at_least(2 * ps, 1024);
      // part bitmap + supplier and year maps + partsupp staging + partsupp table + groups
      return (uint64_t)(r->q9->pa.key_max / 8 + 64) + (uint64_t)r->q9->su.key_max + (uint64_t)r->q9->od.key_max +
             ps * 4 + cap * 16 + 4096 * 12;
    }
    default: return 0;
  }
}

struct gpudb_server {
  gpudb_serve_config cfg{};
  std::vector<gpudb_ctx*> lanes;
  std::vector<std::thread> workers;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<uint64_t> queue;
  std::unordered_map<uint64_t, Ticket> tickets;
  uint64_t next_ticket = 1;
  uint64_t admitted_bytes = 0;
  bool closing = false;
  bool warming = false;
  gpudb_serve_stats stats{};

  // Completion of request `i` of the lane's running batch (under no lock).
  struct LaneRun {
    gpudb_server* s;
    std::vector<gpudb_request>* batch;
    std::vector<uint64_t>* ids;
    std::vector<char>* done;
  };
  static void on_done(void* arg, int32_t* sink) {
    LaneRun* r = static_cast<LaneRun*>(arg);
    const uintptr_t base = reinterpret_cast<uintptr_t>(&(*r->batch)[0].status), at = reinterpret_cast<uintptr_t>(sink);
    if (at < base || (at - base) % sizeof(gpudb_request)) return;
    const size_t i = (at - base) / sizeof(gpudb_request);
    if (i >= r->batch->size() || (*r->done)[i]) return;
    (*r->done)[i] = 1;
    r->s->complete((*r->ids)[i], (*r->batch)[i]);
  }

  void complete(uint64_t id, const gpudb_request& q) {
    const double t = now_ms();
    {
      std::lock_guard<std::mutex> lk(mu);
      Ticket& tk = tickets[id];
      tk.req->status = q.status;
      tk.req->q9_groups = q.q9_groups;
      tk.t_done = t;
      tk.done = true;
      admitted_bytes -= tk.footprint;
      stats.completed++;
      if (q.status != GPUDB_OK) stats.failed++;
    }
    cv_done.notify_all();
    cv_work.notify_all();
  }

  // Whether `lane` takes ticket `id`: every lane takes everything unless heavy lanes are
  // configured; then the last heavy_lanes lanes take the heavy requests, the others the rest.
  bool takes(size_t lane, uint64_t id) {
    const uint32_t h = cfg.heavy_lanes;
    if (h == 0 || h >= lanes.size()) return true;
    return tickets[id].heavy == (lane >= lanes.size() - h);
  }
  // The first queued request of the lane's class (queue.end() if none).
  std::deque<uint64_t>::iterator first_of(size_t lane) {
    auto it = queue.begin();
    while (it != queue.end() && !takes(lane, *it)) ++it;
    return it;
  }

  void work(size_t lane) {
    gpudb_ctx* ctx = lanes[lane];
    std::vector<gpudb_request> batch;
    std::vector<uint64_t> ids;
    std::vector<char> done;
    LaneRun run{this, &batch, &ids, &done};
    for (;;) {
      {
        std::unique_lock<std::mutex> lk(mu);
        auto ready = [&] {
          if (warming) return false;
          auto it = first_of(lane);
          return it != queue.end() && fits(tickets[*it].footprint);
        };
        cv_work.wait(lk, [&] { return closing || ready(); });
        if (closing && first_of(lane) == queue.end()) return;
        if (!ready()) continue;
        ids.clear();
        uint64_t bytes = 0;
        for (auto it = queue.begin(); it != queue.end() && ids.size() < cfg.max_batch;) {
          if (!takes(lane, *it)) { ++it; continue; }
          const uint64_t fp = tickets[*it].footprint;
          if (!ids.empty() && !fits(bytes + fp)) break;   // keep arrival order: stop at the first misfit
          bytes += fp;
          ids.push_back(*it);
          it = queue.erase(it);
        }
        admitted_bytes += bytes;
        stats.peak_admitted_bytes = std::max(stats.peak_admitted_bytes, admitted_bytes);
        stats.batches++;
        stats.max_batch_seen = std::max<uint64_t>(stats.max_batch_seen, ids.size());
        batch.clear();
        for (uint64_t id : ids) batch.push_back(*tickets[id].req);
      }
      done.assign(batch.size(), 0);
      // each request completes as soon as its own work has finished (hook), not at batch end
      ctx->on_done = &gpudb_server::on_done;
      ctx->on_done_arg = &run;
      gpudb_batch_run(ctx, batch.data(), (uint32_t)batch.size(), nullptr, nullptr);
      ctx->on_done = nullptr;
      ctx->on_done_arg = nullptr;
      for (size_t i = 0; i < batch.size(); i++)   // requests that failed before reaching the GPU
        if (!done[i]) { done[i] = 1; complete(ids[i], batch[i]); }
    }
  }

  bool fits(uint64_t bytes) const {
    return cfg.memory_budget == 0 || admitted_bytes + bytes <= cfg.memory_budget;
  }
};

extern "C" int gpudb_serve_open(const gpudb_serve_config* cfg, gpudb_server** out) {
  if (!cfg || !out || cfg->lanes < 1 || cfg->lanes > 16 || cfg->max_batch < 1) return GPUDB_E_INVALID;
  if (cfg->heavy_lanes && cfg->heavy_lanes >= cfg->lanes) return GPUDB_E_INVALID;
  *out = nullptr;
  gpudb_server* s = new gpudb_server();
  s->cfg = *cfg;
  for (uint32_t i = 0; i < cfg->lanes; i++) {
    gpudb_ctx* c = nullptr;
    int rc = gpudb_create(cfg->device, &c);
    if (rc != GPUDB_OK) {
      for (auto* l : s->lanes) gpudb_destroy(l);
      delete s;
      return rc;
    }
    s->lanes.push_back(c);
  }
  for (size_t i = 0; i < s->lanes.size(); i++) s->workers.emplace_back(&gpudb_server::work, s, i);
  *out = s;
  return GPUDB_OK;
}

extern "C" int gpudb_serve_warmup(gpudb_server* s, gpudb_request* reqs, uint32_t n) {
  if (!s || (n && !reqs)) return GPUDB_E_INVALID;
  std::unique_lock<std::mutex> lk(s->mu);
  if (!s->queue.empty() || s->admitted_bytes) return GPUDB_E_BUSY;   // only before traffic
  s->warming = true;   // workers leave their contexts alone meanwhile
  lk.unlock();
  std::vector<int> rcs(s->lanes.size(), GPUDB_OK);
  // every lane runs its own copy of the requests (copied before any lane starts)
  std::vector<std::vector<gpudb_request>> copies(s->lanes.size(), std::vector<gpudb_request>(reqs, reqs + n));
  std::vector<std::thread> th;
  for (size_t i = 0; i < s->lanes.size(); i++)
    th.emplace_back([&, i] {
      std::vector<gpudb_request>& copy = copies[i];
      // lanes other than the first write into outputs of their own: results are converted
      // in place, so two lanes must never share a result struct
      std::vector<gpudb_q6_result> o6(i ? n : 0);
      std::vector<gpudb_q1_result> o1(i ? n : 0);
      std::vector<gpudb_q3_result> o3(i ? n : 0);
      std::vector<std::vector<gpudb_q9_group>> o9(i ? n : 0);
      for (uint32_t k = 0; i && k < n; k++) {
        gpudb_request& q = copy[k];
        if (q.q6_out) q.q6_out = &o6[k];
        if (q.q1_out) q.q1_out = &o1[k];
        if (q.q3_out) q.q3_out = &o3[k];
        if (q.q9_out) {
          o9[k].resize(q.q9_capacity);
          q.q9_out = o9[k].data();
        }
      }
      rcs[i] = gpudb_batch_run(s->lanes[i], copy.data(), n, nullptr, nullptr);
      for (uint32_t k = 0; k < n && rcs[i] == GPUDB_OK; k++)
        if (copy[k].status != GPUDB_OK) rcs[i] = copy[k].status;
    });
  for (auto& t : th) t.join();
  for (uint32_t k = 0; k < n; k++) { reqs[k].status = copies[0][k].status; reqs[k].q9_groups = copies[0][k].q9_groups; }
  lk.lock();
  s->warming = false;
  lk.unlock();
  s->cv_work.notify_all();
  for (int rc : rcs)
    if (rc != GPUDB_OK) return rc;
  return GPUDB_OK;
}

extern "C" int gpudb_serve_submit(gpudb_server* s, gpudb_request* req, uint64_t* ticket) {
  if (!s || !req || !ticket) return GPUDB_E_INVALID;
  const uint64_t fp = gpudb_request_footprint(req);
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->closing) return GPUDB_E_CLOSED;
    if (s->cfg.memory_budget && fp > s->cfg.memory_budget) return GPUDB_E_BUSY;
    const uint64_t id = s->next_ticket++;
    Ticket& t = s->tickets[id];
    t.req = req;
    t.t_submit = now_ms();
    t.footprint = fp;
    t.heavy = heavy_request(req);
    s->queue.push_back(id);
    s->stats.submitted++;
    *ticket = id;
  }
  s->cv_work.notify_all();   // (with heavy lanes, only a lane of the request's class can take it)
  return GPUDB_OK;
}

extern "C" int gpudb_serve_wait(gpudb_server* s, uint64_t ticket, double timeout_ms, double* latency_ms) {
  if (!s) return GPUDB_E_INVALID;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->tickets.find(ticket);
  if (it == s->tickets.end()) return GPUDB_E_INVALID;
  const bool ok = s->cv_done.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms),
                                      [&] { return s->tickets[ticket].done; });
  if (!ok) return GPUDB_E_TIMEOUT;
  Ticket t = s->tickets[ticket];
  s->tickets.erase(ticket);
  if (latency_ms) *latency_ms = t.t_done - t.t_submit;
  return t.req->status;
}

extern "C" int gpudb_serve_stats_get(gpudb_server* s, gpudb_serve_stats* out) {
  if (!s || !out) return GPUDB_E_INVALID;
  std::lock_guard<std::mutex> lk(s->mu);
  *out = s->stats;
  return GPUDB_OK;
}

extern "C" int gpudb_serve_close(gpudb_server* s) {
  if (!s) return GPUDB_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->closing = true;
  }
  s->cv_work.notify_all();
  for (auto& w : s->workers) w.join();
  for (auto* l : s->lanes) gpudb_destroy(l);
  delete s;
  return GPUDB_OK;
}
