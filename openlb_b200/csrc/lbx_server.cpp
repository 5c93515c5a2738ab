// Native continuous-batching request loop (include/lbx_server.h): host C++ only, no CUDA code.
//
// One std::thread per server runs the loop; submissions, cancellations and record reads come
// from other threads and meet the loop under one mutex.  The engine (the ensemble, or a
// caller's) is touched by the loop thread alone, so its calls need no locking of their own.
#include "../../include/lbx_server.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <limits>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <unordered_set>
#include <vector>

namespace lbx {
int set_error(int code, const std::string& msg);  // lbx_api.cu: the message lbx_last_error returns
}

namespace {

using Clock = std::chrono::steady_clock;
constexpr double kNaN = std::numeric_limits<double>::quiet_NaN();

struct Item {
  lbx_server_request req;
  int64_t seq;  // submission order: ties of arrival time keep it
};

struct Active {
  Item item;
  lbx_server_record rec;
};

}  // namespace

struct lbx_server_s {
  lbx_server_engine eng{};
  void* ctx = nullptr;
  lbx_server_config cfg{};
  lbx_server_finish_fn onFinish = nullptr;
  void* onFinishUser = nullptr;
  // for lbx_server_create: the bound ensemble and stream (ctx points here)
  lbx_ensemble ens = nullptr;
  void* stream = nullptr;

  std::mutex mu;
  std::condition_variable wake;      // the loop: submissions, cancellations, close, stop
  std::condition_variable doneCv;    // waiters: the loop ended
  std::deque<Item> pending;          // submitted, arrival not reached (sorted by arrival, seq)
  std::deque<Item> waiting;          // arrived, not admitted yet
  std::unordered_map<int32_t, Active> active;  // by slot
  std::deque<lbx_server_record> done;
  std::unordered_set<int64_t> cancelRequests;  // ids of running requests to cancel
  int64_t seq = 0, submitted = 0, finished = 0;
  int64_t runs = 0, steps = 0, shortRuns = 0, longRuns = 0;
  double busy = 0.0;
  bool closed = false, started = false, stop = false, ended = false;
  int status = LBX_OK;
  std::string error;
  std::thread th;
  Clock::time_point t0;
  double virtualNow = 0.0;  // realtime == 0
  double stepSeconds = 0.0; // measured seconds per step of the last run (for the chunk choice)

  double now_locked() const {
    if (!started) return 0.0;
    if (cfg.realtime) return std::chrono::duration<double>(Clock::now() - t0).count();
    return virtualNow;
  }
  void loop();
  void finish_locked(Active& a, int32_t state, int64_t steps, double residual, double t);
};

namespace {

int32_t ens_admit(void* ctx, const lbx_ensemble_request* req, int32_t* slot) {
  auto* s = static_cast<lbx_server_s*>(ctx);
  return lbx_ensemble_admit(s->ens, req, slot);
}
int32_t ens_run(void* ctx, int32_t steps) {
  auto* s = static_cast<lbx_server_s*>(ctx);
  return lbx_ensemble_run(s->ens, steps, s->stream);
}
int32_t ens_statuses(void* ctx, lbx_ensemble_status* out, int32_t n) {
  auto* s = static_cast<lbx_server_s*>(ctx);
  return lbx_ensemble_statuses(s->ens, out, n, s->stream);
}
int32_t ens_retire(void* ctx, int32_t slot) {
  auto* s = static_cast<lbx_server_s*>(ctx);
  return lbx_ensemble_retire(s->ens, slot);
}

int check_config(const lbx_server_config* cfg) {
  if (!cfg) return lbx::set_error(LBX_ERR_INVALID, "config is null");
  if (cfg->min_chunk < 1 || cfg->max_chunk < cfg->min_chunk)
    return lbx::set_error(LBX_ERR_INVALID, "need 1 <= min_chunk <= max_chunk");
  return LBX_OK;
}

lbx_server_record blank_record(const Item& it) {
  lbx_server_record r{};
  r.id = it.req.id;
  r.cells = int64_t(it.req.request.core[0]) * it.req.request.core[1] * std::max(1, it.req.request.core[2]);
  r.arrival = it.req.arrival;
  r.admitted = kNaN;
  r.finished = kNaN;
  r.steps = 0;
  r.state = LBX_SERVER_REJECTED;
  r.slot = -1;
  r.residual = kNaN;
  return r;
}

}  // namespace

void lbx_server_s::finish_locked(Active& a, int32_t state, int64_t nsteps, double residual, double t) {
  a.rec.state = state;
  a.rec.steps = nsteps;
  a.rec.residual = residual;
  a.rec.finished = t;
  done.push_back(a.rec);
  ++finished;
}

// The loop.  It holds the mutex except while it calls the engine (admission, run, statuses,
// retirement) or the finish callback, so submissions never wait for a GPU run.
void lbx_server_s::loop() {
  std::unique_lock<std::mutex> lk(mu);
  std::vector<lbx_ensemble_status> st(size_t(std::max(eng.slots, 1)));
  auto fail_loop = [&](int code, const std::string& where) {
    status = code;
    error = where;
  };
  while (!stop) {
    double t = now_locked();
    // 1. arrivals
    while (!pending.empty() && pending.front().req.arrival <= t) {
      waiting.push_back(pending.front());
      pending.pop_front();
    }
    // cancellations of waiting requests
    if (!cancelRequests.empty()) {
      for (auto it = waiting.begin(); it != waiting.end();) {
        if (cancelRequests.erase(it->req.id)) {
          lbx_server_record r = blank_record(*it);
          r.state = LBX_SERVER_CANCELLED;
          r.finished = t;
          done.push_back(r);
          ++finished;
          it = waiting.erase(it);
        } else {
          ++it;
        }
      }
    }
    // 2. admission, first fit in arrival order (the queue stays in place meanwhile, so a
    //    cancellation arriving during admission still finds its request)
    if (!waiting.empty()) {
      std::vector<Item> admitList(waiting.begin(), waiting.end());
      lk.unlock();
      std::vector<std::pair<int64_t, int32_t>> admitted;  // (seq, slot)
      std::vector<int64_t> rejected;                      // seq
      for (const Item& it : admitList) {
        int32_t slot = -1;
        const int rc = eng.admit(ctx, &it.req.request, &slot);
        if (rc == LBX_OK) admitted.emplace_back(it.seq, slot);
        else if (rc != LBX_ERR_OUT_OF_MEMORY) rejected.push_back(it.seq);
      }
      lk.lock();
      t = now_locked();
      for (auto it = waiting.begin(); it != waiting.end();) {
        auto a = std::find_if(admitted.begin(), admitted.end(), [&](const auto& p) { return p.first == it->seq; });
        const bool rej = std::find(rejected.begin(), rejected.end(), it->seq) != rejected.end();
        if (a != admitted.end()) {
          Active act{*it, blank_record(*it)};
          act.rec.state = LBX_SLOT_RUNNING;
          act.rec.admitted = t;
          act.rec.slot = a->second;
          active[a->second] = act;
        } else if (rej) {
          lbx_server_record r = blank_record(*it);
          r.finished = t;
          done.push_back(r);
          ++finished;
        } else {
          ++it;
          continue;
        }
        it = waiting.erase(it);
      }
    }
    if (active.empty()) {
      if (!waiting.empty()) {
        // nothing was admitted, so every waiting request was refused by an empty engine: none of
        // them will ever fit (submissions made meanwhile went to `pending`, not here)
        for (const Item& it : waiting) {
          lbx_server_record r = blank_record(it);
          r.finished = t;
          done.push_back(r);
          ++finished;
        }
        waiting.clear();
        continue;
      }
      if (pending.empty()) {
        if (closed) break;
        wake.wait_for(lk, std::chrono::milliseconds(20));
        continue;
      }
      const double gap = pending.front().req.arrival - t;
      if (cfg.realtime) {
        if (gap > 0) wake.wait_for(lk, std::chrono::duration<double>(std::min(gap, 0.05)));
      } else {
        virtualNow = std::max(virtualNow, pending.front().req.arrival);
      }
      continue;
    }
    // 3. one run; the chunk adapts to what waits
    int chunk = cfg.max_chunk;
    if (!waiting.empty()) {
      chunk = cfg.min_chunk;
    } else if (!pending.empty()) {
      const double gap = pending.front().req.arrival - t;
      if (stepSeconds <= 0.0 || gap < stepSeconds * cfg.max_chunk) chunk = cfg.min_chunk;
    }
    lk.unlock();
    const auto r0 = Clock::now();
    int rc = eng.run(ctx, chunk);
    if (rc == LBX_OK) rc = eng.statuses(ctx, st.data(), int32_t(st.size()));
    const double dt = std::chrono::duration<double>(Clock::now() - r0).count();
    lk.lock();
    if (rc != LBX_OK) {
      fail_loop(rc, "engine run failed");
      break;
    }
    ++runs;
    steps += chunk;
    (chunk == cfg.min_chunk ? shortRuns : longRuns) += 1;
    busy += dt;
    stepSeconds = dt / chunk;
    if (!cfg.realtime) virtualNow += dt;
    t = now_locked();
    // 4. retirement: finished or cancelled slots
    std::vector<int32_t> gone;
    for (auto& [slot, a] : active) {
      if (slot < 0 || slot >= int32_t(st.size())) continue;
      const lbx_ensemble_status& s = st[size_t(slot)];
      const bool cancel = cancelRequests.erase(a.item.req.id) > 0;
      if (s.state == LBX_SLOT_RUNNING && !cancel) continue;
      finish_locked(a, cancel ? LBX_SERVER_CANCELLED : s.state, s.steps, s.residual, t);
      gone.push_back(slot);
    }
    if (!gone.empty()) {
      std::vector<lbx_server_record> recs;
      for (int32_t slot : gone) recs.push_back(active[slot].rec);
      lk.unlock();
      int rrc = LBX_OK;
      for (size_t i = 0; i < gone.size(); ++i) {
        if (onFinish) onFinish(onFinishUser, &recs[i]);
        const int r = eng.retire(ctx, gone[i]);
        if (r != LBX_OK && rrc == LBX_OK) rrc = r;
      }
      lk.lock();
      for (int32_t slot : gone) active.erase(slot);
      if (rrc != LBX_OK) {
        fail_loop(rrc, "engine retire failed");
        break;
      }
    }
  }
  // stopped (destroy) or failed: free what is still admitted
  if (!active.empty()) {
    std::vector<int32_t> slots;
    for (auto& kv : active) slots.push_back(kv.first);
    active.clear();
    lk.unlock();
    for (int32_t s : slots) eng.retire(ctx, s);
    lk.lock();
  }
  ended = true;
  doneCv.notify_all();
}

extern "C" {

int lbx_server_create_with_engine(const lbx_server_engine* engine, void* ctx, const lbx_server_config* cfg,
                                  lbx_server* out) {
  if (!engine || !out) return lbx::set_error(LBX_ERR_INVALID, "null argument");
  if (!engine->admit || !engine->run || !engine->statuses || !engine->retire || engine->slots < 1)
    return lbx::set_error(LBX_ERR_INVALID, "engine needs admit, run, statuses, retire and slots >= 1");
  if (int rc = check_config(cfg)) return rc;
  auto* s = new lbx_server_s();
  s->eng = *engine;
  s->ctx = ctx;
  s->cfg = *cfg;
  *out = s;
  return LBX_OK;
}

int lbx_server_create(lbx_ensemble ens, int32_t max_lattices, const lbx_server_config* cfg, void* stream,
                      lbx_server* out) {
  if (!ens || !out) return lbx::set_error(LBX_ERR_INVALID, "null argument");
  if (max_lattices < 1) return lbx::set_error(LBX_ERR_INVALID, "max_lattices must be >= 1");
  if (int rc = check_config(cfg)) return rc;
  auto* s = new lbx_server_s();
  s->eng = lbx_server_engine{ens_admit, ens_run, ens_statuses, ens_retire, max_lattices, 0};
  s->ctx = s;
  s->cfg = *cfg;
  s->ens = ens;
  s->stream = stream;
  *out = s;
  return LBX_OK;
}

int lbx_server_set_finish_callback(lbx_server s, lbx_server_finish_fn fn, void* user) {
  if (!s) return lbx::set_error(LBX_ERR_INVALID, "null server");
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->started) return lbx::set_error(LBX_ERR_INVALID, "set the callback before lbx_server_start");
  s->onFinish = fn;
  s->onFinishUser = user;
  return LBX_OK;
}

int lbx_server_submit(lbx_server s, const lbx_server_request* requests, int32_t n) {
  if (!s || (n > 0 && !requests) || n < 0) return lbx::set_error(LBX_ERR_INVALID, "bad arguments");
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->closed) return lbx::set_error(LBX_ERR_INVALID, "server is closed to submissions");
  const double t = s->now_locked();
  for (int32_t i = 0; i < n; ++i) {
    Item it{requests[i], s->seq++};
    if (!(it.req.arrival >= 0.0)) it.req.arrival = t;  // negative or NaN: now
    // keep `pending` ordered by (arrival, submission); most submissions append
    auto pos = std::upper_bound(s->pending.begin(), s->pending.end(), it, [](const Item& a, const Item& b) {
      return a.req.arrival < b.req.arrival || (a.req.arrival == b.req.arrival && a.seq < b.seq);
    });
    s->pending.insert(pos, it);
    ++s->submitted;
  }
  s->wake.notify_all();
  return LBX_OK;
}

int lbx_server_start(lbx_server s) {
  if (!s) return lbx::set_error(LBX_ERR_INVALID, "null server");
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->started) return lbx::set_error(LBX_ERR_INVALID, "server already started");
  s->started = true;
  s->t0 = Clock::now();
  s->virtualNow = 0.0;
  s->th = std::thread([s] { s->loop(); });
  return LBX_OK;
}

int lbx_server_close(lbx_server s) {
  if (!s) return lbx::set_error(LBX_ERR_INVALID, "null server");
  std::lock_guard<std::mutex> lk(s->mu);
  s->closed = true;
  s->wake.notify_all();
  return LBX_OK;
}

int lbx_server_cancel(lbx_server s, int64_t id) {
  if (!s) return lbx::set_error(LBX_ERR_INVALID, "null server");
  std::lock_guard<std::mutex> lk(s->mu);
  for (auto it = s->pending.begin(); it != s->pending.end(); ++it) {
    if (it->req.id == id) {
      lbx_server_record r = blank_record(*it);
      r.state = LBX_SERVER_CANCELLED;
      r.finished = s->now_locked();
      s->done.push_back(r);
      ++s->finished;
      s->pending.erase(it);
      return LBX_OK;
    }
  }
  bool known = false;
  for (const Item& it : s->waiting) known = known || it.req.id == id;
  for (const auto& kv : s->active) known = known || kv.second.item.req.id == id;
  if (!known) return lbx::set_error(LBX_ERR_INVALID, "request " + std::to_string(id) + " is not waiting or running");
  s->cancelRequests.insert(id);
  s->wake.notify_all();
  return LBX_OK;
}

int lbx_server_wait(lbx_server s, double timeout_s, int32_t* finished) {
  if (!s) return lbx::set_error(LBX_ERR_INVALID, "null server");
  std::unique_lock<std::mutex> lk(s->mu);
  if (!s->started) return lbx::set_error(LBX_ERR_INVALID, "server not started");
  if (timeout_s < 0) {
    s->doneCv.wait(lk, [s] { return s->ended; });
  } else {
    s->doneCv.wait_for(lk, std::chrono::duration<double>(timeout_s), [s] { return s->ended; });
  }
  if (finished) *finished = s->ended ? 1 : 0;
  if (s->ended && s->status != LBX_OK) return lbx::set_error(s->status, "server loop: " + s->error);
  return LBX_OK;
}

int lbx_server_records(lbx_server s, lbx_server_record* out, int32_t capacity, int32_t* n_out) {
  if (!s || capacity < 0 || (capacity > 0 && !out)) return lbx::set_error(LBX_ERR_INVALID, "bad arguments");
  std::lock_guard<std::mutex> lk(s->mu);
  int32_t n = 0;
  while (n < capacity && !s->done.empty()) {
    out[n++] = s->done.front();
    s->done.pop_front();
  }
  if (n_out) *n_out = n;
  return LBX_OK;
}

int lbx_server_get_stats(lbx_server s, lbx_server_stats* out) {
  if (!s || !out) return lbx::set_error(LBX_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  out->submitted = s->submitted;
  out->pending = int64_t(s->pending.size());
  out->waiting = int64_t(s->waiting.size());
  out->running = int64_t(s->active.size());
  out->finished = s->finished;
  out->runs = s->runs;
  out->steps = s->steps;
  out->short_runs = s->shortRuns;
  out->long_runs = s->longRuns;
  out->busy_seconds = s->busy;
  out->clock = s->now_locked();
  return LBX_OK;
}

int lbx_server_destroy(lbx_server s) {
  if (!s) return LBX_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    s->wake.notify_all();
  }
  if (s->th.joinable()) s->th.join();
  delete s;
  return LBX_OK;
}

}  // extern "C"
