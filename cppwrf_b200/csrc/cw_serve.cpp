// SPDX-License-Identifier: GPL-3.0-or-later
// The served form (include/cw_serve.h): a host request loop over the batch interface of the C ABI.
//
// Three host threads, so that setting up and reading back requests overlaps with stepping the resident ones:
//   - the admitter takes queued requests in FIFO order while the device footprint of every request it holds
//     (being set up, resident or being read back: cw_footprint) plus the next one's fits the budget and a slot
//     is free; it makes each a single-domain handle on its own stream (cw_create + cw_upload_case) and hands it
//     to the stepper;
//   - the stepper moves the ready requests into the batch of their acoustic step count without copying
//     (cw_batch_adopt), launches one batched, graph-captured RK3 step of every batch and then waits for all of
//     them, and moves each request that has done its steps out of its batch, again without copying
//     (cw_batch_release);
//   - the reader downloads a finished request's prognostic state from its released handle on that handle's
//     stream, frees the handle (and with it the request's device memory) and completes the request.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/cw_serve.h"
#include "cw_fields.hpp"

namespace {

using Clock = std::chrono::steady_clock;

// the fields a finished request keeps (its prognostic state)
constexpr int kResultFields[] = {CW_U_2, CW_V_2, CW_W_2, CW_T_2, CW_PH_2, CW_MU_2, CW_P, CW_AL};

struct Request {
  long long id = 0;
  cw_case* c = nullptr;  // owned until set up
  cw_grid g{};
  cw_options o{};
  int nsteps = 0, done = 0, n_sound = 0;
  size_t bytes = 0;
  double gp = 0;         // nx * ny * nz
  int status = 0;        // 0 queued / running, 1 finished, -1 failed
  cw_handle* single = nullptr;  // its own handle while being set up or read back
  Clock::time_point t_submit, t_done;
  std::map<std::pair<int, int>, std::vector<double>> result;  // (field, species) -> whole allocation
  std::string err;
};

struct Group {  // the resident requests with one acoustic step count: one batch handle
  int n_sound = 0;
  cw_handle* h = nullptr;
  std::vector<Request*> members;  // in member-index order
};

}  // namespace

struct cw_server {
  cw_serve_config cfg{};
  std::mutex mu;
  std::condition_variable cv_admit, cv_step, cv_read, cv_done;
  std::deque<Request*> pending;   // queued, FIFO
  std::deque<Request*> ready;     // set up, waiting to join a batch
  std::deque<Request*> finished;  // released from their batch, waiting to be read back
  std::map<long long, std::unique_ptr<Request>> all;
  std::vector<Group> groups;      // stepper thread only
  long long next_id = 1;
  bool stop = false;
  int creates_failed = 0;         // injected batch-handle creation failures so far (cfg.test_fail_creates)
  std::thread admitter, stepper, reader;
  // statistics
  long long submitted = 0, completed = 0, failed = 0, rejected = 0, ticks = 0;
  int held = 0, stepping = 0, max_resident_seen = 0;
  double used = 0, max_used = 0, gp_steps = 0;
  bool any_submit = false;
  Clock::time_point t_first, t_last;
  std::vector<double> latencies;
  std::string err;

  void admit_loop();
  void step_loop();
  void read_loop();
  // under mu: a request that held device memory has let it go
  void release_locked(Request* r) {
    --held;
    used -= double(r->bytes);
    cv_admit.notify_all();
  }
  void fail_locked(Request* r, const std::string& e) {
    r->status = -1;
    r->err = e;
    err = e;
    ++failed;
    cv_done.notify_all();
  }
};

namespace {
std::string last_error(cw_handle* h) {
  const char* e = cw_last_error(h);
  return e && *e ? e : "CUDA error";
}
}  // namespace

// admitter: FIFO admission by footprint and slot, set-up of a single-domain handle per request
void cw_server::admit_loop() {
  cw_use_device(cfg.device);
  for (;;) {
    Request* r = nullptr;
    {
      std::unique_lock<std::mutex> lock(mu);
      cv_admit.wait(lock, [&] {
        if (stop) return true;
        if (pending.empty()) return false;
        const Request* head = pending.front();
        return held < cfg.max_resident && used + double(head->bytes) <= cfg.hbm_budget_bytes;
      });
      if (stop) return;
      r = pending.front();
      pending.pop_front();
      ++held;
      used += double(r->bytes);
      max_resident_seen = std::max(max_resident_seen, held);
      max_used = std::max(max_used, used);
    }
    cw_handle* s = nullptr;
    std::string e;
    if (cw_create(&r->g, &r->o, &s) != 0) e = last_error(nullptr);
    else if (cw_upload_case(s, r->c) != 0 || cw_sync(s) != 0) e = last_error(s);
    cw_case_destroy(r->c);
    r->c = nullptr;
    std::lock_guard<std::mutex> lock(mu);
    if (!e.empty()) {
      cw_destroy(s);
      release_locked(r);
      fail_locked(r, "set-up: " + e);
      continue;
    }
    r->single = s;
    ready.push_back(r);
    cv_step.notify_all();
  }
}

// stepper: ready requests join their batch, every batch steps, finished requests leave
void cw_server::step_loop() {
  cw_use_device(cfg.device);
  for (;;) {
    std::vector<Request*> joining;
    {
      std::unique_lock<std::mutex> lock(mu);
      cv_step.wait(lock, [&] { return stop || !ready.empty() || stepping > 0; });
      if (stop) break;
      joining.assign(ready.begin(), ready.end());
      ready.clear();
    }
    for (Request* r : joining) {
      Group* G = nullptr;
      for (Group& x : groups)
        if (x.n_sound == r->n_sound) G = &x;
      std::string e;
      if (!G) {  // a new acoustic step count: a new batch
        cw_handle* h = nullptr;
        bool inject = false;
        {
          std::lock_guard<std::mutex> lock(mu);
          inject = creates_failed < cfg.test_fail_creates;
          if (inject) ++creates_failed;
        }
        if (inject) e = "injected batch creation failure";
        else if (cw_batch_create(0, nullptr, &r->o, &h) != 0) e = last_error(nullptr);
        else if (cw_set_autotune(h, 1) != 0) e = last_error(h);  // its first steps pick the kernels' shapes
        if (!e.empty() && h) {
          cw_destroy(h);
          h = nullptr;
        }
        if (e.empty()) {
          groups.push_back(Group{r->n_sound, h, {}});
          G = &groups.back();
        }
      }
      if (e.empty() && cw_batch_adopt(G->h, r->single, nullptr) != 0) e = last_error(G->h);
      cw_destroy(r->single);  // empty after a successful adoption
      r->single = nullptr;
      std::lock_guard<std::mutex> lock(mu);
      if (!e.empty()) {
        release_locked(r);
        fail_locked(r, "admission: " + e);
        continue;
      }
      G->members.push_back(r);
      ++stepping;
    }
    // every batch's step is launched before the first wait
    std::vector<std::string> errs(groups.size());
    for (size_t gi = 0; gi < groups.size(); ++gi)
      if (!groups[gi].members.empty() && cw_step(groups[gi].h, 1) != 0) errs[gi] = last_error(groups[gi].h);
    bool stepped = false;
    for (size_t gi = groups.size(); gi-- > 0;) {
      Group& G = groups[gi];
      if (G.members.empty()) continue;
      if (errs[gi].empty() && cw_sync(G.h) != 0) errs[gi] = last_error(G.h);
      if (!errs[gi].empty()) {  // the batch's requests fail; the batch is dropped (a later request makes a new one)
        cw_destroy(G.h);
        std::lock_guard<std::mutex> lock(mu);
        for (Request* r : G.members) {
          --stepping;
          release_locked(r);
          fail_locked(r, "step: " + errs[gi]);
        }
        groups.erase(groups.begin() + std::ptrdiff_t(gi));
        continue;
      }
      stepped = true;
      for (Request* r : G.members) ++r->done;
      for (size_t m = G.members.size(); m-- > 0;) {
        Request* r = G.members[m];
        if (r->done < r->nsteps) continue;
        cw_handle* s = nullptr;
        const int rc = cw_batch_release(G.h, int(m), &s);
        G.members.erase(G.members.begin() + std::ptrdiff_t(m));
        std::lock_guard<std::mutex> lock(mu);
        --stepping;
        if (rc != 0) {
          release_locked(r);
          fail_locked(r, "release: " + last_error(G.h));
          continue;
        }
        r->single = s;
        finished.push_back(r);
        cv_read.notify_all();
      }
    }
    if (stepped) {
      std::lock_guard<std::mutex> lock(mu);
      ++ticks;
    }
  }
}

// reader: a finished request's state back to the host, its device memory freed
void cw_server::read_loop() {
  cw_use_device(cfg.device);
  for (;;) {
    Request* r = nullptr;
    {
      std::unique_lock<std::mutex> lock(mu);
      cv_read.wait(lock, [&] { return stop || !finished.empty(); });
      if (stop) return;
      r = finished.front();
      finished.pop_front();
    }
    std::string e;
    if (cfg.keep_results) {
      auto get = [&](int field, int n) {
        if (!e.empty()) return;
        cw_layout L{};
        if (cw_field_layout(r->single, field, n, &L) != 0) {
          e = last_error(r->single);
          return;
        }
        std::vector<double> v(size_t(L.total));
        if (cw_download(r->single, field, n, v.data(), v.size()) != 0) e = last_error(r->single);
        else r->result[{field, n}] = std::move(v);
      };
      for (int f : kResultFields) get(f, 0);
      for (int n = 0; n < r->o.n_scalars; ++n) get(CW_Q_2, n);
    } else if (cw_sync(r->single) != 0) {
      e = last_error(r->single);
    }
    cw_destroy(r->single);
    r->single = nullptr;
    const Clock::time_point now = Clock::now();
    std::lock_guard<std::mutex> lock(mu);
    release_locked(r);
    if (!e.empty()) {
      fail_locked(r, "read-back: " + e);
      continue;
    }
    r->t_done = now;
    r->status = 1;
    ++completed;
    gp_steps += r->gp * r->nsteps;
    latencies.push_back(std::chrono::duration<double>(now - r->t_submit).count());
    t_last = now;
    cv_done.notify_all();
  }
}

// ------------------------------------------------------------------ C ABI
extern "C" {

int cw_serve_default_config(cw_serve_config* c) {
  if (!c) return -1;
  c->hbm_budget_bytes = 150e9;
  c->max_resident = 256;
  c->precision = CW_MIXED;
  c->device = 0;
  c->keep_results = 1;
  c->test_fail_creates = 0;
  return 0;
}

int cw_serve_create(const cw_serve_config* c, cw_server** out) {
  if (!c || !out) return -1;
  if (c->max_resident < 1 || c->max_resident > 256 || !(c->hbm_budget_bytes > 0) || c->test_fail_creates < 0) return -1;
  if (cw_use_device(c->device) != 0) return -3;  // no device: nothing to serve on
  try {
    auto s = std::make_unique<cw_server>();
    s->cfg = *c;
    s->admitter = std::thread([p = s.get()] { p->admit_loop(); });
    s->stepper = std::thread([p = s.get()] { p->step_loop(); });
    s->reader = std::thread([p = s.get()] { p->read_loop(); });
    *out = s.release();
  } catch (...) {
    return -3;
  }
  return 0;
}

int cw_serve_destroy(cw_server* s) {
  if (!s) return 0;
  {
    std::lock_guard<std::mutex> lock(s->mu);
    s->stop = true;
  }
  s->cv_admit.notify_all();
  s->cv_step.notify_all();
  s->cv_read.notify_all();
  for (std::thread* t : {&s->admitter, &s->stepper, &s->reader})
    if (t->joinable()) t->join();
  for (Group& G : s->groups) cw_destroy(G.h);
  for (auto& kv : s->all) {
    if (kv.second->c) cw_case_destroy(kv.second->c);
    if (kv.second->single) cw_destroy(kv.second->single);
  }
  delete s;
  return 0;
}

int cw_serve_submit(cw_server* s, const cw_case* c, int nsteps, long long* id) {
  if (!s || !c || nsteps <= 0) return -1;
  auto r = std::make_unique<Request>();
  if (cw_case_config(c, &r->g, &r->o) != 0) return -1;
  r->o.precision = s->cfg.precision;
  if (cw_footprint(&r->g, &r->o, &r->bytes) != 0) return -1;
  if (double(r->bytes) > s->cfg.hbm_budget_bytes) {
    std::lock_guard<std::mutex> lock(s->mu);
    ++s->rejected;
    s->err = "the request's footprint exceeds the whole budget";
    return -2;
  }
  if (cw_case_clone(c, &r->c) != 0) return -3;
  r->nsteps = nsteps;
  r->n_sound = cw::sound_steps(r->g, r->o);
  r->gp = double(r->g.nx) * r->g.ny * r->g.nz;
  r->t_submit = Clock::now();
  {
    std::lock_guard<std::mutex> lock(s->mu);
    r->id = s->next_id++;
    if (!s->any_submit) {
      s->any_submit = true;
      s->t_first = r->t_submit;
    }
    ++s->submitted;
    if (id) *id = r->id;
    s->pending.push_back(r.get());
    s->all[r->id] = std::move(r);
  }
  s->cv_admit.notify_all();
  return 0;
}

int cw_serve_wait(cw_server* s, long long id, double seconds) {
  if (!s) return -1;
  std::unique_lock<std::mutex> lock(s->mu);
  auto it = s->all.find(id);
  if (it == s->all.end()) return -1;
  Request* r = it->second.get();
  auto done = [&] { return r->status != 0; };
  if (seconds < 0) s->cv_done.wait(lock, done);
  else if (!s->cv_done.wait_for(lock, std::chrono::duration<double>(seconds), done)) return 1;
  return r->status == 1 ? 0 : -2;
}

int cw_serve_drain(cw_server* s) {
  if (!s) return -1;
  std::unique_lock<std::mutex> lock(s->mu);
  s->cv_done.wait(lock, [&] { return s->completed + s->failed == s->submitted; });
  return 0;
}

int cw_serve_result(cw_server* s, long long id, int field, int n, double* host, size_t count) {
  if (!s || !host) return -1;
  std::lock_guard<std::mutex> lock(s->mu);
  auto it = s->all.find(id);
  if (it == s->all.end() || it->second->status != 1) return -1;
  auto f = it->second->result.find({field, field == CW_Q_2 ? n : 0});
  if (f == it->second->result.end() || f->second.size() != count) return -1;
  std::memcpy(host, f->second.data(), count * sizeof(double));
  return 0;
}

int cw_serve_latency(cw_server* s, long long id, double* seconds) {
  if (!s || !seconds) return -1;
  std::lock_guard<std::mutex> lock(s->mu);
  auto it = s->all.find(id);
  if (it == s->all.end() || it->second->status != 1) return -1;
  *seconds = std::chrono::duration<double>(it->second->t_done - it->second->t_submit).count();
  return 0;
}

int cw_serve_release(cw_server* s, long long id) {
  if (!s) return -1;
  std::lock_guard<std::mutex> lock(s->mu);
  auto it = s->all.find(id);
  if (it == s->all.end() || it->second->status == 0) return -1;
  it->second->result.clear();
  return 0;
}

int cw_serve_stats_get(cw_server* s, cw_serve_stats* out) {
  if (!s || !out) return -1;
  std::lock_guard<std::mutex> lock(s->mu);
  cw_serve_stats t{};
  t.submitted = s->submitted;
  t.completed = s->completed;
  t.failed = s->failed;
  t.rejected = s->rejected;
  t.ticks = s->ticks;
  t.resident = s->held;
  t.pending = int(s->pending.size());
  t.max_resident_seen = s->max_resident_seen;
  t.used_bytes = s->used;
  t.max_used_bytes = s->max_used;
  std::vector<double> v = s->latencies;
  if (!v.empty()) {
    std::sort(v.begin(), v.end());
    auto pct = [&](double q) {  // nearest rank
      size_t k = size_t(q * double(v.size()) + 0.999999);
      k = std::min(std::max<size_t>(k, 1), v.size());
      return v[k - 1];
    };
    t.p50_s = pct(0.50);
    t.p99_s = pct(0.99);
    double sum = 0;
    for (double x : v) sum += x;
    t.mean_s = sum / double(v.size());
    t.max_s = v.back();
  }
  t.gp_steps = s->gp_steps;
  if (s->completed > 0) t.wall_s = std::chrono::duration<double>(s->t_last - s->t_first).count();
  t.gp_steps_per_s = t.wall_s > 0 ? t.gp_steps / t.wall_s : 0;
  *out = t;
  return 0;
}

const char* cw_serve_last_error(cw_server* s) { return s ? s->err.c_str() : "null server"; }

}  // extern "C"
