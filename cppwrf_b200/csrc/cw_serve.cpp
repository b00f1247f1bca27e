// SPDX-License-Identifier: GPL-3.0-or-later
// The served form (include/cw_serve.h): a host request loop over the batch interface of the C ABI.
//
// Requests wait in a FIFO queue and are admitted, in order, while the resident requests' device footprint
// (cw_footprint) plus the next one's fits the budget and a slot is free. An admitted request becomes a
// member of a batch handle (one handle per acoustic step count, since a batch shares it), its state is
// uploaded once and stays on the device; every loop iteration advances all resident requests by one RK3
// step (one batched, graph-captured step per handle). A request that has done its steps is read back and
// leaves the batch, which frees its memory and slot for the next one in the queue.
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
  cw_case* c = nullptr;  // owned until admitted
  cw_grid g{};
  cw_options o{};
  int nsteps = 0, done = 0;
  size_t bytes = 0;
  double gp = 0;  // nx * ny * nz
  int status = 0;  // 0 queued / running, 1 finished, -1 failed
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
  std::condition_variable cv_work, cv_done;
  std::deque<Request*> pending;
  std::map<long long, std::unique_ptr<Request>> all;
  std::vector<Group> groups;
  long long next_id = 1;
  bool stop = false;
  std::thread loop;
  // statistics
  long long submitted = 0, completed = 0, failed = 0, rejected = 0, ticks = 0;
  int resident = 0, max_resident_seen = 0;
  double used = 0, max_used = 0, gp_steps = 0;
  bool any_submit = false;
  Clock::time_point t_first, t_last;
  std::vector<double> latencies;
  std::string err;
  int n_sound_of(const cw_grid& g, const cw_options& o);
  void run();
  bool admit_one();
  void finish(Group& G, size_t idx);
};

int cw_server::n_sound_of(const cw_grid& g, const cw_options& o) { return cw::sound_steps(g, o); }

// admits the head of the queue if it fits; false when nothing was admitted
bool cw_server::admit_one() {
  Request* r = nullptr;
  {
    std::lock_guard<std::mutex> lock(mu);
    if (pending.empty()) return false;
    Request* head = pending.front();
    if (resident >= cfg.max_resident || used + double(head->bytes) > cfg.hbm_budget_bytes) return false;
    pending.pop_front();
    r = head;
    ++resident;
    used += double(r->bytes);
    max_resident_seen = std::max(max_resident_seen, resident);
    max_used = std::max(max_used, used);
  }
  const int ns = n_sound_of(r->g, r->o);
  Group* G = nullptr;
  for (Group& x : groups)
    if (x.n_sound == ns) G = &x;
  int rc = 0;
  if (!G) {
    groups.push_back(Group{ns, nullptr, {}});
    G = &groups.back();
    rc = cw_batch_create(0, nullptr, &r->o, &G->h);
  }
  int m = -1;
  if (rc == 0) rc = cw_batch_add(G->h, &r->g, &r->o, &m);
  if (rc == 0) rc = cw_member_upload_case(G->h, m, r->c);
  cw_case_destroy(r->c);
  r->c = nullptr;
  std::lock_guard<std::mutex> lock(mu);
  if (rc != 0) {
    const char* e = G->h ? cw_last_error(G->h) : cw_last_error(nullptr);
    r->err = e ? e : "admission failed";
    err = r->err;
    r->status = -1;
    ++failed;
    --resident;
    used -= double(r->bytes);
    if (m >= 0) cw_batch_remove(G->h, m);
    cv_done.notify_all();
    return true;
  }
  G->members.push_back(r);
  return true;
}

// reads a finished member back and takes it out of its batch
void cw_server::finish(Group& G, size_t idx) {
  Request* r = G.members[idx];
  const int m = int(idx);
  int rc = 0;
  if (cfg.keep_results) {
    auto get = [&](int field, int n) {
      cw_layout L{};
      if (rc == 0) rc = cw_member_field_layout(G.h, m, field, n, &L);
      if (rc != 0) return;
      std::vector<double> v(size_t(L.total));
      rc = cw_member_download(G.h, m, field, n, v.data(), v.size());
      r->result[{field, n}] = std::move(v);
    };
    for (int f : kResultFields) get(f, 0);
    for (int n = 0; n < r->o.n_scalars; ++n) get(CW_Q_2, n);
  } else {
    rc = cw_sync(G.h);
  }
  const Clock::time_point now = Clock::now();
  if (rc != 0) r->err = cw_last_error(G.h) ? cw_last_error(G.h) : "read-back failed";
  cw_batch_remove(G.h, m);
  G.members.erase(G.members.begin() + m);
  std::lock_guard<std::mutex> lock(mu);
  r->t_done = now;
  r->status = rc == 0 ? 1 : -1;
  --resident;
  used -= double(r->bytes);
  if (rc == 0) {
    ++completed;
    gp_steps += r->gp * r->nsteps;
    latencies.push_back(std::chrono::duration<double>(now - r->t_submit).count());
    t_last = now;
  } else {
    ++failed;
    err = r->err;
  }
  cv_done.notify_all();
}

void cw_server::run() {
  cw_use_device(cfg.device);
  for (;;) {
    {
      std::unique_lock<std::mutex> lock(mu);
      cv_work.wait(lock, [&] { return stop || !pending.empty() || resident > 0; });
      if (stop) break;
    }
    while (admit_one()) {
    }
    bool stepped = false;
    for (Group& G : groups) {
      if (G.members.empty()) continue;
      if (cw_step(G.h, 1) != 0 || cw_sync(G.h) != 0) {
        std::lock_guard<std::mutex> lock(mu);
        err = cw_last_error(G.h) ? cw_last_error(G.h) : "step failed";
        for (Request* r : G.members) {
          r->status = -1;
          r->err = err;
          ++failed;
          --resident;
          used -= double(r->bytes);
        }
        G.members.clear();
        cw_destroy(G.h);
        cw_options o;
        cw_default_options(&o);
        o.precision = cfg.precision;
        G.h = nullptr;
        cw_batch_create(0, nullptr, &o, &G.h);
        cv_done.notify_all();
        continue;
      }
      stepped = true;
      for (Request* r : G.members) ++r->done;
      for (size_t i = G.members.size(); i-- > 0;)
        if (G.members[i]->done >= G.members[i]->nsteps) finish(G, i);
    }
    if (stepped) {
      std::lock_guard<std::mutex> lock(mu);
      ++ticks;
    }
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
  return 0;
}

int cw_serve_create(const cw_serve_config* c, cw_server** out) {
  if (!c || !out) return -1;
  if (c->max_resident < 1 || c->max_resident > 256 || !(c->hbm_budget_bytes > 0)) return -1;
  if (cw_use_device(c->device) != 0) return -3;  // no device: nothing to serve on
  try {
    auto s = std::make_unique<cw_server>();
    s->cfg = *c;
    s->loop = std::thread([p = s.get()] { p->run(); });
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
  s->cv_work.notify_all();
  if (s->loop.joinable()) s->loop.join();
  for (Group& G : s->groups) cw_destroy(G.h);
  for (auto& kv : s->all)
    if (kv.second->c) cw_case_destroy(kv.second->c);
  delete s;
  return 0;
}

int cw_serve_submit(cw_server* s, const cw_case* c, int nsteps, long long* id) {
  if (!s || !c || nsteps < 0) return -1;
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
    Request* raw = r.get();
    s->all[r->id] = std::move(r);
    if (raw->nsteps == 0) {  // nothing to do: finished at once, state as given
      raw->status = -1;
      raw->err = "nsteps = 0";
    } else {
      s->pending.push_back(raw);
    }
  }
  s->cv_work.notify_all();
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
  s->cv_done.wait(lock, [&] { return s->pending.empty() && s->resident == 0; });
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
  t.resident = s->resident;
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
