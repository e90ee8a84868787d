// serve.cpp -- continuous-batching request server behind the C ABI
// (b200fem_server_*), for hosts that drive the served form directly (the
// Java binding, C/C++ callers).  It sits on the engine's own C ABI: every
// resident model lives in a pack (one b200fem_handle per pack); a tick steps
// every resident model with work by one BackwardEuler step, all models of a
// pack in the same launches (the pack's active mask leaves idle models out);
// requests that arrive meanwhile join at the next tick; a model's requests run
// FIFO.  Admission is against a device-memory budget: models without a pack
// are admitted in batches as a new pack when its estimated size fits, idle
// packs are evicted least-recently-used after their states are copied to the
// host, and a re-admitted model continues from its saved state.
//
// The reference has no counterpart (ArtiSynth steps one MechModel at a
// time); each request's result equals its model stepped alone, to rounding.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/b200fem.h"

namespace {

struct PoolModel {
  int elem_type = B200FEM_ELEM_TET, n_nodes = 0, n_elems = 0;
  std::vector<double> rest, fext;
  std::vector<int> conn, fixed;
  int mat_kind = B200FEM_MAT_NEOHOOKEAN;
  double params[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  double density = 1000;
  int incomp = B200FEM_INCOMP_AUTO;
};

struct Request {
  int model = 0, steps = 0, remaining = 0;
  int state = 0;  // 0 queued, 1 running, 2 done, -1 failed
  double t_arrive = 0, t_start = -1, t_done = -1;
};

struct Slot {
  b200fem_handle h = nullptr;
  std::vector<int> models;  // pool indices in pack order
  std::vector<int> mask;
  std::vector<int> node_off, n_nodes;
  double last_used = 0;
  unsigned long long bytes = 0;
};

}  // namespace

struct b200fem_server {
  b200fem_config cfg{};
  double budget = 0;
  int pack_models = 256;
  b200fem_step_params step{};
  std::vector<PoolModel> pool;
  std::vector<std::pair<int, int>> options;  // applied to every pack built
  std::vector<std::unique_ptr<Slot>> slots;
  std::vector<Slot*> where;  // pool index -> resident slot (or null)
  std::vector<int> where_idx;
  std::map<int, std::pair<std::vector<double>, std::vector<double>>> saved;
  std::vector<std::deque<int>> queues;  // per pool model: request ids
  std::deque<int> waiting;              // models with work and no pack
  std::vector<Request> reqs;
  // admission estimate: bytes = overhead + per_elem * elements (fit to builds)
  double per_elem = 4096, overhead = 0;
  std::vector<std::pair<double, double>> sizes;
  b200fem_server_stats st{};
  std::string err;
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
  std::mutex mu;  // calls on one server are serialised

  double now() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
  int fail(int code, const std::string& msg) {
    err = msg;
    return code;
  }
  unsigned long long resident() const {
    unsigned long long b = 0;
    for (auto& s : slots) b += s->bytes;
    return b;
  }
  bool busy(const Slot& s) const {
    for (int m : s.models)
      if (!queues[m].empty()) return true;
    return false;
  }
  double estimate(int m) const { return per_elem * pool[m].n_elems; }

  void calibrate(double elems, double bytes) {
    sizes.push_back({elems, bytes});
    double se = 0, sb = 0, see = 0, seb = 0;
    for (auto& p : sizes) {
      se += p.first;
      sb += p.second;
      see += p.first * p.first;
      seb += p.first * p.second;
    }
    const double n = (double)sizes.size(), den = n * see - se * se;
    if (sizes.size() >= 2 && den > 0) {
      const double slope = (n * seb - se * sb) / den, icpt = (sb - slope * se) / n;
      if (slope > 0) {
        per_elem = slope * 1.02;
        overhead = std::max(0.0, icpt) * 1.02;
        double worst = 0;
        for (auto& p : sizes) worst = std::max(worst, p.second - (overhead + per_elem * p.first));
        overhead += worst;
        return;
      }
    }
    per_elem = std::max(per_elem, bytes / std::max(1.0, elems));
  }

  int evict_idle(double need) {
    std::vector<Slot*> idle;
    for (auto& s : slots)
      if (!busy(*s)) idle.push_back(s.get());
    std::sort(idle.begin(), idle.end(), [](Slot* a, Slot* b) { return a->last_used < b->last_used; });
    for (Slot* s : idle) {
      if (resident() + need <= budget) break;
      size_t total = 0;
      for (int n : s->n_nodes) total += 3 * (size_t)n;
      std::vector<double> x(total), v(total);
      int rc = b200fem_get_state(s->h, x.data(), v.data());
      if (rc != B200FEM_OK) return fail(rc, std::string("evict: ") + b200fem_last_error(s->h));
      for (size_t i = 0; i < s->models.size(); i++) {
        const size_t o = 3 * (size_t)s->node_off[i], k = 3 * (size_t)s->n_nodes[i];
        saved[s->models[i]] = {std::vector<double>(x.begin() + o, x.begin() + o + k),
                               std::vector<double>(v.begin() + o, v.begin() + o + k)};
        where[s->models[i]] = nullptr;
      }
      b200fem_destroy(s->h);
      slots.erase(std::find_if(slots.begin(), slots.end(), [&](const std::unique_ptr<Slot>& p) { return p.get() == s; }));
      st.evictions++;
    }
    return B200FEM_OK;
  }

  int build(const std::vector<int>& batch) {
    auto slot = std::make_unique<Slot>();
    b200fem_handle h = b200fem_create(&cfg);
    if (!h) return fail(B200FEM_ERR_CUDA, std::string("pack: ") + b200fem_last_error(nullptr));
    slot->h = h;
    auto bail = [&](int rc) {
      std::string m = b200fem_last_error(h);
      b200fem_destroy(h);
      return fail(rc, "pack: " + m);
    };
    std::vector<double> fext;
    bool any_fext = false;
    for (int m : batch) {
      const PoolModel& pm = pool[m];
      int idx = 0;
      int rc = b200fem_add_model(h, pm.elem_type, pm.n_nodes, pm.rest.data(), pm.n_elems, pm.conn.data(),
                                 pm.fixed.data(), pm.mat_kind, pm.params, pm.density, pm.incomp, &idx);
      if (rc != B200FEM_OK) return bail(rc);
      if (!pm.fext.empty()) any_fext = true;
    }
    for (auto& kv : options) {
      int rc = b200fem_set_option(h, kv.first, kv.second);
      if (rc != B200FEM_OK) return bail(rc);
    }
    int rc = b200fem_build(h);
    if (rc != B200FEM_OK) return bail(rc);
    size_t total = 0;
    for (size_t i = 0; i < batch.size(); i++) {
      int off = 0, nn = 0, na = 0;
      if ((rc = b200fem_model_range(h, (int)i, &off, &nn, &na)) != B200FEM_OK) return bail(rc);
      slot->node_off.push_back(off);
      slot->n_nodes.push_back(nn);
      total += 3 * (size_t)nn;
    }
    if (any_fext) {
      fext.assign(total, 0.0);
      for (size_t i = 0; i < batch.size(); i++) {
        const PoolModel& pm = pool[batch[i]];
        if (!pm.fext.empty()) std::copy(pm.fext.begin(), pm.fext.end(), fext.begin() + 3 * (size_t)slot->node_off[i]);
      }
      if ((rc = b200fem_set_external_forces(h, fext.data())) != B200FEM_OK) return bail(rc);
    }
    bool restore = false;
    for (int m : batch) restore |= saved.count(m) > 0;
    if (restore) {
      std::vector<double> x(total), v(total, 0.0);
      for (size_t i = 0; i < batch.size(); i++) {
        const int m = batch[i];
        const size_t o = 3 * (size_t)slot->node_off[i];
        auto it = saved.find(m);
        if (it != saved.end()) {
          std::copy(it->second.first.begin(), it->second.first.end(), x.begin() + o);
          std::copy(it->second.second.begin(), it->second.second.end(), v.begin() + o);
          saved.erase(it);
        } else {
          std::copy(pool[m].rest.begin(), pool[m].rest.end(), x.begin() + o);
        }
      }
      if ((rc = b200fem_set_state(h, x.data(), v.data())) != B200FEM_OK) return bail(rc);
    }
    unsigned long long nb = 0;
    b200fem_memory_usage(h, &nb);
    double elems = 0;
    for (int m : batch) elems += pool[m].n_elems;
    calibrate(elems, (double)nb);
    slot->models = batch;
    slot->mask.assign(batch.size(), -1);
    slot->bytes = nb;
    slot->last_used = now();
    for (size_t i = 0; i < batch.size(); i++) {
      where[batch[i]] = slot.get();
      where_idx[batch[i]] = (int)i;
    }
    Slot* raw = slot.get();
    slots.push_back(std::move(slot));
    st.builds++;
    if (resident() > budget) evict_idle(0.0);  // the estimate fell short
    if (raw->bytes > budget) {
      // larger than the whole budget: its requests cannot be served
      for (int m : raw->models) {
        where[m] = nullptr;
        for (int r : queues[m]) {
          reqs[r].state = -1;
          st.failed++;
        }
        queues[m].clear();
      }
      b200fem_destroy(raw->h);
      slots.erase(std::find_if(slots.begin(), slots.end(), [&](const std::unique_ptr<Slot>& p) { return p.get() == raw; }));
    }
    st.peak_bytes = std::max(st.peak_bytes, resident());
    return B200FEM_OK;
  }

  int admit() {
    while (!waiting.empty()) {
      std::vector<int> batch;
      double est = overhead;
      for (int m : waiting) {
        if ((int)batch.size() >= pack_models) break;
        const double e = estimate(m);
        if (!batch.empty() && resident() + est + e > budget) break;
        batch.push_back(m);
        est += e;
      }
      if (resident() + est > budget) {
        int rc = evict_idle(est);
        if (rc != B200FEM_OK) return rc;
      }
      while (!batch.empty() && resident() + est > budget) {
        est -= estimate(batch.back());
        batch.pop_back();
      }
      if (batch.empty()) {
        bool any_busy = false;
        for (auto& s : slots) any_busy |= busy(*s);
        if (any_busy) return B200FEM_OK;  // no room until work finishes
        batch.push_back(waiting.front());  // try the first model by its real size
      }
      for (int m : batch) waiting.erase(std::find(waiting.begin(), waiting.end(), m));
      int rc = build(batch);
      if (rc != B200FEM_OK) return rc;
    }
    return B200FEM_OK;
  }
};

#define SRV(s)                                  \
  if (!(s)) return B200FEM_ERR_INVALID_ARG;     \
  std::lock_guard<std::mutex> lock_((s)->mu);   \
  b200fem_server& S = *(s)

extern "C" {

b200fem_server_handle b200fem_server_create(const b200fem_config* cfg, double budget_bytes, int pack_models,
                                            const b200fem_step_params* step) {
  if (!step || !(budget_bytes > 0) || pack_models <= 0) return nullptr;
  auto* s = new b200fem_server();
  if (cfg) s->cfg = *cfg;
  s->budget = budget_bytes;
  s->pack_models = pack_models;
  s->step = *step;
  return s;
}

int b200fem_server_destroy(b200fem_server_handle s) {
  if (!s) return B200FEM_OK;
  for (auto& sl : s->slots) b200fem_destroy(sl->h);
  delete s;
  return B200FEM_OK;
}

const char* b200fem_server_last_error(b200fem_server_handle s) { return s ? s->err.c_str() : "null server"; }

double b200fem_server_clock(b200fem_server_handle s) { return s ? s->now() : 0.0; }

int b200fem_server_set_option(b200fem_server_handle s, int key, int value) {
  SRV(s);
  for (auto& kv : S.options)
    if (kv.first == key) {
      kv.second = value;
      return B200FEM_OK;
    }
  S.options.push_back({key, value});
  return B200FEM_OK;
}

int b200fem_server_add_model(b200fem_server_handle s, int elem_type, int n_nodes, const double* rest_xyz,
                             int n_elems, const int* conn, const int* fixed, int mat_kind, const double* params,
                             double density, int incomp_method, const double* fext, int* model_id) {
  SRV(s);
  if (elem_type < B200FEM_ELEM_TET || elem_type > B200FEM_ELEM_QUADPYRAMID || n_nodes <= 0 || n_elems <= 0 ||
      !rest_xyz || !conn || !params || !(density > 0))
    return S.fail(B200FEM_ERR_INVALID_ARG, "invalid model");
  PoolModel m;
  // tet, hex, wedge, pyramid and their quadratic forms
  static const int kNen[8] = {4, 8, 6, 5, 10, 20, 15, 13};
  const int nen = kNen[elem_type];
  m.elem_type = elem_type;
  m.n_nodes = n_nodes;
  m.n_elems = n_elems;
  m.rest.assign(rest_xyz, rest_xyz + 3 * (size_t)n_nodes);
  m.conn.assign(conn, conn + (size_t)nen * n_elems);
  m.fixed.assign(n_nodes, 0);
  if (fixed) std::copy(fixed, fixed + n_nodes, m.fixed.begin());
  if (fext) m.fext.assign(fext, fext + 3 * (size_t)n_nodes);
  m.mat_kind = mat_kind;
  std::copy(params, params + 8, m.params);
  m.density = density;
  m.incomp = incomp_method;
  S.pool.push_back(std::move(m));
  S.where.push_back(nullptr);
  S.where_idx.push_back(0);
  S.queues.emplace_back();
  if (model_id) *model_id = (int)S.pool.size() - 1;
  return B200FEM_OK;
}

int b200fem_server_submit(b200fem_server_handle s, int model, int steps, double t_arrive, int* request_id) {
  SRV(s);
  if (model < 0 || model >= (int)S.pool.size() || steps <= 0) return S.fail(B200FEM_ERR_INVALID_ARG, "invalid request");
  Request r;
  r.model = model;
  r.steps = r.remaining = steps;
  r.t_arrive = t_arrive >= 0 ? t_arrive : S.now();
  S.reqs.push_back(r);
  const int id = (int)S.reqs.size() - 1;
  S.queues[model].push_back(id);
  if (!S.where[model] && std::find(S.waiting.begin(), S.waiting.end(), model) == S.waiting.end())
    S.waiting.push_back(model);
  if (request_id) *request_id = id;
  return B200FEM_OK;
}

int b200fem_server_preload(b200fem_server_handle s) {
  SRV(s);
  for (int m = 0; m < (int)S.pool.size(); m++)
    if (!S.where[m] && std::find(S.waiting.begin(), S.waiting.end(), m) == S.waiting.end()) S.waiting.push_back(m);
  return S.admit();
}

int b200fem_server_tick(b200fem_server_handle s, int* model_steps) {
  SRV(s);
  if (model_steps) *model_steps = 0;
  int rc = S.admit();
  if (rc != B200FEM_OK) return rc;
  int taken = 0;
  std::vector<Slot*> order;
  for (auto& sl : S.slots) order.push_back(sl.get());
  for (Slot* sl : order) {
    std::vector<int> mask(sl->models.size(), 0);
    bool any = false, all = true;
    for (size_t i = 0; i < sl->models.size(); i++) {
      mask[i] = S.queues[sl->models[i]].empty() ? 0 : 1;
      any |= mask[i] != 0;
      all &= mask[i] != 0;
    }
    if (!any) continue;
    if (mask != sl->mask) {
      if ((rc = b200fem_set_active_models(sl->h, all ? nullptr : mask.data())) != B200FEM_OK)
        return S.fail(rc, std::string("tick: ") + b200fem_last_error(sl->h));
      sl->mask = mask;
    }
    const double t_start = S.now();
    for (size_t i = 0; i < mask.size(); i++)
      if (mask[i]) {
        Request& r = S.reqs[S.queues[sl->models[i]].front()];
        if (r.t_start < 0) {
          r.t_start = t_start;
          r.state = 1;
        }
      }
    b200fem_stats stats{};
    rc = b200fem_backward_euler_step(sl->h, &S.step, 1, &stats);
    if (rc != B200FEM_OK) return S.fail(rc, std::string("tick: ") + b200fem_last_error(sl->h));
    const double t_end = S.now();
    sl->last_used = t_end;
    S.st.slot_steps++;
    for (size_t i = 0; i < mask.size(); i++) {
      if (!mask[i]) continue;
      auto& q = S.queues[sl->models[i]];
      Request& r = S.reqs[q.front()];
      if (--r.remaining == 0) {
        r.t_done = t_end;
        r.state = 2;
        q.pop_front();
        S.st.completed++;
      }
      taken++;
    }
  }
  S.st.ticks++;
  S.st.model_steps += taken;
  if (model_steps) *model_steps = taken;
  return B200FEM_OK;
}

int b200fem_server_poll(b200fem_server_handle s, int request_id, int* state, double* latency_s) {
  SRV(s);
  if (request_id < 0 || request_id >= (int)S.reqs.size()) return S.fail(B200FEM_ERR_INVALID_ARG, "unknown request");
  const Request& r = S.reqs[request_id];
  if (state) *state = r.state;
  if (latency_s) *latency_s = r.state == 2 ? r.t_done - r.t_arrive : -1.0;
  return B200FEM_OK;
}

int b200fem_server_get_state(b200fem_server_handle s, int model, double* x, double* v) {
  SRV(s);
  if (model < 0 || model >= (int)S.pool.size()) return S.fail(B200FEM_ERR_INVALID_ARG, "unknown model");
  const size_t k = 3 * (size_t)S.pool[model].n_nodes;
  if (Slot* sl = S.where[model]) {
    size_t total = 0;
    for (int n : sl->n_nodes) total += 3 * (size_t)n;
    std::vector<double> xs(total), vs(total);
    int rc = b200fem_get_state(sl->h, xs.data(), vs.data());
    if (rc != B200FEM_OK) return S.fail(rc, b200fem_last_error(sl->h));
    const size_t o = 3 * (size_t)sl->node_off[S.where_idx[model]];
    if (x) std::copy(xs.begin() + o, xs.begin() + o + k, x);
    if (v) std::copy(vs.begin() + o, vs.begin() + o + k, v);
    return B200FEM_OK;
  }
  auto it = S.saved.find(model);
  if (it != S.saved.end()) {
    if (x) std::copy(it->second.first.begin(), it->second.first.end(), x);
    if (v) std::copy(it->second.second.begin(), it->second.second.end(), v);
  } else {
    if (x) std::copy(S.pool[model].rest.begin(), S.pool[model].rest.end(), x);
    if (v) std::fill(v, v + k, 0.0);
  }
  return B200FEM_OK;
}

int b200fem_server_get_stats(b200fem_server_handle s, b200fem_server_stats* out) {
  SRV(s);
  if (!out) return S.fail(B200FEM_ERR_INVALID_ARG, "null stats");
  S.st.resident_bytes = S.resident();
  int pending = 0, res = 0;
  for (auto& q : S.queues) pending += (int)q.size();
  for (Slot* p : S.where) res += p != nullptr;
  S.st.pending = pending;
  S.st.resident_models = res;
  *out = S.st;
  return B200FEM_OK;
}

}  // extern "C"
