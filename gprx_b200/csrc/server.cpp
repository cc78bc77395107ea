// server.cpp — a request loop over resident exact-GPR models on one GPU.
//
// Requests (fit, predict, online add, online remove) arrive from any host
// thread; each names a model, and a fit creates one.  A pool of worker
// threads runs them continuously: a request is admitted as soon as a worker is
// free, its model is not busy and — for a fit — the model's device memory fits
// in the HBM budget (idle models are evicted least-recently-used to make
// room).  Every model owns a CUDA stream (its gprx_exact handle), so the work
// of different models overlaps on the device.  Same-phase work is batched:
//  - fits of up to SERVE_BATCH_FIT_MAX_N points always run on the batched
//    evaluator (gprx_batch_fit: one persistent launch per L-BFGS round, one
//    CTA per problem); the fits waiting at the heads of different models'
//    queues that share a kernel tree, d and optimizer settings are admitted
//    together into one such launch, and a fit that arrives alone runs the
//    same kernels as a batch of one;
//  - small predicts (at most SERVE_GROUP_MAX_Q points against a fitted model
//    of at most SERVE_GROUP_MAX_N points) always run as a grouped launch
//    (gprx_exact_predict_group, one CTA per request tile): those waiting at
//    the heads of several models' queues, and a model's consecutive ones,
//    share one launch; larger consecutive predicts of one model with the
//    same variance kind are merged into one predict launch and split back.
// Requests on one model run in submission order; each model's results do
// not depend on what else is running (a batched problem is evaluated by one
// CTA in a fixed order whatever the batch holds).
//
// The per-request device work is the exact path of this library (the
// reference's Gpr::fit / FittedGpr::predict_with / OnlineGpr insert and
// delete, src/gpr/trainer.rs:533-613, src/gpr/shared.rs:754-820,
// src/gpr/online.rs:564-611,794-900); the loop itself has no counterpart in
// the reference.

#include <algorithm>
#include <atomic>
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

#include <cuda_runtime.h>

#include "../../include/gprx_cuda.h"

namespace {

enum Kind { FIT = 0, PREDICT = 1, ADD = 2, REMOVE = 3 };

int64_t now_ns() {
  return std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

struct Request {
  uint64_t id = 0;
  int kind = FIT;
  uint64_t model = 0;
  // fit
  std::vector<double> x, y, theta;
  std::vector<gprx_kernel_node> nodes;
  uint64_t n = 0, d = 0;
  gprx_options opt{};
  gprx_lbfgs_options lopt{};
  int optimize = 1;
  // predict
  std::vector<double> xs;
  uint64_t q = 0;
  int vkind = GPRX_VARIANCE_OBSERVATION;
  double* mean_out = nullptr;
  double* var_out = nullptr;
  // add / remove
  uint64_t* ids_out = nullptr;
  std::vector<uint64_t> ids;
  // result
  gprx_status status = GPRX_OK;
  std::string message;
  int64_t t_submit = 0, t_start = 0, t_end = 0;
  int merged = 1;  // requests that shared this request's launch
  bool done = false;
};

struct Model {
  gprx_exact* h = nullptr;
  uint64_t d = 0;
  uint64_t n = 0;      // training points of the fitted model
  uint64_t fit_req = 0;  // the fit request (its kernel tree)
  uint64_t bytes = 0;
  bool busy = false;
  bool ready = false;  // fitted and resident
  bool online = false;
  bool failed = false;
  int64_t last_used = 0;
  std::deque<uint64_t> queue;  // request ids, submission order
};

// fits of at most this many points run on the batched evaluator (one CTA per
// problem: beyond it the blocked factor on the whole GPU has lower latency)
constexpr uint64_t SERVE_BATCH_FIT_MAX_N = 512;
// problems per batched fit launch (one CTA each on the 148 SMs)
constexpr size_t SERVE_BATCH_FIT_MAX = 148;

bool batched_fit(const Request* r) { return r->kind == FIT && r->optimize && r->n <= SERVE_BATCH_FIT_MAX_N; }

// Fits that may share one batched launch: the same tree, d, θ length,
// jitter policy and optimizer settings (each problem keeps its own data and θ0).
bool fit_compatible(const Request* a, const Request* b) {
  if (a->d != b->d || a->nodes.size() != b->nodes.size() || a->theta.size() != b->theta.size()) return false;
  for (size_t i = 0; i < a->nodes.size(); ++i)
    if (a->nodes[i].kind != b->nodes[i].kind || a->nodes[i].arg != b->nodes[i].arg) return false;
  const gprx_options &oa = a->opt, &ob = b->opt;
  if (oa.jitter_kind != ob.jitter_kind || oa.jitter_initial != ob.jitter_initial ||
      oa.jitter_multiplier != ob.jitter_multiplier || oa.jitter_max_retries != ob.jitter_max_retries ||
      oa.jitter_max != ob.jitter_max)
    return false;
  return std::memcmp(&a->lopt, &b->lopt, sizeof(gprx_lbfgs_options)) == 0;
}

// predicts of at most this many points against a fitted (not online) model
// of at most SERVE_GROUP_MAX_N points and SERVE_GROUP_MAX_D features run as
// one grouped launch (gprx_exact_predict_group) with the other models' small
// predicts waiting at the same time, alone or not
constexpr uint64_t SERVE_GROUP_MAX_Q = 256;
constexpr uint64_t SERVE_GROUP_MAX_N = 1024;
constexpr uint64_t SERVE_GROUP_MAX_D = 16;
constexpr size_t SERVE_GROUP_MAX = 64;

uint64_t model_bytes(uint64_t n, uint64_t d) {
  const uint64_t ld = (n + 31) / 32 * 32, cap = std::max<uint64_t>(n, 1);
  // K/L, L⁻¹ (the gradient path), x, diagonal-block inverses, vectors
  return 2 * ld * cap * 8 + cap * d * 8 + ((n + 127) / 128) * 128 * 128 * 8 + 16 * cap * 8 + (1u << 20);
}

}  // namespace

struct gprx_server {
  gprx_server_options opt{};
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::map<uint64_t, std::unique_ptr<Request>> reqs;
  std::map<uint64_t, Model> models;
  uint64_t next_id = 1;
  uint64_t used_bytes = 0;
  bool stopping = false;
  std::vector<std::thread> workers;
  // latency records of finished requests (ns): per kind
  std::vector<int64_t> lat[4];
  uint64_t completed = 0, merged_launches = 0, merged_fit_launches = 0;

  void run_worker();
  // picks a runnable request under the lock; returns its id (0: none)
  uint64_t pick(std::vector<uint64_t>& batch);
  bool admit_fit(uint64_t model, Request* r);
  bool small_predict(const Request* r);
  bool same_tree(uint64_t a, uint64_t b);
  void execute_predict_group(std::vector<uint64_t>& batch);
  void execute(std::vector<uint64_t>& batch);
  void execute_fit_batch(std::vector<uint64_t>& batch);
  void finish(Request* r, gprx_status st, const char* why);
};

bool gprx_server::small_predict(const Request* r) {
  if (r->kind != PREDICT) return false;
  const Model& m = models[r->model];
  return m.ready && !m.online && !m.failed && m.n <= SERVE_GROUP_MAX_N && m.d <= SERVE_GROUP_MAX_D &&
         r->q <= SERVE_GROUP_MAX_Q;
}

// Models fitted with the same kernel tree (so one grouped launch serves both).
bool gprx_server::same_tree(uint64_t a, uint64_t b) {
  auto ra = reqs.find(models[a].fit_req), rb = reqs.find(models[b].fit_req);
  if (ra == reqs.end() || rb == reqs.end()) return false;
  const auto &na = ra->second->nodes, &nb = rb->second->nodes;
  if (na.size() != nb.size() || models[a].d != models[b].d) return false;
  for (size_t i = 0; i < na.size(); ++i)
    if (na[i].kind != nb[i].kind || na[i].arg != nb[i].arg) return false;
  return true;
}

// Makes room for a fit of r's size in the HBM budget (evicting idle resident
// models, least recently used first) and accounts it; false if it does not fit.
bool gprx_server::admit_fit(uint64_t model, Request* r) {
  const uint64_t need = model_bytes(r->n, r->d);
  if (used_bytes + need > opt.hbm_budget_bytes) {
    std::vector<std::pair<int64_t, uint64_t>> idle;
    for (auto& o : models)
      if (o.first != model && o.second.ready && !o.second.busy && o.second.queue.empty())
        idle.push_back({o.second.last_used, o.first});
    std::sort(idle.begin(), idle.end());
    uint64_t freeable = 0;
    for (auto& e : idle) freeable += models[e.second].bytes;
    if (used_bytes - std::min(used_bytes, freeable) + need > opt.hbm_budget_bytes) return false;
    for (auto& e : idle) {
      if (used_bytes + need <= opt.hbm_budget_bytes) break;
      Model& o = models[e.second];
      gprx_exact_destroy(o.h);
      o.h = nullptr;
      o.ready = false;
      o.failed = true;  // later requests on an evicted model fail
      used_bytes -= o.bytes;
      o.bytes = 0;
    }
  }
  Model& m = models[model];
  m.bytes = need;
  used_bytes += need;
  return true;
}

uint64_t gprx_server::pick(std::vector<uint64_t>& batch) {
  batch.clear();
  // oldest runnable head across models (a fit must fit in the HBM budget,
  // possibly after evicting idle models)
  uint64_t best = 0;
  int64_t best_t = INT64_MAX;
  for (auto& kv : models) {
    Model& m = kv.second;
    if (m.busy || m.queue.empty()) continue;
    Request* r = reqs[m.queue.front()].get();
    if (r->t_submit >= best_t) continue;
    if (r->kind == FIT && used_bytes + model_bytes(r->n, r->d) > opt.hbm_budget_bytes) {
      uint64_t freeable = 0;
      for (auto& o : models)
        if (o.first != kv.first && o.second.ready && !o.second.busy && o.second.queue.empty()) freeable += o.second.bytes;
      if (used_bytes - std::min(used_bytes, freeable) + model_bytes(r->n, r->d) > opt.hbm_budget_bytes) continue;
    }
    best_t = r->t_submit;
    best = kv.first;
  }
  if (!best) return 0;
  Model& m = models[best];
  Request* head = reqs[m.queue.front()].get();
  if (head->kind == FIT && !admit_fit(best, head)) return 0;
  batch.push_back(head->id);
  m.queue.pop_front();
  m.busy = true;
  if (head->kind == PREDICT && small_predict(head)) {
    // small predicts: this model's consecutive ones, then the other models'
    // waiting at the heads of their queues, share one grouped launch
    while (!m.queue.empty() && batch.size() < SERVE_GROUP_MAX) {
      Request* nx = reqs[m.queue.front()].get();
      if (!small_predict(nx) || nx->vkind != head->vkind) break;
      batch.push_back(nx->id);
      m.queue.pop_front();
    }
    std::vector<std::pair<int64_t, uint64_t>> cand;
    for (auto& kv : models) {
      Model& o = kv.second;
      if (kv.first == best || o.busy || o.queue.empty()) continue;
      Request* r = reqs[o.queue.front()].get();
      if (small_predict(r) && r->vkind == head->vkind && same_tree(best, kv.first))
        cand.push_back({r->t_submit, kv.first});
    }
    std::sort(cand.begin(), cand.end());
    for (auto& c : cand) {
      Model& o = models[c.second];
      bool took = false;
      while (!o.queue.empty() && batch.size() < SERVE_GROUP_MAX) {
        Request* r = reqs[o.queue.front()].get();
        if (!small_predict(r) || r->vkind != head->vkind) break;
        batch.push_back(r->id);
        o.queue.pop_front();
        took = true;
      }
      if (took) o.busy = true;
      if (batch.size() >= SERVE_GROUP_MAX) break;
    }
  } else if (head->kind == PREDICT) {
    // consecutive predicts of the same kind share one launch
    while (!m.queue.empty()) {
      Request* nx = reqs[m.queue.front()].get();
      if (nx->kind != PREDICT || nx->vkind != head->vkind || small_predict(nx)) break;
      batch.push_back(nx->id);
      m.queue.pop_front();
    }
  } else if (batched_fit(head)) {
    // other models' waiting small fits join the same batched launch, oldest first
    std::vector<std::pair<int64_t, uint64_t>> cand;
    for (auto& kv : models) {
      Model& o = kv.second;
      if (kv.first == best || o.busy || o.queue.empty()) continue;
      Request* r = reqs[o.queue.front()].get();
      if (batched_fit(r) && fit_compatible(head, r)) cand.push_back({r->t_submit, kv.first});
    }
    std::sort(cand.begin(), cand.end());
    for (auto& c : cand) {
      if (batch.size() >= SERVE_BATCH_FIT_MAX) break;
      Model& o = models[c.second];
      Request* r = reqs[o.queue.front()].get();
      if (!admit_fit(c.second, r)) continue;
      batch.push_back(r->id);
      o.queue.pop_front();
      o.busy = true;
    }
  }
  const int64_t t = now_ns();
  for (uint64_t id : batch) reqs[id]->t_start = t;
  return best;
}

void gprx_server::finish(Request* r, gprx_status st, const char* why) {
  r->status = st;
  if (st != GPRX_OK) {
    gprx_error_info info;
    gprx_last_error(&info);
    r->message = why ? why : info.message;
  }
}

// Small fits (one or several models): the batched evaluator fits every
// problem (device L-BFGS, one CTA per problem), then each model is factored
// at its fitted θ on its own handle for the requests that follow.
void gprx_server::execute_fit_batch(std::vector<uint64_t>& batch) {
  std::vector<Request*> rs;
  {
    std::lock_guard<std::mutex> lock(mu);
    for (uint64_t id : batch) rs.push_back(reqs[id].get());
  }
  const Request* h0 = rs[0];
  const size_t k = rs.size();
  const uint64_t d = h0->d, p = h0->theta.size();
  std::vector<uint64_t> ns(k);
  std::vector<double> xall, yall, th0(k * p), thf(k * p);
  for (size_t i = 0; i < k; ++i) {
    ns[i] = rs[i]->n;
    xall.insert(xall.end(), rs[i]->x.begin(), rs[i]->x.end());
    yall.insert(yall.end(), rs[i]->y.begin(), rs[i]->y.end());
    std::copy(rs[i]->theta.begin(), rs[i]->theta.end(), th0.begin() + i * p);
  }
  std::vector<gprx_fit_report> reps(k);
  std::vector<int32_t> pst(k, GPRX_OK);
  gprx_batch* b = nullptr;
  gprx_options bo = h0->opt;
  bo.device = opt.device;
  gprx_status st = gprx_batch_create(xall.data(), yall.data(), ns.data(), k, d, h0->nodes.data(),
                                     (int32_t)h0->nodes.size(), (int32_t)p, &bo, &b);
  std::string why;
  if (st == GPRX_OK) st = gprx_batch_fit(b, th0.data(), p, &h0->lopt, thf.data(), reps.data(), pst.data());
  if (st != GPRX_OK) {
    gprx_error_info info;
    gprx_last_error(&info);
    why = info.message;
  }
  if (b) gprx_batch_destroy(b);
  std::vector<gprx_exact*> hs(k, nullptr);
  std::vector<gprx_status> sts(k, st);
  for (size_t i = 0; i < k; ++i) {
    Request* r = rs[i];
    if (st == GPRX_OK) {
      sts[i] = (gprx_status)pst[i];
      if (sts[i] == GPRX_OK)
        sts[i] = gprx_exact_create(r->x.data(), r->n, r->d, r->y.data(), r->nodes.data(), (int32_t)r->nodes.size(),
                                   thf.data() + i * p, (int32_t)p, &r->opt, &hs[i]);
      if (sts[i] == GPRX_OK) sts[i] = gprx_exact_factor(hs[i]);
      if (sts[i] != GPRX_OK && hs[i]) {
        gprx_exact_destroy(hs[i]);
        hs[i] = nullptr;
      }
      finish(r, sts[i], nullptr);
    } else {
      finish(r, st, why.c_str());
    }
    r->merged = (int)k;
  }
  std::lock_guard<std::mutex> lock(mu);
  const int64_t t = now_ns();
  if (k > 1) ++merged_fit_launches;
  for (size_t i = 0; i < k; ++i) {
    Request* r = rs[i];
    Model& m = models[r->model];
    m.h = hs[i];
    m.d = r->d;
    m.n = r->n;
    m.fit_req = r->id;
    m.ready = hs[i] != nullptr;
    m.failed = hs[i] == nullptr;
    if (m.failed && m.bytes) {
      used_bytes -= m.bytes;
      m.bytes = 0;
    }
    m.busy = false;
    m.last_used = t;
    r->t_end = t;
    r->done = true;
    lat[r->kind].push_back(r->t_end - r->t_submit);
    ++completed;
  }
  cv_done.notify_all();
  cv_work.notify_all();
}

// Small predicts of one or several models in one grouped launch.
void gprx_server::execute_predict_group(std::vector<uint64_t>& batch) {
  std::vector<Request*> rs;
  std::vector<gprx_exact*> hs;
  {
    std::lock_guard<std::mutex> lock(mu);
    for (uint64_t id : batch) {
      rs.push_back(reqs[id].get());
      hs.push_back(models[rs.back()->model].h);
    }
  }
  const size_t k = rs.size();
  std::vector<const double*> xs(k);
  std::vector<uint64_t> qs(k);
  std::vector<double*> means(k), vars(k);
  for (size_t i = 0; i < k; ++i) {
    xs[i] = rs[i]->xs.data();
    qs[i] = rs[i]->q;
    means[i] = rs[i]->mean_out;
    vars[i] = rs[i]->var_out;
  }
  const gprx_status st =
      gprx_exact_predict_group(hs.data(), k, xs.data(), qs.data(), rs[0]->vkind, means.data(), vars.data());
  for (Request* r : rs) {
    r->merged = (int)k;
    finish(r, st, nullptr);
  }
  std::lock_guard<std::mutex> lock(mu);
  const int64_t t = now_ns();
  if (k > 1) ++merged_launches;
  for (Request* r : rs) {
    Model& m = models[r->model];
    m.busy = false;
    m.last_used = t;
    r->t_end = t;
    r->done = true;
    lat[r->kind].push_back(r->t_end - r->t_submit);
    ++completed;
  }
  cv_done.notify_all();
  cv_work.notify_all();
}

void gprx_server::execute(std::vector<uint64_t>& batch) {
  bool small_fit, group;
  {
    std::lock_guard<std::mutex> lock(mu);
    small_fit = batched_fit(reqs[batch[0]].get());
    group = small_predict(reqs[batch[0]].get());
  }
  if (small_fit) {
    execute_fit_batch(batch);
    return;
  }
  if (group) {
    execute_predict_group(batch);
    return;
  }
  std::vector<Request*> rs;
  Model* mp;
  gprx_exact* h;
  uint64_t md;
  bool failed, online;
  {
    std::lock_guard<std::mutex> lock(mu);
    for (uint64_t id : batch) rs.push_back(reqs[id].get());
    mp = &models[rs[0]->model];
    h = mp->h;
    md = mp->d;
    failed = mp->failed;
    online = mp->online;
  }
  Request* head = rs[0];
  bool ready = false;
  uint64_t n_now = 0;
  if (failed && head->kind != FIT) {
    for (Request* r : rs) finish(r, GPRX_INVALID_CONFIG, "the model is not resident");
  } else if (head->kind == FIT) {
    gprx_exact* nh = nullptr;
    gprx_status st = gprx_exact_create(head->x.data(), head->n, head->d, head->y.data(), head->nodes.data(),
                                       (int32_t)head->nodes.size(), head->theta.data(), (int32_t)head->theta.size(),
                                       &head->opt, &nh);
    if (st == GPRX_OK) {
      if (head->optimize) {
        gprx_fit_report rep;
        st = gprx_exact_fit(nh, &head->lopt, &rep);
      } else {
        st = gprx_exact_factor(nh);
      }
    }
    finish(head, st, nullptr);
    if (st == GPRX_OK) {
      h = nh;
      md = head->d;
      ready = true;
    } else {
      if (nh) gprx_exact_destroy(nh);
      failed = true;
    }
  } else if (head->kind == PREDICT) {
    uint64_t total = 0;
    for (Request* r : rs) total += r->q;
    std::vector<double> xs(total * md), mean(total), var(total);
    uint64_t off = 0;
    for (Request* r : rs) {
      for (uint64_t f = 0; f < md; ++f)
        std::memcpy(xs.data() + f * total + off, r->xs.data() + f * r->q, sizeof(double) * r->q);
      off += r->q;
    }
    gprx_status st = gprx_exact_predict(h, xs.data(), total, head->vkind, mean.data(), var.data());
    off = 0;
    for (Request* r : rs) {
      if (st == GPRX_OK) {
        std::memcpy(r->mean_out, mean.data() + off, sizeof(double) * r->q);
        std::memcpy(r->var_out, var.data() + off, sizeof(double) * r->q);
      }
      r->merged = (int)rs.size();
      off += r->q;
      finish(r, st, nullptr);
    }
  } else {
    gprx_status st = GPRX_OK;
    if (!online) {
      st = gprx_online_begin(h);
      if (st == GPRX_OK) online = true;
    }
    if (head->kind == ADD) {
      std::vector<double> xi(md);
      for (uint64_t i = 0; i < head->n && st == GPRX_OK; ++i) {
        for (uint64_t f = 0; f < md; ++f) xi[f] = head->x[f * head->n + i];
        st = gprx_online_insert(h, xi.data(), head->y[i], head->ids_out ? head->ids_out + i : nullptr);
      }
    } else {
      for (size_t i = 0; i < head->ids.size() && st == GPRX_OK; ++i) st = gprx_online_delete(h, head->ids[i]);
    }
    n_now = gprx_online_n(h);
    finish(head, st, nullptr);
  }
  std::lock_guard<std::mutex> lock(mu);
  Model& m = *mp;
  if (head->kind == FIT) {
    m.h = ready ? h : nullptr;
    m.d = md;
    m.n = head->n;
    m.fit_req = head->id;
    m.ready = ready;
  }
  if (online && n_now) m.n = n_now;
  m.failed = failed;
  m.online = online;
  const int64_t t = now_ns();
  if (rs.size() > 1) ++merged_launches;
  for (Request* r : rs) {
    r->t_end = t;
    r->done = true;
    lat[r->kind].push_back(r->t_end - r->t_submit);
    ++completed;
  }
  if (m.failed && m.bytes) {
    used_bytes -= m.bytes;
    m.bytes = 0;
  }
  if (online && n_now) {
    // online growth: account the model at its current size
    const uint64_t nb = model_bytes(n_now, m.d);
    if (nb > m.bytes) {
      used_bytes += nb - m.bytes;
      m.bytes = nb;
    }
  }
  m.busy = false;
  m.last_used = t;
  cv_done.notify_all();
  cv_work.notify_all();
}

void gprx_server::run_worker() {
  std::vector<uint64_t> batch;
  cudaSetDevice(opt.device);
  for (;;) {
    {
      std::unique_lock<std::mutex> lock(mu);
      for (;;) {
        if (stopping) return;
        if (pick(batch)) break;
        cv_work.wait(lock);
      }
    }
    execute(batch);
  }
}

extern "C" {

void gprx_server_options_default(gprx_server_options* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->device = 0;
  o->workers = 8;
  o->hbm_budget_bytes = 150ull << 30;
}

gprx_status gprx_server_create(const gprx_server_options* o, gprx_server** out) {
  if (!out) return GPRX_INVALID_ARGUMENT;
  std::unique_ptr<gprx_server> s(new (std::nothrow) gprx_server());
  if (!s) return GPRX_OUT_OF_MEMORY;
  if (o) s->opt = *o;
  else gprx_server_options_default(&s->opt);
  if (s->opt.workers < 1 || s->opt.workers > 64) return GPRX_INVALID_CONFIG;
  for (int i = 0; i < s->opt.workers; ++i) s->workers.emplace_back([p = s.get()] { p->run_worker(); });
  *out = s.release();
  return GPRX_OK;
}

gprx_status gprx_server_destroy(gprx_server* s) {
  if (!s) return GPRX_INVALID_ARGUMENT;
  {
    std::lock_guard<std::mutex> lock(s->mu);
    s->stopping = true;
  }
  s->cv_work.notify_all();
  for (auto& t : s->workers) t.join();
  for (auto& kv : s->models)
    if (kv.second.h) gprx_exact_destroy(kv.second.h);
  delete s;
  return GPRX_OK;
}

static uint64_t enqueue(gprx_server* s, std::unique_ptr<Request> r) {
  std::lock_guard<std::mutex> lock(s->mu);
  const uint64_t id = s->next_id++;
  r->id = id;
  if (r->kind == FIT) {
    r->model = id;
    s->models[id] = Model();
  }
  r->t_submit = now_ns();
  s->models[r->model].queue.push_back(id);
  s->reqs[id] = std::move(r);
  s->cv_work.notify_one();
  return id;
}

gprx_status gprx_server_fit(gprx_server* s, const double* x, uint64_t n, uint64_t d, const double* y,
                            const gprx_kernel_node* nodes, int32_t n_nodes, const double* theta, int32_t n_theta,
                            const gprx_options* options, const gprx_lbfgs_options* lbfgs, int32_t optimize,
                            uint64_t* request_id) {
  if (!s || !x || !y || !nodes || !theta || !request_id || n_nodes <= 0 || n_theta <= 0)
    return GPRX_INVALID_ARGUMENT;
  if (n == 0 || d == 0) return GPRX_EMPTY_INPUT;
  std::unique_ptr<Request> r(new Request());
  r->kind = FIT;
  r->x.assign(x, x + n * d);
  r->y.assign(y, y + n);
  r->nodes.assign(nodes, nodes + n_nodes);
  r->theta.assign(theta, theta + n_theta);
  r->n = n;
  r->d = d;
  if (options) r->opt = *options;
  else gprx_options_default(&r->opt);
  r->opt.device = s->opt.device;
  if (lbfgs) r->lopt = *lbfgs;
  else gprx_lbfgs_options_default(&r->lopt);
  r->optimize = optimize;
  if (model_bytes(n, d) > s->opt.hbm_budget_bytes) return GPRX_OUT_OF_MEMORY;
  *request_id = enqueue(s, std::move(r));
  return GPRX_OK;
}

static gprx_status check_model(gprx_server* s, uint64_t model, uint64_t d_given, bool check_d) {
  std::lock_guard<std::mutex> lock(s->mu);
  auto it = s->models.find(model);
  if (it == s->models.end()) return GPRX_INVALID_ARGUMENT;
  if (check_d) {
    auto rq = s->reqs.find(model);  // the model's fit request holds d
    if (rq != s->reqs.end() && rq->second->d != d_given) return GPRX_SHAPE_MISMATCH;
  }
  return GPRX_OK;
}

gprx_status gprx_server_predict(gprx_server* s, uint64_t model, const double* xs, uint64_t q, uint64_t d,
                                int32_t variance_kind, double* mean, double* var, uint64_t* request_id) {
  if (!s || !xs || !mean || !var || !request_id) return GPRX_INVALID_ARGUMENT;
  if (q == 0) return GPRX_EMPTY_INPUT;
  gprx_status st = check_model(s, model, d, true);
  if (st != GPRX_OK) return st;
  std::unique_ptr<Request> r(new Request());
  r->kind = PREDICT;
  r->model = model;
  r->xs.assign(xs, xs + q * d);
  r->q = q;
  r->vkind = variance_kind;
  r->mean_out = mean;
  r->var_out = var;
  *request_id = enqueue(s, std::move(r));
  return GPRX_OK;
}

gprx_status gprx_server_add(gprx_server* s, uint64_t model, const double* x, const double* y, uint64_t k, uint64_t d,
                            uint64_t* ids_out, uint64_t* request_id) {
  if (!s || !x || !y || !request_id) return GPRX_INVALID_ARGUMENT;
  if (k == 0) return GPRX_EMPTY_INPUT;
  gprx_status st = check_model(s, model, d, true);
  if (st != GPRX_OK) return st;
  std::unique_ptr<Request> r(new Request());
  r->kind = ADD;
  r->model = model;
  r->x.assign(x, x + k * d);
  r->y.assign(y, y + k);
  r->n = k;
  r->ids_out = ids_out;
  *request_id = enqueue(s, std::move(r));
  return GPRX_OK;
}

gprx_status gprx_server_remove(gprx_server* s, uint64_t model, const uint64_t* ids, uint64_t k,
                               uint64_t* request_id) {
  if (!s || !ids || !request_id) return GPRX_INVALID_ARGUMENT;
  if (k == 0) return GPRX_EMPTY_INPUT;
  gprx_status st = check_model(s, model, 0, false);
  if (st != GPRX_OK) return st;
  std::unique_ptr<Request> r(new Request());
  r->kind = REMOVE;
  r->model = model;
  r->ids.assign(ids, ids + k);
  *request_id = enqueue(s, std::move(r));
  return GPRX_OK;
}

gprx_status gprx_server_wait(gprx_server* s, uint64_t request_id, gprx_request_info* info) {
  if (!s) return GPRX_INVALID_ARGUMENT;
  std::unique_lock<std::mutex> lock(s->mu);
  auto it = s->reqs.find(request_id);
  if (it == s->reqs.end()) return GPRX_INVALID_ARGUMENT;
  Request* r = it->second.get();
  s->cv_done.wait(lock, [r] { return r->done; });
  if (info) {
    std::memset(info, 0, sizeof(*info));
    info->status = r->status;
    info->model = r->model;
    info->kind = r->kind;
    info->submit_ns = r->t_submit;
    info->start_ns = r->t_start;
    info->end_ns = r->t_end;
    info->merged = r->merged;
    std::strncpy(info->message, r->message.c_str(), sizeof(info->message) - 1);
  }
  const gprx_status st = r->status;
  if (r->kind != FIT) s->reqs.erase(it);  // a fit request stays: it describes its model
  return st;
}

gprx_status gprx_server_stats(gprx_server* s, gprx_server_stats_t* out) {
  if (!s || !out) return GPRX_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(s->mu);
  std::memset(out, 0, sizeof(*out));
  out->completed = s->completed;
  out->merged_launches = s->merged_launches;
  out->merged_fit_launches = s->merged_fit_launches;
  out->used_bytes = s->used_bytes;
  uint64_t resident = 0;
  for (auto& kv : s->models)
    if (kv.second.ready) ++resident;
  out->resident_models = resident;
  return GPRX_OK;
}

}  // extern "C"
