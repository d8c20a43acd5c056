// lbm_server.cpp — the serving form: a request queue over one batch.
//
// Requests (one solve each: a case, its storage options, a step budget and
// an optional residual tolerance) arrive with lbm_server_submit and wait in
// a queue.  lbm_server_progress drives the loop one chunk at a time:
//   1. admission: queued requests become batch members while their state
//      fits the batch's HBM pool (lbm_batch_add reports LBM_ERR_BUDGET when
//      it does not) and, optionally, while the resident backlog (lattice
//      updates still owed) stays under backlog_horizon_s seconds of work at
//      nominal_mlups.  FIFO admits in arrival order and stops at the first
//      request that does not fit (no overtaking); SHORTEST admits the
//      queued requests with the least work (nodes x steps) first and skips
//      those that do not fit;
//   2. one chunk of steps for every resident request (continuous batching:
//      members join and leave between chunks, lbm_batch_step);
//   3. retirement: a request that reached its step budget, or whose density
//      residual sum |rho_k - rho_(k-1)| (the quantity kernel.cu:232-248
//      prints) fell to its tolerance at a check (every check_every steps),
//      has its rho and u copied to host buffers and its device memory
//      returned to the pool.
// Time stamps (arrival, admission, result on the host) come from one
// steady clock; lbm_server_stats reports p50/p99 of time-to-solution
// (arrival -> result) and of service time (admission -> result) over the
// completed requests, with the lattice updates executed and completed.
//
// Chunk issue is paced: at most kInflight chunks are queued on the batch
// stream ahead of the GPU (an event after each), so a request admitted now
// starts behind at most that much work instead of behind every step the
// resident requests still owe.
//
// The residual check reduces the member's density fields through
// lbm_field_diagnostics_static (no allocation; it synchronises the batch
// stream, so checks are spaced by check_every steps).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <deque>
#include <map>
#include <new>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/lbm_b200.h"
#include "lbm_internal.h"

namespace {

enum { kQueued = LBM_REQ_QUEUED, kResident = LBM_REQ_RESIDENT, kDone = LBM_REQ_DONE };
constexpr int kInflight = 2;

struct Request {
  Inputval in;
  lbm_options opt;
  long long steps = 0;
  double tol = 0.0;
  double t_arrive = 0, t_admit = -1, t_done = -1;
  long long nodes = 0;
  size_t bytes = 0;
  int member = -1;
  int state = kQueued;
  long long steps_done = 0;
  long long next_check = 0;
  double residual = -1.0;
  int converged = 0;
  std::vector<float> den, ux, uy, uz;
};

double percentile(std::vector<double> v, double p) {
  if (v.empty()) return 0.0;
  std::sort(v.begin(), v.end());
  const double r = p / 100.0 * (double)(v.size() - 1);
  const size_t i = (size_t)std::floor(r);
  const double f = r - (double)i;
  return i + 1 < v.size() ? v[i] * (1.0 - f) + v[i + 1] * f : v[i];
}

}  // namespace

struct lbm_server {
  lbm_server_options opt;
  lbm_batch* b = nullptr;
  std::chrono::steady_clock::time_point t0;
  std::map<int, Request> reqs;
  std::deque<int> queue;
  std::map<int, int> by_member;  // batch member id -> request id
  int next_id = 1;
  long long submitted = 0, admitted = 0, completed = 0, converged = 0;
  double executed_lups = 0, completed_lups = 0;
  std::vector<double> tts, service;
  // smallest request that did not fit since memory was last returned
  size_t fail_bytes = SIZE_MAX;
  std::deque<cudaEvent_t> inflight;  // one event after each queued chunk
  std::vector<cudaEvent_t> spare;
  double now() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
};

namespace {

int chunk_of(const lbm_server* s) {
  return s->opt.batch.chunk_steps > 0 ? s->opt.batch.chunk_steps : 32;
}

// resident backlog: lattice updates the resident requests still owe
double backlog(const lbm_server* s) {
  double r = 0;
  for (auto& kv : s->by_member) {
    const Request& q = s->reqs.at(kv.second);
    r += (double)q.nodes * (double)(q.steps - q.steps_done);
  }
  return r;
}

// copy rho, u of a resident request to its host buffers, release its
// member and mark it done
int retire(lbm_server* s, int rid, bool at_target) {
  Request& q = s->reqs.at(rid);
  q.den.resize(q.nodes);
  q.ux.resize(q.nodes);
  q.uy.resize(q.nodes);
  q.uz.resize(q.nodes);
  int rc;
  if (at_target) {
    rc = lbm_batch_fetch(s->b, q.member, q.den.data(), q.ux.data(), q.uy.data(), q.uz.data());
  } else {
    lbm_domain* d = nullptr;
    rc = lbm_batch_domain(s->b, q.member, &d);
    if (!rc) rc = lbm_get_macroscopic(d, q.den.data(), q.ux.data(), q.uy.data(), q.uz.data());
  }
  if (rc) return rc;
  if ((rc = lbm_batch_remove(s->b, q.member))) return rc;
  s->fail_bytes = SIZE_MAX;
  s->by_member.erase(q.member);
  q.member = -1;
  q.state = kDone;
  q.t_done = s->now();
  ++s->completed;
  if (!at_target) ++s->converged;
  s->completed_lups += (double)q.nodes * (double)q.steps_done;
  s->tts.push_back(q.t_done - q.t_arrive);
  s->service.push_back(q.t_done - q.t_admit);
  return LBM_OK;
}

// try to make queued request rid a batch member; LBM_ERR_BUDGET if its state
// does not fit the pool now
int admit(lbm_server* s, int rid) {
  Request& q = s->reqs.at(rid);
  if (q.bytes >= s->fail_bytes) return LBM_ERR_BUDGET;  // a smaller one already failed
  int member = 0;
  const int rc = lbm_batch_add(s->b, &q.in, &q.opt, q.steps, &member);
  if (rc == LBM_ERR_BUDGET) {
    s->fail_bytes = std::min(s->fail_bytes, q.bytes);
    lbm::clear_error();
  }
  if (rc) return rc;
  q.member = member;
  q.state = kResident;
  q.t_admit = s->now();
  q.next_check = s->opt.check_every;
  s->by_member[member] = rid;
  ++s->admitted;
  return LBM_OK;
}

int admit_queued(lbm_server* s) {
  const double cap = s->opt.backlog_horizon_s > 0 && s->opt.nominal_mlups > 0
                         ? s->opt.backlog_horizon_s * s->opt.nominal_mlups * 1e6
                         : HUGE_VAL;
  double owed = backlog(s);
  if (s->opt.policy == LBM_SERVE_FIFO) {
    while (!s->queue.empty() && owed < cap) {
      const int rid = s->queue.front();
      const int rc = admit(s, rid);
      if (rc == LBM_ERR_BUDGET) break;  // head-of-line: no overtaking
      if (rc) return rc;
      s->queue.pop_front();
      const Request& q = s->reqs.at(rid);
      owed += (double)q.nodes * (double)q.steps;
    }
    return LBM_OK;
  }
  // SHORTEST: least work first, skipping what does not fit
  std::vector<int> order(s->queue.begin(), s->queue.end());
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
    const Request& x = s->reqs.at(a);
    const Request& y = s->reqs.at(b);
    return (double)x.nodes * (double)x.steps < (double)y.nodes * (double)y.steps;
  });
  for (int rid : order) {
    if (owed >= cap) break;
    const int rc = admit(s, rid);
    if (rc == LBM_ERR_BUDGET) continue;
    if (rc) return rc;
    s->queue.erase(std::find(s->queue.begin(), s->queue.end(), rid));
    const Request& q = s->reqs.at(rid);
    owed += (double)q.nodes * (double)q.steps;
  }
  return LBM_OK;
}

// wait until fewer than kInflight chunks are queued ahead of the GPU
int pace(lbm_server* s) {
  while ((int)s->inflight.size() >= kInflight) {
    cudaEvent_t e = s->inflight.front();
    if (cudaEventSynchronize(e) != cudaSuccess)
      return lbm::set_error(LBM_ERR_CUDA, "waiting for a chunk: %s",
                            cudaGetErrorString(cudaGetLastError()));
    s->inflight.pop_front();
    s->spare.push_back(e);
  }
  return LBM_OK;
}

// record an event after the chunk just issued on the batch stream
int mark_chunk(lbm_server* s) {
  cudaEvent_t e = nullptr;
  if (!s->spare.empty()) {
    e = s->spare.back();
    s->spare.pop_back();
  } else if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
    return lbm::set_error(LBM_ERR_CUDA, "event creation failed");
  }
  if (cudaEventRecord(e, (cudaStream_t)lbm::batch_stream(s->b)) != cudaSuccess) {
    cudaEventDestroy(e);
    return lbm::set_error(LBM_ERR_CUDA, "event record failed");
  }
  s->inflight.push_back(e);
  return LBM_OK;
}

void free_events(lbm_server* s) {
  if (!s->b) return;
  cudaSetDevice(lbm::batch_device(s->b));
  for (cudaEvent_t e : s->inflight) cudaEventDestroy(e);
  for (cudaEvent_t e : s->spare) cudaEventDestroy(e);
  s->inflight.clear();
  s->spare.clear();
}

}  // namespace

extern "C" {

void lbm_server_default_options(lbm_server_options* so) {
  if (!so) return;
  std::memset(so, 0, sizeof(*so));
  lbm_batch_default_options(&so->batch);
  so->policy = LBM_SERVE_FIFO;
  so->check_every = 256;
}

int lbm_server_create(const lbm_server_options* so, lbm_server** out) {
  if (!out) return lbm::set_error(LBM_ERR_INVALID, "NULL out");
  *out = nullptr;
  lbm_server_options o;
  if (so)
    o = *so;
  else
    lbm_server_default_options(&o);
  if (o.policy != LBM_SERVE_FIFO && o.policy != LBM_SERVE_SHORTEST)
    return lbm::set_error(LBM_ERR_INVALID, "unknown admission policy %d", o.policy);
  const int chunk = o.batch.chunk_steps > 0 ? o.batch.chunk_steps : 32;
  if (o.check_every < chunk || o.check_every % chunk)
    return lbm::set_error(LBM_ERR_INVALID,
                          "check_every (%d) must be a positive multiple of the chunk (%d steps)",
                          o.check_every, chunk);
  if (!(o.backlog_horizon_s >= 0) || !(o.nominal_mlups >= 0))
    return lbm::set_error(LBM_ERR_INVALID, "bad backlog horizon");
  lbm_server* s = new (std::nothrow) lbm_server();
  if (!s) return lbm::set_error(LBM_ERR_OOM, "host allocation failed");
  s->opt = o;
  const int rc = lbm_batch_create(&o.batch, &s->b);
  if (rc) {
    delete s;
    return rc;
  }
  s->t0 = std::chrono::steady_clock::now();
  *out = s;
  return LBM_OK;
}

int lbm_server_destroy(lbm_server* s) {
  if (!s) return lbm::set_error(LBM_ERR_INVALID, "NULL server");
  free_events(s);
  const int rc = lbm_batch_destroy(s->b);
  delete s;
  return rc;
}

int lbm_server_submit(lbm_server* s, const Inputval* pinput, const lbm_options* opt,
                      long long steps, double tol, int* id) {
  if (!s || !pinput || !id) return lbm::set_error(LBM_ERR_INVALID, "NULL argument");
  if (steps < 1) return lbm::set_error(LBM_ERR_INVALID, "a request needs at least one step");
  if (!(tol >= 0)) return lbm::set_error(LBM_ERR_INVALID, "tolerance must be >= 0");
  size_t bytes = 0;
  int rc = lbm_batch_domain_bytes(pinput, opt, &bytes);
  if (rc) return rc;
  if (bytes > s->opt.batch.hbm_budget)
    return lbm::set_error(LBM_ERR_BUDGET, "request of %zu bytes exceeds the HBM budget", bytes);
  if (tol > 0 && (long long)pinput->nx * pinput->ny * pinput->nz > 67108864)
    return lbm::set_error(LBM_ERR_INVALID,
                          "a residual tolerance needs a domain of at most 67,108,864 nodes");
  Request q;
  q.in = *pinput;
  if (opt)
    q.opt = *opt;
  else
    lbm_default_options(&q.opt);
  q.steps = steps;
  q.tol = tol;
  q.nodes = (long long)pinput->nx * pinput->ny * pinput->nz;
  q.bytes = bytes;
  q.t_arrive = s->now();
  const int rid = s->next_id++;
  s->reqs.emplace(rid, std::move(q));
  s->queue.push_back(rid);
  ++s->submitted;
  *id = rid;
  return LBM_OK;
}

int lbm_server_progress(lbm_server* s, int* completed) {
  if (!s) return lbm::set_error(LBM_ERR_INVALID, "NULL server");
  const long long before = s->completed;
  int rc = admit_queued(s);
  if (rc) return rc;
  if (!s->by_member.empty()) {
    const int chunk = chunk_of(s);
    if ((rc = pace(s))) return rc;
    if ((rc = lbm_batch_step(s->b, chunk))) return rc;
    if ((rc = mark_chunk(s))) return rc;
    for (auto& kv : s->by_member) {
      Request& q = s->reqs.at(kv.second);
      const long long took = std::min<long long>(chunk, q.steps - q.steps_done);
      q.steps_done += took;
      s->executed_lups += (double)q.nodes * (double)took;
    }
    // residual checks of the requests with a tolerance
    std::vector<int> early;
    for (auto& kv : s->by_member) {
      Request& q = s->reqs.at(kv.second);
      if (q.tol <= 0 || q.steps_done >= q.steps || q.steps_done < q.next_check) continue;
      q.next_check += s->opt.check_every;
      lbm_domain* d = nullptr;
      float *den = nullptr, *prev = nullptr, *ux = nullptr, *uy = nullptr, *uz = nullptr;
      double diag[8];
      if ((rc = lbm_batch_domain(s->b, kv.first, &d)) ||
          (rc = lbm_device_fields(d, &den, &prev, &ux, &uy, &uz)) ||
          (rc = lbm_field_diagnostics_static(den, prev, ux, uy, uz, q.nodes, diag,
                                             lbm_get_stream(d))))
        return rc;
      q.residual = diag[4];
      if (diag[4] <= q.tol) {
        q.converged = 1;
        early.push_back(kv.second);
      }
    }
    for (int rid : early)
      if ((rc = retire(s, rid, false))) return rc;
    // requests at their step budget
    int ids[256];
    for (;;) {
      int n = 0;
      if ((rc = lbm_batch_poll(s->b, ids, 256, &n))) return rc;
      if (n == 0) break;
      for (int i = 0; i < n; ++i) {
        auto it = s->by_member.find(ids[i]);
        if (it == s->by_member.end()) continue;
        if ((rc = retire(s, it->second, true))) return rc;
      }
      if (n < 256) break;
    }
  }
  if (completed) *completed = (int)(s->completed - before);
  return LBM_OK;
}

int lbm_server_wait(lbm_server* s, int id) {
  if (!s) return lbm::set_error(LBM_ERR_INVALID, "NULL server");
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return lbm::set_error(LBM_ERR_INVALID, "no request %d", id);
  while (it->second.state != kDone) {
    const int rc = lbm_server_progress(s, nullptr);
    if (rc) return rc;
    if (it->second.state == kQueued && s->by_member.empty())
      return lbm::set_error(LBM_ERR_STATE, "request %d cannot be admitted", id);
  }
  return LBM_OK;
}

int lbm_server_result(lbm_server* s, int id, float* den, float* velx, float* vely, float* velz,
                      lbm_server_request* info) {
  if (!s) return lbm::set_error(LBM_ERR_INVALID, "NULL server");
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return lbm::set_error(LBM_ERR_INVALID, "no request %d", id);
  const Request& q = it->second;
  if (info) {
    std::memset(info, 0, sizeof(*info));
    info->state = q.state;
    info->steps_done = q.steps_done;
    info->residual = q.residual;
    info->converged = q.converged;
    info->t_arrive = q.t_arrive;
    info->t_admit = q.t_admit;
    info->t_done = q.t_done;
  }
  if (den || velx || vely || velz) {
    if (q.state != kDone) return lbm::set_error(LBM_ERR_STATE, "request %d is not done", id);
    const size_t nb = (size_t)q.nodes * sizeof(float);
    if (den) std::memcpy(den, q.den.data(), nb);
    if (velx) std::memcpy(velx, q.ux.data(), nb);
    if (vely) std::memcpy(vely, q.uy.data(), nb);
    if (velz) std::memcpy(velz, q.uz.data(), nb);
  }
  return LBM_OK;
}

int lbm_server_release(lbm_server* s, int id) {
  if (!s) return lbm::set_error(LBM_ERR_INVALID, "NULL server");
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return lbm::set_error(LBM_ERR_INVALID, "no request %d", id);
  if (it->second.state != kDone)
    return lbm::set_error(LBM_ERR_STATE, "request %d is not done", id);
  s->reqs.erase(it);
  return LBM_OK;
}

int lbm_server_stats(lbm_server* s, lbm_server_summary* st) {
  if (!s || !st) return lbm::set_error(LBM_ERR_INVALID, "NULL argument");
  std::memset(st, 0, sizeof(*st));
  st->submitted = s->submitted;
  st->admitted = s->admitted;
  st->completed = s->completed;
  st->converged = s->converged;
  st->queued = (long long)s->queue.size();
  st->resident = (long long)s->by_member.size();
  st->elapsed_s = s->now();
  st->tts_p50_s = percentile(s->tts, 50);
  st->tts_p99_s = percentile(s->tts, 99);
  st->service_p50_s = percentile(s->service, 50);
  st->service_p99_s = percentile(s->service, 99);
  st->executed_lups = s->executed_lups;
  st->completed_lups = s->completed_lups;
  st->aggregate_mlups = st->elapsed_s > 0 ? s->executed_lups / st->elapsed_s / 1e6 : 0.0;
  size_t used = 0, largest = 0;
  int nd = 0;
  const int rc = lbm_batch_usage(s->b, &used, &largest, &nd);
  if (rc) return rc;
  st->pool_used_bytes = used;
  return LBM_OK;
}

int lbm_server_batch(lbm_server* s, lbm_batch** b) {
  if (!s || !b) return lbm::set_error(LBM_ERR_INVALID, "NULL argument");
  *b = s->b;
  return LBM_OK;
}

}  // extern "C"
