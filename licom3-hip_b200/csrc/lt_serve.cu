// lt_serve.cu - request server for tracer integrations on one device:
// admission by free HBM, resident state, continuous batching.
//
// One scheduling iteration:
//   1. step every resident request through one batch by k steps, k the
//      smallest remaining step count capped at chunk_steps (enqueued, async);
//   2. meanwhile on the host: queue the requests that have arrived, start
//      building their inputs from the generators on worker threads (at most
//      one per host core in flight), and admit from the head of the queue
//      while their arenas fit the HBM budget (arena allocated, inputs
//      uploaded on the new domain's own stream); they join the batch at the
//      next iteration;
//   3. wait for the step, retire the requests that reached their step count
//      (content sums, optional host copy of the state), free their arenas.
// The queue is first come, first served; a request larger than the whole
// budget is refused.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <deque>
#include <future>
#include <new>
#include <thread>
#include <vector>
#include "lt_domain.h"
#include "../../include/licom_batch.h"
#include "../../include/licom_serve.h"

using namespace lt;

namespace {

struct Req {
  lt_request r;
  lt_request_status st;
  lt_grid grid;
  lt_domain* dom = nullptr;
  int remaining = 0;
  std::vector<double> final_at;
  std::future<std::pair<int, lt_synth*>> inputs;   // generator build on a worker thread
  bool building = false;
};

std::pair<int, lt_synth*> build_inputs(lt_synth_config cfg) {
  lt_synth* syn = nullptr;
  const int rc = lt_synth_build(&cfg, &syn);
  return {rc, syn};
}

}  // namespace

struct lt_server {
  lt_server_config cfg;
  std::chrono::steady_clock::time_point t0;
  std::vector<Req> reqs;        // by id
  std::vector<int> pending;     // not yet arrived, in order of arrival
  size_t next_pending = 0;
  std::deque<int> queue;        // arrived, waiting for memory
  std::vector<int> active;      // resident
  size_t used = 0;
  lt_batch* batch = nullptr;
  std::vector<int> batch_ids;   // membership of `batch`
  lt_server_stats stats{};
  int builders = 4;             // input builds in flight at most
};

namespace {

double now_s(const lt_server* s) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - s->t0).count();
}

void drop_batch(lt_server* s) {
  if (s->batch) lt_batch_destroy(s->batch);
  s->batch = nullptr;
  s->batch_ids.clear();
}

// Arrivals into the queue, then admission from its head.
int admit(lt_server* s) {
  const double t = now_s(s);
  while (s->next_pending < s->pending.size() && s->reqs[s->pending[s->next_pending]].r.arrival <= t) {
    const int id = s->pending[s->next_pending++];
    s->reqs[id].st.state = LT_REQ_QUEUED;
    s->queue.push_back(id);
  }
  // start input builds for the head of the queue
  int in_flight = 0;
  for (int id : s->queue) in_flight += s->reqs[id].building;
  for (int id : s->queue) {
    if (in_flight >= s->builders) break;
    Req& q = s->reqs[id];
    if (q.building || q.st.bytes > s->cfg.hbm_budget) continue;
    q.inputs = std::async(std::launch::async, build_inputs, q.r.domain);
    q.building = true;
    ++in_flight;
  }
  while (!s->queue.empty() && (int)s->active.size() < s->cfg.max_active) {
    Req& q = s->reqs[s->queue.front()];
    if (q.st.bytes > s->cfg.hbm_budget) {
      q.st.state = LT_REQ_REFUSED;
      s->stats.requests_refused++;
      s->queue.pop_front();
      continue;
    }
    if (s->used + q.st.bytes > s->cfg.hbm_budget) break;
    if (!q.building) {
      q.inputs = std::async(std::launch::async, build_inputs, q.r.domain);
      q.building = true;
    }
    // with requests resident, the device keeps stepping them while the head
    // request's inputs are still being built: admit it at a later iteration
    // rather than wait here (first come, first served is kept)
    if (!s->active.empty() && q.inputs.wait_for(std::chrono::seconds(0)) != std::future_status::ready) break;
    auto built = q.inputs.get();
    q.building = false;
    lt_synth* syn = built.second;
    lt_params prm;
    int rc = built.first;
    if (!rc) rc = lt_synth_params(syn, &prm);
    if (!rc) rc = lt_create(&q.grid, &prm, &q.dom);
    if (!rc) rc = lt_synth_upload(syn, q.dom);
    if (syn) lt_synth_free(syn);
    if (rc) {
      if (q.dom) lt_destroy(q.dom);
      q.dom = nullptr;
      if (rc == LT_E_OOM && !s->active.empty()) break;   // wait for memory to free up
      q.st.state = LT_REQ_REFUSED;
      s->stats.requests_refused++;
      s->queue.pop_front();
      continue;
    }
    q.st.state = LT_REQ_RESIDENT;
    q.st.admitted = now_s(s);
    q.remaining = q.r.steps;
    s->used += q.st.bytes;
    s->stats.peak_bytes = std::max(s->stats.peak_bytes, s->used);
    s->active.push_back(s->queue.front());
    s->queue.pop_front();
  }
  s->stats.max_resident = std::max(s->stats.max_resident, (int)s->active.size());
  return LT_OK;
}

void latency_stats(lt_server* s) {
  std::vector<double> lat;
  for (const Req& q : s->reqs)
    if (q.st.state == LT_REQ_DONE) lat.push_back(q.st.finished - q.st.arrival);
  if (lat.empty()) return;
  std::sort(lat.begin(), lat.end());
  auto pct = [&](double p) {
    const double x = p * (lat.size() - 1);
    const size_t i = (size_t)std::floor(x);
    const size_t j = std::min(i + 1, lat.size() - 1);
    return lat[i] + (lat[j] - lat[i]) * (x - i);
  };
  s->stats.latency_p50 = pct(0.50);
  s->stats.latency_p99 = pct(0.99);
  s->stats.latency_max = lat.back();
}

}  // namespace

extern "C" {

int lt_server_create(const lt_server_config* cfg, lt_server** out) {
  if (!cfg || !out) return LT_E_INVALID;
  if (cfg->precision != LT_PREC_FP64 && cfg->precision != LT_PREC_MIXED) return LT_E_INVALID;
  lt_server* s = new (std::nothrow) lt_server;
  if (!s) return LT_E_OOM;
  s->cfg = *cfg;
  if (s->cfg.max_active <= 0) s->cfg.max_active = 512;
  if (s->cfg.chunk_steps <= 0) s->cfg.chunk_steps = 10;
  s->builders = std::max(4, (int)std::thread::hardware_concurrency());
  if (s->cfg.hbm_budget == 0) {
    size_t free_b = 0, total_b = 0;
    LT_CUDA_OK(cudaMemGetInfo(&free_b, &total_b));
    const size_t reserve = (size_t)8 << 30;
    s->cfg.hbm_budget = free_b > reserve ? free_b - reserve : 0;
  }
  s->t0 = std::chrono::steady_clock::now();
  *out = s;
  return LT_OK;
}

int lt_server_destroy(lt_server* s) {
  if (!s) return LT_E_INVALID;
  drop_batch(s);
  for (Req& q : s->reqs) {
    if (q.building) {
      auto built = q.inputs.get();
      if (built.second) lt_synth_free(built.second);
    }
    if (q.dom) lt_destroy(q.dom);
  }
  delete s;
  return LT_OK;
}

double lt_server_clock(lt_server* s) { return s ? now_s(s) : 0.0; }

int lt_server_submit(lt_server* s, const lt_request* r, int* id) {
  if (!s || !r || r->steps < 1) return LT_E_INVALID;
  Req q;
  q.r = *r;
  q.st = lt_request_status{};
  q.st.state = LT_REQ_PENDING;
  q.st.arrival = r->arrival;
  lt_synth_config c = r->domain;
  q.grid = lt_grid{c.nx, c.ny, c.km, s->cfg.precision, 0, c.ew_cyclic, c.tripole};
  q.st.cells = (long long)c.nx * c.ny * c.km;
  q.st.bytes = lt_domain_bytes(&q.grid);
  if (q.st.bytes == 0) {
    set_error("lt_server_submit: grid %d x %d x %d not accepted for this precision", c.nx, c.ny, c.km);
    return LT_E_INVALID;
  }
  const int nid = (int)s->reqs.size();
  s->reqs.push_back(std::move(q));
  // keep the not-yet-arrived list in arrival order (stable for equal times)
  auto pos = std::upper_bound(s->pending.begin() + s->next_pending, s->pending.end(), nid, [&](int a, int b) {
    return s->reqs[a].r.arrival < s->reqs[b].r.arrival;
  });
  s->pending.insert(pos, nid);
  if (id) *id = nid;
  return LT_OK;
}

int lt_server_run_once(lt_server* s, int* busy) {
  if (!s) return LT_E_INVALID;
  int rc;
  int k = 0;
  // 1. enqueue one chunk of steps for every resident request
  if (!s->active.empty()) {
    k = s->cfg.chunk_steps;
    for (int id : s->active) k = std::min(k, s->reqs[id].remaining);
    if (s->batch_ids != s->active) {
      drop_batch(s);
      std::vector<lt_domain*> doms;
      for (int id : s->active) doms.push_back(s->reqs[id].dom);
      if ((rc = lt_batch_create(doms.data(), (int)doms.size(), &s->batch))) return rc;
      s->batch_ids = s->active;
    }
    if ((rc = lt_batch_step(s->batch, k))) return rc;
  }
  // 2. host work while the device steps: arrivals and admission
  if ((rc = admit(s))) return rc;
  // 3. wait, account, retire
  if (k > 0) {
    if ((rc = lt_batch_sync(s->batch))) return rc;
    float ms = 0.f;
    lt_batch_last_ms(s->batch, &ms);
    s->stats.busy_s += ms * 1e-3;
    s->stats.iterations++;
    bool retired = false;
    for (int id : s->batch_ids) {
      Req& q = s->reqs[id];
      q.remaining -= k;
      q.st.steps_done += k;
      s->stats.cell_steps += (double)q.st.cells * k;
      if (q.remaining == 0) retired = true;
    }
    if (retired) {
      drop_batch(s);
      std::vector<int> keep;
      for (int id : s->active) {
        Req& q = s->reqs[id];
        if (q.remaining > 0) { keep.push_back(id); continue; }
        if ((rc = lt_tracer_content(q.dom, q.st.content))) return rc;
        if (q.r.keep_state) {
          q.final_at.resize((size_t)lt_field_count(LT_F_AT, q.grid.nx, q.grid.ny, q.grid.km));
          if ((rc = lt_get_field(q.dom, LT_F_AT, q.final_at.data(), q.final_at.size() * sizeof(double)))) return rc;
        }
        q.st.finished = now_s(s);
        q.st.state = LT_REQ_DONE;
        lt_destroy(q.dom);
        q.dom = nullptr;
        s->used -= q.st.bytes;
        s->stats.requests_done++;
      }
      s->active.swap(keep);
      latency_stats(s);
    }
  }
  s->stats.wall_s = now_s(s);
  if (busy) *busy = !(s->active.empty() && s->queue.empty() && s->next_pending >= s->pending.size());
  return LT_OK;
}

int lt_server_drain(lt_server* s) {
  if (!s) return LT_E_INVALID;
  for (;;) {
    int busy = 0;
    const int rc = lt_server_run_once(s, &busy);
    if (rc) return rc;
    if (!busy) return LT_OK;
    if (s->active.empty() && s->queue.empty() && s->next_pending < s->pending.size()) {
      const double wait = s->reqs[s->pending[s->next_pending]].r.arrival - now_s(s);
      if (wait > 0) std::this_thread::sleep_for(std::chrono::duration<double>(std::min(wait, 1.0)));
    }
  }
}

int lt_server_status(lt_server* s, int id, lt_request_status* st) {
  if (!s || !st || id < 0 || id >= (int)s->reqs.size()) return LT_E_INVALID;
  *st = s->reqs[id].st;
  return LT_OK;
}

int lt_server_state(lt_server* s, int id, double* host_at, size_t nbytes) {
  if (!s || !host_at || id < 0 || id >= (int)s->reqs.size()) return LT_E_INVALID;
  const Req& q = s->reqs[id];
  if (q.st.state != LT_REQ_DONE || q.final_at.empty()) {
    set_error("lt_server_state: request %d is not finished or was not submitted with keep_state", id);
    return LT_E_STATE;
  }
  if (nbytes != q.final_at.size() * sizeof(double)) {
    set_error("lt_server_state: %zu bytes given, %zu needed", nbytes, q.final_at.size() * sizeof(double));
    return LT_E_INVALID;
  }
  std::copy(q.final_at.begin(), q.final_at.end(), host_at);
  return LT_OK;
}

int lt_server_stats_get(lt_server* s, lt_server_stats* st) {
  if (!s || !st) return LT_E_INVALID;
  *st = s->stats;
  return LT_OK;
}

}  // extern "C"
