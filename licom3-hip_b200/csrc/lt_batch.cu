// lt_batch.cu - several tracer domains stepped together on one device: the
// batched launches, CUDA-graph replay and the launch-shape autotuner.
//
// A batch step is the tracer_ sequence of every member (surface fluxes, SSS
// norm, net halo, continuity, column march, state halo), each small kernel
// one launch over every member, and the two heavy kernels batched in mixed
// precision: one continuity launch over every member's tiles and one
// persistent column launch over the concatenated (member, tile) work
// list.  A kernel's parameters are frozen when a
// graph is captured, and each step reads the ping-pong state buffer `cur` and
// writes the other, so two graphs are kept: parity 0 (every member at the
// `cur` it had when the descriptors were built) and parity 1 (flipped).
#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <vector>
#include "lt_domain.h"
#include "../../include/licom_batch.h"

using namespace lt;

struct lt_batch {
  std::vector<lt_domain*> m;
  std::vector<int> base_cur;        // member cur when the descriptors were built
  std::vector<const double*> base_forcing;   // member forcing set (lt_step_host_async swaps it)
  int dev = 0, sms = 148;
  bool mixed = false;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, evx = nullptr;
  lt_batch_config cfg{kMixedCtasPerSm, 8, 1};
  MemberDesc* d_desc[2] = {nullptr, nullptr};   // per parity
  double* scratch = nullptr;                     // column scratch, kMixedCtasPerSm CTAs per SM
  int km_max = 0, max_imt = 0, max_jmt = 0;
  long max_cols = 0;                             // largest member's nx * ny
  long total_items = 0;
  int parity = 0;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  int graph_kernels = 0;                         // kernels in one step's graph
  bool graphs_valid = false;
};

namespace {

std::mutex g_tune_mutex;
std::map<std::string, lt_batch_config> g_tuned;   // member shapes -> chosen launch shape

std::string shape_key(const lt_batch* b) {
  std::string k = b->mixed ? "m" : "d";
  for (const lt_domain* d : b->m)
    k += ":" + std::to_string(d->a.nx) + "x" + std::to_string(d->a.ny) + "x" + std::to_string(d->a.km);
  return k;
}

// Both run between steps: the batch stream is drained first, so no launch in
// flight reads a graph or descriptor being replaced.
void drop_graphs(lt_batch* b) {
  if (b->stream) cudaStreamSynchronize(b->stream);
  for (auto& g : b->graph)
    if (g) { cudaGraphExecDestroy(g); g = nullptr; }
  b->graphs_valid = false;
}

// Member descriptors for both parities from the members' current state.
int build_descriptors(lt_batch* b) {
  const int n = (int)b->m.size();
  std::vector<MemberDesc> h[2];
  h[0].resize(n);
  h[1].resize(n);
  long item = 0;
  b->km_max = b->max_imt = b->max_jmt = 0;
  b->max_cols = 0;
  b->base_cur.resize(n);
  b->base_forcing.resize(n);
  for (int i = 0; i < n; ++i) {
    lt_domain* d = b->m[i];
    const Arena& a = d->a;
    const int ntx = (a.imt + TX - 1) / TX;
    const long ntiles = (long)ntx * ((a.jmt + kMixedTileY - 1) / kMixedTileY);
    b->base_cur[i] = a.cur;
    b->base_forcing[i] = a.swv;
    for (int p = 0; p < 2; ++p) {
      MemberDesc& e = h[p][i];
      std::memset(&e, 0, sizeof(e));
      e.maps = d->maps;
      e.a = a;
      e.a.cur = a.cur ^ p;
      e.item0 = item;
      e.ntiles = ntiles;
      e.ntx = ntx;
      e.tma = d->use_tma ? 1 : 0;
    }
    item += ntiles;   // one work item per tile (both tracers)
    b->km_max = std::max(b->km_max, a.km);
    b->max_imt = std::max(b->max_imt, a.imt);
    b->max_jmt = std::max(b->max_jmt, a.jmt);
    b->max_cols = std::max(b->max_cols, (long)a.nx * a.ny);
  }
  b->total_items = item;
  if (b->stream) LT_CUDA_OK(cudaStreamSynchronize(b->stream));
  for (int p = 0; p < 2; ++p) {
    if (!b->d_desc[p]) LT_CUDA_OK(cudaMalloc(&b->d_desc[p], sizeof(MemberDesc) * n));
    LT_CUDA_OK(cudaMemcpy(b->d_desc[p], h[p].data(), sizeof(MemberDesc) * n, cudaMemcpyHostToDevice));
  }
  b->parity = 0;
  drop_graphs(b);
  return LT_OK;
}

// Members stepped outside the batch since the descriptors were built (their
// cur moved without the batch's parity, or their forcing set was swapped)
// need new descriptors.
bool descriptors_stale(const lt_batch* b) {
  for (size_t i = 0; i < b->m.size(); ++i)
    if (b->m[i]->a.cur != (b->base_cur[i] ^ b->parity) || b->m[i]->a.swv != b->base_forcing[i]) return true;
  return false;
}

// One step of every member at parity p, enqueued on the batch stream.
int enqueue_step(lt_batch* b, int p) {
  cudaStream_t s = b->stream;
  const int nmem = (int)b->m.size();
  int rc;
  if ((rc = launch_small_batch_pre(b->d_desc[p], nmem, b->max_imt, b->max_jmt, b->max_cols, s))) return rc;
  if (b->mixed) {
    if ((rc = launch_continuity_mixed_batch(b->d_desc[p], (int)b->m.size(), b->max_imt, b->max_jmt,
                                            b->cfg.continuity_tile_y, s)))
      return rc;
    if ((rc = launch_tracer_mixed_batch(b->d_desc[p], (int)b->m.size(), b->total_items, b->scratch, b->km_max,
                                        b->sms * b->cfg.column_ctas_per_sm, s)))
      return rc;
  } else {
    for (size_t i = 0; i < b->m.size(); ++i) {
      lt_domain* d = b->m[i];
      Arena a = d->a;
      a.cur = b->base_cur[i] ^ p;
      if ((rc = launch_continuity_fp64(a, s))) return rc;
      rc = a.p.adv_tracer == LT_ADV_TSPAS ? launch_tracer_tma64(a, d->maps, s, d->tma_grid, d->use_tma)
                                          : launch_tracer_fp64(a, s, d->slots);
      if (rc) return rc;
    }
  }
  return launch_halo_state_batch(b->d_desc[p], nmem, b->max_imt, b->km_max, s);
}

int capture_graphs(lt_batch* b) {
  drop_graphs(b);
  for (int p = 0; p < 2; ++p) {
    cudaGraph_t g = nullptr;
    LT_CUDA_OK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    const long long n0 = launch_counter();
    const int rc = enqueue_step(b, p);
    // captured kernels are counted when a replay launches them, not here
    b->graph_kernels = (int)(launch_counter() - n0);
    count_launches(-b->graph_kernels);
    const cudaError_t e = cudaStreamEndCapture(b->stream, &g);
    if (rc) { if (g) cudaGraphDestroy(g); return rc; }
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
    const cudaError_t ei = cudaGraphInstantiate(&b->graph[p], g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) return cuda_fail(ei, "cudaGraphInstantiate");
  }
  b->graphs_valid = true;
  return LT_OK;
}

bool config_ok(const lt_batch* b, const lt_batch_config& c) {
  if (c.use_graph != 0 && c.use_graph != 1) return false;
  if (!b->mixed) return true;
  return c.column_ctas_per_sm >= 1 && c.column_ctas_per_sm <= kMixedCtasPerSm &&
         (c.continuity_tile_y == 4 || c.continuity_tile_y == 8 || c.continuity_tile_y == 16);
}

// Order the batch after every member's own stream (uploads, earlier steps)
// and, after the batch, every member's stream after the batch.
int join_members(lt_batch* b, bool before) {
  for (lt_domain* d : b->m) {
    if (before) {
      LT_CUDA_OK(cudaEventRecord(b->evx, d->stream));
      LT_CUDA_OK(cudaStreamWaitEvent(b->stream, b->evx, 0));
    } else {
      LT_CUDA_OK(cudaEventRecord(b->evx, b->stream));
      LT_CUDA_OK(cudaStreamWaitEvent(d->stream, b->evx, 0));
    }
  }
  return LT_OK;
}

int step_n(lt_batch* b, int nsteps, bool timed) {
  int rc;
  if (descriptors_stale(b) && (rc = build_descriptors(b))) return rc;
  if (b->cfg.use_graph && !b->graphs_valid && (rc = capture_graphs(b))) return rc;
  if ((rc = join_members(b, true))) return rc;
  if (timed) LT_CUDA_OK(cudaEventRecord(b->ev0, b->stream));
  for (int k = 0; k < nsteps; ++k) {
    if (b->cfg.use_graph) {
      LT_CUDA_OK(cudaGraphLaunch(b->graph[b->parity], b->stream));
      count_launches(b->graph_kernels);
    } else if ((rc = enqueue_step(b, b->parity))) {
      return rc;
    }
    b->parity ^= 1;
    for (lt_domain* d : b->m) {
      d->a.cur ^= 1;
      d->steps_done++;
    }
  }
  if (timed) LT_CUDA_OK(cudaEventRecord(b->ev1, b->stream));
  return join_members(b, false);
}

}  // namespace

extern "C" {

int lt_batch_create(lt_domain* const* members, int n, lt_batch** out) {
  if (!members || n <= 0 || !out) return LT_E_INVALID;
  *out = nullptr;
  lt_batch* b = new (std::nothrow) lt_batch;
  if (!b) return LT_E_OOM;
  LT_CUDA_OK(cudaGetDevice(&b->dev));
  cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, b->dev);
  b->mixed = members[0] && members[0]->a.precision == LT_PREC_MIXED;
  for (int i = 0; i < n; ++i) {
    lt_domain* d = members[i];
    if (!d || (d->a.precision == LT_PREC_MIXED) != b->mixed) {
      set_error("lt_batch_create: member %d is missing or of another precision", i);
      delete b;
      return LT_E_INVALID;
    }
    b->m.push_back(d);
  }
  int rc = LT_OK;
  auto fail = [&](int code) { lt_batch_destroy(b); return code; };
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&b->ev0) != cudaSuccess || cudaEventCreate(&b->ev1) != cudaSuccess ||
      cudaEventCreateWithFlags(&b->evx, cudaEventDisableTiming) != cudaSuccess)
    return fail(LT_E_CUDA);
  if ((rc = build_descriptors(b))) return fail(rc);
  if (b->mixed) {
    const size_t bytes =
        sizeof(double) * (size_t)b->sms * kMixedCtasPerSm * b->km_max * kMixedScratchPerLevel * kMixedThreads;
    if (cudaMalloc(&b->scratch, bytes) != cudaSuccess) {
      set_error("lt_batch_create: cudaMalloc(%zu) for the column scratch failed", bytes);
      return fail(LT_E_OOM);
    }
    if ((rc = prepare_tracer_mixed_batch())) return fail(rc);
  }
  {
    std::lock_guard<std::mutex> g(g_tune_mutex);
    auto it = g_tuned.find(shape_key(b));
    if (it != g_tuned.end()) b->cfg = it->second;
  }
  *out = b;
  return LT_OK;
}

int lt_batch_destroy(lt_batch* b) {
  if (!b) return LT_E_INVALID;
  if (b->stream) cudaStreamSynchronize(b->stream);
  drop_graphs(b);
  for (auto& p : b->d_desc)
    if (p) cudaFree(p);
  if (b->scratch) cudaFree(b->scratch);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  if (b->evx) cudaEventDestroy(b->evx);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return LT_OK;
}

int lt_batch_size(lt_batch* b, int* n) {
  if (!b || !n) return LT_E_INVALID;
  *n = (int)b->m.size();
  return LT_OK;
}

int lt_batch_get_config(lt_batch* b, lt_batch_config* cfg) {
  if (!b || !cfg) return LT_E_INVALID;
  *cfg = b->cfg;
  return LT_OK;
}

int lt_batch_set_config(lt_batch* b, const lt_batch_config* cfg) {
  if (!b || !cfg || !config_ok(b, *cfg)) {
    set_error("lt_batch_set_config: launch shape out of range");
    return LT_E_INVALID;
  }
  b->cfg = *cfg;
  return build_descriptors(b);   // also takes the members' current parameters
}

int lt_batch_step(lt_batch* b, int nsteps) {
  if (!b || nsteps < 0) return LT_E_INVALID;
  return step_n(b, nsteps, true);
}

int lt_batch_sync(lt_batch* b) {
  if (!b) return LT_E_INVALID;
  LT_CUDA_OK(cudaStreamSynchronize(b->stream));
  int rc = LT_OK;
  for (lt_domain* d : b->m) {
    LT_CUDA_OK(cudaStreamSynchronize(d->stream));
    const int r = timeout_status(d);
    if (r && !rc) rc = r;
  }
  return rc;
}

int lt_batch_last_ms(lt_batch* b, float* ms) {
  if (!b || !ms) return LT_E_INVALID;
  LT_CUDA_OK(cudaEventSynchronize(b->ev1));
  LT_CUDA_OK(cudaEventElapsedTime(ms, b->ev0, b->ev1));
  return LT_OK;
}

int lt_batch_autotune(lt_batch* b, int trial_steps, lt_batch_config* chosen) {
  if (!b || trial_steps < 1) return LT_E_INVALID;
  int rc = lt_batch_sync(b);
  if (rc) return rc;
  // keep every member's current state (both tracers, with halos) to restore
  const size_t nm = b->m.size();
  std::vector<double*> keep(nm, nullptr);
  std::vector<int> cur0(nm), done0(nm);
  auto release = [&]() { for (double* p : keep) if (p) cudaFree(p); };
  for (size_t i = 0; i < nm; ++i) {
    const Arena& a = b->m[i]->a;
    cur0[i] = a.cur;
    done0[i] = b->m[i]->steps_done;
    if (cudaMalloc(&keep[i], sizeof(double) * 2 * (a.F + a.FB)) != cudaSuccess) {
      release();
      set_error("lt_batch_autotune: no room to keep the member states");
      return LT_E_OOM;
    }
    LT_CUDA_OK(cudaMemcpy(keep[i], a.at[a.cur], sizeof(double) * 2 * a.F, cudaMemcpyDeviceToDevice));
    LT_CUDA_OK(cudaMemcpy(keep[i] + 2 * a.F, a.atb[a.cur], sizeof(double) * 2 * a.FB, cudaMemcpyDeviceToDevice));
  }
  std::vector<lt_batch_config> cands;
  if (b->mixed) {
    for (int ctas = 1; ctas <= kMixedCtasPerSm; ++ctas)
      for (int ty : {4, 8, 16}) cands.push_back({ctas, ty, 1});
  } else {
    cands.push_back({b->cfg.column_ctas_per_sm, b->cfg.continuity_tile_y, 1});
  }
  cands.push_back({cands.back().column_ctas_per_sm, cands.back().continuity_tile_y, 0});
  float best = 1e30f;
  lt_batch_config best_cfg = b->cfg;
  for (const lt_batch_config& c : cands) {
    b->cfg = c;
    drop_graphs(b);
    if ((rc = step_n(b, 1, false)) || (rc = step_n(b, trial_steps, true)) || (rc = lt_batch_sync(b))) break;
    float ms = 0.f;
    if ((rc = lt_batch_last_ms(b, &ms))) break;
    if (ms < best) { best = ms; best_cfg = c; }
  }
  // restore the states into the buffers they came from
  cudaDeviceSynchronize();
  for (size_t i = 0; i < nm; ++i) {
    Arena& a = b->m[i]->a;
    a.cur = cur0[i];
    b->m[i]->steps_done = done0[i];
    cudaMemcpy(a.at[a.cur], keep[i], sizeof(double) * 2 * a.F, cudaMemcpyDeviceToDevice);
    cudaMemcpy(a.atb[a.cur], keep[i] + 2 * a.F, sizeof(double) * 2 * a.FB, cudaMemcpyDeviceToDevice);
  }
  release();
  if (rc) return rc;
  b->cfg = best_cfg;
  if ((rc = build_descriptors(b))) return rc;
  {
    std::lock_guard<std::mutex> g(g_tune_mutex);
    g_tuned[shape_key(b)] = best_cfg;
  }
  if (chosen) *chosen = best_cfg;
  return LT_OK;
}

}  // extern "C"
