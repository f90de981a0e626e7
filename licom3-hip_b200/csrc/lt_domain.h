// lt_domain.h - the per-domain state behind the C ABI handle (private to the
// library: lt_api.cu and lt_batch.cu).
#pragma once
#include <vector>
#include "lt_common.cuh"
#include "lt_tracer_tma.cuh"

constexpr int LT_NPHASE = 6;       // surface, sss sum, net halo, continuity, tracer, state halo
// launch order of the phases in a step (continuity first: it needs no
// forcing, so it runs while lt_step_host's forcing copies are in flight)
constexpr int LT_PHASE_ORDER[LT_NPHASE] = {3, 0, 1, 2, 4, 5};
constexpr int LT_PROF_STEPS = 512;  // steps whose phase events are kept

struct lt_domain {
  lt::Arena a;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaStream_t copy_stream = nullptr;          // lt_step_host's forcing copies
  cudaEvent_t ev_free = nullptr, ev_forcing = nullptr;
  // lt_step_host_async: two sets of the six forcing fields (set 0 the
  // arena's, set 1 allocated on first use), the set the current step reads,
  // and per set an event after its last reader and one after its copies
  double* forcing_set[2][6] = {};
  int forcing_cur = 0;
  cudaEvent_t ev_set_used[2] = {}, ev_set_ready[2] = {};
  int profile = 0;
  int prof_steps = 0;
  std::vector<cudaEvent_t> prof_ev;   // [LT_PROF_STEPS][LT_NPHASE + 1]
  std::vector<void*> allocations;
  int slots = 0;
  int steps_done = 0;
  bool have_state = false;
  bool owns_stream = false;
  bool use_tma = false;       // tracer kernel fed by TMA boxes (needs 16-byte row pitch)
  int tma_grid = 0;           // persistent CTAs of the TMA tracer kernel
  lt::TracerMaps maps;
};

namespace lt {
// one tracer step of a domain on its own stream (the tracer_ body); the
// surface fluxes wait for forcing_ready when it is given
int run_step(lt_domain* d, cudaEvent_t forcing_ready = nullptr);
// after the stream has drained: LT_E_TIMEOUT once if a column kernel's
// bounded wait ran out since the last check
int timeout_status(lt_domain* d);
// allocate the turbulence closure's / momentum friction's fields of a domain
// if not yet done
int ensure_turb(lt_domain* d);
int ensure_mom(lt_domain* d);
}  // namespace lt
