// lt_tracer_tma.cuh - what the TMA-fed column kernels share: the tensor maps
// of a domain's level boxes, the FP64 kernel's level slot and its issue, the
// box index helpers and the batch member descriptor.
//
// Both column kernels (k_tracer_tma64 in FP64, k_tracer_mixed) march a tile
// of columns from the bottom level up.  The data of one level arrive as 3-D
// TMA boxes (no multicast) into one of three shared-memory level slots
// guarded by mbarriers, issued one step ahead of their first use.  At step k
// a CTA computes the tspas predictor and masked extrema at level k-1 on the
// tile plus a 1-cell halo and the first Laplacian of the biharmonic operator
// at level k (tracer.cpp:291-547, 1238-1293), then per column the limited
// flux divergence at level k, the second Laplacian, shortwave, the explicit
// half of the vertical diffusion, surface fluxes, the explicit update and
// one elimination step of the implicit tridiagonal sweep, which runs upward
// with the march (tracer.cpp:549-921, 1295-1699, 923-978).  A final downward
// pass substitutes through the sweep and writes the new state of the inner
// cells; ghost cells and the fold are done by the halo kernel afterwards.
#pragma once
#include "lt_common.cuh"
#include "lt_tma.cuh"

namespace lt {

constexpr int SW = 40;      // row width of loaded boxes: columns x0-4 .. x0+35
constexpr int HQX = TX + 2, HQY = TY + 2;   // tile plus 1-cell halo
constexpr int HN = HQX * HQY;

struct TracerMaps {
  CUtensorMap at[2], atb[2], ws, uw, vs, akt;
  CUtensorMap vel[4];   // mixed: utf, vtf, utl, vtl (f32) in the continuity march's boxes
};

template <class VT>
struct alignas(128) LevelSlot {
  alignas(128) double at[(TY + 4) * SW];   // rows y0-2 .. y0+TY+1
  alignas(128) double atb[(TY + 4) * SW];  // tracer level L of the previous time level
  alignas(128) VT ws[(TY + 2) * SW];       // rows y0-1 .. y0+TY
  alignas(128) VT uw[(TY + 2) * SW];       // rows y0-1 .. y0+TY
  alignas(128) VT vs[(TY + 3) * SW];       // rows y0-2 .. y0+TY
  alignas(128) VT akt[TY * TX];            // the tile itself, columns x0 .. x0+TX-1
};

template <class VT>
constexpr uint32_t level_bytes() {
  return (uint32_t)(2 * (TY + 4) * SW * sizeof(double) +
                    ((TY + 2) * SW * 2 + (TY + 3) * SW + TY * TX) * sizeof(VT));
}

// index helpers (shared-memory layouts)
__device__ __forceinline__ int r2(int hj, int hi) { return (hj + 1) * SW + hi + 3; }  // H1 point -> at/atb/kmt box
__device__ __forceinline__ int ru(int hj, int hi) { return hj * SW + hi + 3; }        // H1 point -> ws/uw box
__device__ __forceinline__ int rv(int hj, int hi) { return (hj + 1) * SW + hi + 3; }  // H1 point -> vs box (row j)

// Issue the six boxes of level L of tracer n into a slot (one thread).
template <class VT>
__device__ __forceinline__ void issue_level(LevelSlot<VT>& sl, uint64_t* bar, const TracerMaps& m, int cur, int n,
                                            int km, int L, int x0, int y0) {
  mbar_expect_tx(bar, level_bytes<VT>());
  tma_load_3d(sl.at, &m.at[cur], x0 - 4, y0 - 2, n * km + L, bar);
  tma_load_3d(sl.atb, &m.atb[cur], x0 - 4, y0 - 2, n * (km + 1) + L + 1, bar);
  tma_load_3d(sl.ws, &m.ws, x0 - 4, y0 - 1, L, bar);
  tma_load_3d(sl.uw, &m.uw, x0 - 4, y0 - 1, L, bar);
  tma_load_3d(sl.vs, &m.vs, x0 - 4, y0 - 2, L, bar);
  tma_load_3d(sl.akt, &m.akt, x0, y0, n * km + L, bar);
}

// One member of a batched launch, in device memory.  The tensor maps come
// first: a map read from global memory must be 64-byte aligned.
struct alignas(64) MemberDesc {
  TracerMaps maps;
  Arena a;
  long item0;    // first work item (a tile, both tracers) of this member in the batch list
  long ntiles;   // column tiles of this member
  int ntx;       // tiles along i
  int tma;       // 1: level boxes by TMA; 0: by per-thread copies (row pitch TMA cannot take)
};

// The FP64 column kernel of the tspas scheme; tma: its level boxes by TMA (else
// per-thread copies, for row pitches TMA cannot take)
int launch_tracer_tma64(const Arena& a, const TracerMaps& maps, cudaStream_t s, int grid, bool tma);
// Batched forms (mixed precision): nmem members, total work items, one
// persistent column launch of `grid` CTAs with per-CTA scratch of km_max
// levels; continuity over every member's tiles with tiles of 32 x cby columns.
int launch_tracer_mixed_batch(const MemberDesc* mem, int nmem, long total, double* scratch, int km_max, int grid,
                              cudaStream_t s);
int launch_continuity_mixed_batch(const MemberDesc* mem, int nmem, int max_imt, int max_jmt, int cby,
                                  cudaStream_t s);
// The small kernels of a batch step for every member in one launch each:
// surface fluxes, the SSS-norm tree (one launch per tree pass; max_cols is
// the largest member's nx * ny) and its finish, the net halo; and the state
// halo (two launches, temperature first).
int launch_small_batch_pre(const MemberDesc* mem, int nmem, int max_imt, int max_jmt, long max_cols,
                           cudaStream_t s);
int launch_halo_state_batch(const MemberDesc* mem, int nmem, int max_imt, int km_max, cudaStream_t s);
// sets the batched column kernel's shared-memory size on the current device
int prepare_tracer_mixed_batch();
// The mixed column kernel; tma: its level boxes by TMA (else per-thread copies)
int launch_tracer_tma_mixed(const Arena& a, const TracerMaps& maps, bool tma, cudaStream_t s, int grid);
// The mixed continuity: TMA-fed when the domain has its maps (tma), else
// plain loads.
int launch_continuity_mixed(const Arena& a, const TracerMaps& maps, bool tma, cudaStream_t s);
// Build the tensor maps of a domain; false if the layout does not allow TMA
// (row pitch not a multiple of 16 bytes for some field).
bool build_tracer_maps(const Arena& a, TracerMaps* maps);

// Records a timed-out wait and drains this CTA's outstanding loads (bounded).
template <class SM>
__device__ __forceinline__ void tma_bail(SM& S, const Arena& a, uint32_t par, uint32_t outstanding) {
  constexpr int ns = sizeof(S.bar) / sizeof(S.bar[0]);
  if (threadIdx.x == 0) {
    atomicExch(a.status + 1, 1);
    for (int s = 0; s < ns; ++s)
      if (outstanding & (1u << s)) mbar_wait(&S.bar[s], (par >> s) & 1u);
  }
  __syncthreads();
}

}  // namespace lt
