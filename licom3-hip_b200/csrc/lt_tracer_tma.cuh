// lt_tracer_tma.cuh - the fused tracer column kernel with a TMA level pipeline.
//
// A CTA owns a TX x TY tile of columns and one tracer (work items are
// interleaved T,S per tile and strided over a persistent grid).  It marches
// the levels from the bottom up.  The data of one level - the tracer and its
// previous time level over the tile plus a 2-cell halo, w, the face
// transports and the mixing coefficient - arrive together as six 3-D TMA boxes
// into one of NSLOT shared-memory slots; levels are prefetched two steps ahead
// of their first use.  At step k the CTA
//   B: computes the tspas predictor and masked extrema at level k-1 on the
//      tile plus a 1-cell halo, and the first Laplacian of the biharmonic
//      operator at level k (tracer.cpp:291-547, 1238-1293);
//   C: per column, the limited flux divergence at level k, the second
//      Laplacian, shortwave, the explicit half of the vertical diffusion,
//      surface fluxes, the explicit update and one elimination step of the
//      implicit tridiagonal sweep, which runs upward with the march
//      (tracer.cpp:549-921, 1295-1699, 923-978).
// A final downward pass substitutes through the sweep and writes the new
// state of the inner cells.  Ghost cells and the fold are done by the halo
// kernel afterwards.
//
// The arithmetic comes from a policy: TmaExact (FP64, the reference's
// operation order, bit-exact with the oracle) or TmaMixed (FP32 flux
// arithmetic on FP64 differences, FP64 state, predictor and sweep).
#pragma once
#include "lt_common.cuh"
#include "lt_tma.cuh"

namespace lt {

constexpr int SW = 40;      // row width of loaded boxes: columns x0-4 .. x0+35
constexpr int NSLOT = 5;    // levels resident: k+1 .. k-2 in use, one in flight
constexpr int HQX = TX + 2, HQY = TY + 2;   // tile plus 1-cell halo
constexpr int HN = HQX * HQY;

struct TracerMaps {
  CUtensorMap at[2], atb[2], ws, uw, vs, akt;
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

template <class VT, class CT>
struct TracerSmem {
  LevelSlot<VT> slot[NSLOT];
  double a00[3][HN], amx[3][HN], amn[3][HN];
  CT d2[HN];
  CT tr[HN], dtn[HN], dts[HN], dte[HN], dtw[HN], ahf[HN];
  CT hw[(TY + 2) * SW];   // htw*hun (exact policy) or its reciprocal (mixed) at uw positions
  CT hs[(TY + 3) * SW];   // hts*hue or its reciprocal at vs positions
  int kmt[(TY + 4) * SW];
  uint64_t bar[NSLOT];
};

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

// Per-tile 2-D data: kmt with a 2-cell halo, metric terms with a 1-cell halo.
// hwv(htw, hun) / hsv(hts, hue) give the policy's form of the face divisors.
template <class SM, class HW>
__device__ __forceinline__ void load_tile_statics(SM& S, const Arena& a, int x0, int y0, HW hwv) {
  const int imt = a.imt, jmt = a.jmt;
  for (int m = threadIdx.x; m < (TY + 4) * SW; m += TTHREADS) {
    const int gj = y0 - 2 + m / SW, gi = x0 - 4 + m % SW;
    S.kmt[m] = (gj >= 0 && gj < jmt && gi >= 0 && gi < imt) ? a.kmt[(long)gj * imt + gi] : 0;
  }
  for (int m = threadIdx.x; m < HN; m += TTHREADS) {
    const int gj = y0 - 1 + m / HQX, gi = x0 - 1 + m % HQX;
    const bool in = (gj >= 0 && gj < jmt && gi >= 0 && gi < imt);
    const long q = in ? (long)gj * imt + gi : 0;
    S.tr[m] = in ? a.tarea_r[q] : 0.0;
    S.dtn[m] = in ? a.dtn[q] : 0.0;
    S.dts[m] = in ? a.dts[q] : 0.0;
    S.dte[m] = in ? a.dte[q] : 0.0;
    S.dtw[m] = in ? a.dtw[q] : 0.0;
    S.ahf[m] = in ? a.ahf[q] : 0.0;
  }
  for (int m = threadIdx.x; m < (TY + 2) * SW; m += TTHREADS) {
    const int gj = y0 - 1 + m / SW, gi = x0 - 4 + m % SW;
    const bool in = (gj >= 0 && gj < jmt && gi >= 0 && gi < imt);
    S.hw[m] = in ? hwv(a.htw[(long)gj * imt + gi], a.hun[(long)gj * imt + gi]) : hwv(1.0, 1.0);
  }
  for (int m = threadIdx.x; m < (TY + 3) * SW; m += TTHREADS) {
    const int gj = y0 - 2 + m / SW, gi = x0 - 4 + m % SW;
    const bool in = (gj >= 0 && gj < jmt && gi >= 0 && gi < imt);
    S.hs[m] = in ? hwv(a.hts[(long)gj * imt + gi], a.hue[(long)gj * imt + gi]) : hwv(1.0, 1.0);
  }
}

// One member of a batched launch, in device memory.  The tensor maps come
// first: a map read from global memory must be 64-byte aligned.
struct alignas(64) MemberDesc {
  TracerMaps maps;
  Arena a;
  long item0;    // first work item (a tile, both tracers) of this member in the batch list
  long ntiles;   // column tiles of this member
  int ntx;       // tiles along i
};

int launch_tracer_tma64(const Arena& a, const TracerMaps& maps, cudaStream_t s, int grid);
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
int launch_tracer_tma_mixed(const Arena& a, const TracerMaps& maps, cudaStream_t s, int grid);
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
