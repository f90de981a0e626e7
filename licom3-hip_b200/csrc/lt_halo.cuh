// lt_halo.cuh - in-GPU ghost-cell fill with the semantics of LICOM's
// POP_HaloUpdate for one block covering the global domain
// (POP_HaloMod.F90:2716-3139 message order, addresses :5602-5680, ghost
// indices POP_BlocksMod.F90:284-375):
//   * east-west cyclic: physical rows copy columns nx,nx+1 -> 0,1 and 2,3 -> nx+2,nx+3
//   * tripole north fold (cell centres, scalars): ghost rows 0,1 take the
//     mirrored physical rows 4,3; the top physical row 2 is replaced by the
//     average of each point with its mirror (global i <-> nx-i for
//     i = 1..nx/2-1; i = nx/2 and i = nx keep their value) and its ghost
//     columns follow the same mirror map
//   * closed sides (south always, east-west/north when not cyclic/tripole):
//     no message, the ghost cell keeps whatever it held.
// One thread block handles one horizontal level; the top physical row is
// staged in shared memory first so the in-place fold never reads a value
// another thread already rewrote.
#pragma once
#include <cuda_runtime.h>

namespace lt {

// POP global column of local column i (0-based local, 1-based global),
// 0 for a closed-boundary ghost.
__device__ __forceinline__ int halo_iglobal(int i, int nx, int ew_cyclic) {
  int g = i - 1;
  if (g < 1) g = ew_cyclic ? g + nx : 0;
  else if (g > nx) g = ew_cyclic ? g - nx : 0;
  return g;
}

// Source column (global, 1..nx) in the tripole buffer for local column i.
__device__ __forceinline__ int halo_fold_src(int i, int nx, int ew_cyclic) {
  int s = nx - halo_iglobal(i, nx, ew_cyclic);
  return s == 0 ? nx : s;
}

// Averaged top-row value at global column g given the staged row (local
// columns, top[g+1] is global g).
__device__ __forceinline__ double halo_fold_top(const double* top, int g, int nx) {
  const int h = nx / 2;
  if (g >= 1 && g <= h - 1) return 0.5 * (top[g + 1] + top[nx - g + 1]);
  if (g >= h + 1 && g <= nx - 1) return 0.5 * (top[nx - g + 1] + top[g + 1]);
  return top[g + 1];
}

// Number of cells of one level that are not interior (i in [2,imt-2), j in [2,jmt-2))
// plus the top physical row when the fold rewrites it.  Enumeration order:
//   [0, 2*imt)            rows 0,1
//   [2*imt, 3*imt)        row 2 (all columns) when tripole, else skipped
//   then 4 ghost/edge columns of the remaining physical rows
//   then rows jmt-2, jmt-1
struct HaloCells {
  int imt, jmt, tripole;
  __device__ __forceinline__ int first_side_row() const { return tripole ? 3 : 2; }
  __device__ __forceinline__ long count() const {
    const int side_rows = (jmt - 2) - first_side_row();
    return 2L * imt + (tripole ? imt : 0) + 4L * side_rows + 2L * imt;
  }
  __device__ __forceinline__ void cell(long m, int& j, int& i) const {
    if (m < 2L * imt) { j = (int)(m / imt); i = (int)(m % imt); return; }
    m -= 2L * imt;
    if (tripole) {
      if (m < imt) { j = 2; i = (int)m; return; }
      m -= imt;
    }
    const int side_rows = (jmt - 2) - first_side_row();
    if (m < 4L * side_rows) {
      j = first_side_row() + (int)(m / 4);
      const int c = (int)(m % 4);
      i = c < 2 ? c : imt - 4 + c;
      return;
    }
    m -= 4L * side_rows;
    j = jmt - 2 + (int)(m / imt);
    i = (int)(m % imt);
  }
};

// New value of halo cell (j,i) of a level whose top physical row is staged in
// `top` (local columns).  Returns false when the halo leaves the cell alone.
__device__ __forceinline__ bool halo_cell_value(const double* lvl, const double* top, int j, int i, int imt,
                                                int jmt, int ew_cyclic, int tripole, double& v) {
  const int nx = imt - 4;
  if (j <= 2 && tripole) {
    const int g = halo_fold_src(i, nx, ew_cyclic);
    if (j == 2) v = halo_fold_top(top, g, nx);
    else v = lvl[(long)(4 - j) * imt + g + 1];  // row 0 <- row 4, row 1 <- row 3
    return true;
  }
  if (j >= 2 && j < jmt - 2 && ew_cyclic) {
    if (i < 2) { v = lvl[(long)j * imt + nx + i]; return true; }
    if (i >= imt - 2) { v = lvl[(long)j * imt + i - nx]; return true; }
  }
  return false;
}

}  // namespace lt
