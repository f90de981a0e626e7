// lt_step_mixed.cu - the mixed-precision tracer step.
//
// Storage: the prognostic state (at, atb) stays f64; the dynamics inputs, the
// mixing coefficient and the derived fields (w, face transports, scaled
// utf/vtf) are f32.  Arithmetic: the flux, stencil and diffusion terms are
// computed in f32 from f64 differences of the state (predictor, limiter
// fluxes, Lax-Wendroff and upwind parts, both Laplacians, explicit vertical
// diffusion, shortwave); the tspas bound test compares the f32 predictor
// increment with the f32 differences between the cell and its six
// neighbours, so the limiter decisions are those of an f64 run except at
// near-ties.  f64 remains where
// the global tracer content needs it: the centred advective product d*u of
// the final update (both cells of a face add it with the same sign, so its
// rounding would not cancel), the face-flux sums and their metric weights,
// the surface fluxes, the explicit update and the tridiagonal sweep.
//
// The tspas terms of tracer.cpp:291-921 are regrouped per face.  For a face
// between cells L (lower index) and R with difference d = a_R - a_L (for the
// horizontal faces) and transport u, the centred part A = d*u and the
// Lax-Wendroff part B = 2*dts*u*u*d/(face metric) (horizontal) or
// B = w*w*odzt*dts*d (vertical, d = a_upper - a_lower) enter
//    L: -(A - X), R: -(A + X)   horizontally,  upper: -(A + X), lower: -(A - X) vertically,
// times tarea_r (0.5*odzp vertically), with X = B, or X = |u|*d where the
// predictor leaves the local bounds at either cell (the upwind fallback).
// This is the reference's advective form algebraically (the centred and
// divergence terms x0 + c1 combine to d*u per face); each face is evaluated
// once for both cells.
#include <cstdio>
#include "lt_common.cuh"
#include "lt_halo.cuh"
#include "lt_tracer_tma.cuh"

namespace lt {
namespace {

__global__ void k_f64_to_f32(const double* __restrict__ x, float* __restrict__ y, long n) {
  for (long m = (long)blockIdx.x * blockDim.x + threadIdx.x; m < n; m += (long)gridDim.x * blockDim.x)
    y[m] = (float)x[m];
}

__global__ void k_f32_to_f64(const float* __restrict__ x, double* __restrict__ y, long n) {
  for (long m = (long)blockIdx.x * blockDim.x + threadIdx.x; m < n; m += (long)gridDim.x * blockDim.x)
    y[m] = (double)x[m];
}

// Face transports from the U-point means (u_wface, v_sface of
// advection_tracer_1_0, tracer.cpp:83-119):
//   uw(j,i) = (wkd(j-1,i) + wkd(j,i)) * htw(j,i) / 4
//   vs(j,i) = (wkb(j,i) + wkb(j,i+1)) * hts(j,i) / 4
// The f64 forms are the one expression the continuity march and the tracer
// march's centred term both use, so the divergence that builds w and the
// transports that advect the tracer agree to f64 rounding.  The f32 forms
// feed the predictor, the Lax-Wendroff and the upwind parts.
__device__ __forceinline__ double face_x64(float wn, float wc, double htw) {
  return ((double)wn + (double)wc) * htw * 0.25;
}
__device__ __forceinline__ double face_y64(float wc, float we, double hts) {
  return ((double)wc + (double)we) * hts * 0.25;
}
__device__ __forceinline__ float face32(float w1, float w2, float h) { return (w1 + w2) * h * 0.25f; }
// Lax-Wendroff part of a face flux, d*u*u*(2 dts / (h_t h_u)): one expression
// wherever a face is used, so both cells of the face get the same value
__device__ __forceinline__ float lw_part(float d, float u, float c) { return d * u * u * c; }


// ------------------------------------------------------------- continuity
// As the f64 k_cont_march64 (tracer_1, upwell_2..4,
// operators_div, advection_tracer_1_0) with f32 storage.  The tracer march
// uses the advective form, whose content change is sum(T * 3-D divergence of
// the transports it advects with); to keep that divergence zero in exact
// arithmetic where the flow is non-divergent, both marches form the face
// transports in f64 from the same stored f32 U-point means (face_x64,
// face_y64), the free-surface factor enters the divergence as an additive
// correction that vanishes with the surface height, and w is integrated in
// f64 and rounded once.  Rounding w to f32 then costs f32 precision of w
// only, not of the transports.
//
// One CTA marches a 32 x CBY column tile down the levels: the 2-D metric and
// free-surface factors are read once per tile, each level's U-point means
// (with a one-point halo north and east) pass through shared memory, and the
// vertical recurrence of upwell_4,
//   raw(k) = raw(k-1) + dzp(k-1) * (W * ohbt + wka(k-1)),  ws(k) = fac * raw(k),
// with W = -sum dzp*wka over the wet levels, is evaluated after the march
// from the partial sums P(k) = sum_{k'<k} dzp*wka as
//   raw(k) = ws(0) + W * ohbt * Z(k) + P(k),  Z(k) = sum_{k'<k} dzp,
// with P(k) parked in the ws field between the two passes.
constexpr int CBX = 32;
template <int CBY>
__device__ __forceinline__ void cont_tile(const Arena& a, int bx, int by) {
  constexpr int UX = CBX + 1, UY = CBY + 1, UN = UX * UY, NT = CBX * CBY;
  // wkd/wkb: mean velocities at U points, double-buffered over levels;
  // fm1: free-surface factor minus one (-1 where the reference's uk/vk are zero)
  __shared__ float s_wkd[2][UN], s_wkb[2][UN], s_fm1[UN];
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * CBX + tx;
  const int x0 = bx * CBX, y0 = by * CBY;
  const int imt = a.imt, jmt = a.jmt, km = a.km;
  const long A = a.A;
  const float oncc = (float)a.p.oncc;
  for (int m = tid; m < UN; m += NT) {
    const int uj = y0 - 1 + m / UX, ui = x0 + m % UX;
    float fm1 = -1.f;
    if (uj >= 0 && uj < jmt - 1 && ui >= 1 && ui < imt) {
      const long q = (long)uj * imt + ui;
      const double work = a.au0[q] * a.stf_ssh[q] + a.aus[q] * a.stf_ssh[q + imt] +
                          a.auw[q] * a.stf_ssh[q - 1] + a.ausw[q] * a.stf_ssh[q + imt - 1];
      fm1 = (float)(work * a.ohbu[q]);
    }
    s_fm1[m] = fm1;
  }
  const int i = x0 + tx, j = y0 + ty;
  const bool own = i < imt && j < jmt;
  const bool div_here = own && j >= 1 && i < imt - 1;
  const bool col_here = own && j >= 1 && j < jmt - 1 && i >= 1 && i < imt - 1;
  const long qo = own ? (long)j * imt + i : 0;
  const int kz = own ? a.kmt[qo] : 0;
  const double htw_cd = own ? a.htw[qo] : 0.0, hts_cd = own ? a.hts[qo] : 0.0;
  const double htw_ed = div_here ? a.htw[qo + 1] : 0.0, hts_nd = div_here ? a.hts[qo - imt] : 0.0;
  const double tr = div_here ? a.tarea_r[qo] : 0.0;
  const int m0 = (ty + 1) * UX + tx, mn = ty * UX + tx;
  double P = 0.0;
  // U-point means of the region at one level: each thread loads the raw f32
  // velocities of up to two region points into registers one level ahead, so
  // the loads of level k+1 are in flight while level k is computed
  constexpr int NPT = (UN + NT - 1) / NT;
  static_assert(NPT <= 2, "region points per thread");
  float ruf[NPT], rul[NPT], rvf[NPT], rvl[NPT];
  long rc[NPT];
  bool rin[NPT];
#pragma unroll
  for (int p = 0; p < NPT; ++p) {
    const int m = tid + p * NT;
    const int uj = y0 - 1 + m / UX, ui = x0 + m % UX;
    rin[p] = m < UN && uj >= 0 && uj < jmt && ui < imt;
    rc[p] = rin[p] ? (long)uj * imt + ui : 0;
  }
  auto fetch = [&](int k) {
    const long lvl = (long)k * A;
#pragma unroll
    for (int p = 0; p < NPT; ++p) {
      ruf[p] = rul[p] = rvf[p] = rvl[p] = 0.f;
      if (rin[p]) {
        const long c = lvl + rc[p];
        ruf[p] = a.utf32[c]; rul[p] = a.utl32[c];
        rvf[p] = a.vtf32[c]; rvl[p] = a.vtl32[c];
      }
    }
  };
  auto park = [&](int b) {
#pragma unroll
    for (int p = 0; p < NPT; ++p) {
      const int m = tid + p * NT;
      if (m < UN) {
        s_wkd[b][m] = rin[p] ? 0.5f * (ruf[p] * oncc) + 0.5f * rul[p] : 0.f;
        s_wkb[b][m] = rin[p] ? 0.5f * (rvf[p] * oncc) + 0.5f * rvl[p] : 0.f;
      }
    }
  };
  fetch(0);
  park(0);
  for (int k = 0; k < km; ++k) {
    const int b = k & 1;
    const long lvl = (long)k * A;
    __syncthreads();
    if (k + 1 < km) fetch(k + 1);
    if (own) {
      const long c = lvl + qo;
      const float* wd = s_wkd[b];
      const float* wb = s_wkb[b];
      a.utf_out32[c] = a.utf32[c] * oncc;
      a.vtf_out32[c] = a.vtf32[c] * oncc;
      a.wkd32[c] = wd[m0];
      a.wkb32[c] = wb[m0];
      if (col_here && k < kz) {
        // the four faces, as the tracer kernel forms them (face_x64/face_y64)
        const double uw_w = face_x64(wd[mn], wd[m0], htw_cd);
        const double uw_e = face_x64(wd[mn + 1], wd[m0 + 1], htw_ed);
        const double vs_s = face_y64(wb[m0], wb[m0 + 1], hts_cd);
        const double vs_n = face_y64(wb[mn], wb[mn + 1], hts_nd);
        // (uk_1 + uk_2) * htw = 4 * uw + htw * (fm1_1 * wkd_1 + fm1_2 * wkd_2)
        auto corr = [&](const float* s, int m1, int m2) {
          return (double)s_fm1[m1] * (double)s[m1] + (double)s_fm1[m2] * (double)s[m2];
        };
        const double east = 4.0 * uw_e + htw_ed * corr(wd, m0 + 1, mn + 1);
        const double west = 4.0 * uw_w + htw_cd * corr(wd, m0, mn);
        const double south = 4.0 * vs_s + hts_cd * corr(wb, m0 + 1, m0);
        const double north = 4.0 * vs_n + hts_nd * corr(wb, mn + 1, mn);
        const double wka = 0.5 * (east - west + south - north) * tr;
        if (k >= 1) a.ws32[c] = (float)P;
        P += a.dzp[k] * wka;
      }
    }
    // buffer b^1 was last read in step k-1, before this step's barrier
    if (k + 1 < km) park(b ^ 1);
  }
  if (!col_here) return;
  const double ohbt = a.ohbt[qo];
  const double fac = 1.0 / (1.0 + a.stf_ssh[qo] * ohbt);
  const double W = -P;
  const double ws0 = a.ws32[qo];
  double Z = 0.0;
  for (int k = 1; k < km; ++k) {
    Z += a.dzp[k - 1];
    const long c = (long)k * A + qo;
    a.ws32[c] = (k < kz) ? (float)(fac * (ws0 + W * ohbt * Z + (double)a.ws32[c])) : 0.f;
  }
}

constexpr int kContTileY = 4;   // tile height of the single-domain continuity march

__global__ void __launch_bounds__(CBX * kContTileY) k_cont_march32(Arena a) {
  cont_tile<kContTileY>(a, blockIdx.x, blockIdx.y);
}

// every member's tiles in one launch: blockIdx.z is the member; tiles beyond
// a smaller member's grid leave at once
// (the member's arena is read from a shared-memory copy, which the march's
// global stores cannot alias, so its fields stay in registers across levels)
template <int CBY>
__global__ void __launch_bounds__(CBX * CBY) k_cont_batch(const MemberDesc* __restrict__ mem) {
  __shared__ __align__(16) unsigned char s_arena[sizeof(Arena)];
  const Arena& g = mem[blockIdx.z].a;
  if ((int)blockIdx.x * CBX >= g.imt || (int)blockIdx.y * CBY >= g.jmt) return;
  const int tid = threadIdx.y * CBX + threadIdx.x;
  for (int t = tid; t < (int)(sizeof(Arena) / 16); t += CBX * CBY)
    reinterpret_cast<uint4*>(s_arena)[t] = reinterpret_cast<const uint4*>(&g)[t];
  __syncthreads();
  cont_tile<CBY>(*reinterpret_cast<const Arena*>(s_arena), blockIdx.x, blockIdx.y);
}

}  // namespace

int launch_f64_to_f32(const double* x, float* y, long n, cudaStream_t s) {
  k_f64_to_f32<<<1184, 256, 0, s>>>(x, y, n);
  LT_LAUNCHED();
  return LT_OK;
}

int launch_f32_to_f64(const float* x, double* y, long n, cudaStream_t s) {
  k_f32_to_f64<<<1184, 256, 0, s>>>(x, y, n);
  LT_LAUNCHED();
  return LT_OK;
}

namespace {

// ------------------------------------------------------------ column march
// Tile of the mixed march: TX x MY columns, one thread per column.  Taller
// than the FP64 kernel's 32 x 4 tile: the 1-cell halo the predictor, the first
// Laplacian and the faces are computed on grows less than the tile.
constexpr int MY = kMixedTileY;
constexpr int MTH = kMixedThreads;
constexpr int MHQY = MY + 2;          // tile plus 1-cell halo, rows
constexpr int MHN = HQX * MHQY;
// Level slots.  Step k (the march runs downward) reads levels k-2, k-1 and
// k only, so at the end of step k the slot of level k takes level k-3: three
// slots keep one step of lead time for every box.
constexpr int NSM = 3;
constexpr int FXN = (MY + 2) * (TX + 3);   // x faces of the 1-halo region
constexpr int FYN = (MY + 3) * (TX + 2);   // y faces of the 1-halo region

// One level of the column tile, filled by five TMA boxes (the mixing
// coefficient of the own column comes by plain loads, a step ahead).  The f32 fields
// are w and the U-point means wkd, wkb from which the kernel forms the face
// transports (face32, face_x64, face_y64).
struct alignas(128) MxSlot {
  alignas(128) double at[(MY + 4) * SW];   // rows y0-2 .. y0+MY+1
  alignas(128) double atb[(MY + 4) * SW];  // tracer level L of the previous time level
  alignas(128) float ws[(MY + 2) * SW];    // rows y0-1 .. y0+MY
  alignas(128) float wkd[(MY + 3) * SW];   // rows y0-2 .. y0+MY
  alignas(128) float wkb[(MY + 3) * SW];   // rows y0-2 .. y0+MY
};
constexpr uint32_t kMxLevelBytes =
    (uint32_t)(2 * (MY + 4) * SW * sizeof(double) + ((MY + 2) * SW + 2 * (MY + 3) * SW) * sizeof(float));

struct MxSmem {
  MxSlot slot[NSM];
  float fxd[2][FXN];                  // per level parity: face difference d
  float fyd[2][FYN];
  unsigned char flag[3][MHN];          // predictor outside its local bounds
  float d2[MHN];                       // first Laplacian (times ahf)
  float tr[MHN], dtn[MHN], dts[MHN], dte[MHN], dtw[MHN], ahf[MHN];
  float kx[MHN], ky[MHN];               // del4 face weights tarea*dte (east face), tarea*dts (south face)
  float cxf[FXN], cyf[FYN];           // 2*dts/(htw*hun), 2*dts/(hts*hue) at the faces
  float fxu[2][FXN], fyv[2][FYN];    // per level parity: f32 face transports uw, vs
  float hwx[FXN], hsy[FYN];           // htw, hts at the faces (f32)
  uint16_t kmt[(MY + 4) * SW];        // bottom level of the tile's columns and their 2-cell halo
  uint64_t bar[NSM];
};
// four CTAs per SM: 228 KB of shared memory, 1 KB of it reserved per CTA
// kMixedCtasPerSm CTAs per SM: 228 KB of shared memory, 1 KB of it reserved per CTA
static_assert(kMixedCtasPerSm * (sizeof(MxSmem) + 1024) <= 228 * 1024,
              "mixed tracer tile no longer fits kMixedCtasPerSm CTAs per SM");

// Issue the boxes of level L of tracer n into a slot (one thread).
__device__ __forceinline__ void issue_mx(MxSlot& sl, uint64_t* bar, const TracerMaps& m, int cur, int n, int km,
                                         int L, int x0, int y0) {
  mbar_expect_tx(bar, kMxLevelBytes);
  tma_load_3d(sl.at, &m.at[cur], x0 - 4, y0 - 2, n * km + L, bar);
  tma_load_3d(sl.atb, &m.atb[cur], x0 - 4, y0 - 2, n * (km + 1) + L + 1, bar);
  tma_load_3d(sl.ws, &m.ws, x0 - 4, y0 - 1, L, bar);
  tma_load_3d(sl.wkd, &m.uw, x0 - 4, y0 - 2, L, bar);
  tma_load_3d(sl.wkb, &m.vs, x0 - 4, y0 - 2, L, bar);
}


// x face (fj, fi): row y0-1+fj, west side of column x0-1+fi
// y face (fj, fi): south side of row y0-2+fj, column x0-1+fi
__device__ __forceinline__ int fx(int fj, int fi) { return fj * (TX + 3) + fi; }
__device__ __forceinline__ int fy(int fj, int fi) { return fj * (TX + 2) + fi; }

// Face quantities of level kk for the 1-halo region, once per face: the f32
// transport (face32 on the U-point means) and the difference d.  Every later
// use reads these, so both cells of a face see the same f32 values.
//
// A face is described by (kind, index in its array, box index r): an x face
// by its east cell R = r, a y face by its north cell r.  Each thread forms the
// west x face and the north y face of its own cell, and up to two of the 192
// faces on the region's border (FaceSet).
__device__ __forceinline__ void face_one(MxSmem& S, const MxSlot& L, int kk, bool is_x, int m, int r) {
  if (is_x) {
    S.fxd[kk & 1][m] = (float)(L.at[r] - L.at[r - 1]);
    S.fxu[kk & 1][m] = face32(L.wkd[r - SW], L.wkd[r], S.hwx[m]);
  } else {
    S.fyd[kk & 1][m] = (float)(L.at[r + SW] - L.at[r]);
    S.fyv[kk & 1][m] = face32(L.wkb[r], L.wkb[r + 1], S.hsy[m]);
  }
}

constexpr int FX_OWN = TX * MY, FX_EXTRA = FXN - FX_OWN, FY_EXTRA = FYN - TX * MY;
constexpr int F_EXTRA = FX_EXTRA + FY_EXTRA;   // border faces of the region

struct FaceSet {
  int own_x, own_y, own_r;   // own cell's west x face, north y face, box index of the cell
  uint32_t e[2];             // border faces: bit 31 = y face, bits 16..30 index, bits 0..15 box index
  int ne;
};

__device__ __forceinline__ uint32_t face_desc(bool is_y, int m, int r) {
  return (is_y ? 0x80000000u : 0u) | ((uint32_t)m << 16) | (uint32_t)r;
}

// border face q (0 .. F_EXTRA-1): x faces of the top and bottom rows, x faces
// of the west column and the two east columns, y faces of rows 0, MY+1, MY+2,
// y faces of the west and east columns
__device__ __forceinline__ uint32_t border_face(int q) {
  int fj, fi;
  if (q < 2 * (TX + 3)) {
    fj = q < TX + 3 ? 0 : MY + 1;
    fi = q % (TX + 3);
    return face_desc(false, fx(fj, fi), (fj + 1) * SW + fi + 3);
  }
  q -= 2 * (TX + 3);
  if (q < 3 * MY) {
    const int c = q % 3;
    fj = 1 + q / 3;
    fi = c == 0 ? 0 : TX + c;
    return face_desc(false, fx(fj, fi), (fj + 1) * SW + fi + 3);
  }
  q -= 3 * MY;
  if (q < 3 * (TX + 2)) {
    const int row = q / (TX + 2);
    fj = row == 0 ? 0 : MY + row;
    fi = q % (TX + 2);
    return face_desc(true, fy(fj, fi), fj * SW + fi + 3);
  }
  q -= 3 * (TX + 2);
  fj = 1 + q / 2;
  fi = (q % 2) ? TX + 1 : 0;
  return face_desc(true, fy(fj, fi), fj * SW + fi + 3);
}

__device__ __forceinline__ FaceSet face_set(int tid) {
  const int tx = tid % TX, ty = tid / TX;
  FaceSet f;
  f.own_x = fx(ty + 1, tx + 1);
  f.own_y = fy(ty + 1, tx + 1);
  f.own_r = (ty + 2) * SW + tx + 4;
  f.ne = 0;
  for (int q = tid; q < F_EXTRA && f.ne < 2; q += MTH) f.e[f.ne++] = border_face(q);
  if (f.ne < 2) f.e[1] = 0;
  if (f.ne < 1) f.e[0] = 0;
  return f;
}

// sk: the slot of level kk (kk % NSM, carried through the level loop)
__device__ __forceinline__ void faces_level(MxSmem& S, int kk, int sk, const FaceSet& f) {
  const MxSlot& L = S.slot[sk];
  face_one(S, L, kk, true, f.own_x, f.own_r);
  face_one(S, L, kk, false, f.own_y, f.own_r - SW);
#pragma unroll
  for (int i = 0; i < 2; ++i)
    if (i < f.ne) {
      const uint32_t d = f.e[i];
      face_one(S, L, kk, !(d >> 31), (int)((d >> 16) & 0x7fffu), (int)(d & 0xffffu));
    }
}
static_assert(F_EXTRA <= 2 * MTH, "border faces: at most two per thread");

// A cell of the 1-halo region as one thread handles it: its index m in the
// region, box index r (at, atb, kmt boxes), u (ws box), its west x face fw and
// north y face fn (the east and south faces are fw + 1 and fn + HQX); valid:
// inside the rows and columns the reference computes (1 .. imt-2, 1 .. jmt-2).
// Every thread owns the interior cell above its column; the 76 ring cells of
// the region go to threads 0 .. 75, one each.
struct HCell {
  int m, r, u, fw, fn;
  bool valid;
};
constexpr int RING = MHN - TX * MY;

__device__ __forceinline__ HCell hcell(int hj, int hi, int x0, int y0, int imt, int jmt) {
  HCell c;
  c.m = hj * HQX + hi;
  c.r = r2(hj, hi);
  c.u = ru(hj, hi);
  c.fw = fx(hj, hi);
  c.fn = fy(hj, hi);
  const int gj = y0 - 1 + hj, gi = x0 - 1 + hi;
  c.valid = gi >= 1 && gi < imt - 1 && gj >= 1 && gj < jmt - 1;
  return c;
}

// ring cell q (0 .. RING-1): top row, bottom row, west column, east column
__device__ __forceinline__ HCell ring_hcell(int q, int x0, int y0, int imt, int jmt) {
  int hj, hi;
  if (q < HQX) { hj = 0; hi = q; }
  else if (q < 2 * HQX) { hj = MHQY - 1; hi = q - HQX; }
  else if (q < 2 * HQX + MY) { hj = q - 2 * HQX + 1; hi = 0; }
  else { hj = q - 2 * HQX - MY + 1; hi = HQX - 1; }
  return hcell(hj, hi, x0, y0, imt, jmt);
}

// Per-level constants of the predictor at level kk.
struct PredLevel {
  const double *at_c, *at_u, *at_d;
  const float *ws_c, *ws_d, *dx, *dy, *ux, *vy;
  float hodz, odzt_k, odzt_k1, dts;
  int kk, km;
  bool up, dn;   // level kk has a level above / below
};

// sc, su, sd: the slots of levels kk, kk-1, kk+1
__device__ __forceinline__ PredLevel pred_level(const MxSmem& S, const Arena& a, int kk, int sc, int su, int sd) {
  PredLevel P;
  const int km = a.km;
  P.kk = kk;
  P.km = km;
  // at the top and bottom levels the missing neighbour level is replaced by
  // level kk itself: its differences are then exactly zero, and so are the
  // vertical terms they carry (pred_cell needs no branch on the level)
  P.up = kk > 0;
  P.dn = kk < km - 1;
  P.at_c = S.slot[sc].at;
  P.at_u = P.up ? S.slot[su].at : P.at_c;
  P.at_d = P.dn ? S.slot[sd].at : P.at_c;
  P.ws_c = S.slot[sc].ws;
  P.ws_d = P.dn ? S.slot[sd].ws : P.ws_c;
  P.dx = S.fxd[kk & 1];
  P.dy = S.fyd[kk & 1];
  P.ux = S.fxu[kk & 1];
  P.vy = S.fyv[kk & 1];
  P.hodz = 0.5f * (float)a.odzp[kk];
  P.odzt_k = (float)a.odzt[kk];
  P.odzt_k1 = kk < km - 1 ? (float)a.odzt[kk + 1] : 0.f;
  P.dts = (float)a.p.dts;
  return P;
}

// Predictor and bound test of one cell: true if the predictor leaves the
// local bounds (the reference's a00 > amax or a00 < amin).
__device__ __forceinline__ bool pred_cell(const MxSmem& S, const PredLevel& P, const HCell& h) {
  if (!h.valid) return false;
  const int kk = P.kk, r = h.r, u = h.u;
  const int fw = h.fw, fe = fw + 1, fn = h.fn, fs = fn + HQX;
  const float* dx = P.dx;
  const float* dy = P.dy;
  const float dts = P.dts;
  // horizontal: east/west x faces, south/north y faces
  const float ue = P.ux[fe], uwv = P.ux[fw];
  const float vs = P.vy[fs], vn = P.vy[fn];
  const float sx = (dx[fe] * ue - lw_part(dx[fe], ue, S.cxf[fe])) + (dx[fw] * uwv + lw_part(dx[fw], uwv, S.cxf[fw]));
  const float sy = (dy[fs] * vs - lw_part(dy[fs], vs, S.cyf[fs])) + (dy[fn] * vn + lw_part(dy[fn], vn, S.cyf[fn]));
  // vertical faces: above (kk-1|kk) with w(kk), below (kk|kk+1) with w(kk+1)
  // (at a missing level the difference is 0, the term +-0, and sz stays +0)
  float sz = 0.f;
  const double c = P.at_c[r];
  const float dup = (float)(P.at_u[r] - c);   // a_above - c
  {
    const float w = P.ws_c[u];
    const float A = w * dup;
    sz += A - A * w * P.odzt_k * dts;
  }
  const float d = (float)(c - P.at_d[r]);
  const float ddn = -d;                         // a_below - c
  {
    const float w = P.ws_d[u];
    const float A = w * d;
    sz += A + A * w * P.odzt_k1 * dts;
  }
  const float inc = -(S.tr[h.m] * (sx + sy) + P.hodz * sz) * dts;
  // Bound test of the predictor c + inc against the masked 7-point extrema
  // (land excluded: -1e10 for the max, +1e10 for the min), done on
  // differences from c: c + inc > max_p a_p  <=>  inc > max_p (a_p - c).
  // The horizontal differences are the face differences already formed;
  // with no wet point the reference's extrema flag the cell, as -inf does.
  const uint16_t* kt = S.kmt;
  float dmax = -INFINITY, dmin = INFINITY;
  auto acc = [&](bool wet, float d) {
    if (wet) { dmax = fmaxf(dmax, d); dmin = fminf(dmin, d); }
  };
  acc(kk < kt[r], 0.f);
  acc(kk < kt[r + 1], dx[fe]);
  acc(kk < kt[r - 1], -dx[fw]);
  acc(kk < kt[r + SW], dy[fs]);
  acc(kk < kt[r - SW], -dy[fn]);
  acc(P.up && kk - 1 < kt[r], dup);
  acc(P.dn && kk + 1 < kt[r], ddn);
  return inc > dmax || inc < dmin;
}

// Predictor flags of level kk for the thread's own cell and ring cell;
// returns the own cell's flag.
__device__ __forceinline__ bool predictor_mixed(MxSmem& S, const Arena& a, int kk, int sc, int su, int sd,
                                                const HCell& own, const HCell& ring, bool has_ring) {
  const PredLevel P = pred_level(S, a, kk, sc, su, sd);
  unsigned char* fl = S.flag[sc];   // flags kept per level modulo 3, as the slots
  const bool f = pred_cell(S, P, own);
  fl[own.m] = f ? 1 : 0;
  if (has_ring) fl[ring.m] = pred_cell(S, P, ring) ? 1 : 0;
  return f;
}

// first Laplacian of atb at level kk (f32 on f64 differences), masked
__device__ __forceinline__ float d2_cell(const MxSmem& S, const double* atb, int kk, const HCell& h) {
  if (!h.valid) return 0.f;
  const int r = h.r, m = h.m;
  const double c = atb[r];
  if (kk > S.kmt[r] - 1) return 0.f;
  float v = 0.f;
  if (kk <= S.kmt[r - SW] - 1) v += S.dtn[m] * (float)(atb[r - SW] - c);
  if (kk <= S.kmt[r + SW] - 1) v += S.dts[m] * (float)(atb[r + SW] - c);
  if (kk <= S.kmt[r + 1] - 1) v += S.dte[m] * (float)(atb[r + 1] - c);
  if (kk <= S.kmt[r - 1] - 1) v += S.dtw[m] * (float)(atb[r - 1] - c);
  return S.ahf[m] * v;
}

__device__ __forceinline__ void del4_first_mixed(MxSmem& S, int kk, int sk, const HCell& own, const HCell& ring,
                                                 bool has_ring) {
  const double* atb = S.slot[sk].atb;
  S.d2[own.m] = d2_cell(S, atb, kk, own);
  if (has_ring) S.d2[ring.m] = d2_cell(S, atb, kk, ring);
}

// Per-tile 2-D data of the mixed march (kmt with a 2-cell halo, the metric
// and biharmonic terms of the 1-halo region, the face factors) with fixed
// trip counts and read-only loads, so a thread's loads of a loop are in
// flight together.  The batched kernel, whose work items are short and change
// member often, stages its tiles this way; the single-domain kernel keeps the
// plain loops in mixed_item, with which it compiles better.
__device__ __forceinline__ void stage_tile_statics_ahead(MxSmem& S, const Arena& a, int x0, int y0, double dts) {
  const int tid = threadIdx.x;
  const int imt = a.imt, jmt = a.jmt;
#pragma unroll
  for (int it = 0; it < ((MY + 4) * SW + MTH - 1) / MTH; ++it) {
    const int m = tid + it * MTH;
    if (m < (MY + 4) * SW) {
      const int gj = y0 - 2 + m / SW, gi = x0 - 4 + m % SW;
      S.kmt[m] = (gj >= 0 && gj < jmt && gi >= 0 && gi < imt) ? __ldg(a.kmt + (long)gj * imt + gi) : 0;
    }
}
#pragma unroll
for (int it = 0; it < (MHN + MTH - 1) / MTH; ++it) {
  const int m = tid + it * MTH;
  if (m < MHN) {
    const int gj = y0 - 1 + m / HQX, gi = x0 - 1 + m % HQX;
    const bool in = (gj >= 0 && gj < jmt && gi >= 0 && gi < imt);
    const long q = in ? (long)gj * imt + gi : 0;
    const double tarea = __ldg(a.tarea + q), dte = __ldg(a.dte + q), dtsq = __ldg(a.dts + q);
    S.tr[m] = in ? (float)__ldg(a.tarea_r + q) : 0.f;
    S.dtn[m] = in ? (float)__ldg(a.dtn + q) : 0.f;
    S.dts[m] = in ? (float)dtsq : 0.f;
    S.dte[m] = in ? (float)dte : 0.f;
    S.dtw[m] = in ? (float)__ldg(a.dtw + q) : 0.f;
    S.ahf[m] = in ? (float)__ldg(a.ahf + q) : 0.f;
    S.kx[m] = in ? (float)(tarea * dte) : 0.f;
    S.ky[m] = in ? (float)(tarea * dtsq) : 0.f;
  }
}
#pragma unroll
for (int it = 0; it < (FXN + FYN + MTH - 1) / MTH; ++it) {
  const int m = tid + it * MTH;
  if (m < FXN + FYN) {
    int gj, gi;
    if (m < FXN) { gj = y0 - 1 + m / (TX + 3); gi = x0 - 1 + m % (TX + 3); }
    else { gj = y0 - 2 + (m - FXN) / (TX + 2); gi = x0 - 1 + (m - FXN) % (TX + 2); }
    const bool inb = gj >= 0 && gj < jmt && gi >= 0 && gi < imt;
    const long q = inb ? (long)gj * imt + gi : 0;
    const double h = (m < FXN) ? __ldg(a.htw + q) : __ldg(a.hts + q);
    const double hu = (m < FXN) ? __ldg(a.hun + q) : __ldg(a.hue + q);
    const float v = inb ? (float)(2.0 * dts / (h * hu)) : 0.f;
    const float hf = inb ? (float)h : 0.f;
    if (m < FXN) { S.cxf[m] = v; S.hwx[m] = hf; }
    else { S.cyf[m - FXN] = v; S.hsy[m - FXN] = hf; }
  }
}
}

// One work item (tile, tracer) of the mixed column march.  Returns false if
// a level wait gave up: the CTA has then recorded the timeout and drained
// its boxes, and must return.
template <bool kLoadsAhead>
__device__ __forceinline__ bool mixed_item(MxSmem& S, const Arena& a, const TracerMaps& maps, double* scr, int ntx,
                                           long tile, int n, uint32_t& par, uint32_t& outstanding) {
  const int tid = threadIdx.x, tx = tid % TX, ty = tid / TX;
  const int imt = a.imt, jmt = a.jmt, km = a.km;
  const long A = a.A, F = a.F, FB = a.FB;
  const lt_params& p = a.p;
  const double dts = p.dts;
  const float dtsf = (float)dts;
  const double* __restrict__ odzp = a.odzp;
  const double* __restrict__ odzt = a.odzt;
  {
    const int x0 = (int)(tile % ntx) * TX, y0 = (int)(tile / ntx) * MY;
    const int i = x0 + tx, j = y0 + ty;
    double* at_out = a.at[a.cur ^ 1] + n * F;
    double* atb_out = a.atb[a.cur ^ 1] + n * FB;

    __syncthreads();
    // level L goes to slot s = L % NSM
    auto issue = [&](int L, int s) {
      if (tid == 0) issue_mx(S.slot[s], &S.bar[s], maps, a.cur, n, km, L, x0, y0);
      outstanding |= 1u << s;
    };
    auto wait = [&](int s) -> bool {
      const bool ok = mbar_wait(&S.bar[s], (par >> s) & 1u, a.wait_limit);
      if (ok) { par ^= 1u << s; outstanding &= ~(1u << s); }
      return ok;
    };
    for (int L = km - 1; L >= (km - NSM > 0 ? km - NSM : 0); --L) issue(L, L % NSM);
    if constexpr (kLoadsAhead) {
      stage_tile_statics_ahead(S, a, x0, y0, dts);
    } else {
      for (int m = tid; m < (MY + 4) * SW; m += MTH) {
        const int gj = y0 - 2 + m / SW, gi = x0 - 4 + m % SW;
        S.kmt[m] = (gj >= 0 && gj < jmt && gi >= 0 && gi < imt) ? a.kmt[(long)gj * imt + gi] : 0;
      }
      for (int m = tid; m < MHN; m += MTH) {
        const int gj = y0 - 1 + m / HQX, gi = x0 - 1 + m % HQX;
        const bool in = (gj >= 0 && gj < jmt && gi >= 0 && gi < imt);
        const long q = in ? (long)gj * imt + gi : 0;
        S.tr[m] = in ? (float)a.tarea_r[q] : 0.f;
        S.dtn[m] = in ? (float)a.dtn[q] : 0.f;
        S.dts[m] = in ? (float)a.dts[q] : 0.f;
        S.dte[m] = in ? (float)a.dte[q] : 0.f;
        S.dtw[m] = in ? (float)a.dtw[q] : 0.f;
        S.ahf[m] = in ? (float)a.ahf[q] : 0.f;
        S.kx[m] = in ? (float)(a.tarea[q] * a.dte[q]) : 0.f;
        S.ky[m] = in ? (float)(a.tarea[q] * a.dts[q]) : 0.f;
      }
      for (int m = tid; m < FXN + FYN; m += MTH) {
        int gj, gi;
        if (m < FXN) { gj = y0 - 1 + m / (TX + 3); gi = x0 - 1 + m % (TX + 3); }
        else { gj = y0 - 2 + (m - FXN) / (TX + 2); gi = x0 - 1 + (m - FXN) % (TX + 2); }
        float v = 0.f;
        if (gj >= 0 && gj < jmt && gi >= 0 && gi < imt) {
          const long q = (long)gj * imt + gi;
          v = (m < FXN) ? (float)(2.0 * dts / (a.htw[q] * a.hun[q])) : (float)(2.0 * dts / (a.hts[q] * a.hue[q]));
        }
        if (m < FXN) S.cxf[m] = v; else S.cyf[m - FXN] = v;
        const bool inb = gj >= 0 && gj < jmt && gi >= 0 && gi < imt;
        if (m < FXN) S.hwx[m] = inb ? (float)a.htw[(long)gj * imt + gi] : 0.f;
        else S.hsy[m - FXN] = inb ? (float)a.hts[(long)gj * imt + gi] : 0.f;
      }
    }

    const bool own = (i < imt && j < jmt);
    const bool inner = own && i >= 2 && i < imt - 2 && j >= 2 && j < jmt - 2;
    const long qo = own ? (long)j * imt + i : 0;
    const int kz = own ? a.kmt[qo] : 0;
    const int hc = (ty + 1) * HQX + (tx + 1);
    const int rc = r2(ty + 1, tx + 1), uc = ru(ty + 1, tx + 1);
    const HCell own_cell = hcell(ty + 1, tx + 1, x0, y0, imt, jmt);
    const bool has_ring = tid < RING;
    const HCell ring_cell = ring_hcell(has_ring ? tid : 0, x0, y0, imt, jmt);
    const FaceSet fset = face_set(tid);
    const int fe = fx(ty + 1, tx + 2), fwi = fx(ty + 1, tx + 1), fs = fy(ty + 2, tx + 1), fn = fy(ty + 1, tx + 1);
    const float swv = (inner && n == 0) ? (float)a.swv[qo] : 0.f;
    const double stf = own ? a.stf_n[n * A + qo] : 0.0;
    const double err_norm2 = a.scalars[0];
    const double ah64 = p.ah;
    const double trc = inner ? a.tarea_r[qo] : 0.0;
    const double htw_w64 = inner ? a.htw[qo] : 0.0, htw_e64 = inner ? a.htw[qo + 1] : 0.0;
    const double hts_s64 = inner ? a.hts[qo] : 0.0, hts_n64 = inner ? a.hts[qo - imt] : 0.0;
    double e_prev = 0.0, f_prev = 0.0;
    double carry = 0.0;  // lower face of the level below, as seen by the level above: A + X
    float w_below = 0.f;  // explicit diffusion flux through the bottom face, from the level below
    // own column's mixing coefficient: level k in akt_here, level k-1 loaded a step ahead
    const float* akt_col = a.akt32 + n * F + qo;
    float akt_here = inner ? __ldg(akt_col + (long)(km - 1) * A) : 0.f;

    // slots of levels k, k-1, k+1 (NSM == 3: level k-2 shares k+1's)
    static_assert(NSM == 3, "slot rotation below assumes three slots");
    int sk = (km - 1) % NSM;
    int sm1 = sk == 0 ? 2 : sk - 1, sp1 = sk == 2 ? 0 : sk + 1;
    {
      const bool ok = wait(sk) && wait(sm1);
      if (__syncthreads_or(!ok)) { tma_bail(S, a, par, outstanding); return false; }
    }
    faces_level(S, km - 1, sk, fset);
    __syncthreads();
    predictor_mixed(S, a, km - 1, sk, sm1, sp1, own_cell, ring_cell, has_ring);

    // Level slots: after step k the slot of level k takes level k-NSM.
    for (int k = km - 1; k >= 0; --k) {
      const float akt_above = (inner && k >= 1) ? __ldg(akt_col + (long)(k - 1) * A) : 0.f;
      // ---- phase B1: faces one level up, first Laplacian here (levels k-1, k
      // arrived in earlier steps; the previous step ended with a barrier)
      if (k >= 1) faces_level(S, k - 1, sm1, fset);
      del4_first_mixed(S, k, sk, own_cell, ring_cell, has_ring);
      const bool ok = (k >= 2) ? wait(sp1) : true;   // level k-2
      if (__syncthreads_or(!ok)) { tma_bail(S, a, par, outstanding); return false; }
      // ---- phase B2: predictor one level up.  The column phase below reads
      // the flags of level k (written in the previous step) and, of level
      // k-1, only its own cell's flag, which this thread computes: no barrier
      // between the two phases.
      const bool flag_up = (k >= 1) ? predictor_mixed(S, a, k - 1, sm1, sp1, sk, own_cell, ring_cell, has_ring) : false;
      // ---- phase C: own column at level k
      if (inner) {
        const MxSlot& Lk = S.slot[sk];
        const unsigned char* fl = S.flag[sk];
        const bool self = fl[hc] != 0;
        const float* dx = S.fxd[k & 1];
        const float* dy = S.fyd[k & 1];
        const float ue = S.fxu[k & 1][fe], uwv = S.fxu[k & 1][fwi];
        const float vsv = S.fyv[k & 1][fs], vnv = S.fyv[k & 1][fn];
        // the same faces in f64, as the continuity march formed them
        const int xw = (ty + 1) * SW + tx + 4;   // wkd of U point (j-1, i); (j, i) is one row down
        const double ue64 = face_x64(Lk.wkd[xw + 1], Lk.wkd[xw + 1 + SW], htw_e64);
        const double uw64 = face_x64(Lk.wkd[xw], Lk.wkd[xw + SW], htw_w64);
        const int ys = (ty + 2) * SW + tx + 4;   // wkb of U point (j, i); (j, i+1) is next
        const double vs64 = face_y64(Lk.wkb[ys], Lk.wkb[ys + 1], hts_s64);
        const double vn64 = face_y64(Lk.wkb[ys - SW], Lk.wkb[ys - SW + 1], hts_n64);
        // Content bookkeeping.  Both cells of a face receive its centred part
        // A = d*u with the same sign (the advective form), so any rounding of
        // A adds up over the domain instead of cancelling: A is formed in f64
        // from the exact f64 state difference and the f32 transport.  The
        // upwind / Lax-Wendroff part X (f32) enters the two cells with
        // opposite signs and cancels exactly in the f64 face sums.
        const double c = Lk.at[rc];
        const double dE = Lk.at[rc + 1] - c, dW = c - Lk.at[rc - 1];
        const double dS = Lk.at[rc + SW] - c, dN = c - Lk.at[rc - SW];
        float t;
        t = dx[fe];                                   // east face: this cell is L
        const float Xe = (self || fl[hc + 1]) ? fabsf(ue) * t : lw_part(t, ue, S.cxf[fe]);
        t = dx[fwi];
        const float Xw = (self || fl[hc - 1]) ? fabsf(uwv) * t : lw_part(t, uwv, S.cxf[fwi]);
        t = dy[fs];
        const float Xs = (self || fl[hc + HQX]) ? fabsf(vsv) * t : lw_part(t, vsv, S.cyf[fs]);
        t = dy[fn];
        const float Xn = (self || fl[hc - HQX]) ? fabsf(vnv) * t : lw_part(t, vnv, S.cyf[fn]);
        double sh = dE * ue64 + dW * uw64 + dS * vs64 + dN * vn64;
        sh += ((double)Xw - (double)Xe) + ((double)Xn - (double)Xs);
        // vertical: face above (k-1|k) computed here, face below carried
        // (at the top level the level itself stands in for the missing one
        // above: the difference and both face terms are 0, sz keeps carry)
        double sz = carry;
        {
          const float wv = Lk.ws[uc];
          const double d64 = (k > 0 ? S.slot[sm1].at : Lk.at)[rc] - c;
          const float d = (float)d64;
          const bool up = self || flag_up;
          const float Xv = up ? fabsf(wv) * d : (wv * d) * wv * (float)odzt[k] * dtsf;
          const double Av = (double)wv * d64;
          sz += Av - (double)Xv;
          carry = Av + (double)Xv;
        }
        // Face-flux sums are weighted by tarea_r (horizontal) and odzp
        // (vertical) in f64, so a flux leaves one cell and enters the next
        // with weights that cancel against the cell volumes to f64 rounding.
        const float vit_k = k < kz ? 1.f : 0.f;
        const float vit_kp1 = (k + 1 < kz) ? 1.f : 0.f;
        sh *= (double)vit_k;                          // horizontal advection, times -tarea_r
        const double vadv = -0.5 * sz * (double)vit_k;  // vertical advection, times odzp
        double vz = 0.0;                              // other vertical face-flux differences, times odzp
        float tf = 0.f;                               // the remaining tendency terms
        // second Laplacian as face fluxes K*(d2_R - d2_L), K = tarea*dte
        // (x) or tarea*dts (y): one f32 value per face, the same in both of
        // its cells, summed in f64 (dtn/dts/dte/dtw are K*tarea_r of the
        // cell, hmix_del4.F90:368-385)
        double hd = 0.0;
        if (k <= S.kmt[rc] - 1) {
          const float dc = S.d2[hc];
          if (k <= S.kmt[rc + 1] - 1) hd += (double)(S.kx[hc] * (S.d2[hc + 1] - dc));
          if (k <= S.kmt[rc - 1] - 1) hd -= (double)(S.kx[hc - 1] * (dc - S.d2[hc - 1]));
          if (k <= S.kmt[rc + SW] - 1) hd += (double)(S.ky[hc] * (S.d2[hc + HQX] - dc));
          if (k <= S.kmt[rc - SW] - 1) hd -= (double)(S.ky[hc - HQX] * (dc - S.d2[hc - HQX]));
        }
        const double atb_k = Lk.atb[rc];
        const double atb_km1 = k >= 1 ? S.slot[sm1].atb[rc] : 0.0;
        const float wkc_k = akt_here;
        const float wkc_km1 = akt_above;
        // shortwave through the faces above and below (tracer.cpp:1430-1474)
        // and the explicit half of the vertical diffusion: each face flux is
        // the same f32 expression in the cells above and below it, summed in f64
        if (n == 0) {
          if (k >= 1) vz += (double)(swv * (float)a.pen[k - 1] * vit_k);
          if (k < km - 1) vz -= (double)(swv * (float)a.pen[k] * vit_kp1);
        }
        const float w1 = k >= 1 ? wkc_km1 * (float)(atb_km1 - atb_k) * (float)odzt[k] * vit_k : 0.f;
        const float w2 = w_below;   // = wkc_k * (atb_k - atb_kp1) * odzt[k+1] * vit_kp1, as formed at level k+1
        w_below = w1;
        vz += 0.5 * ((double)w1 - (double)w2);
        // surface flux and the freshwater-norm correction stay f64: the
        // correction cancels the global salt flux, which f32 would leave at
        // f32 precision of the flux
        double sfc = 0.0;
        if (k == 0) {
          if (kz > 0) sfc = stf * 0.5 * odzp[0];
          if (n == 1) sfc += err_norm2 * (double)vit_k;
        }
        if (p.boundary_restore == 1 && k >= 1)
          tf += vit_k * (float)(a.restore[n * F + (long)k * A + qo] - atb_k) * (float)(1.0 / (15.0 * 86400.0));
        const double d8 = c + dts * ((double)tf - trc * sh + odzp[k] * (vz + vadv) + sfc + ah64 * trc * hd);
        double ev = 0.0, fv = d8;
        if (k < kz) {
          double a8, c8, b8;
          if (k >= 1) a8 = (double)wkc_km1 * odzt[k] * odzp[k] * dts * 0.5;
          else a8 = odzp[0] * dts * 0.5;
          if (k == kz - 1) {
            c8 = odzp[kz - 1] * dts * 0.5;
            b8 = 1.0 + a8;
          } else if (k >= 1) {
            c8 = (double)wkc_k * odzt[k + 1] * odzp[k] * dts * 0.5;
            b8 = 1.0 + a8 + c8;
          } else {
            c8 = (double)wkc_k * odzt[k + 1] * odzp[k] * dts * 0.5;
            b8 = 1.0 + c8;
          }
          if (k == kz - 1) { e_prev = 0.0; f_prev = 0.0; }
          const double g0 = 1.0 / (b8 - c8 * e_prev);
          ev = a8 * g0;
          fv = (d8 + c8 * f_prev) * g0;
          e_prev = ev;
          f_prev = fv;
        }
        double* sl = scr + (long)k * 2 * MTH;
        sl[tid] = ev;
        sl[MTH + tid] = fv;
      }
      akt_here = akt_above;
      __syncthreads();
      if (k - NSM >= 0) issue(k - NSM, sk);   // level k-3 takes level k's slot
      // one level down: the slots of k-1, k-2, k
      sp1 = sk;
      sk = sm1;
      sm1 = sk == 0 ? 2 : sk - 1;
    }
    // substitution, top down: the elimination coefficients of SUB levels are
    // loaded together ahead of their stores (one scratch round trip per SUB
    // levels)
    if (inner) {
      double x = 0.0;
      constexpr int SUB = 8;
      for (int k0 = 0; k0 < km; k0 += SUB) {
        double evs[SUB], fvs[SUB];
#pragma unroll
        for (int c = 0; c < SUB; ++c) {
          const double* sl = scr + (long)(k0 + c) * 2 * MTH;
          evs[c] = k0 + c < km ? sl[tid] : 0.0;
          fvs[c] = k0 + c < km ? sl[MTH + tid] : 0.0;
        }
#pragma unroll
      for (int c = 0; c < SUB; ++c) {
        const int k = k0 + c;
        if (k >= km) break;
        const double ev = evs[c], fv = fvs[c];
        double v;
        if (k < kz) {
          v = (k == 0) ? ev * stf + fv : ev * x + fv;
          x = v;
        } else {
          v = fv;
        }
        const long cg = (long)k * A + qo;
        at_out[cg] = v;
        atb_out[(long)(k + 1) * A + qo] = v;
      }
      }
    }
  }
  return true;
}

__device__ __forceinline__ MxSmem& mixed_smem_init() {
  extern __shared__ __align__(128) unsigned char smem_mx[];
  MxSmem& S = *reinterpret_cast<MxSmem*>(smem_mx);
  if (threadIdx.x == 0) {
    for (int s = 0; s < NSM; ++s) mbar_init(&S.bar[s], 1);
    mbar_fence_init();
  }
  __syncthreads();
  return S;
}

__global__ void __launch_bounds__(MTH, kMixedCtasPerSm)
    k_tracer_mixed(Arena a, const __grid_constant__ TracerMaps maps, int ntx, long ntiles) {
  MxSmem& S = mixed_smem_init();
  uint32_t par = 0, outstanding = 0;
  double* scr = a.col_scratch + (long)blockIdx.x * a.km * 2 * MTH;
  for (long w = blockIdx.x; w < 2 * ntiles; w += gridDim.x)
    if (!mixed_item<false>(S, a, maps, scr, ntx, w >> 1, (int)(w & 1), par, outstanding)) return;
}

// Several domains (ensemble members, serving requests; any sizes) in one
// persistent launch: the work list is the concatenation of every member's
// (tile, tracer) items, member after member, so neighbouring CTAs work on
// neighbouring tiles of the same member.  Each CTA's items ascend, so its
// member index only moves forward.
// The current member's arena is copied into shared memory behind MxSmem:
// read from there, its fields cannot alias the kernel's global stores, so
// the compiler keeps them across the level loop instead of reloading them
// from global memory at every level.
constexpr size_t kBatchArenaOff = (sizeof(MxSmem) + 15) / 16 * 16;
constexpr size_t kBatchSmem = kBatchArenaOff + sizeof(Arena);
static_assert(sizeof(Arena) % 16 == 0, "arena copied as 16-byte words");
static_assert(kMixedCtasPerSm * (kBatchSmem + 1024) <= 228 * 1024,
              "batched mixed tracer tile no longer fits kMixedCtasPerSm CTAs per SM");

__global__ void __launch_bounds__(MTH, kMixedCtasPerSm)
    k_tracer_mixed_batch(const MemberDesc* __restrict__ mem, int nmem, long total, double* scratch, int km_max) {
  MxSmem& S = mixed_smem_init();
  extern __shared__ __align__(128) unsigned char smem_mx[];
  Arena& sa = *reinterpret_cast<Arena*>(smem_mx + kBatchArenaOff);
  uint32_t par = 0, outstanding = 0;
  double* scr = scratch + (long)blockIdx.x * km_max * 2 * MTH;
  int m = 0, staged = -1;
  for (long w = blockIdx.x; w < total; w += gridDim.x) {
    while (m + 1 < nmem && mem[m + 1].item0 <= w) ++m;
    const MemberDesc& d = mem[m];
    if (m != staged) {
      __syncthreads();   // the previous item no longer reads the staged arena
      const uint4* src = reinterpret_cast<const uint4*>(&d.a);
      uint4* dst = reinterpret_cast<uint4*>(&sa);
      for (int t = threadIdx.x; t < (int)(sizeof(Arena) / 16); t += MTH) dst[t] = src[t];
      __syncthreads();
      staged = m;
    }
    const long local = w - d.item0;
    if (!mixed_item<true>(S, sa, d.maps, scr, d.ntx, local >> 1, (int)(local & 1), par, outstanding)) return;
  }
}

}  // namespace

int launch_tracer_tma_mixed(const Arena& a, const TracerMaps& maps, cudaStream_t s, int grid) {
  const int ntx = (a.imt + TX - 1) / TX;
  const long ntiles = (long)ntx * ((a.jmt + MY - 1) / MY);
  const size_t sm = sizeof(MxSmem);
  static bool attr = false;
  if (!attr) {
    LT_CUDA_OK(cudaFuncSetAttribute(k_tracer_mixed, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    attr = true;
  }
  k_tracer_mixed<<<grid, MTH, sm, s>>>(a, maps, ntx, ntiles);
  LT_LAUNCHED();
  return LT_OK;
}

int prepare_tracer_mixed_batch() {
  LT_CUDA_OK(cudaFuncSetAttribute(k_tracer_mixed_batch, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)kBatchSmem));
  return LT_OK;
}

// prepare_tracer_mixed_batch() must have run on this device (it cannot run
// inside a stream capture)
int launch_tracer_mixed_batch(const MemberDesc* mem, int nmem, long total, double* scratch, int km_max, int grid,
                              cudaStream_t s) {
  k_tracer_mixed_batch<<<grid, MTH, kBatchSmem, s>>>(mem, nmem, total, scratch, km_max);
  LT_LAUNCHED();
  return LT_OK;
}

int launch_continuity_mixed_batch(const MemberDesc* mem, int nmem, int max_imt, int max_jmt, int cby,
                                  cudaStream_t s) {
  const unsigned gx = (max_imt + CBX - 1) / CBX;
  switch (cby) {
    case 4: k_cont_batch<4><<<dim3(gx, (max_jmt + 3) / 4, nmem), dim3(CBX, 4), 0, s>>>(mem); break;
    case 8: k_cont_batch<8><<<dim3(gx, (max_jmt + 7) / 8, nmem), dim3(CBX, 8), 0, s>>>(mem); break;
    case 16: k_cont_batch<16><<<dim3(gx, (max_jmt + 15) / 16, nmem), dim3(CBX, 16), 0, s>>>(mem); break;
    default: set_error("continuity tile height %d not built (4, 8, 16)", cby); return LT_E_INVALID;
  }
  LT_LAUNCHED();
  return LT_OK;
}

int launch_continuity_mixed(const Arena& a, cudaStream_t s) {
  dim3 b(CBX, kContTileY), g((a.imt + CBX - 1) / CBX, (a.jmt + kContTileY - 1) / kContTileY);
  k_cont_march32<<<g, b, 0, s>>>(a);
  LT_LAUNCHED();
  return LT_OK;
}

}  // namespace lt
