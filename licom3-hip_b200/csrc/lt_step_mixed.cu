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

// The U-point mean velocity wkd = (utf*oncc + utl)/2 (wkb likewise), with
// every rounding spelled out: the plain-load and the TMA-fed march form it
// in different code, and must give the same bits.
__device__ __forceinline__ float u_mean32(float f, float l, float oncc) {
  return __fadd_rn(__fmul_rn(0.5f, __fmul_rn(f, oncc)), __fmul_rn(0.5f, l));
}

// Horizontal divergence of one T cell at one level (tracer_1, upwell_2,
// operators_div; the four faces as the tracer kernel forms them, face_x64 /
// face_y64, with the free-surface correction: (uk_1 + uk_2) * htw = 4 * uw +
// htw * (fm1_1 * wkd_1 + fm1_2 * wkd_2)), roundings spelled out for the same
// reason.  d*: wkd at the U points (j-1,i), (j,i), (j-1,i+1), (j,i+1); b*:
// wkb at the same points; f*: the free-surface factors minus one there.
struct ContCell {
  double htw_c, htw_e, hts_c, hts_n, tr;
};
__device__ __forceinline__ double cont_wka(const ContCell& g, float dn, float d0, float dn1, float d01, float bn,
                                           float b0, float bn1, float b01, float fn, float f0, float fn1,
                                           float f01) {
  auto corr = [](float f1, float w1, float f2, float w2) {
    return __dadd_rn(__dmul_rn((double)f1, (double)w1), __dmul_rn((double)f2, (double)w2));
  };
  const double uw_w = face_x64(dn, d0, g.htw_c);
  const double uw_e = face_x64(dn1, d01, g.htw_e);
  const double vs_s = face_y64(b0, b01, g.hts_c);
  const double vs_n = face_y64(bn, bn1, g.hts_n);
  const double east = __fma_rn(g.htw_e, corr(f01, d01, fn1, dn1), __dmul_rn(4.0, uw_e));
  const double west = __fma_rn(g.htw_c, corr(f0, d0, fn, dn), __dmul_rn(4.0, uw_w));
  const double south = __fma_rn(g.hts_c, corr(f01, b01, f0, b0), __dmul_rn(4.0, vs_s));
  const double north = __fma_rn(g.hts_n, corr(fn1, bn1, fn, bn), __dmul_rn(4.0, vs_n));
  return __dmul_rn(__dmul_rn(0.5, __dadd_rn(__dsub_rn(east, west), __dsub_rn(south, north))), g.tr);
}

// Final pass of the march: ws(k) from the partial sums P(k), parked in the ws
// field (ps null) or in shared memory (ps[k * ps_stride]), eight levels'
// loads ahead of their stores.
__device__ __forceinline__ void cont_finish(const Arena& a, long qo, int kz, double P, const float* ps = nullptr,
                                            int ps_stride = 0) {
  const int km = a.km;
  const long A = a.A;
  const double ohbt = a.ohbt[qo];
  const double fac = 1.0 / (1.0 + a.stf_ssh[qo] * ohbt);
  const double W = -P;
  float* __restrict__ ws = a.ws32;
  const double ws0 = ws[qo];
  const double* __restrict__ dzp = a.dzp;
  double Z = 0.0;
  for (int k0 = 1; k0 < km; k0 += 8) {
    float pk[8];
#pragma unroll
    for (int c = 0; c < 8; ++c)
      pk[c] = (k0 + c < km && k0 + c < kz) ? (ps ? ps[(k0 + c) * ps_stride] : ws[(long)(k0 + c) * A + qo]) : 0.f;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const int k = k0 + c;
      if (k >= km) break;
      Z = __dadd_rn(Z, dzp[k - 1]);
      ws[(long)k * A + qo] =
          (k < kz) ? (float)__dmul_rn(fac, __dadd_rn(__fma_rn(__dmul_rn(W, ohbt), Z, ws0), (double)pk[c])) : 0.f;
    }
  }
}

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
        s_wkd[b][m] = rin[p] ? u_mean32(ruf[p], rul[p], oncc) : 0.f;
        s_wkb[b][m] = rin[p] ? u_mean32(rvf[p], rvl[p], oncc) : 0.f;
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
        const ContCell g{htw_cd, htw_ed, hts_cd, hts_nd, tr};
        const double wka = cont_wka(g, wd[mn], wd[m0], wd[mn + 1], wd[m0 + 1], wb[mn], wb[m0], wb[mn + 1],
                                    wb[m0 + 1], s_fm1[mn], s_fm1[m0], s_fm1[mn + 1], s_fm1[m0 + 1]);
        if (k >= 1) a.ws32[c] = (float)P;
        P = __fma_rn(a.dzp[k], wka, P);
      }
    }
    // buffer b^1 was last read in step k-1, before this step's barrier
    if (k + 1 < km) park(b ^ 1);
  }
  if (!col_here) return;
  cont_finish(a, qo, kz, P);
}

constexpr int kContTileY = kMixedContTileY;   // tile height of the single-domain continuity march

// The single-domain march fed by TMA: each level's raw U-point velocities
// (utf, vtf, utl, vtl over the tile plus a row above and a column east) come
// as four boxes into a ring of kContRing level slots, so kContRing levels of
// loads are in flight; each thread forms the U-point means it needs from
// them (u_mean32, the same bits as the plain-load march).  The partial sums
// P(k) of the upward integration stay in shared memory behind the ring (km
// floats per column) instead of making a round trip through the ws field
// (through ws: 3.77 -> 3.93 ms per 0.1-degree step, the round trip reaches
// DRAM).  The ring's depth and the boxes' width set how many CTAs fit on an
// SM: six slots of 40-column boxes, four CTAs (3.77 ms); four slots, five
// CTAs (3.55 ms); three slots of 36-column boxes with the free-surface
// factors in registers, six CTAs (3.54 ms: the march runs at about 72 % of
// the measured copy bandwidth in either of the last two shapes).
constexpr int kContRing = 3;
constexpr int CRW = kMixedContBoxW, CRR = kMixedContTileY + 1;
// A tiled TMA load writes to a 128-byte aligned shared-memory address: every
// box starts on a 128-byte boundary (a 16-byte aligned box faulted with a
// misaligned address).
struct alignas(128) ContSlot {
  struct alignas(128) Box { float v[CRR * CRW]; };
  Box f[4];   // utf, vtf, utl, vtl
};
struct ContSmem {
  ContSlot slot[kContRing];
  uint64_t bar[kContRing];
};
constexpr uint32_t kContLevelBytes = 4 * CRR * CRW * sizeof(float);

__global__ void __launch_bounds__(CBX * kContTileY) k_cont_tma32(Arena a, const __grid_constant__ TracerMaps maps) {
  extern __shared__ __align__(128) unsigned char smem_ct[];
  ContSmem& S = *reinterpret_cast<ContSmem*>(smem_ct);
  constexpr int NT = CBX * kContTileY;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * CBX + tx;
  float* ps = reinterpret_cast<float*>(smem_ct + sizeof(ContSmem)) + tid;   // P(k) at ps[k * NT]
  const int x0 = blockIdx.x * CBX, y0 = blockIdx.y * kContTileY;
  const int imt = a.imt, jmt = a.jmt, km = a.km;
  const long A = a.A;
  const float oncc = (float)a.p.oncc;
  if (tid == 0) {
    for (int r = 0; r < kContRing; ++r) mbar_init(&S.bar[r], 1);
    mbar_fence_init();
  }
  __syncthreads();
  auto issue = [&](int k) {
    if (tid == 0 && k < km) {
      const int r = k % kContRing;
      mbar_expect_tx(&S.bar[r], kContLevelBytes);
      for (int v = 0; v < 4; ++v) tma_load_3d(S.slot[r].f[v].v, &maps.vel[v], x0, y0 - 1, k, &S.bar[r]);
    }
  };
  for (int k = 0; k < kContRing; ++k) issue(k);
  // the free-surface factor minus one at U point (uj, ui), -1 where the
  // reference's uk/vk are zero (as cont_tile forms it for its region)
  auto fm1_at = [&](int uj, int ui) {
    float fm1 = -1.f;
    if (uj >= 0 && uj < jmt - 1 && ui >= 1 && ui < imt) {
      const long q = (long)uj * imt + ui;
      const double work = a.au0[q] * a.stf_ssh[q] + a.aus[q] * a.stf_ssh[q + imt] +
                          a.auw[q] * a.stf_ssh[q - 1] + a.ausw[q] * a.stf_ssh[q + imt - 1];
      fm1 = (float)(work * a.ohbu[q]);
    }
    return fm1;
  };
  const int i = x0 + tx, j = y0 + ty;
  const bool own = i < imt && j < jmt;
  const bool div_here = own && j >= 1 && i < imt - 1;
  const bool col_here = own && j >= 1 && j < jmt - 1 && i >= 1 && i < imt - 1;
  const long qo = own ? (long)j * imt + i : 0;
  const int kz = own ? a.kmt[qo] : 0;
  const ContCell g{own ? a.htw[qo] : 0.0, div_here ? a.htw[qo + 1] : 0.0, own ? a.hts[qo] : 0.0,
                   div_here ? a.hts[qo - imt] : 0.0, div_here ? a.tarea_r[qo] : 0.0};
  // box index of U point (j, i) and (j-1, i)
  const int b0 = (ty + 1) * CRW + tx, bn = ty * CRW + tx;
  const float fn = fm1_at(j - 1, i), f0 = fm1_at(j, i), fn1 = fm1_at(j - 1, i + 1), f01 = fm1_at(j, i + 1);
  // outside the domain the boxes read zeros, as the plain-load march does
  const bool in_n = j >= 1 && i < imt, in_0 = own, in_n1 = j >= 1 && i + 1 < imt, in_01 = j < jmt && i + 1 < imt;
  double P = 0.0;
  // level k is the (k / kContRing)-th use of its slot: that use's phase parity
  auto parity = [](int k) { return (uint32_t)((k / kContRing) & 1); };
  for (int k = 0; k < km; ++k) {
    const int r = k % kContRing;
    const bool ok = mbar_wait(&S.bar[r], parity(k), a.wait_limit);
    if (__syncthreads_or(!ok)) {
      // a wait ran out: record it, let the boxes still in flight land
      // (bounded) and leave together
      if (tid == 0) {
        atomicExch(a.status + 1, 1);
        for (int l = k; l < km && l < k + kContRing; ++l)
          mbar_wait(&S.bar[l % kContRing], parity(l));   // the full bound, whatever a.wait_limit is
      }
      __syncthreads();
      return;
    }
    const ContSlot& L = S.slot[r];
    auto mean = [&](int f, int l, int b, bool in) { return in ? u_mean32(L.f[f].v[b], L.f[l].v[b], oncc) : 0.f; };
    if (own) {
      const long c = (long)k * A + qo;
      const float d0 = mean(0, 2, b0, in_0), e0 = mean(1, 3, b0, in_0);
      a.utf_out32[c] = L.f[0].v[b0] * oncc;
      a.vtf_out32[c] = L.f[1].v[b0] * oncc;
      a.wkd32[c] = d0;
      a.wkb32[c] = e0;
      if (col_here && k < kz) {
        const double wka = cont_wka(g, mean(0, 2, bn, in_n), d0, mean(0, 2, bn + 1, in_n1), mean(0, 2, b0 + 1, in_01),
                                    mean(1, 3, bn, in_n), e0, mean(1, 3, bn + 1, in_n1), mean(1, 3, b0 + 1, in_01),
                                    fn, f0, fn1, f01);
        if (k >= 1) ps[k * NT] = (float)P;
        P = __fma_rn(a.dzp[k], wka, P);
      }
    }
    __syncthreads();   // level k's slot is read: it takes level k + kContRing
    issue(k + kContRing);
  }
  if (!col_here) return;
  cont_finish(a, qo, kz, P, ps, NT);
}

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
// Tile of the mixed march: TX x MY columns, one thread per column, and both
// tracers in every thread.  T and S move through the same faces with the
// same transports, masks and metric terms, so those are formed and read once
// for the two; the f32 arithmetic of the predictor runs on (T, S) pairs with
// the packed sm_100 instructions (fma/add/mul .f32x2).  The column phase, the
// first and second Laplacians and the sweep compute in f64: on this part the
// f64 pipe is cheaper than rounding every f64 state difference to f32 and
// every f32 term back (conversions issue at a quarter of the f64 rate), and
// the f32 inputs (U-point means, w, the mixing coefficient) are converted
// once where they enter.
constexpr int MY = kMixedTileY;
constexpr int MTH = kMixedThreads;
constexpr int MHQY = MY + 2;          // tile plus 1-cell halo, rows
constexpr int MHN = HQX * MHQY;
// Level slots.  Step k (the march runs upward) reads levels k-2, k-1 and k
// only, so at the end of step k the slot of level k takes level k-3: three
// slots keep one step of lead time for every box.
constexpr int NSM = 3;
// f64 boxes (state): columns x0-2 .. x0+TX+1, so that the x start stays a
// multiple of two elements (16 bytes); f32 boxes: columns x0-4 .. x0+TX+3 (SW)
constexpr int SW64 = kMixedBoxW64;
constexpr int FXN = (MY + 2) * (TX + 3);   // x faces of the 1-halo region
constexpr int FYN = (MY + 3) * (TX + 2);   // y faces of the 1-halo region
constexpr int FN = FXN + FYN;
constexpr int OXN = MY * (TX + 1);         // x faces of the tile (west sides of columns x0 .. x0+TX)
constexpr int OYN = (MY + 1) * TX;         // y faces of the tile (north sides of rows y0 .. y0+MY)

// One level of the column tile, filled by seven TMA boxes: T and S of the
// state and of its previous time level, w and the U-point means wkd, wkb
// from which the kernel forms the face transports (face32, face_x64,
// face_y64).
struct alignas(128) MxSlot {
  alignas(128) double at[2][(MY + 4) * SW64];    // rows y0-2 .. y0+MY+1
  alignas(128) double atb[2][(MY + 4) * SW64];   // tracer level L of the previous time level
  alignas(128) float ws[(MY + 2) * SW];          // rows y0-1 .. y0+MY
  alignas(128) float wkd[(MY + 3) * SW];         // rows y0-2 .. y0+MY
  alignas(128) float wkb[(MY + 3) * SW];         // rows y0-2 .. y0+MY
  alignas(128) float akt[2][TX * MY];            // mixing coefficient of the tile's columns (T, S)
};
static_assert(((MY + 4) * SW64 * sizeof(double)) % 128 == 0, "each tracer's box starts 128-byte aligned");
constexpr uint32_t kMxLevelBytes =
    (uint32_t)(4 * (MY + 4) * SW64 * sizeof(double) + ((MY + 2) * SW + 2 * (MY + 3) * SW + 2 * TX * MY) * sizeof(float));

// per-level constants of the march (the 1-D vertical grid)
struct MxLevel {
  double odzp, odzt;   // odzp(k), odzt(k)
  double ka, kc;       // odzt(k)*odzp(k)*dts/2, odzt(k+1)*odzp(k)*dts/2 (0 at the bottom)
  double pu, pd;       // pen(k-1) (0 at the top), pen(k) (0 at the bottom)
  float hodz, odzt1;   // f32 forms for the predictor: odzp(k)/2, odzt(k+1) (0 at the bottom)
};

struct MxSmem {
  MxSlot slot[NSM];
  // predictor's level, per face: the difference (T, S), 0 where a side is
  // land, and u + u*u*cf, u - u*u*cf of the f32 transport u (the cell east /
  // south of the face takes the first, the other cell the second)
  float4 fdq[FN];
  double ou[OXN + OYN], oq[OXN + OYN]; // column phase's level: the tile's f64 transports and u*u*cf
  double d2[2][MHN];                   // column phase's level: first Laplacian times ahf (T, S)
  unsigned char flag[NSM][MHN];        // bit n: tracer n's predictor leaves its local bounds
  float tr[MHN], dtn[MHN], dts[MHN], dte[MHN], dtw[MHN], ahf[MHN];
  float cf[FN];                        // 2*dts/(htw*hun) at x faces, 2*dts/(hts*hue) at y faces
  float hw[FN];                        // htw at x faces, hts at y faces
  uint16_t kmt[(MY + 4) * SW64];       // bottom level of the tile's columns and their 2-cell halo
  int wmax[MTH / 32];                  // per-warp maxima of the region's bottom level
  uint64_t bar[NSM];
};
// followed by the km level constants (dynamic shared memory)
constexpr size_t kMxLevOff = (sizeof(MxSmem) + 15) / 16 * 16;
__host__ __device__ constexpr size_t mx_smem_bytes(int km) { return kMxLevOff + (size_t)km * sizeof(MxLevel); }
// kMixedCtasPerSm CTAs per SM: 228 KB of shared memory, 1 KB of it reserved
// per CTA; the largest km a mixed domain may have must still fit
static_assert(kMixedCtasPerSm * (mx_smem_bytes(kMixedMaxLevels) + sizeof(Arena) + 16 + 1024) <= 228 * 1024,
              "mixed tracer tile no longer fits kMixedCtasPerSm CTAs per SM");

// x face (fj, fi): row y0-1+fj, west side of column x0-1+fi
// y face (fj, fi): south side of row y0-2+fj, column x0-1+fi (index FXN + ...)
__device__ __forceinline__ int fx(int fj, int fi) { return fj * (TX + 3) + fi; }
__device__ __forceinline__ int fy(int fj, int fi) { return FXN + fj * (TX + 2) + fi; }
// region cell (hj, hi) = row y0-1+hj, column x0-1+hi in the boxes
__device__ __forceinline__ int b64(int hj, int hi) { return (hj + 1) * SW64 + hi + 1; }   // at, atb, kmt
__device__ __forceinline__ int bws(int hj, int hi) { return hj * SW + hi + 3; }           // ws (rows from y0-1)
__device__ __forceinline__ int b32(int hj, int hi) { return (hj + 1) * SW + hi + 3; }     // wkd, wkb (rows from y0-2)

// Issue the boxes of level L of both tracers into a slot (one thread).
__device__ __forceinline__ void issue_mx(MxSlot& sl, uint64_t* bar, const TracerMaps& m, int cur, int km, int L,
                                         int x0, int y0) {
  mbar_expect_tx(bar, kMxLevelBytes);
  tma_load_3d(sl.at[0], &m.at[cur], x0 - 2, y0 - 2, L, bar);
  tma_load_3d(sl.at[1], &m.at[cur], x0 - 2, y0 - 2, km + L, bar);
  tma_load_3d(sl.atb[0], &m.atb[cur], x0 - 2, y0 - 2, L + 1, bar);
  tma_load_3d(sl.atb[1], &m.atb[cur], x0 - 2, y0 - 2, (km + 1) + L + 1, bar);
  tma_load_3d(sl.ws, &m.ws, x0 - 4, y0 - 1, L, bar);
  tma_load_3d(sl.wkd, &m.uw, x0 - 4, y0 - 2, L, bar);
  tma_load_3d(sl.wkb, &m.vs, x0 - 4, y0 - 2, L, bar);
  tma_load_3d(sl.akt[0], &m.akt, x0, y0, L, bar);
  tma_load_3d(sl.akt[1], &m.akt, x0, y0, km + L, bar);
}

// The same level by per-thread asynchronous copies, for grids whose row
// pitch TMA cannot take (not a multiple of 16 bytes): every thread copies
// its share of the boxes' elements (zeros outside the domain, as TMA fills)
// and the slot's mbarrier counts one arrival per thread once its copies have
// landed.  The slot layout and the waits are the TMA path's.
constexpr int kF64Elems = 4 * (MY + 4) * SW64;
constexpr int kWsElems = (MY + 2) * SW, kWkElems = (MY + 3) * SW, kAktElems = TX * MY;
constexpr int kF32Elems = kWsElems + 2 * kWkElems + 2 * kAktElems;
__device__ __forceinline__ void copy_level_mx(MxSlot& sl, uint64_t* bar, const Arena& a, int km, int L, int x0,
                                              int y0) {
  const int imt = a.imt, jmt = a.jmt;
  const long A = a.A, F = a.F, FB = a.FB;
  for (int e = threadIdx.x; e < kF64Elems; e += MTH) {
    constexpr int BOX = (MY + 4) * SW64;
    const int b = e / BOX, r = e % BOX;
    const int gj = y0 - 2 + r / SW64, gi = x0 - 2 + r % SW64;
    const bool in = gj >= 0 && gj < jmt && gi >= 0 && gi < imt;
    const int n = b & 1;
    const double* src = (b < 2) ? a.at[a.cur] + n * F + (long)L * A : a.atb[a.cur] + n * FB + (long)(L + 1) * A;
    double* dst = (b < 2) ? sl.at[n] : sl.atb[n];
    cp_async8z(dst + r, src + (in ? (long)gj * imt + gi : 0), in);
  }
  for (int e = threadIdx.x; e < kF32Elems; e += MTH) {
    const float* base;
    float* dst;
    int r, w, gj0, gi0;
    if (e < kWsElems) {
      r = e; w = SW; gj0 = y0 - 1; gi0 = x0 - 4; base = a.ws32 + (long)L * A; dst = sl.ws;
    } else if (e < kWsElems + 2 * kWkElems) {
      const int q = e - kWsElems, b = q / kWkElems;
      r = q % kWkElems; w = SW; gj0 = y0 - 2; gi0 = x0 - 4;
      base = (b == 0 ? a.wkd32 : a.wkb32) + (long)L * A;
      dst = b == 0 ? sl.wkd : sl.wkb;
    } else {
      const int q = e - kWsElems - 2 * kWkElems, n = q / kAktElems;
      r = q % kAktElems; w = TX; gj0 = y0; gi0 = x0;
      base = a.akt32 + n * F + (long)L * A;
      dst = sl.akt[n];
    }
    const int gj = gj0 + r / w, gi = gi0 + r % w;
    const bool in = gj >= 0 && gj < jmt && gi >= 0 && gi < imt;
    cp_async4z(dst + r, base + (in ? (long)gj * imt + gi : 0), in);
  }
  cp_async_mbar_arrive(bar);
}

// ---- f32 faces of the 1-halo region (the predictor's level)
// A face is described by (kind, index, box index of its east / north cell
// in the f64 boxes, index of its first U point in the f32 boxes).
struct FaceRef {
  int f, r, w;
  bool x;
};

__device__ __forceinline__ FaceRef face_x_ref(int fj, int fi) {
  // west side of cell (fj, fi): cells (fj, fi-1) | (fj, fi); U points (fj-1, fi), (fj, fi) of rows y0-2+..
  return {fx(fj, fi), b64(fj, fi), b32(fj - 1, fi), true};
}
__device__ __forceinline__ FaceRef face_y_ref(int fj, int fi) {
  // south side of region row fj-1: cells (fj-1, fi) (north) | (fj, fi) (south); U points (fj-1, fi), (fj-1, fi+1)
  return {fy(fj, fi), b64(fj - 1, fi), b32(fj - 1, fi), false};
}

// Difference a(east) - a(west) for x faces and a(south) - a(north) for y
// faces (the face's cell of higher index minus the other, j running south)
// masked to 0 where either cell is land at level kk: the transport through
// such a face is 0, and a 0 difference stands for the excluded neighbour in
// the masked extrema.
__device__ __forceinline__ void face_f32(MxSmem& S, const MxSlot& L, int kk, const FaceRef& q, int k1 = -1,
                                         int k2 = -1) {
  int r1, r2;    // the two cells: r1 the one whose value is subtracted
  float u;
  if (q.x) {
    r1 = q.r - 1; r2 = q.r;
    u = face32(L.wkd[q.w], L.wkd[q.w + SW], S.hw[q.f]);
  } else {
    r1 = q.r; r2 = q.r + SW64;
    u = face32(L.wkb[q.w], L.wkb[q.w + 1], S.hw[q.f]);
  }
  const bool wet = kk < (k1 >= 0 ? k1 : (int)S.kmt[r1]) && kk < (k2 >= 0 ? k2 : (int)S.kmt[r2]);
  float2 d;
  d.x = wet ? (float)(L.at[0][r2] - L.at[0][r1]) : 0.f;
  d.y = wet ? (float)(L.at[1][r2] - L.at[1][r1]) : 0.f;
  const float lw = u * u * S.cf[q.f];
  S.fdq[q.f] = make_float4(d.x, d.y, u + lw, u - lw);
}

// border faces of the region beyond each thread's own west x face and north
// y face (the faces of cell (ty+1, tx+1)): x faces of region rows 0 and MY+1
// (all TX+3 columns), x faces of rows 1..MY at columns 0, TX+1, TX+2, y faces
// of rows 0, MY+1, MY+2 (all TX+2 columns), y faces of rows 1..MY at columns
// 0 and TX+1
constexpr int F_EXTRA = FN - 2 * TX * MY;

__device__ __forceinline__ FaceRef border_face(int q) {
  if (q < 2 * (TX + 3)) return face_x_ref(q < TX + 3 ? 0 : MY + 1, q % (TX + 3));
  q -= 2 * (TX + 3);
  if (q < 3 * MY) {
    const int c = q % 3;
    return face_x_ref(1 + q / 3, c == 0 ? 0 : TX + c);
  }
  q -= 3 * MY;
  if (q < 3 * (TX + 2)) {
    const int row = q / (TX + 2);
    return face_y_ref(row == 0 ? 0 : MY + row, q % (TX + 2));
  }
  q -= 3 * (TX + 2);
  return face_y_ref(1 + q / 2, (q % 2) ? TX + 1 : 0);
}

// ---- f64 faces of the tile (the column phase's level), as the continuity
// march formed them: uw(j,i) = (wkd(j-1,i) + wkd(j,i)) * htw(j,i) / 4,
// vs(j,i) = (wkb(j,i) + wkb(j,i+1)) * hts(j,i) / 4 (face_x64, face_y64)
struct OwnFace {
  int o;       // index in ou/oq
  int w;       // first U point in the f32 boxes
  int f;       // the same face in the region arrays (for cf)
  bool x;
  double h;    // htw or hts of the face
};

// o index of the tile's x face west of column tx in row ty, and of the y
// face north of row ty at column tx
__device__ __forceinline__ int ox(int ty, int tx) { return ty * (TX + 1) + tx; }
__device__ __forceinline__ int oy(int ty, int tx) { return OXN + ty * TX + tx; }

__device__ __forceinline__ void face_f64(MxSmem& S, const MxSlot& L, const OwnFace& q) {
  double u;
  if (q.x) u = face_x64(L.wkd[q.w], L.wkd[q.w + SW], q.h);
  else u = face_y64(L.wkb[q.w], L.wkb[q.w + 1], q.h);
  S.ou[q.o] = u;
  S.oq[q.o] = u * u * (double)S.cf[q.f];
}

// A cell of the 1-halo region as one thread handles it: its index m in the
// region, box indices (f64 boxes r, ws box u), its west x face and north y
// face; valid: inside the rows and columns the reference computes
// (1 .. imt-2, 1 .. jmt-2).  Every thread owns the interior cell above its
// column; the ring cells of the region go to the last RING threads, one each.
struct HCell {
  int m, r, u, fw, fn;
  bool valid;
};
constexpr int RING = MHN - TX * MY;
static_assert(RING <= MTH, "ring cells: at most one per thread");

__device__ __forceinline__ HCell hcell(int hj, int hi, int x0, int y0, int imt, int jmt) {
  HCell c;
  c.m = hj * HQX + hi;
  c.r = b64(hj, hi);
  c.u = bws(hj, hi);
  c.fw = fx(hj, hi);
  c.fn = fy(hj, hi);
  const int gj = y0 - 1 + hj, gi = x0 - 1 + hi;
  c.valid = gi >= 1 && gi < imt - 1 && gj >= 1 && gj < jmt - 1;
  return c;
}

__device__ __forceinline__ HCell ring_hcell(int q, int x0, int y0, int imt, int jmt) {
  int hj, hi;
  if (q < HQX) { hj = 0; hi = q; }
  else if (q < 2 * HQX) { hj = MHQY - 1; hi = q - HQX; }
  else if (q < 2 * HQX + MY) { hj = q - 2 * HQX + 1; hi = 0; }
  else { hj = q - 2 * HQX - MY + 1; hi = HQX - 1; }
  return hcell(hj, hi, x0, y0, imt, jmt);
}

__device__ __forceinline__ float fmax3f(float a, float b, float c) {
  float r;
  asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
}
__device__ __forceinline__ float fmin3f(float a, float b, float c) {
  float r;
  asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
}
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }

// Predictor of level kk for one cell, both tracers: bit n set where tracer
// n's predictor leaves its local bounds (the reference's a00 > amax or
// a00 < amin).  sc, su, sd: the slots of levels kk, kk-1, kk+1 (at the top
// and bottom level the missing neighbour level is replaced by kk itself,
// whose differences are then 0, and so are the vertical terms they carry).
__device__ __forceinline__ unsigned pred_cell(const MxSmem& S, const HCell& h, int kk, int km, int sc, int su,
                                              int sd, const MxLevel& lv, float dts, int kself = -1) {
  const int r = h.r;
  const int kr = kself >= 0 ? kself : (int)S.kmt[r];
  // land cells need no flag: every face of a land cell carries no transport
  if (!h.valid || kk >= kr) return 0u;
  const int fe = h.fw + 1, fw = h.fw, fs = h.fn + HQX, fn = h.fn;
  const float4 qe = S.fdq[fe], qw = S.fdq[fw], qs = S.fdq[fs], qn = S.fdq[fn];
  const float2 de = make_float2(qe.x, qe.y), dw = make_float2(qw.x, qw.y);
  const float2 ds = make_float2(qs.x, qs.y), dn = make_float2(qn.x, qn.y);
  // east face: this cell is the lower one, d*(u - q); west face: upper, d*(u + q)
  const float2 sx = __ffma2_rn(dw, f2(qw.z), __fmul2_rn(de, f2(qe.w)));
  const float2 sy = __ffma2_rn(dn, f2(qn.z), __fmul2_rn(ds, f2(qs.w)));
  // vertical faces: above (kk-1|kk) with w(kk), below (kk|kk+1) with w(kk+1)
  const MxSlot& C = S.slot[sc];
  const MxSlot& U = S.slot[kk > 0 ? su : sc];
  const MxSlot& D = S.slot[kk < km - 1 ? sd : sc];
  const double cT = C.at[0][r], cS = C.at[1][r];
  const float2 dup = make_float2((float)(U.at[0][r] - cT), (float)(U.at[1][r] - cS));   // a_above - c
  const float2 dlo = make_float2((float)(cT - D.at[0][r]), (float)(cS - D.at[1][r]));   // c - a_below
  const float wc = C.ws[h.u], wd = D.ws[h.u];
  const float cu = wc - wc * wc * (float)lv.odzt * dts;
  const float cd = wd + wd * wd * lv.odzt1 * dts;
  const float2 sz = __ffma2_rn(dup, f2(cu), __fmul2_rn(dlo, f2(cd)));
  // inc = -(tr*(sx+sy) + hodz*sz)*dts
  const float2 inc = __fmul2_rn(__ffma2_rn(f2(lv.hodz), sz, __fmul2_rn(f2(S.tr[h.m]), __fadd2_rn(sx, sy))),
                                f2(-dts));
  // Bound test of the predictor c + inc against the masked 7-point extrema,
  // on differences from c: c + inc > max_p a_p  <=>  inc > max_p (a_p - c).
  // Land neighbours enter as 0 (the cell itself): horizontally through the
  // masked face differences, below through the test here; the level above a
  // wet cell is wet.  The flags of land cells are never used: every face of
  // a land cell carries no transport.
  const bool below_wet = kk + 1 < kr;
  const float lx = below_wet ? -dlo.x : 0.f, ly = below_wet ? -dlo.y : 0.f;
  const float mxT = fmax3f(fmax3f(0.f, de.x, -dw.x), fmax3f(ds.x, -dn.x, dup.x), lx);
  const float mnT = fmin3f(fmin3f(0.f, de.x, -dw.x), fmin3f(ds.x, -dn.x, dup.x), lx);
  const float mxS = fmax3f(fmax3f(0.f, de.y, -dw.y), fmax3f(ds.y, -dn.y, dup.y), ly);
  const float mnS = fmin3f(fmin3f(0.f, de.y, -dw.y), fmin3f(ds.y, -dn.y, dup.y), ly);
  return ((inc.x > mxT || inc.x < mnT) ? 1u : 0u) | ((inc.y > mxS || inc.y < mnS) ? 2u : 0u);
}

// First Laplacian of atb at level kk for one cell, both tracers (f64 on the
// state differences), masked: land neighbours drop out, a land cell is 0.
struct Kmt5 {
  int c, n, s, e, w;
};
__device__ __forceinline__ void d2_cell(MxSmem& S, const MxSlot& L, int kk, const HCell& h,
                                        const Kmt5* kq = nullptr) {
  double vT = 0.0, vS = 0.0;
  const int r = h.r, m = h.m;
  if (h.valid && kk < (kq ? kq->c : (int)S.kmt[r])) {
    const double cT = L.atb[0][r], cS = L.atb[1][r];
    auto term = [&](int rn, float coef, int kn) {
      if (kk < (kq ? kn : (int)S.kmt[rn])) {
        const double c = (double)coef;
        vT = fma(c, L.atb[0][rn] - cT, vT);
        vS = fma(c, L.atb[1][rn] - cS, vS);
      }
    };
    term(r - SW64, S.dtn[m], kq ? kq->n : 0);
    term(r + SW64, S.dts[m], kq ? kq->s : 0);
    term(r + 1, S.dte[m], kq ? kq->e : 0);
    term(r - 1, S.dtw[m], kq ? kq->w : 0);
    const double ah = (double)S.ahf[m];
    vT *= ah;
    vS *= ah;
  }
  S.d2[0][m] = vT;
  S.d2[1][m] = vS;
}

// Per-tile 2-D data of the march: kmt with a 2-cell halo (stage_kmt), the
// metric and biharmonic terms of the 1-halo region and the face factors
// (stage_tile).  kLoadsAhead:
// fixed trip counts and read-only loads, so a thread's loads of a loop are in
// flight together (the batched kernel, whose short work items change member
// often, stages its tiles this way).
template <bool kLoadsAhead>
__device__ __forceinline__ void stage_kmt(MxSmem& S, const Arena& a, int x0, int y0) {
  const int tid = threadIdx.x;
  const int imt = a.imt, jmt = a.jmt;
#pragma unroll
  for (int it = 0; it < ((MY + 4) * SW64 + MTH - 1) / MTH; ++it) {
    const int m = tid + it * MTH;
    if (m < (MY + 4) * SW64) {
      const int gj = y0 - 2 + m / SW64, gi = x0 - 2 + m % SW64;
      const bool in = gj >= 0 && gj < jmt && gi >= 0 && gi < imt;
      S.kmt[m] = in ? (uint16_t)(kLoadsAhead ? __ldg(a.kmt + (long)gj * imt + gi) : a.kmt[(long)gj * imt + gi]) : 0;
    }
  }
}

template <bool kLoadsAhead>
__device__ __forceinline__ void stage_tile(MxSmem& S, const Arena& a, int x0, int y0, double dts) {
  const int tid = threadIdx.x;
  const int imt = a.imt, jmt = a.jmt;
  auto ld = [&](const double* p) { return kLoadsAhead ? __ldg(p) : *p; };
#pragma unroll
  for (int it = 0; it < (MHN + MTH - 1) / MTH; ++it) {
    const int m = tid + it * MTH;
    if (m < MHN) {
      const int gj = y0 - 1 + m / HQX, gi = x0 - 1 + m % HQX;
      const bool in = gj >= 0 && gj < jmt && gi >= 0 && gi < imt;
      const long q = in ? (long)gj * imt + gi : 0;
      S.tr[m] = in ? (float)ld(a.tarea_r + q) : 0.f;
      S.dtn[m] = in ? (float)ld(a.dtn + q) : 0.f;
      S.dts[m] = in ? (float)ld(a.dts + q) : 0.f;
      S.dte[m] = in ? (float)ld(a.dte + q) : 0.f;
      S.dtw[m] = in ? (float)ld(a.dtw + q) : 0.f;
      S.ahf[m] = in ? (float)ld(a.ahf + q) : 0.f;
    }
  }
#pragma unroll
  for (int it = 0; it < (FN + MTH - 1) / MTH; ++it) {
    const int m = tid + it * MTH;
    if (m < FN) {
      int gj, gi;
      if (m < FXN) { gj = y0 - 1 + m / (TX + 3); gi = x0 - 1 + m % (TX + 3); }
      else { gj = y0 - 2 + (m - FXN) / (TX + 2); gi = x0 - 1 + (m - FXN) % (TX + 2); }
      const bool in = gj >= 0 && gj < jmt && gi >= 0 && gi < imt;
      const long q = in ? (long)gj * imt + gi : 0;
      const double h = in ? ((m < FXN) ? ld(a.htw + q) : ld(a.hts + q)) : 1.0;
      const double hu = in ? ((m < FXN) ? ld(a.hun + q) : ld(a.hue + q)) : 1.0;
      S.cf[m] = in ? (float)(2.0 * dts / (h * hu)) : 0.f;
      S.hw[m] = in ? (float)h : 0.f;
    }
  }
}

// The km level constants, once per CTA.
__device__ __forceinline__ void stage_levels(MxLevel* lv, const Arena& a) {
  const int km = a.km;
  const double dts = a.p.dts;
  for (int k = threadIdx.x; k < km; k += MTH) {
    MxLevel L;
    L.odzp = a.odzp[k];
    L.odzt = a.odzt[k];
    L.ka = a.odzt[k] * a.odzp[k] * dts * 0.5;
    L.kc = k < km - 1 ? a.odzt[k + 1] * a.odzp[k] * dts * 0.5 : 0.0;
    L.pu = k >= 1 ? a.pen[k - 1] : 0.0;
    L.pd = k < km - 1 ? a.pen[k] : 0.0;
    L.hodz = 0.5f * (float)a.odzp[k];
    L.odzt1 = k < km - 1 ? (float)a.odzt[k + 1] : 0.f;
    lv[k] = L;
  }
}

// Column-phase state of one tracer carried up the levels.
struct ColState {
  double e, f;      // the sweep's elimination coefficients of the level below
  double carry;     // vertical face below as seen from above: A + X
  double wbelow;    // explicit diffusion flux through the face below
  double stf;       // surface flux
};

// the thread that issues the level boxes (in a warp with a single border face)
constexpr int kIssueThread = 4 * TX;

// One work item (a tile, both tracers) of the mixed column march.  Returns
// false if a level wait gave up: the CTA has then recorded the timeout and
// drained its boxes, and must return.
template <bool kLoadsAhead>
__device__ __forceinline__ bool mixed_item(bool tma, MxSmem& S, const MxLevel* __restrict__ lvs, const Arena& a,
                                           const TracerMaps& maps, double* scr, int ntx, long tile, uint32_t& par,
                                           uint32_t& outstanding) {
  const int tid = threadIdx.x, tx = tid % TX, ty = tid / TX;
  const int imt = a.imt, jmt = a.jmt, km = a.km;
  const long A = a.A, F = a.F, FB = a.FB;
  const lt_params& p = a.p;
  const double dts = p.dts;
  const float dtsf = (float)dts;
  const int x0 = (int)(tile % ntx) * TX, y0 = (int)(tile / ntx) * MY;
  const int i = x0 + tx, j = y0 + ty;

  __syncthreads();   // the previous item no longer reads the slots or the tile data
  // level L goes to slot s = L % NSM
  // every thread arrives on the slot's barrier once per level: by TMA (the
  // issuing thread with the level's byte count) or after its own copies
  auto issue = [&](int L, int s) {
    if (tma) {
      if (tid == kIssueThread) issue_mx(S.slot[s], &S.bar[s], maps, a.cur, km, L, x0, y0);
      else mbar_arrive(&S.bar[s]);
    } else {
      copy_level_mx(S.slot[s], &S.bar[s], a, km, L, x0, y0);
    }
    outstanding |= 1u << s;
  };
  auto wait = [&](int s) -> bool {
    const bool ok = mbar_wait(&S.bar[s], (par >> s) & 1u, a.wait_limit);
    if (ok) { par ^= 1u << s; outstanding &= ~(1u << s); }
    return ok;
  };
  const bool own = i < imt && j < jmt;
  const bool inner = own && i >= 2 && i < imt - 2 && j >= 2 && j < jmt - 2;
  const long qo = own ? (long)j * imt + i : 0;
  const int hc = (ty + 1) * HQX + (tx + 1);
  const int rc = b64(ty + 1, tx + 1), uc = bws(ty + 1, tx + 1);
  const HCell own_cell = hcell(ty + 1, tx + 1, x0, y0, imt, jmt);
  const bool has_ring = tid >= MTH - RING;
  const HCell ring_cell = ring_hcell(has_ring ? tid - (MTH - RING) : 0, x0, y0, imt, jmt);
  // Levels at and below the deepest bottom of the tile's own columns are land
  // for every cell the march updates there: the step leaves them as they
  // are.  The march starts at the first of them (or the bottom level), and
  // the inner cells' values below it are copied.  (A wetter halo cell's flag
  // at that level, formed without the level below, meets the tile's cells
  // only through faces and a w that carry no transport there.)
  stage_kmt<kLoadsAhead>(S, a, x0, y0);
  __syncthreads();
  const Kmt5 kq = {S.kmt[rc], S.kmt[rc - SW64], S.kmt[rc + SW64], S.kmt[rc + 1], S.kmt[rc - 1]};
  int kmax = kq.c;
  kmax = __reduce_max_sync(0xffffffffu, kmax);
  if (tx == 0) S.wmax[ty] = kmax;
  __syncthreads();
#pragma unroll
  for (int w = 0; w < MTH / 32; ++w) kmax = max(kmax, S.wmax[w]);
  const int ks = min(km - 1, kmax);   // the march's first (deepest) level
  for (int L = ks; L >= (ks - NSM + 1 > 0 ? ks - NSM + 1 : 0); --L) issue(L, L % NSM);
  stage_tile<kLoadsAhead>(S, a, x0, y0, dts);
  if (inner) {
    // eight levels' loads in flight ahead of their stores
    const double* __restrict__ at_in = a.at[a.cur];
    double* __restrict__ at_out = a.at[a.cur ^ 1];
    double* __restrict__ atb_out = a.atb[a.cur ^ 1];
    for (int k0 = ks + 1; k0 < km; k0 += 8) {
      double v[8][2];
#pragma unroll
      for (int c = 0; c < 8; ++c)
#pragma unroll
        for (int n = 0; n < 2; ++n) v[c][n] = k0 + c < km ? at_in[n * F + (long)(k0 + c) * A + qo] : 0.0;
#pragma unroll
      for (int c = 0; c < 8; ++c)
        if (k0 + c < km)
#pragma unroll
          for (int n = 0; n < 2; ++n) {
            __stcs(at_out + n * F + (long)(k0 + c) * A + qo, v[c][n]);
            __stcs(atb_out + n * FB + (long)(k0 + c + 1) * A + qo, v[c][n]);
          }
    }
  }

  const int kz = own ? a.kmt[qo] : 0;
  // The region's extra cells and faces are spread so that no warp carries
  // much more than the others between two barriers: the ring cells (first
  // Laplacian and predictor) go to the last warps, the border faces to the
  // first ones (two per thread where needed), the TMA issue to a thread of a
  // warp with a single border face.
  // f32 faces: the own cell's west x face and north y face, and one border face
  const FaceRef fo_x = face_x_ref(ty + 1, tx + 1), fo_y = face_y_ref(ty + 1, tx + 1);
  constexpr int kFaceThreads = MTH - RING - (MTH - RING) % TX;   // the warps without ring cells
  static_assert(F_EXTRA <= 2 * kFaceThreads, "border faces: at most two per thread");
  const bool has_fb = tid < kFaceThreads && tid < F_EXTRA;
  const bool has_fb2 = tid < F_EXTRA - kFaceThreads;
  const FaceRef fo_b = border_face(has_fb ? tid : 0);
  const FaceRef fo_b2 = border_face(has_fb2 ? tid + kFaceThreads : 0);
  // f64 faces of the tile: the own cell's west and north faces, and the east
  // column's x faces and the bottom row's y faces (threads kOwnB .. kOwnB+MY-1
  // and kOwnB+MY .. kOwnB+MY+TX-1, in warps with a single border face)
  auto hval = [&](const double* h, int gj, int gi) {
    return (gj >= 0 && gj < jmt && gi >= 0 && gi < imt) ? h[(long)gj * imt + gi] : 0.0;
  };
  const OwnFace of_x = {ox(ty, tx), b32(ty, tx + 1), fx(ty + 1, tx + 1), true, hval(a.htw, j, i)};
  const OwnFace of_y = {oy(ty, tx), b32(ty, tx + 1), fy(ty + 1, tx + 1), false, hval(a.hts, j - 1, i)};
  constexpr int kOwnB = 2 * TX;
  static_assert(F_EXTRA - kFaceThreads <= kOwnB && kOwnB + MY + TX <= kFaceThreads, "f64 border faces");
  const int tb = tid - kOwnB;
  const bool has_ob = tb >= 0 && tb < MY + TX;
  OwnFace of_b;
  if (tb >= 0 && tb < MY) of_b = {ox(tb, TX), b32(tb, TX + 1), fx(tb + 1, TX + 1), true, hval(a.htw, y0 + tb, x0 + TX)};
  else if (has_ob) of_b = {oy(MY, tb - MY), b32(MY, tb - MY + 1), fy(MY + 1, tb - MY + 1), false,
                           hval(a.hts, y0 + MY - 1, x0 + tb - MY)};
  else of_b = of_x;
  const int oe = ox(ty, tx + 1), ow = ox(ty, tx), os = oy(ty + 1, tx), on = oy(ty, tx);
  // second Laplacian face weights K = tarea*dte (x faces), tarea*dts (y faces)
  // of the own cell's four faces, f64: the same expression in both cells of a face
  auto kxw = [&](int gj, int gi) {
    return (gj >= 0 && gj < jmt && gi >= 0 && gi < imt) ? a.tarea[(long)gj * imt + gi] * a.dte[(long)gj * imt + gi]
                                                      : 0.0;
  };
  auto kys = [&](int gj, int gi) {
    return (gj >= 0 && gj < jmt && gi >= 0 && gi < imt) ? a.tarea[(long)gj * imt + gi] * a.dts[(long)gj * imt + gi]
                                                      : 0.0;
  };
  const double kxE = inner ? kxw(j, i) : 0.0, kxW = inner ? kxw(j, i - 1) : 0.0;
  const double kyS = inner ? kys(j, i) : 0.0, kyN = inner ? kys(j - 1, i) : 0.0;
  const double swv = (inner) ? a.swv[qo] : 0.0;
  const double err_norm2 = a.scalars[0];
  const double ah64 = p.ah;
  const double trc = inner ? a.tarea_r[qo] : 0.0;
  ColState cs[2];
  cs[0] = {0.0, 0.0, 0.0, 0.0, own ? a.stf_n[qo] : 0.0};
  cs[1] = {0.0, 0.0, 0.0, 0.0, own ? a.stf_n[A + qo] : 0.0};

  // slots of levels k, k-1, k+1 (NSM == 3: level k-2 shares k+1's)
  static_assert(NSM == 3, "slot rotation below assumes three slots");
  // (below ks the slot of level ks+1 holds nothing of this tile: the
  // predictor of level ks, a land level everywhere, does not read it)
  int sk = ks % NSM;
  int sm1 = sk == 0 ? 2 : sk - 1, sp1 = sk == 2 ? 0 : sk + 1;
  {
    // every level the prologue issued is waited before any of them is used
    // (as in the FP64 kernel)
    const bool ok = wait(sk) && (ks == 0 || wait(sm1)) && (ks < 2 || wait(sp1));
    if (__syncthreads_or(!ok)) { tma_bail(S, a, par, outstanding); return false; }
  }
  {
    const MxSlot& L = S.slot[sk];
    face_f32(S, L, ks, fo_x, kq.w, kq.c);
    face_f32(S, L, ks, fo_y, kq.n, kq.c);
    if (has_fb) face_f32(S, L, ks, fo_b);
    if (has_fb2) face_f32(S, L, ks, fo_b2);
  }
  __syncthreads();
  {
    const MxLevel lv = lvs[ks];
    S.flag[sk][own_cell.m] = (unsigned char)pred_cell(S, own_cell, ks, km, sk, sm1, sp1, lv, dtsf, kq.c);
    if (has_ring) S.flag[sk][ring_cell.m] = (unsigned char)pred_cell(S, ring_cell, ks, km, sk, sm1, sp1, lv, dtsf);
  }
  // The first step's phase B1 overwrites the face arrays these predictors
  // read (its faces are of level ks-1).  Without this barrier a warp that
  // finished its predictors early changed a neighbouring cell's faces while
  // that cell's predictor still read them: the limiter flags of level ks came
  // out different from run to run in tiles whose level ks is wet (a column
  // reaching the bottom level), at the tile's edge columns.
  __syncthreads();

  // Level slots: after step k the slot of level k takes level k-NSM.
  for (int k = ks; k >= 0; --k) {
    // ---- phase B1: f32 faces one level up (the predictor's), the tile's f64
    // faces and the first Laplacian here (levels k-1, k arrived in earlier
    // steps; the previous step ended with a barrier)
    const MxSlot& Lk = S.slot[sk];
    if (k >= 1) {
      const MxSlot& Lu = S.slot[sm1];
      face_f32(S, Lu, k - 1, fo_x, kq.w, kq.c);
      face_f32(S, Lu, k - 1, fo_y, kq.n, kq.c);
      if (has_fb) face_f32(S, Lu, k - 1, fo_b);
      if (has_fb2) face_f32(S, Lu, k - 1, fo_b2);
    }
    face_f64(S, Lk, of_x);
    face_f64(S, Lk, of_y);
    if (has_ob) face_f64(S, Lk, of_b);
    d2_cell(S, Lk, k, own_cell, &kq);
    if (has_ring) d2_cell(S, Lk, k, ring_cell);
    const bool ok = (k >= 2 && k != ks) ? wait(sp1) : true;   // level k-2 (the prologue waited ks-2)
    if (__syncthreads_or(!ok)) { tma_bail(S, a, par, outstanding); return false; }
    // ---- phase B2: predictor one level up.  The column phase below reads
    // the flags of level k (written in the previous step) and, of level k-1,
    // only its own cell's, which this thread computes: no barrier between
    // the two phases.
    unsigned flag_up = 0;
    if (k >= 1) {
      const MxLevel lv = lvs[k - 1];
      flag_up = pred_cell(S, own_cell, k - 1, km, sm1, sp1, sk, lv, dtsf, kq.c);
      S.flag[sm1][own_cell.m] = (unsigned char)flag_up;
      if (has_ring) S.flag[sm1][ring_cell.m] = (unsigned char)pred_cell(S, ring_cell, k - 1, km, sm1, sp1, sk, lv, dtsf);
    }
    // ---- phase C: own column at level k, both tracers.  Below the column's
    // bottom every term of the step is masked (vit = 0): the new value is the
    // old one and no face flux leaves the level.
    if (inner && k >= kz) {
#pragma unroll
      for (int n = 0; n < 2; ++n) {
        const double c = Lk.at[n][rc];
        __stcs(a.at[a.cur ^ 1] + n * F + (long)k * A + qo, c);
        __stcs(a.atb[a.cur ^ 1] + n * FB + (long)(k + 1) * A + qo, c);
        cs[n].carry = 0.0;
        cs[n].wbelow = 0.0;
      }
    } else if (inner) {
      const MxLevel lv = lvs[k];
      const unsigned char* fl = S.flag[sk];
      const unsigned fself = fl[hc];
      const unsigned fE = fself | fl[hc + 1], fW = fself | fl[hc - 1];
      const unsigned fS = fself | fl[hc + HQX], fN = fself | fl[hc - HQX];
      const unsigned fV = fself | flag_up;
      const double uE = S.ou[oe], uW = S.ou[ow], vS = S.ou[os], vN = S.ou[on];
      const double qE = S.oq[oe], qW = S.oq[ow], qS = S.oq[os], qN = S.oq[on];
      const double wv = (double)Lk.ws[uc];
      const double wq = wv * wv * lv.odzt * dts;       // vertical Lax-Wendroff factor
      const double vit_kp1 = (k + 1 < kz) ? 1.0 : 0.0;
      // masks of the second Laplacian's faces (hmix_del4.F90:626-757)
      const bool mself = k <= kq.c - 1;
      const bool mE = mself && k <= kq.e - 1, mW = mself && k <= kq.w - 1;
      const bool mS = mself && k <= kq.s - 1, mN = mself && k <= kq.n - 1;
      const MxSlot& Lu = S.slot[k > 0 ? sm1 : sk];
#pragma unroll
      for (int n = 0; n < 2; ++n) {
        ColState& st = cs[n];
        const unsigned bit = 1u << n;
        const double* at = Lk.at[n];
        // Content bookkeeping.  Both cells of a face receive its centred
        // part A = d*u with the same sign (the advective form), and the
        // upwind / Lax-Wendroff part X = c*d with opposite signs: every face
        // term is one f64 value formed from the same operands in both cells,
        // weighted by tarea_r (horizontal) and odzp (vertical) in f64, so a
        // flux leaves one cell and enters the next with weights that cancel
        // against the cell volumes to f64 rounding.
        const double c = at[rc];
        const double dE = at[rc + 1] - c, dW = c - at[rc - 1];
        const double dS = at[rc + SW64] - c, dN = c - at[rc - SW64];
        const double Xe = ((fE & bit) ? fabs(uE) : qE) * dE;
        const double Xw = ((fW & bit) ? fabs(uW) : qW) * dW;
        const double Xs = ((fS & bit) ? fabs(vS) : qS) * dS;
        const double Xn = ((fN & bit) ? fabs(vN) : qN) * dN;
        double sh = dE * uE + dW * uW + dS * vS + dN * vN;
        sh += (Xw - Xe) + (Xn - Xs);
        // vertical: face above (k-1|k) computed here, face below carried (at
        // the top level the level itself stands in for the missing one above:
        // the difference and both face terms are 0)
        const double dv = Lu.at[n][rc] - c;
        const double Xv = ((fV & bit) ? fabs(wv) : wq) * dv;
        const double Av = wv * dv;
        const double sz = st.carry + (Av - Xv);
        st.carry = Av + Xv;
        const double vadv = -0.5 * sz;                 // vertical advection, times odzp
        // second Laplacian as face fluxes K*(d2_R - d2_L)
        double hd = 0.0;
        {
          const double* d2 = S.d2[n];
          const double dc = d2[hc];
          if (mE) hd += kxE * (d2[hc + 1] - dc);
          if (mW) hd -= kxW * (dc - d2[hc - 1]);
          if (mS) hd += kyS * (d2[hc + HQX] - dc);
          if (mN) hd -= kyN * (dc - d2[hc - HQX]);
        }
        // shortwave through the faces above and below (tracer.cpp:1430-1474)
        // and the explicit half of the vertical diffusion: each face flux is
        // one f64 expression in the cells above and below it
        double vz = 0.0;
        if (n == 0) vz = swv * lv.pu - swv * lv.pd * vit_kp1;
        const double atb_k = Lk.atb[n][rc];
        const double wkc_km1 = k >= 1 ? (double)S.slot[sm1].akt[n][tid] : 0.0;
        const double w1 = k >= 1 ? wkc_km1 * (S.slot[sm1].atb[n][rc] - atb_k) * lv.odzt : 0.0;
        vz += 0.5 * (w1 - st.wbelow);
        st.wbelow = w1;
        // surface flux and the freshwater-norm correction
        double sfc = 0.0;
        if (k == 0) {
          sfc = st.stf * 0.5 * lv.odzp;
          if (n == 1) sfc += err_norm2;
        }
        double tf = 0.0;
        if (p.boundary_restore == 1 && k >= 1)
          tf = (a.restore[n * F + (long)k * A + qo] - atb_k) * (1.0 / (15.0 * 86400.0));
        const double d8 = c + dts * (tf - trc * sh + lv.odzp * (vz + vadv) + sfc + ah64 * trc * hd);
        // one elimination step of the implicit half of the vertical
        // diffusion (invtrit, tracer.cpp:923-978)
        {
          const double wkc_k = (double)Lk.akt[n][tid];
          const double a8 = k >= 1 ? wkc_km1 * lv.ka : lv.odzp * dts * 0.5;
          double c8, b8;
          if (k == kz - 1) {
            c8 = lv.odzp * dts * 0.5;
            b8 = 1.0 + a8;
            st.e = 0.0;
            st.f = 0.0;
          } else {
            c8 = wkc_k * lv.kc;
            b8 = k >= 1 ? 1.0 + a8 + c8 : 1.0 + c8;
          }
          const double g0 = 1.0 / (b8 - c8 * st.e);
          st.e = a8 * g0;
          st.f = (d8 + c8 * st.f) * g0;
          st_l2(reinterpret_cast<double2*>(scr) + ((long)k * 2 + n) * MTH + tid, make_double2(st.e, st.f),
                l2_evict_last());
        }
      }
    }
    __syncthreads();
    if (k - NSM >= 0) issue(k - NSM, sk);   // level k-3 takes level k's slot
    // one level down: the slots of k-1, k-2, k
    sp1 = sk;
    sk = sm1;
    sm1 = sk == 0 ? 2 : sk - 1;
  }
  // substitution, top down through the wet levels: the elimination
  // coefficients of SUB levels are loaded together ahead of their stores (one
  // scratch round trip per SUB levels)
  if (inner) {
    double* at_out = a.at[a.cur ^ 1];
    double* atb_out = a.atb[a.cur ^ 1];
    double x[2] = {0.0, 0.0};
    constexpr int SUB = 4;
    const double2* sc2 = reinterpret_cast<const double2*>(scr);
    const uint64_t pf = l2_evict_first();
    for (int k0 = 0; k0 < kz; k0 += SUB) {
      double2 ef[SUB][2];
#pragma unroll
      for (int c = 0; c < SUB; ++c)
#pragma unroll
        for (int n = 0; n < 2; ++n)
          ef[c][n] = k0 + c < kz ? ld_l2(sc2 + ((long)(k0 + c) * 2 + n) * MTH + tid, pf) : make_double2(0.0, 0.0);
#pragma unroll
      for (int c = 0; c < SUB; ++c) {
        const int k = k0 + c;
        if (k >= kz) break;
#pragma unroll
        for (int n = 0; n < 2; ++n) {
          const double v = (k == 0) ? ef[c][n].x * cs[n].stf + ef[c][n].y : ef[c][n].x * x[n] + ef[c][n].y;
          x[n] = v;
          __stcs(at_out + n * F + (long)k * A + qo, v);
          __stcs(atb_out + n * FB + (long)(k + 1) * A + qo, v);
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
    for (int s = 0; s < NSM; ++s) mbar_init(&S.bar[s], MTH);   // one arrival per thread and level
    mbar_fence_init();
  }
  __syncthreads();
  return S;
}

__device__ __forceinline__ MxLevel* mixed_levels() {
  extern __shared__ __align__(128) unsigned char smem_mx[];
  return reinterpret_cast<MxLevel*>(smem_mx + kMxLevOff);
}

__global__ void __launch_bounds__(MTH, kMixedCtasPerSm)
    k_tracer_mixed(Arena a, const __grid_constant__ TracerMaps maps, int ntx, long ntiles, int tma) {
  MxSmem& S = mixed_smem_init();
  MxLevel* lv = mixed_levels();
  stage_levels(lv, a);
  uint32_t par = 0, outstanding = 0;
  double* scr = a.col_scratch + (long)blockIdx.x * a.km * kMixedScratchPerLevel * MTH;
  for (long w = blockIdx.x; w < ntiles; w += gridDim.x)
    if (!mixed_item<false>(tma != 0, S, lv, a, maps, scr, ntx, w, par, outstanding)) return;
}

// Several domains (ensemble members, serving requests; any sizes) in one
// persistent launch: the work list is the concatenation of every member's
// tiles, member after member, so neighbouring CTAs work on neighbouring tiles
// of the same member.  Each CTA's items ascend, so its member index only
// moves forward.
// The current member's arena is copied into shared memory behind the level
// constants: read from there, its fields cannot alias the kernel's global
// stores, so the compiler keeps them across the level loop instead of
// reloading them from global memory at every level.
__host__ __device__ constexpr size_t mx_batch_arena_off(int km) { return (mx_smem_bytes(km) + 15) / 16 * 16; }
__host__ __device__ constexpr size_t mx_batch_smem(int km) { return mx_batch_arena_off(km) + sizeof(Arena); }
static_assert(sizeof(Arena) % 16 == 0, "arena copied as 16-byte words");

__global__ void __launch_bounds__(MTH, kMixedCtasPerSm)
    k_tracer_mixed_batch(const MemberDesc* __restrict__ mem, int nmem, long total, double* scratch, int km_max) {
  MxSmem& S = mixed_smem_init();
  extern __shared__ __align__(128) unsigned char smem_mx[];
  MxLevel* lv = mixed_levels();
  Arena& sa = *reinterpret_cast<Arena*>(smem_mx + mx_batch_arena_off(km_max));
  uint32_t par = 0, outstanding = 0;
  double* scr = scratch + (long)blockIdx.x * km_max * kMixedScratchPerLevel * MTH;
  int m = 0, staged = -1;
  for (long w = blockIdx.x; w < total; w += gridDim.x) {
    while (m + 1 < nmem && mem[m + 1].item0 <= w) ++m;
    const MemberDesc& d = mem[m];
    if (m != staged) {
      __syncthreads();   // the previous item no longer reads the staged arena or levels
      const uint4* src = reinterpret_cast<const uint4*>(&d.a);
      uint4* dst = reinterpret_cast<uint4*>(&sa);
      for (int t = threadIdx.x; t < (int)(sizeof(Arena) / 16); t += MTH) dst[t] = src[t];
      __syncthreads();
      stage_levels(lv, sa);
      staged = m;
    }
    if (!mixed_item<true>(d.tma != 0, S, lv, sa, d.maps, scr, d.ntx, w - d.item0, par, outstanding)) return;
  }
}

}  // namespace

int launch_tracer_tma_mixed(const Arena& a, const TracerMaps& maps, bool tma, cudaStream_t s, int grid) {
  const int ntx = (a.imt + TX - 1) / TX;
  const long ntiles = (long)ntx * ((a.jmt + MY - 1) / MY);
  const size_t sm = mx_smem_bytes(a.km);
  static int attr_dev = -1;
  int dev = 0;
  LT_CUDA_OK(cudaGetDevice(&dev));
  if (attr_dev != dev) {
    LT_CUDA_OK(cudaFuncSetAttribute(k_tracer_mixed, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)mx_smem_bytes(kMixedMaxLevels)));
    attr_dev = dev;
  }
  k_tracer_mixed<<<grid, MTH, sm, s>>>(a, maps, ntx, ntiles, tma ? 1 : 0);
  LT_LAUNCHED();
  return LT_OK;
}

int prepare_tracer_mixed_batch() {
  LT_CUDA_OK(cudaFuncSetAttribute(k_tracer_mixed_batch, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)mx_batch_smem(kMixedMaxLevels)));
  return LT_OK;
}

// prepare_tracer_mixed_batch() must have run on this device (it cannot run
// inside a stream capture)
int launch_tracer_mixed_batch(const MemberDesc* mem, int nmem, long total, double* scratch, int km_max, int grid,
                              cudaStream_t s) {
  k_tracer_mixed_batch<<<grid, MTH, mx_batch_smem(km_max), s>>>(mem, nmem, total, scratch, km_max);
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

int launch_continuity_mixed(const Arena& a, const TracerMaps& maps, bool tma, cudaStream_t s) {
  dim3 b(CBX, kContTileY), g((a.imt + CBX - 1) / CBX, (a.jmt + kContTileY - 1) / kContTileY);
  if (tma) {
    static int attr_dev = -1;
    int dev = 0;
    LT_CUDA_OK(cudaGetDevice(&dev));
    const size_t psm = sizeof(float) * CBX * kContTileY;   // partial sums per level
    if (attr_dev != dev) {
      LT_CUDA_OK(cudaFuncSetAttribute(k_cont_tma32, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)(sizeof(ContSmem) + psm * kMixedMaxLevels)));
      attr_dev = dev;
    }
    k_cont_tma32<<<g, b, sizeof(ContSmem) + psm * a.km, s>>>(a, maps);
  } else {
    k_cont_march32<<<g, b, 0, s>>>(a);
  }
  LT_LAUNCHED();
  return LT_OK;
}

}  // namespace lt
