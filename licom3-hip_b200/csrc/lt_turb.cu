// lt_turb.cu - the Canuto 2002 turbulence closure that produces the tracer
// step's vertical mixing (turb_cu with turb_device, interp1d_expabs,
// interp2d_expabs, formld and eplatidepend_fun, readyc.cpp:880-1612, with
// TIDEMIX as the reference is configured).  Compiled with -fmad=false: the
// operation order is the reference's term for term; the transcendental
// functions (log, atan, sin, cos, acosh) are CUDA's, so results agree with the
// reference to a few units in the last place, not bit for bit.
//
// One thread per column.  Where the reference first fills per-column work
// arrays (wp1, wp3, wp7, wp8 in [i][j][k] order) and then walks them, this
// kernel makes three passes down and up the column straight from the level
// fields, which a warp reads coalesced (i fastest):
//   1. upward from the deepest interface: the tidal mixing with the
//      reference's bottom-up minimum, and the tidal diagnostics;
//   2. downward: the mixed-layer depth (formld);
//   3. downward: the closure itself, level by level, keeping the few
//      neighbouring levels it looks at in registers, and the diffusivities
//      written as soon as a level is done (level 0 last: the wind-mixing floor
//      applies to it once the column is complete).
#include "lt_common.cuh"
#include "lt_domain.h"

struct lt_turb_tab {
  lt::TurbTabDev t;
  void* base = nullptr;
  int dev = 0;
};

namespace lt {
namespace {

constexpr int MT = LT_TURB_MT, MT0 = LT_TURB_MT0, NTH = LT_TURB_NTHETA;
constexpr int N1 = LT_TURB_N1;

// pconst_mod.h:242-247 and canuto_mod.h constants of the configuration
constexpr double kBackTidal = 1.0e-6, kMaxTidal = 1.0e-2, kMixingEf = 0.20, kLocalFrac = 0.33;
constexpr double kEpson2 = 0.288e0, kEplatMin = 7.0e-2, kS2min = 1.0e-14;

__device__ __forceinline__ double sgn(double x, double y) { return y >= 0.0 ? fabs(x) : -fabs(x); }
__device__ __forceinline__ int sgn_i(int x, int y) { return y >= 0 ? abs(x) : -abs(x); }

// Values the reference recomputes at every call from constants: atan(1),
// the denominator of eplatidepend_fun, the logarithms of the geometric table
// parts.  Computed once per thread with the same functions, so the bits are
// those of the per-call evaluation.
struct TurbConst {
  double pi4;               // atan(1.0)
  double eplat_den;         // wavelat(f_30, an0)
  double log_gm, log_rri;   // 2-D tables: log(rib[mt + mt0]), log(rri)
  double log_gm1, log_rnd;  // zero-shear table: log(and2on2a1[mt + mt0]), log(rnd2on2)
};

// wavelat / eplatidepend_fun (readyc.cpp:880-896)
__device__ __forceinline__ double eplat(const TurbConst& C, double f, double an) {
  const double anum = f * acosh(an / f);
  return anum / C.eplat_den;
}

// Table index of x on an "expabs" grid (linear spacing delta up to
// grid[mt + mt0], geometric ratio rat beyond), as interp1d_expabs and
// interp2d_expabs find it (readyc.cpp:922-941, 1014-1031).  Sets l0, l1.
__device__ __forceinline__ void expabs_index(double x, const double* g, double delta, double log_gm, double log_rat,
                                             int& l0, int& l1) {
  const double gm = g[MT + MT0], gmax = g[2 * MT];
  if (fabs(x) >= gm && fabs(x) >= gmax) {
    l0 = (int)sgn((double)MT, x);
    l1 = l0;
    return;
  }
  if (fabs(x) < gm) {
    l1 = (int)(x / delta) + (int)sgn(1.0, x);
  } else {
    const double ti = sgn((double)MT0 + ((log(fabs(x)) - log_gm) / log_rat), x);
    l1 = (int)ti + (int)sgn(1.0, x);
  }
  // a rounding of the logarithms could put x's index one past the table
  // end, where the reference reads beyond its array; stay inside
  l1 = max(-MT, min(MT, l1));
  if (fabs(g[MT + l1]) < fabs(x)) l1 += sgn_i(1, l1);
  else if (fabs(g[MT + l1 - sgn_i(1, l1)]) > fabs(x)) l1 += -sgn_i(1, l1);
  l0 = l1 - (int)sgn(1.0, x);
}

// interp1d_expabs (readyc.cpp:915-973): outputs left as they were when x
// falls outside the bracketing entries
__device__ void interp1d(double x, const TurbTabDev& T, const TurbConst& C, double& slq2, double& sm, double& sh,
                         double& ss) {
  const double* x1 = T.and2on2a1;
  if (x > x1[2 * MT]) x = x1[2 * MT];
  else if (x < x1[0]) x = x1[0];
  int l0, l1;
  const double gm = x1[MT + MT0], gmax = x1[2 * MT];
  if (fabs(x) >= gm && fabs(x) >= gmax) {
    l0 = (int)sgn((double)MT, x);
    l1 = l0;
  } else {
    expabs_index(x, x1, T.dand2on2, C.log_gm1, C.log_rnd, l0, l1);
    if (fabs(x) <= 0.0e0) l1 = 1;
  }
  if ((x > 0.0e0 && (x < x1[MT + l0] || x > x1[MT + l1])) || (x < 0.0e0 && (x > x1[MT + l0] || x < x1[MT + l1])))
    return;
  const double dta = x1[MT + l1] - x1[MT + l0];
  const double dx = x - x1[MT + l0];
  double d_slq2, d_sm, d_sh, d_ss;
  if (l1 == l0) {
    d_slq2 = d_sm = d_sh = d_ss = 0.0e0;
  } else {
    d_slq2 = (T.amtaun2a1[MT + l1] - T.amtaun2a1[MT + l0]) / dta;
    d_sm = (T.sma1[MT + l1] - T.sma1[MT + l0]) / dta;
    d_sh = (T.sha1[MT + l1] - T.sha1[MT + l0]) / dta;
    d_ss = (T.ssa1[MT + l1] - T.ssa1[MT + l0]) / dta;
  }
  slq2 = T.amtaun2a1[MT + l0] + d_slq2 * dx;
  sm = T.sma1[MT + l0] + d_sm * dx;
  sh = T.sha1[MT + l0] + d_sh * dx;
  ss = T.ssa1[MT + l0] + d_ss * dx;
}

// interp2d_expabs (readyc.cpp:975-1114): ri, rid clipped to the table in
// place; outputs left as they were on the reference's early returns
__device__ void interp2d(double& ri, double& rid, const TurbTabDev& T, const TurbConst& C, double& slq2, double& sm,
                         double& sh, double& ss) {
  const double* rib = T.rib;
  const double rmax = rib[2 * MT], rmin = rib[0];
  if (ri > rmax) {
    if (fabs(rid) <= ri) {
      rid = rmax * (rid / ri);
      ri = rmax;
    } else if (rid > ri) {
      ri = rmax * (ri / rid);
      rid = rmax;
    } else if (rid < -ri) {
      ri = rmin * (ri / rid);
      rid = rmin;
    }
  } else if (ri < rmin) {
    if (fabs(rid) <= -ri) {
      rid = rmin * (rid / ri);
      ri = rmin;
    } else if (rid > -ri) {
      ri = rmax * (ri / rid);
      rid = rmax;
    } else if (rid < ri) {
      ri = rmin * (ri / rid);
      rid = rmin;
    }
  } else if (rid > rmax) {
    ri = rmax * (ri / rid);
    rid = rmax;
  } else if (rid < rmin) {
    ri = rmin * (ri / rid);
    rid = rmin;
  }
  const double x_ri = ri, x_rid = rid;
  const double gm = rib[MT + MT0];
  int d0, d1, r0, r1;
  if (fabs(x_rid) >= gm && fabs(x_rid) >= rmax) {
    d0 = (int)sgn((double)MT, x_rid);
    d1 = d0;
  } else {
    expabs_index(x_rid, rib, T.dri, C.log_gm, C.log_rri, d0, d1);
    if (x_rid == 0.0e0) d1 = 1;
  }
  if ((x_rid > 0.0e0 && (x_rid < rib[MT + d0] || x_rid > rib[MT + d1])) ||
      (x_rid < 0.0e0 && (x_rid > rib[MT + d0] || x_rid < rib[MT + d1])))
    return;
  if (x_ri > fmin(rib[MT + T.irimax[MT + d0]], rib[MT + T.irimax[MT + d1]])) {
    slq2 = 0.0e0;
    sm = 0.0e0;
    sh = 0.0e0;
    ss = 0.0e0;
    return;
  }
  if (fabs(x_ri) >= gm && fabs(x_ri) >= rmax) {
    r0 = (int)sgn((double)MT, x_ri);
    r1 = r0;
  } else {
    expabs_index(x_ri, rib, T.dri, C.log_gm, C.log_rri, r0, r1);
    if (x_ri == 0.0e0) r1 = 1;
  }
  if ((x_ri > 0.0e0 && (x_ri < rib[MT + r0] || x_ri > rib[MT + r1])) ||
      (x_ri < 0.0e0 && (x_ri > rib[MT + r0] || x_ri < rib[MT + r1])))
    return;
  const double dridta = rib[MT + d1] - rib[MT + d0];
  const double drita = rib[MT + r1] - rib[MT + r0];
  const double drid = x_rid - rib[MT + d0];
  const double dri = x_ri - rib[MT + r0];
  const long c00 = (long)N1 * (d0 + MT) + r0 + MT;
  const long c10 = (long)N1 * (d1 + MT) + r0 + MT;
  const long c01 = (long)N1 * (d0 + MT) + r1 + MT;
  double a_rid[4], a_ri[4];
  const double* tab[4] = {T.slq2b, T.smb, T.shb, T.ssb};
#pragma unroll
  for (int m = 0; m < 4; ++m) {
    if (d1 == d0) {
      a_rid[m] = 0.0e0;
      a_ri[m] = 0.0e0;
    } else {
      a_rid[m] = (tab[m][c10] - tab[m][c00]) / dridta;
      a_ri[m] = (tab[m][c01] - tab[m][c00]) / drita;
    }
  }
  slq2 = T.slq2b[c00] + a_ri[0] * dri + a_rid[0] * drid;
  sm = T.smb[c00] + a_ri[1] * dri + a_rid[1] * drid;
  sh = T.shb[c00] + a_ri[2] * dri + a_rid[2] * drid;
  ss = T.ssb[c00] + a_ri[3] * dri + a_rid[3] * drid;
}

// The column's interface values (the reference's wp1, wp3, wp8 at level k,
// k < kmt-1): temperature and density interpolated to the interface below
// level k, and its depth in cm
struct Iface {
  const double *T, *pd, *dzp, *zkp;
  long A;
  __device__ double t(int k) const {
    return T[k * A] - (T[k * A] - T[(k + 1) * A]) * dzp[k] / (dzp[k] + dzp[k + 1]);
  }
  __device__ double rh(int k) const {
    return (pd[k * A] + (pd[(k + 1) * A] - pd[k * A]) * dzp[k] / (dzp[k] + dzp[k + 1])) * 1.0e-3;
  }
  __device__ double z(int k) const { return -zkp[k + 1] * 1.0e+2; }
};

__global__ void __launch_bounds__(128, 5) k_turb(Arena a, TurbTabDev T, double ncc_f, double fricmx, double wndmix) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= a.imt || j >= a.jmt) return;
  const long q = (long)j * a.imt + i;
  const long A = a.A;
  const int km = a.km;
  const int kz = a.kmt[q];
  if (!(i > 0 && i < a.imt - 1 && j > 0 && j < a.jmt - 1 && kz > 0)) {
    // not a column of turb_cu: what the reference's memsets leave
    for (int k = 0; k < km; ++k) {
      a.akmt[k * A + q] = 0.0;
      a.ak_tide[k * A + q] = 0.0;
    }
    a.amld[q] = 0.0;
    return;
  }
  const int n = kz - 1;   // interfaces of the column (iwk)
  Iface f{a.at[a.cur] + q, a.pdensity + q, a.dzp, a.zkp, A};
  const double* rict = a.rict + q;

  // ---- 1. tidal mixing, bottom-up minimum (readyc.cpp:1534-1557)
  {
    double below = 0.0;
    const double wd = a.wave_dis[q];
    for (int k = km - 1; k >= n; --k) a.ak_tide[k * A + q] = 0.0;
    for (int k = n - 1; k >= 0; --k) {
      const double wp3 = f.rh(k);
      const double rc = rict[k * A];
      const double fz = a.fz_tide[k * A + q];
      double v = kBackTidal + kMixingEf * kLocalFrac * wd * fz / (fmax(rc, 1.0e-8) * (wp3 * 1000.0));
      if (v > kMaxTidal) v = kMaxTidal;
      if (k <= n - 2) v = fmin(v, below);
      below = v;
      a.ak_tide[k * A + q] = v;
      a.richardson[k * A + q] = rc;
      a.fztidal[k * A + q] = fz;
      a.wp3_tidal[k * A + q] = wp3;
    }
  }

  // ---- 2. mixed-layer depth (formld, readyc.cpp:902-913)
  double amld;
  if (n > 0) {
    amld = f.z(n - 1);
    const double t0 = f.t(0);
    double tp = t0, zp = f.z(0);
    for (int k = 1; k < n; ++k) {
      const double tk = f.t(k), zk = f.z(k);
      if (fabs(tk - t0) > 0.1) {
        const double tm = t0 - sgn(0.1e0, t0 - tk);
        amld = zk + (zp - zk) * (tm - tk) / (tp - tk + 1.0e-20);
        break;
      }
      tp = tk;
      zp = zk;
    }
  } else {
    amld = 0.0;   // z[0] of an empty column (the work array is zeroed)
  }
  a.amld[q] = amld * 1.0e-2;

  // ---- 3. the closure, level by level (turb_device, readyc.cpp:1116-1454)
  TurbConst C;
  C.pi4 = atan(1.0e0);
  {
    const double an0 = 5.24e-3, f30 = 4.0e0 * C.pi4 / 43082.0e0;
    C.eplat_den = f30 * acosh(an0 / f30);
  }
  C.log_gm = log(T.rib[MT + MT0]);
  C.log_rri = log(T.rri);
  C.log_gm1 = log(T.and2on2a1[MT + MT0]);
  C.log_rnd = log(T.rnd2on2);
  const double coriol = a.fcort[q];
  const double buoytot = a.buoytur[q] * 1.0e+4 + a.buoysol[q] * 1.0e+4;
  const double b1 = T.b1;
  const double al0 = 0.17 * amld;
  double ifbelow = 0.0;
  double an = 0.0;                     // unset in the reference until N^2 >= 0 is met
  double slq2 = 0.0, sm = 0.0, sh = 0.0, ss = 0.0, amtaun2 = 0.0;
  double slq2_back = 0.0, sm_back = 0.0, sh_back = 0.0, ss_back = 0.0;
  double back_ri1 = 0.0, tmp = 0.0;
  double km0 = 0.0, kh0 = 0.0, ks0 = 0.0;   // level 0, written last
  double* akt_t = a.precision == LT_PREC_MIXED ? nullptr : a.akt + q;
  float* akt_t32 = a.precision == LT_PREC_MIXED ? a.akt32 + q : nullptr;
  const long F = a.F;
  auto put = [&](int k, double akm, double akh, double aks) {
    const double tide = a.ak_tide[k * A + q];
    a.akmt[k * A + q] = akm * 1.0e-4 + tide * 5.0;
    const double t_ = (akh * 1.0e-4 + tide) / ncc_f;
    const double s_ = (aks * 1.0e-4 + tide) / ncc_f;
    if (akt_t) {
      akt_t[k * A] = t_;
      akt_t[F + k * A] = s_;
    } else {
      akt_t32[k * A] = (float)t_;
      akt_t32[F + k * A] = (float)s_;
    }
  };
  // rolling window of interface depths and densities: k-2 .. k+1
  double z_m1 = 0.0, z_0 = n > 0 ? f.z(0) : 0.0, z_p1 = n > 1 ? f.z(1) : 0.0;
  double rh_m2 = 0.0, rh_m1 = 0.0, rh_0 = n > 0 ? f.rh(0) : 0.0, rh_p1 = n > 1 ? f.rh(1) : 0.0;
  int done = 0;   // levels whose diffusivities the closure set
  bool quit = false;
  for (int k = 0; k < n; ++k) {
    const double an2 = rict[k * A];
    const double rik = a.rit[k * A + q];
    const double ridk = a.ricdttms[k * A + q];
    double s2 = a.s2t[k * A + q];
    double ifnofsmall = 0.0;
    if (an2 >= 0.0e0) an = sqrt(an2);
    if (an < fabs(coriol)) ifnofsmall = 1.0;
    double ri1 = rik, rid1 = ridk;
    const double and2 = ridk / (rik + 1.0e-25) * an2;
    const double and2on2 = and2 / (an2 + 1.0e-25);
    const int ifpureshear = (an2 < T.rib[0] * s2) ? 1 : 0;
    if (ifpureshear == 1) {
      interp1d(and2on2, T, C, amtaun2, sm, sh, ss);
      slq2 = (-amtaun2) / ((b1 * b1) * rik + 1.0e-25);
    } else {
      interp2d(ri1, rid1, T, C, slq2, sm, sh, ss);
      if (slq2 < 0.0e0) { quit = true; break; }
      if (slq2 == 0.0e0) ifbelow = 1.0;
    }
    const bool lifupper = ((ifbelow == 0.0 || ifnofsmall == 1.0 || ((ri1 < 0.0e0) && (k <= 1))) && (slq2 > 0.0e0));
    double epsy = 0.0e0;
    bool lifepsy = false;
    if (slq2 == 0.0e0) epsy = 0.0e0;
    else epsy = -buoytot / ((1.0e0 / ((b1 * b1) * (slq2))) - 0.5e0 * sm);
    lifepsy = ((epsy >= 0.0e0) && lifupper);
    const double akz = 0.4 * z_0;
    const double al = akz * al0 / (al0 + akz);
    double al2 = al * al;
    if (ifbelow != 1.0 && !lifepsy) {
      if (ri1 > 0.0e0) {
        const double anlq2 = slq2 * ri1;
        if (anlq2 > 0.281e0) {
          al2 *= 0.281e0 / anlq2;
          slq2 = 0.281e0 / (ri1 + 1.0e-20);
        }
      }
    }
    double epson2;
    if (an2 < 0.0e0) {
      epson2 = kEpson2;
    } else {
      double ep = ifnofsmall == 1.0 ? 0.0e0 : eplat(C, fabs(coriol), an);
      ep = fmax(ep, kEplatMin);
      epson2 = kEpson2 * ep;
    }
    double back_ra_r1 = 0.0, back_rit1 = 0.0, back_ric1 = 0.0, back_rid1 = 0.0;
    if (rik > 0.0e0) {
      const double rit = (rik + ridk) / 2.0e0;
      const double ric = (rik - ridk) / 2.0e0;
      const double ra_r = sqrt((rit * rit) + (ric * ric));
      double theta_r;
      if (fabs(rit) <= 0.0e0) theta_r = (fabs(ric) <= 0.0e0) ? C.pi4 : 2.0e0 * C.pi4;
      else theta_r = atan(ric / rit);
      if (fabs(theta_r) > 2.0e0 * C.pi4) { quit = true; break; }
      if (theta_r < -C.pi4) theta_r += 4.0e0 * C.pi4;
      const int jt0 = (int)((theta_r + C.pi4) / T.deltheta_r);
      int it0 = jt0 - NTH, it1 = it0 + 1;
      double th0 = it0 * T.deltheta_r, th1 = it1 * T.deltheta_r;
      if ((th0 <= T.theta_rcrp) && (theta_r > T.theta_rcrp)) {
        theta_r = th1;
        th0 = th1;
        it0 = it1;
        ++it1;
        th1 += T.deltheta_r;
      } else if ((th1 >= T.theta_rcrn) && (theta_r < T.theta_rcrn)) {
        theta_r = th0;
        th1 = th0;
        it1 = it0;
        --it0;
        th0 += -T.deltheta_r;
      }
      if ((it1 > 3 * NTH) || (it0 < -NTH)) { quit = true; break; }
      double dth = theta_r - th0;
      const double del = T.back_ra_r[NTH + it1] - T.back_ra_r[NTH + it0];
      back_ra_r1 = T.back_ra_r[NTH + it0] + dth * (del / T.deltheta_r);
      int ifrafglt = 0;
      if ((theta_r <= T.theta_rcrp) || (theta_r >= T.theta_rcrn)) {
        if (back_ra_r1 > ra_r) {
          ifrafglt = 1;
          back_ra_r1 = ra_r;
        }
      }
      if (back_ra_r1 < 0.0e0) { quit = true; break; }
      back_rit1 = cos(theta_r) * back_ra_r1;
      back_ric1 = sin(theta_r) * back_ra_r1;
      back_ri1 = back_rit1 + back_ric1;
      back_rid1 = back_rit1 - back_ric1;
      if (ifrafglt == 1) {
        interp2d(back_ri1, back_rid1, T, C, slq2_back, sm_back, sh_back, ss_back);
      } else {
        dth = theta_r - it0 * T.deltheta_r;
        sm_back = T.sm_r1[NTH + it0] + dth * ((T.sm_r1[NTH + it1] - T.sm_r1[NTH + it0]) / T.deltheta_r);
        sh_back = T.sh_r1[NTH + it0] + dth * ((T.sh_r1[NTH + it1] - T.sh_r1[NTH + it0]) / T.deltheta_r);
        ss_back = T.ss_r1[NTH + it0] + dth * ((T.ss_r1[NTH + it1] - T.ss_r1[NTH + it0]) / T.deltheta_r);
        slq2_back = T.slq2_r1[NTH + it0] + dth * ((T.slq2_r1[NTH + it1] - T.slq2_r1[NTH + it0]) / T.deltheta_r);
      }
      if (slq2_back < 0.0e0) { quit = true; break; }
    }
    if (rik <= 0.0e0) back_ri1 = 0.0e0;
    if (ri1 <= 0.0e0) {
      sm_back = 0.0e0;
      sh_back = 0.0e0;
      ss_back = 0.0e0;
    }
    if ((sm_back < 0.0e0) || (sh_back < 0.0e0) || (ss_back < 0.0e0)) { quit = true; break; }
    const double tmp_back = 0.5e0 * b1 * b1 * back_ri1 * slq2_back * epson2;
    const double v_back = tmp_back * sm_back, t_back = tmp_back * sh_back, s_back = tmp_back * ss_back;
    if ((v_back < 0.0e0) || (t_back < 0.0e0) || (s_back < 0.0e0)) { quit = true; break; }
    if ((rik > 0.0e0) && ((fabs(v_back) <= 0.0e0) || (fabs(t_back) <= 0.0e0) || (fabs(s_back) < 0.0e0))) {
      quit = true;
      break;
    }
    if (ifbelow == 1.0) {
      if (ri1 >= 0.0e0) {
        tmp = 0.5e0 * b1 * b1 * ri1 * slq2 * epson2;
      } else if (k >= 2) {
        double delz, delrh, del2rh;
        if (k == n - 1) {
          delz = z_0 - z_m1;
          delrh = rh_0 - rh_m1;
          del2rh = rh_0 - 2.0e0 * rh_m1 + rh_m2;
        } else {
          delz = z_p1 - z_m1;
          delrh = rh_p1 - rh_m1;
          del2rh = rh_p1 - 2.0e0 * rh_0 + rh_m1;
        }
        const double dzrh = delrh / delz;
        const double d2zrh = 4.0e0 * del2rh / (delz * delz);
        const double rdzlndzrh = dzrh / d2zrh;
        const double al0deep = 0.17e0 * fabs(rdzlndzrh);
        const double akz2 = 0.4e0 * z_0;
        const double aldeep = akz2 * al0deep / (al0deep + akz2);
        al2 = aldeep * aldeep;
        if (ifpureshear != 1) {
          s2 = fmax(s2, kS2min);
          tmp = 0.5e0 * b1 * al2 * sqrt(s2 / (slq2 + 1.0e-40));
        }
      } else {
        if (ifpureshear != 1) {
          s2 = fmax(s2, kS2min);
          if (lifepsy) tmp = 0.5e0 * epsy / (s2 + 1.0e-40);
          else tmp = 0.5e0 * b1 * al2 * sqrt(s2 / (slq2 + 1.0e-40));
        }
      }
    } else {
      if (ifpureshear != 1) {
        s2 = fmax(s2, kS2min);
        if (lifepsy) tmp = 0.5e0 * epsy / (s2 + 1.0e-40);
        else tmp = 0.5e0 * b1 * al2 * sqrt(s2 / (slq2 + 1.0e-40));
      }
    }
    if (ifpureshear == 1) tmp = 0.5e0 * (b1 * b1) * al2 * sqrt(-an2 / amtaun2);
    const double akm = fmin(tmp * sm + v_back, fricmx);
    const double akh = fmin(tmp * sh + t_back, fricmx);
    const double aks = fmin(tmp * ss + s_back, fricmx);
    if (k == 0) {
      km0 = akm;
      kh0 = akh;
      ks0 = aks;
    } else {
      put(k, akm, akh, aks);
    }
    done = k + 1;
    // slide the window
    z_m1 = z_0;
    z_0 = z_p1;
    z_p1 = (k + 2 < n) ? f.z(k + 2) : 0.0;
    rh_m2 = rh_m1;
    rh_m1 = rh_0;
    rh_0 = rh_p1;
    rh_p1 = (k + 2 < n) ? f.rh(k + 2) : 0.0;
  }
  // the reference returns early on an inconsistent table value: the levels
  // from there on keep their zeroed work arrays and the surface floor is skipped
  if (!quit && n > 0) {
    if (km0 < wndmix) km0 = wndmix;
    if (kh0 < wndmix) kh0 = wndmix;
    if (ks0 < wndmix) ks0 = wndmix;
  }
  put(0, km0, kh0, ks0);
  for (int k = done > 1 ? done : 1; k < km - 1; ++k) put(k, 0.0, 0.0, 0.0);
  a.akmt[(long)(km - 1) * A + q] = 0.0;
}

}  // namespace

int launch_turb(const Arena& a, const TurbTabDev& T, int ncc, double dfricmx, cudaStream_t s) {
  dim3 b(32, 4), g((a.imt + 31) / 32, (a.jmt + 3) / 4);
  k_turb<<<g, b, 0, s>>>(a, T, (double)(float)ncc, dfricmx * 1.0e+4, a.p.dwndmix * 1.0e+4);
  LT_LAUNCHED();
  return LT_OK;
}

}  // namespace lt

using namespace lt;

extern "C" {

int lt_turb_tables_create(const lt_turb_tables* h, lt_turb_tab** out) {
  if (!h || !out || !h->rib || !h->irimax || !h->slq2b || !h->smb || !h->shb || !h->ssb || !h->and2on2a1 ||
      !h->amtaun2a1 || !h->sma1 || !h->sha1 || !h->ssa1 || !h->back_ra_r || !h->sm_r1 || !h->sh_r1 || !h->ss_r1 ||
      !h->slq2_r1) {
    set_error("lt_turb_tables_create: a table pointer is missing");
    return LT_E_INVALID;
  }
  if (!(h->dri > 0.0) || !(h->rri > 1.0) || !(h->dand2on2 > 0.0) || !(h->rnd2on2 > 1.0) || !(h->deltheta_r > 0.0)) {
    set_error("lt_turb_tables_create: grid steps must be positive and ratios above 1");
    return LT_E_INVALID;
  }
  for (int m = 0; m < N1; ++m)
    if (h->irimax[m] < -MT || h->irimax[m] > MT) {
      set_error("lt_turb_tables_create: irimax[%d] = %d outside -%d..%d", m, h->irimax[m], MT, MT);
      return LT_E_INVALID;
    }
  const size_t n1 = N1, n2 = (size_t)N1 * N1, nb = LT_TURB_NB;
  struct Item { const void* src; size_t bytes; const void** dst; };
  lt_turb_tab* t = new (std::nothrow) lt_turb_tab;
  if (!t) return LT_E_OOM;
  TurbTabDev& T = t->t;
  const Item items[] = {
      {h->rib, n1 * 8, (const void**)&T.rib},         {h->irimax, n1 * 4, (const void**)&T.irimax},
      {h->slq2b, n2 * 8, (const void**)&T.slq2b},     {h->smb, n2 * 8, (const void**)&T.smb},
      {h->shb, n2 * 8, (const void**)&T.shb},         {h->ssb, n2 * 8, (const void**)&T.ssb},
      {h->and2on2a1, n1 * 8, (const void**)&T.and2on2a1}, {h->amtaun2a1, n1 * 8, (const void**)&T.amtaun2a1},
      {h->sma1, n1 * 8, (const void**)&T.sma1},       {h->sha1, n1 * 8, (const void**)&T.sha1},
      {h->ssa1, n1 * 8, (const void**)&T.ssa1},       {h->back_ra_r, nb * 8, (const void**)&T.back_ra_r},
      {h->sm_r1, nb * 8, (const void**)&T.sm_r1},     {h->sh_r1, nb * 8, (const void**)&T.sh_r1},
      {h->ss_r1, nb * 8, (const void**)&T.ss_r1},     {h->slq2_r1, nb * 8, (const void**)&T.slq2_r1}};
  size_t total = 0;
  for (const Item& it : items) total += (it.bytes + 255) / 256 * 256;
  char* base = nullptr;
  cudaError_t e = cudaMalloc(&base, total);
  if (e != cudaSuccess) {
    delete t;
    set_error("lt_turb_tables_create: cudaMalloc(%zu) failed: %s", total, cudaGetErrorString(e));
    return LT_E_OOM;
  }
  size_t off = 0;
  for (const Item& it : items) {
    *it.dst = base + off;
    e = cudaMemcpy(base + off, it.src, it.bytes, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      cudaFree(base);
      delete t;
      return cuda_fail(e, "lt_turb_tables_create");
    }
    off += (it.bytes + 255) / 256 * 256;
  }
  T.rri = h->rri;
  T.rnd2on2 = h->rnd2on2;
  T.dri = h->dri;
  T.deltheta_r = h->deltheta_r;
  T.b1 = h->b1;
  T.theta_rcrp = h->theta_rcrp;
  T.theta_rcrn = h->theta_rcrn;
  T.dand2on2 = h->dand2on2;
  t->base = base;
  cudaGetDevice(&t->dev);
  *out = t;
  return LT_OK;
}

int lt_turb_tables_destroy(lt_turb_tab* t) {
  if (!t) return LT_E_INVALID;
  cudaFree(t->base);
  delete t;
  return LT_OK;
}

int lt_turb(lt_domain* d, const lt_turb_tab* t, const lt_turb_params* p) {
  if (!d || !t || !p || p->ncc < 1) {
    set_error("lt_turb: invalid arguments");
    return LT_E_INVALID;
  }
  int rc = ensure_turb(d);
  if (rc) return rc;
  return launch_turb(d->a, t->t, p->ncc, p->dfricmx, d->stream);
}

}  // extern "C"
