// licom_oracle.cpp - CPU FP64 restatement of the LICOM3-HIP baroclinic tracer
// step.  TEST INFRASTRUCTURE ONLY: it is the checker the GPU path is compared
// against, never part of the product.
//
// What it follows (paths are within the reference project):
//   orchestration and index ranges: tracer.cpp:1701-1903 (tracer_)
//   continuity                      tracer.cpp:980-1150 (tracer_1_0, tracer_1,
//                                   upwell_2, operators_div, upwell_3, upwell_4),
//                                   upwell.F90:26-109, grid.F90:1936-1993
//   tspas advection                 tracer.cpp:83-119, 291-921, advection.F90:153-431
//   biharmonic tracer diffusion     tracer.cpp:1238-1362, hmix_del4.F90:626-757
//   vertical terms, forcing         tracer.cpp:1395-1699
//   implicit vertical diffusion     tracer.cpp:923-978, invtri.F90:5-65
//   halo and tripole fold           POP_HaloMod.F90:2716-3139, 5602-5680,
//                                   POP_BlocksMod.F90:284-375
//   convective adjustment           convadj.cpp:29-288
//   sea-ice adjustment              icesnow.cpp:15-85
//   momentum biharmonic friction    readyc.cpp:343-577, 1754-1775 (hdel4_div,
//                                   hdel4_grad, hdel4_zcurl, hdiffu_del4_0/1)
//   Canuto turbulence closure       readyc.cpp:880-1612 (turb_cu, turb_device,
//                                   interp1d_expabs, interp2d_expabs, formld,
//                                   eplatidepend_fun), TIDEMIX configuration
//
// Arithmetic keeps the reference's operation order term by term (so that a
// build with -ffp-contract=off reproduces the reference's own code compiled
// the same way bit for bit); the loop structure, storage and naming are this
// file's own.  The only reduction, the SSS-normalisation sum, runs in the
// reference's sequential j-major order.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <vector>
#include <algorithm>
#include "../include/licom_tracer.h"

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

enum Kind { K3N = 0, KB3N, K3, KW, K2, K2N, K2I, K1, K1C, K3M1, K1P };

struct FieldInfo { int kind; bool is_int; };

FieldInfo field_info(int f) {
  switch (f) {
    case LT_F_AT: case LT_F_AKT: case LT_F_RESTORE: case LT_F_RESTORE_AT: case LT_F_DT_RESTORE:
    case LT_F_AX: case LT_F_AY: case LT_F_AZ: case LT_F_DZ: case LT_F_TEND: case LT_F_DT_DIFF: case LT_F_DT_CONV:
      return {K3N, false};
    case LT_F_ATB: return {KB3N, false};
    case LT_F_UTF: case LT_F_VTF: case LT_F_UTL: case LT_F_VTL: case LT_F_UTF_OUT: case LT_F_VTF_OUT:
    case LT_F_PENETRATE: case LT_F_FZ_TIDE: case LT_F_AKMT: case LT_F_AK_TIDE: case LT_F_RICHARDSON:
    case LT_F_FZTIDAL: case LT_F_WP3_TIDAL: case LT_F_UP: case LT_F_VP: case LT_F_DLU: case LT_F_DLV:
    case LT_F_WKA_DRAG:
      return {K3, false};
    case LT_F_RIT: case LT_F_RICDTTMS: case LT_F_S2T: case LT_F_RICT: return {K3M1, false};
    case LT_F_ZKP: return {K1P, false};
    case LT_F_WS: case LT_F_PDENSITY: return {KW, false};
    case LT_F_NET: return {K2N, false};
    case LT_F_KMT: case LT_F_KMU: case LT_F_KMTN: case LT_F_KMTS: case LT_F_KMTE: case LT_F_KMTW:
      return {K2I, true};
    case LT_F_DZP: case LT_F_ODZP: case LT_F_ODZT: case LT_F_PEN: case LT_F_TO: case LT_F_SO:
      return {K1, false};
    case LT_F_C: return {K1C, false};
    default: return {K2, false};
  }
}

// tracer_7 (tracer.cpp:1571-1626) for tracer n: the nudging toward
// restore_at of the levels k < ktv (simple_assm), whose rate is 1/(5 days)
// down to level 45 and smaller by ((k+1)/5)^2 below, with its term also
// written to dt_restore; then the 15-day restoring toward restore
// (boundary_restore == 1) of the levels k >= 1.  Inner cells only.  tf, vit:
// [km][jmt][imt]; atbn: this tracer's [km+1][jmt][imt]; restore, restore_at,
// dt_restore: [2][km][jmt][imt].
void tracer7(const lt_params& p, int n, int imt, int jmt, int km, double* tf, const double* vit, const double* atbn,
             const double* restore, const double* restore_at, double* dt_restore) {
  const long A = (long)imt * jmt, F = A * km;
  if (p.simple_assm) {
#pragma omp parallel for
    for (int k = 0; k < std::min(p.ktv, km); ++k) {
      const double lamda1 = k < 45 ? 1.0e0 / (5.e0 * 86400.e0)
                                   : 1.0e0 / (5.e0 * 86400.e0) / ((k + 1) * (k + 1) / 5.0 / 5.0);
      for (int j = 2; j < jmt - 2; ++j)
        for (int i = 2; i < imt - 2; ++i) {
          const long c = (long)k * A + (long)j * imt + i;
          tf[c] = tf[c] + vit[c] * (restore_at[n * F + c] - atbn[c + A]) * lamda1;
          dt_restore[n * F + c] = vit[c] * (restore_at[n * F + c] - atbn[c + A]) * lamda1;
        }
    }
  }
  if (p.boundary_restore == 1) {
    const double lamda = 1.0 / (15.0 * 86400.0);
#pragma omp parallel for
    for (int k = 1; k < km; ++k)
      for (int j = 2; j < jmt - 2; ++j)
        for (int i = 2; i < imt - 2; ++i) {
          const long c = (long)k * A + (long)j * imt + i;
          tf[c] = tf[c] + vit[c] * (restore[n * F + c] - atbn[c + A]) * lamda;
        }
  }
}

struct Oracle {
  int nx, ny, km, imt, jmt;
  long A, F, FB;
  int ew_cyclic = 1, tripole = 1, diagnostics = 1;
  lt_params p{};
  std::vector<double> fd[LT_F_COUNT];
  std::vector<int> fi[LT_F_COUNT];
  // scratch of the reference kernels
  std::vector<double> vit, at00, atmax, atmin, uk, vk, wka, wkb, wkd, wkc, work, stf, tf, adv_tt, d2tk,
      u_wface, v_sface, ori, temp11, vtl_work;
  double fw_norm2 = 0.0;
  int ist = 0;
  bool tree_sum = false;  // SSS-norm sum in the device's tree order instead of sequential

  long count(int f) const {
    switch (field_info(f).kind) {
      case K3N: return 2 * F;
      case KB3N: return 2 * FB;
      case K3: return F;
      case KW: return FB;
      case K2N: return 2 * A;
      case K2: case K2I: return A;
      case K1: return km;
      case K1C: return 9L * km;
      case K3M1: return A * (km - 1);
      case K1P: return km + 1;
    }
    return 0;
  }

  // copies of the dynamics inputs that or_step restores before every step
  std::vector<double> dyn0[5];

  // Fields of the tracer step are allocated at creation; the diagnostics
  // only while diagnostics are on; the restoring target, the closure's and
  // the momentum friction's fields on first use (a 0.1-degree oracle then
  // fits the host memory of one GPU's share of a node).
  Oracle(int nx_, int ny_, int km_) : nx(nx_), ny(ny_), km(km_) {
    imt = nx + 4; jmt = ny + 4;
    A = (long)imt * jmt; F = A * km; FB = A * (km + 1);
    for (int f = 0; f < LT_F_COUNT; ++f) {
      const int kd = field_info(f).kind;
      const bool small = kd == K2 || kd == K2I || kd == K2N || kd == K1 || kd == K1C || kd == K1P;
      const bool step = f == LT_F_AT || f == LT_F_ATB || f == LT_F_UTF || f == LT_F_VTF || f == LT_F_UTL ||
                        f == LT_F_VTL || f == LT_F_AKT || f == LT_F_WS || f == LT_F_UTF_OUT || f == LT_F_VTF_OUT;
      if (small || step) ensure(f);
    }
    set_diagnostics(1);
    for (auto* v : {&vit, &at00, &atmax, &atmin, &uk, &vk, &wka, &wkb, &wkd, &wkc, &tf, &adv_tt, &d2tk,
                    &u_wface, &v_sface, &ori})
      v->assign(F, 0.0);
    work.assign(A, 0.0); stf.assign(A, 0.0); temp11.assign(A, 0.0);
  }

  void ensure(int f) {
    if (field_info(f).is_int) {
      if (fi[f].empty()) fi[f].assign(count(f), 0);
    } else if (fd[f].empty()) {
      fd[f].assign(count(f), 0.0);
    }
  }
  void ensure_all() {
    for (int f = 0; f < LT_F_COUNT; ++f) ensure(f);
  }
  void set_diagnostics(int on) {
    diagnostics = on;
    if (on)
      for (int f : {LT_F_AX, LT_F_AY, LT_F_AZ, LT_F_DZ, LT_F_TEND, LT_F_DT_DIFF, LT_F_DT_CONV, LT_F_PENETRATE})
        ensure(f);
  }

  // index helpers
  long c3(int k, int j, int i) const { return (long)k * A + (long)j * imt + i; }
  long c2(int j, int i) const { return (long)j * imt + i; }
};

// The device's deterministic sum order (alternative to the reference's
// sequential loop): blocks of 2048 consecutive terms zero-padded, each reduced
// by pairing element t with t+stride for stride = 1024, 512, ..., 1; the
// block sums are reduced the same way until one value remains.
double device_tree_sum(std::vector<double> x) {
  const size_t RB = 1024;
  if (x.empty()) x.push_back(0.0);
  for (;;) {
    const size_t nb = (x.size() + 2 * RB - 1) / (2 * RB);
    std::vector<double> part(nb);
    std::vector<double> s(2 * RB);
    for (size_t b = 0; b < nb; ++b) {
      for (size_t t = 0; t < 2 * RB; ++t) s[t] = (b * 2 * RB + t < x.size()) ? x[b * 2 * RB + t] : 0.0;
      for (size_t stride = RB; stride > 0; stride >>= 1)
        for (size_t t = 0; t < stride; ++t) s[t] = s[t] + s[t + stride];
      part[b] = s[0];
    }
    if (nb == 1) return part[0];
    x.swap(part);
  }
}

// ------------------------------------------------------------------ halo
// Global-domain, single-block ghost update (POP_HaloUpdate3DR8 with
// POP_gridHorzLocCenter / POP_fieldKindScalar).  Message order of the
// reference: east/west local copies of physical rows, then the tripole buffer
// (top haloWidth+1 physical rows), symmetric averaging of its first row for
// i = 1..nx/2-1 with partner nx-i, and the copy-out into ghost rows j=1,2 and
// the top physical row j=3 (1-based) for every column including E-W ghosts.
// A closed boundary sends no message, so its ghost cells are left as they are.
void halo_r8(double* a, int nz, int imt, int jmt, int ew_cyclic, int tripole) {
  const int nx = imt - 4;
  std::vector<double> buf((size_t)(nx + 1) * 3);
  for (int z = 0; z < nz; ++z) {
    double* s = a + (long)z * imt * jmt;
    if (ew_cyclic) {
      for (int jf = 3; jf <= jmt - 2; ++jf) {        // physical rows, Fortran numbering
        double* row = s + (long)(jf - 1) * imt;
        for (int h = 1; h <= 2; ++h) {
          row[h - 1] = row[(nx + 2) - 2 + h - 1];      // east msg: ie-hw+h -> h
          row[(nx + 2) + h - 1] = row[3 + h - 2];      // west msg: ib+h-1 -> ie+h
        }
      }
    }
    if (!tripole) continue;
    for (int r = 1; r <= 3; ++r)
      for (int g = 1; g <= nx; ++g) buf[(size_t)(r - 1) * (nx + 1) + g] = s[(long)(2 + r - 1) * imt + (g + 2) - 1];
    for (int g = 1; g <= nx / 2 - 1; ++g) {
      const int gd = nx - g;
      const double x1 = buf[g], x2 = buf[gd];
      const double xavg = 0.5 * (x1 + x2);
      buf[g] = xavg;
      buf[gd] = xavg;
    }
    buf[nx] = 1.0 * buf[nx];
    for (int jf = 1; jf <= 3; ++jf) {
      for (int iF = 1; iF <= imt; ++iF) {
        int ig = iF - 2;                            // POP_BlocksMod global index
        if (ig < 1) ig = ew_cyclic ? ig + nx : 0;
        else if (ig > nx) ig = ew_cyclic ? ig - nx : 0;
        int isrc = nx - ig + 1 - 1;
        const int jsrc = (2 + 3 - jf) - 1;
        if (isrc == 0) isrc = nx;
        if (jsrc > 0) s[(long)(jf - 1) * imt + iF - 1] = buf[(size_t)(jsrc - 1) * (nx + 1) + isrc];
      }
    }
  }
}

// advection_tracer_1 for Str 0 (centered) and Str 1 (flux), tracer.cpp:120-289:
// adv_tt on the inner cells (2 <= j < jmt-2, 2 <= i < imt-2) of every level.
// The centred form also accumulates the diagnostics ax, ay, az with weight
// 1/nss.  The reference writes its top- and bottom-level statements without a
// level guard, so every thread of the launch's level dimension repeats them
// and their diagnostic accumulations race; here each level is accumulated
// once (adv_tt itself gets the same value from every repetition).
void advect_simple(Oracle& o, int n, const double* atn, const double* uw, const double* vs, const double* ws,
                   double* adv_tt, bool dg) {
  const int km = o.km, imt = o.imt, jmt = o.jmt;
  const long A = o.A, F = o.F;
  const double* tarea_r = o.fd[LT_F_TAREA_R].data();
  const double* odzp = o.fd[LT_F_ODZP].data();
  double* ax = o.fd[LT_F_AX].data();
  double* ay = o.fd[LT_F_AY].data();
  double* az = o.fd[LT_F_AZ].data();
  const double nss = (double)o.p.nss;
  const bool centered = o.p.adv_tracer == LT_ADV_CENTERED;
#pragma omp parallel for
  for (int k = 0; k < km; ++k)
    for (int j = 2; j < jmt - 2; ++j)
      for (int i = 2; i < imt - 2; ++i) {
        const long c = (long)k * A + (long)j * imt + i;
        const double tr = tarea_r[(long)j * imt + i];
        const double ac = atn[c], ae = atn[c + 1], aw = atn[c - 1], as = atn[c + imt], an = atn[c - imt];
        if (centered) {
          const double h = (-uw[c] * (ac - aw) - uw[c + 1] * (ae - ac) - vs[c] * (as - ac) - vs[c - imt] * (ac - an)) * tr;
          if (dg) {
            ax[n * F + c] = ax[n * F + c] + (-uw[c] * (ac - aw) - uw[c + 1] * (ae - ac)) * tr / nss;
            ay[n * F + c] = ay[n * F + c] + (-vs[c] * (as - ac) - vs[c - imt] * (ac - an)) * tr / nss;
          }
          double z;
          if (k == 0) {
            const double z2 = ws[c + A] * (ac - atn[c + A]);
            z = 0.5 * odzp[0] * z2;
          } else if (k == km - 1) {
            const double z1 = ws[c] * (atn[c - A] - ac);
            z = 0.5 * odzp[km - 1] * z1;
          } else {
            const double z1 = ws[c] * (atn[c - A] - ac);
            const double z2 = ws[c + A] * (ac - atn[c + A]);
            z = 0.5 * odzp[k] * (z1 + z2);
          }
          adv_tt[c] = h - z;
          if (dg) az[n * F + c] = az[n * F + c] - z / nss;
        } else {
          const double h = (-uw[c] * (ac + aw) + uw[c + 1] * (ae + ac) - vs[c - imt] * (ac + an) + vs[c] * (as + ac)) * tr;
          const double z1 = k == 0 ? 0.0 : ws[c] * (atn[c - A] + ac) * 0.5;
          const double z2 = k == km - 1 ? 0.0 : ws[c + A] * (ac + atn[c + A]) * 0.5;
          adv_tt[c] = h - odzp[k] * (z2 - z1);
        }
      }
}

// ------------------------------------------------------------ the step
void tracer_call(Oracle& o) {
  const int km = o.km, imt = o.imt, jmt = o.jmt;
  const long A = o.A, F = o.F, FB = o.FB;
  const lt_params& p = o.p;
  double* at = o.fd[LT_F_AT].data();
  double* atb = o.fd[LT_F_ATB].data();
  double* utf = o.fd[LT_F_UTF].data();
  double* vtf = o.fd[LT_F_VTF].data();
  double* utl = o.fd[LT_F_UTL].data();
  double* vtl = o.fd[LT_F_VTL].data();
  double* h0f = o.fd[LT_F_H0F].data();
  double* h0l = o.fd[LT_F_H0L].data();
  double* akt = o.fd[LT_F_AKT].data();
  double* ws = o.fd[LT_F_WS].data();
  double* net = o.fd[LT_F_NET].data();
  const double* swv = o.fd[LT_F_SWV].data();
  const double* nswv = o.fd[LT_F_NSWV].data();
  const double* sst = o.fd[LT_F_SST].data();
  const double* sss = o.fd[LT_F_SSS].data();
  const double* fresh = o.fd[LT_F_FRESH].data();
  const double* seaice = o.fd[LT_F_SEAICE].data();
  const double* tarea = o.fd[LT_F_TAREA].data();
  const double* tarea_r = o.fd[LT_F_TAREA_R].data();
  const double* htw = o.fd[LT_F_HTW].data();
  const double* hts = o.fd[LT_F_HTS].data();
  const double* hun = o.fd[LT_F_HUN].data();
  const double* hue = o.fd[LT_F_HUE].data();
  const double* dxu = o.fd[LT_F_DXU].data();
  const double* dyu = o.fd[LT_F_DYU].data();
  const double* ahf = o.fd[LT_F_AHF].data();
  const double* dtn = o.fd[LT_F_DTN].data();
  const double* dts_c = o.fd[LT_F_DTS].data();
  const double* dte = o.fd[LT_F_DTE].data();
  const double* dtw = o.fd[LT_F_DTW].data();
  const double* ohbt = o.fd[LT_F_OHBT].data();
  const double* ohbu = o.fd[LT_F_OHBU].data();
  const double* au0 = o.fd[LT_F_AU0].data();
  const double* aus = o.fd[LT_F_AUS].data();
  const double* auw = o.fd[LT_F_AUW].data();
  const double* ausw = o.fd[LT_F_AUSW].data();
  const int* kmt = o.fi[LT_F_KMT].data();
  const int* kmtn = o.fi[LT_F_KMTN].data();
  const int* kmts = o.fi[LT_F_KMTS].data();
  const int* kmte = o.fi[LT_F_KMTE].data();
  const int* kmtw = o.fi[LT_F_KMTW].data();
  const double* dzp = o.fd[LT_F_DZP].data();
  const double* odzp = o.fd[LT_F_ODZP].data();
  const double* odzt = o.fd[LT_F_ODZT].data();
  const double* pen = o.fd[LT_F_PEN].data();
  if (o.p.boundary_restore == 1) o.ensure(LT_F_RESTORE);
  const double* restore = o.fd[LT_F_RESTORE].data();
  if (o.p.simple_assm) { o.ensure(LT_F_RESTORE_AT); o.ensure(LT_F_DT_RESTORE); }
  const double* restore_at = o.fd[LT_F_RESTORE_AT].data();
  double* dt_restore = o.fd[LT_F_DT_RESTORE].data();
  const bool dg = o.diagnostics != 0;   // diagnostic fields are written only while on
  double* ax = o.fd[LT_F_AX].data();
  double* ay = o.fd[LT_F_AY].data();
  double* az = o.fd[LT_F_AZ].data();
  double* dzd = o.fd[LT_F_DZ].data();
  double* tend = o.fd[LT_F_TEND].data();
  double* dt_diff = o.fd[LT_F_DT_DIFF].data();
  double* penetrate = o.fd[LT_F_PENETRATE].data();
  double* vit = o.vit.data();
  double *at00 = o.at00.data(), *atmax = o.atmax.data(), *atmin = o.atmin.data();
  double *uk = o.uk.data(), *vk = o.vk.data(), *wka = o.wka.data(), *wkb = o.wkb.data(), *wkd = o.wkd.data();
  double *wkc = o.wkc.data(), *work = o.work.data(), *stf = o.stf.data(), *tf = o.tf.data();
  double *adv_tt = o.adv_tt.data(), *d2tk = o.d2tk.data(), *uw = o.u_wface.data(), *vs = o.v_sface.data();
  double *ori = o.ori.data(), *temp11 = o.temp11.data();
  const double dts = p.dts;

  // vit from kmt (boundary.F90:44-52)
#pragma omp parallel for
  for (int k = 0; k < km; ++k)
    for (long a = 0; a < A; ++a) vit[(long)k * A + a] = (k < kmt[a]) ? 1.0 : 0.0;

  auto C = [&](int k, int j, int i) { return (long)k * A + (long)j * imt + i; };
  auto Q = [&](int j, int i) { return (long)j * imt + i; };

  std::fill(o.at00.begin(), o.at00.end(), 0.0);
  std::fill(o.atmax.begin(), o.atmax.end(), 0.0);
  std::fill(o.atmin.begin(), o.atmin.end(), 0.0);
  std::fill(o.uk.begin(), o.uk.end(), 0.0);
  std::fill(o.vk.begin(), o.vk.end(), 0.0);

  // tracer_1_0: h0f *= onbc; stf = mean sea level of the two time levels
  for (long a = 0; a < A; ++a) {
    h0f[a] = h0f[a] * p.onbc;
    stf[a] = 0.5 * h0f[a] + 0.5 * h0l[a];
  }
  // tracer_1: scale utf/vtf, time-mean velocities, T->U interpolation of stf
#pragma omp parallel for
  for (int k = 0; k < km; ++k)
    for (int j = 0; j < jmt; ++j)
      for (int i = 0; i < imt; ++i) {
        const long c = C(k, j, i);
        utf[c] = utf[c] * p.oncc;
        vtf[c] = vtf[c] * p.oncc;
        wkd[c] = 0.5 * utf[c] + 0.5 * utl[c];
        wkb[c] = 0.5 * vtf[c] + 0.5 * vtl[c];
        wka[c] = 0.0;
      }
  for (int j = 0; j < jmt; ++j)
    for (int i = 0; i < imt; ++i) {
      double v = 0.0;
      if (j < jmt - 1 && i >= 1)
        v = au0[Q(j, i)] * stf[Q(j, i)] + aus[Q(j, i)] * stf[Q(j + 1, i)] + auw[Q(j, i)] * stf[Q(j, i - 1)] +
            ausw[Q(j, i)] * stf[Q(j + 1, i - 1)];
      work[Q(j, i)] = v;
    }
  // upwell_2: U-point velocities corrected for the free surface
#pragma omp parallel for
  for (int k = 0; k < km; ++k)
    for (int j = 0; j < jmt - 1; ++j)
      for (int i = 1; i < imt; ++i) {
        const long c = C(k, j, i);
        uk[c] = (1.0 + work[Q(j, i)] * ohbu[Q(j, i)]) * wkd[c];
        vk[c] = (1.0 + work[Q(j, i)] * ohbu[Q(j, i)]) * wkb[c];
      }
  // operators_div: horizontal divergence on T cells above the bottom
#pragma omp parallel for
  for (int k = 0; k < km; ++k)
    for (int j = 1; j < jmt; ++j)
      for (int i = 0; i < imt - 1; ++i) {
        if (!(k <= kmt[Q(j, i)] - 1)) continue;
        const double east = (uk[C(k, j, i + 1)] + uk[C(k, j - 1, i + 1)]) * htw[Q(j, i + 1)];
        const double west = (uk[C(k, j, i)] + uk[C(k, j - 1, i)]) * htw[Q(j, i)];
        const double south = (vk[C(k, j, i + 1)] + vk[C(k, j, i)]) * hts[Q(j, i)];
        const double north = (vk[C(k, j - 1, i + 1)] + vk[C(k, j - 1, i)]) * hts[Q(j - 1, i)];
        wka[C(k, j, i)] = 0.5 * (east - west + south - north) * tarea_r[Q(j, i)];
      }
  // upwell_3 / upwell_4: column divergence, w by upward integration, rescale
#pragma omp parallel for
  for (int j = 0; j < jmt; ++j)
    for (int i = 0; i < imt; ++i) {
      const long a = Q(j, i);
      work[a] = 0.0;
      if (!(j >= 1 && j < jmt - 1 && i >= 1 && i < imt - 1)) continue;
      for (int k = 0; k < km; ++k) work[a] = work[a] - dzp[k] * wka[k * A + a] * vit[k * A + a];
      for (int k = 1; k < km; ++k)
        ws[k * A + a] = vit[k * A + a] * (ws[(k - 1) * A + a] + dzp[k - 1] * (work[a] * ohbt[a] + wka[(k - 1) * A + a]));
      work[a] = 1.0 / (1.0 + stf[a] * ohbt[a]);
      for (int k = 1; k < km; ++k) ws[k * A + a] = ws[k * A + a] * work[a];
    }
  o.ist += 1;

  for (int n = 0; n < 2; ++n) {
    const double* atn = at + n * F;
    double* atbn = atb + n * FB;
    std::fill(o.tf.begin(), o.tf.end(), 0.0);
    std::fill(o.adv_tt.begin(), o.adv_tt.end(), 0.0);
    // advection_tracer_1_0: face transports, the U-point means times the
    // face lengths (tspas, centered) or times dxu / dyu before the mean (flux)
    const bool flux_faces = p.adv_tracer == LT_ADV_FLUX;
#pragma omp parallel for
    for (int k = 0; k < km; ++k)
      for (int j = 0; j < jmt; ++j)
        for (int i = 0; i < imt; ++i) {
          if (flux_faces) {
            if (i >= 1 && i < imt - 1)
              vs[C(k, j, i)] = (wkb[C(k, j, i)] * dxu[Q(j, i)] + wkb[C(k, j, i + 1)] * dxu[Q(j, i + 1)]) * 0.25;
            if (j >= 1 && j < jmt - 1)
              uw[C(k, j, i)] = (wkd[C(k, j - 1, i)] * dyu[Q(j - 1, i)] + wkd[C(k, j, i)] * dyu[Q(j, i)]) * 0.25;
          } else {
            if (i >= 1 && i < imt - 1) vs[C(k, j, i)] = (wkb[C(k, j, i)] + wkb[C(k, j, i + 1)]) * hts[Q(j, i)] * 0.25;
            if (j >= 1 && j < jmt - 1) uw[C(k, j, i)] = (wkd[C(k, j - 1, i)] + wkd[C(k, j, i)]) * htw[Q(j, i)] * 0.25;
          }
        }
    if (p.adv_tracer != LT_ADV_TSPAS) advect_simple(o, n, atn, uw, vs, ws, adv_tt, dg);
    else {
    // advection_tracer_2: predictor at00 and masked 7-point extrema
#pragma omp parallel for
    for (int k = 0; k < km; ++k)
      for (int j = 1; j < jmt - 1; ++j)
        for (int i = 1; i < imt - 1; ++i) {
          const long c = C(k, j, i), a = Q(j, i);
          const double tr = tarea_r[a];
          const double x0 = (atn[c + 1] + atn[c]) * uw[c + 1] * tr - (atn[c] + atn[c - 1]) * uw[c] * tr;
          const double y0 = ((atn[c + imt] + atn[c]) * vs[c] - (atn[c] + atn[c - imt]) * vs[c - imt]) * tr;
          const double xy1 = -dts * (atn[c + 1] - atn[c]) * 2.0 * tr * uw[c + 1] * uw[c + 1] / (htw[a + 1] * hun[a + 1]);
          const double xy2 = dts * (atn[c] - atn[c - 1]) * 2.0 * tr * uw[c] * uw[c] / (htw[a] * hun[a]);
          const double xy3 = -dts * (atn[c + imt] - atn[c]) * 2.0 * tr * vs[c] * vs[c] / (hts[a] * hue[a]);
          const double xy4 = dts * (atn[c] - atn[c - imt]) * 2.0 * tr * vs[c - imt] * vs[c - imt] / (hts[a - imt] * hue[a - imt]);
          const double cx = -atn[c] * (uw[c + 1] - uw[c]) * tr * 2.0;
          const double cy = -atn[c] * (vs[c] - vs[c - imt]) * tr * 2.0;
          double za, zb1, zb2, zc;
          if (k == 0) {
            za = -0.5 * odzp[0] * ws[A + a] * (atn[A + a] + atn[a]);
            zb1 = 0.0;
            zb2 = 0.5 * odzp[0] * ws[A + a] * ws[A + a] * odzt[1] * (atn[a] - atn[A + a]) * dts;
            zc = odzp[0] * atn[a] * ws[A + a];
          } else if (k == km - 1) {
            za = 0.5 * odzp[km - 1] * ws[c] * (atn[c] + atn[c - A]);
            zb1 = -0.5 * odzp[km - 1] * ws[c] * ws[c] * odzt[km - 1] * (atn[c - A] - atn[c]) * dts;
            zb2 = 0.0;
            zc = -odzp[km - 1] * atn[c] * ws[c];
          } else {
            za = 0.5 * odzp[k] * ws[c] * (atn[c] + atn[c - A]) - 0.5 * odzp[k] * ws[c + A] * (atn[c] + atn[c + A]);
            zb1 = -0.5 * odzp[k] * ws[c] * ws[c] * odzt[k] * (atn[c - A] - atn[c]) * dts;
            zb2 = 0.5 * odzp[k] * ws[c + A] * ws[c + A] * odzt[k + 1] * (atn[c] - atn[c + A]) * dts;
            zc = -odzp[k] * atn[c] * (ws[c] - ws[c + A]);
          }
          const double xx = -(x0 + xy1 + xy2 + cx);
          const double yy = -(y0 + xy3 + xy4 + cy);
          const double zz = -(zb1 + zb2 + za + zc);
          at00[c] = atn[c] + (xx + yy + zz) * dts;
          // masked extrema: land contributes -1e10 to the max, +1e10 to the min
          auto mx = [&](long q) { return atn[q] * vit[q] + (1.0 - vit[q]) * -1.0e10; };
          auto mn = [&](long q) { return atn[q] * vit[q] + (1.0 - vit[q]) * 1.0e10; };
          const long nb[4] = {c - imt, c + imt, c - 1, c + 1};
          double vmax = mx(c), vmin = mn(c);
          for (long q : nb) { const double v = mx(q); if (vmax < v) vmax = v; }
          for (long q : nb) { const double v = mn(q); if (vmin > v) vmin = v; }
          if (k == 0) {
            const double v = mx(c + A); if (vmax < v) vmax = v;
            const double w = mn(c + A); if (vmin > w) vmin = w;
          } else if (k == km - 1) {
            const double v = mx(c - A); if (vmax < v) vmax = v;
            const double w = mn(c - A); if (vmin > w) vmin = w;
          } else {
            const double v = mx(c - A); if (vmax < v) vmax = v;
            const double w = mn(c - A); if (vmin > w) vmin = w;
            const double v2 = mx(c + A); if (vmax < v2) vmax = v2;
            const double w2 = mn(c + A); if (vmin > w2) vmin = w2;
          }
          atmax[c] = vmax;
          atmin[c] = vmin;
        }
    // advection_tracer_3: limited fluxes (upwind where the predictor leaves
    // the local bounds at this cell or the neighbour across the face)
#pragma omp parallel for
    for (int k = 0; k < km; ++k)
      for (int j = 1; j < jmt - 1; ++j)
        for (int i = 1; i < imt - 1; ++i) {
          const long c = C(k, j, i), a = Q(j, i);
          const double tr = tarea_r[a];
          auto out = [&](long q) { return at00[q] > atmax[q] || at00[q] < atmin[q]; };
          const bool self = out(c);
          const bool edge_k = (k == 0 || k == km - 1);
          // horizontal faces: at the top and bottom level the neighbour test is
          // guarded alone; at inner levels the guard covers the whole test
          auto lim = [&](long q, bool guard) { return edge_k ? (self || (out(q) && guard)) : ((self || out(q)) && guard); };
          double xy1, xy2, xy3, xy4, zb1, zb2;
          if (lim(c + 1, i <= imt - 3)) xy1 = -(atn[c + 1] - atn[c]) * std::fabs(uw[c + 1]) * tr;
          else xy1 = -dts * (atn[c + 1] - atn[c]) * 2.0 * tr * uw[c + 1] * uw[c + 1] / (htw[a + 1] * hun[a + 1]);
          if (lim(c - 1, i >= 2)) xy2 = (atn[c] - atn[c - 1]) * std::fabs(uw[c]) * tr;
          else xy2 = dts * (atn[c] - atn[c - 1]) * 2.0 * tr * uw[c] * uw[c] / (htw[a] * hun[a]);
          if (lim(c + imt, j <= jmt - 3)) xy3 = -(atn[c + imt] - atn[c]) * std::fabs(vs[c]) * tr;
          else xy3 = -dts * (atn[c + imt] - atn[c]) * 2.0 * tr * vs[c] * vs[c] / (hts[a] * hue[a]);
          if (lim(c - imt, j >= 2)) xy4 = (atn[c] - atn[c - imt]) * std::fabs(vs[c - imt]) * tr;
          else xy4 = dts * (atn[c] - atn[c - imt]) * 2.0 * tr * vs[c - imt] * vs[c - imt] / (hts[a - imt] * hue[a - imt]);
          double za, zc;
          if (k == 0) {
            zb1 = 0.0;
            if (self || (out(c + A) && k <= km - 2)) zb2 = 0.5 * std::fabs(ws[c + A]) * odzp[k] * (atn[c] - atn[c + A]);
            else zb2 = 0.5 * odzp[0] * ws[A + a] * ws[A + a] * odzt[1] * (atn[a] - atn[A + a]) * dts;
            za = -0.5 * odzp[0] * ws[A + a] * (atn[A + a] + atn[a]);
            zc = odzp[0] * atn[a] * ws[A + a];
          } else if (k == km - 1) {
            if (self || out(c - A)) zb1 = -0.5 * std::fabs(ws[c]) * odzp[k] * (atn[c - A] - atn[c]);
            else zb1 = -0.5 * odzp[k] * ws[c] * ws[c] * odzt[k] * (atn[c - A] - atn[c]) * dts;
            zb2 = 0.0;
            za = 0.5 * odzp[km - 1] * ws[c] * (atn[c] + atn[c - A]);
            zc = -odzp[km - 1] * atn[c] * ws[c];
          } else {
            if ((self || out(c - A)) && k >= 1) zb1 = -0.5 * std::fabs(ws[c]) * odzp[k] * (atn[c - A] - atn[c]);
            else zb1 = -0.5 * odzp[k] * ws[c] * ws[c] * odzt[k] * (atn[c - A] - atn[c]) * dts;
            if ((self || out(c + A)) && k <= km - 2) zb2 = 0.5 * std::fabs(ws[c + A]) * odzp[k] * (atn[c] - atn[c + A]);
            else zb2 = 0.5 * odzp[k] * ws[c + A] * ws[c + A] * odzt[k + 1] * (atn[c] - atn[c + A]) * dts;
            za = 0.5 * odzp[k] * ws[c] * (atn[c] + atn[c - A]) - 0.5 * odzp[k] * ws[c + A] * (atn[c] + atn[c + A]);
            zc = -odzp[k] * atn[c] * (ws[c] - ws[c + A]);
          }
          const double cx = -atn[c] * (uw[c + 1] - uw[c]) * tr * 2.0;
          const double cy = -atn[c] * (vs[c] - vs[c - imt]) * tr * 2.0;
          const double x0 = (atn[c + 1] + atn[c]) * uw[c + 1] * tr - (atn[c] + atn[c - 1]) * uw[c] * tr;
          const double y0 = ((atn[c + imt] + atn[c]) * vs[c] - (atn[c] + atn[c - imt]) * vs[c - imt]) * tr;
          const double xx = -(x0 + xy1 + xy2 + cx);
          const double yy = -(y0 + xy3 + xy4 + cy);
          const double zz = -(za + zb1 + zb2 + zc);
          adv_tt[c] = xx + yy + zz;
          if (dg) {
            ax[n * F + c] = xx;
            ay[n * F + c] = yy;
            az[n * F + c] = zz;
          }
        }
    }  // tspas
    // tracer_del4_1: first masked Laplacian of atb, scaled by ahf
    std::fill(o.d2tk.begin(), o.d2tk.end(), 0.0);
    auto lap = [&](const double* fld, long c, long a, int k) {
      double h = 0.0, cc = 0.0;
      if (k <= kmt[a] - 1) {
        if (k <= kmtn[a] - 1) { h += dtn[a] * fld[c - imt]; cc -= dtn[a]; }
        if (k <= kmts[a] - 1) { h += dts_c[a] * fld[c + imt]; cc -= dts_c[a]; }
        if (k <= kmte[a] - 1) { h += dte[a] * fld[c + 1]; cc -= dte[a]; }
        if (k <= kmtw[a] - 1) { h += dtw[a] * fld[c - 1]; cc -= dtw[a]; }
      }
      return std::pair<double, double>(h, cc);
    };
#pragma omp parallel for
    for (int k = 0; k < km; ++k)
      for (int j = 1; j < jmt - 1; ++j)
        for (int i = 1; i < imt - 1; ++i) {
          const long c = C(k, j, i), a = Q(j, i);
          const double* lvl = atbn + A;  // tracer level k lives at atb level k+1
          auto hc = lap(lvl, c, a, k);
          d2tk[c] = ahf[a] * (hc.second * lvl[c] + hc.first);
        }
    // tracer_del4_2: advective tendency, surface mixing floor, second Laplacian
    double* aktn = akt + n * F;
#pragma omp parallel for
    for (int k = 0; k < km; ++k)
      for (int j = 1; j < jmt - 1; ++j)
        for (int i = 1; i < imt - 1; ++i) {
          const long c = C(k, j, i), a = Q(j, i);
          const bool inner = (j >= 2 && j < jmt - 2 && i >= 2 && i < imt - 2);
          if (inner) tf[c] = adv_tt[c] * vit[c];
          if (n == 0 && aktn[a] < p.dwndmix) aktn[a] = p.dwndmix;
          wkc[c] = aktn[c];
          auto hc = lap(d2tk, c, a, k);
          const double h = inner ? p.ah * (hc.second * d2tk[c] + hc.first) : 0.0;
          tf[c] += h;
        }
    // tracer_5: shortwave penetration (T), explicit half of vertical
    // diffusion (aidif = 0.5), salt surface flux (S)
    const double aidif = 0.5;
#pragma omp parallel for
    for (int j = 2; j < jmt - 2; ++j)
      for (int i = 2; i < imt - 2; ++i) {
        const long a = Q(j, i);
        if (n == 0) {
          for (int k = 1; k < km - 1; ++k) {
            const long c = C(k, j, i);
            const double w1 = swv[a] * pen[k - 1] * vit[c];
            const double w2 = swv[a] * pen[k] * vit[c + A];
            tf[c] = tf[c] + (w1 - w2) * odzp[k];
            if (dg) penetrate[c] = (w1 - w2) * odzp[k];
          }
          const double w1 = swv[a] * pen[0] * vit[A + a];
          const double w2 = swv[a] * pen[km - 2] * vit[(km - 1) * A + a];
          tf[a] = tf[a] - odzp[0] * w1;
          tf[(km - 1) * A + a] = tf[(km - 1) * A + a] + odzp[km - 1] * w2;
          if (dg) {
            penetrate[a] = -w1 * odzp[0];
            penetrate[(km - 1) * A + a] = w2 * odzp[km - 1];
          }
        }
        for (int k = 1; k < km - 1; ++k) {
          const long c = C(k, j, i);
          const double w1 = wkc[c - A] * (atbn[c] - atbn[c + A]) * odzt[k] * vit[c];
          const double w2 = wkc[c] * (atbn[c + A] - atbn[c + 2 * A]) * odzt[k + 1] * vit[c + A];
          tf[c] = tf[c] + odzp[k] * (w1 - w2) * 0.5;
          if (dg) dzd[n * F + c] = odzp[k] * (w1 - w2) * 0.5;
        }
        const double w1 = wkc[a] * (atbn[A + a] - atbn[2 * A + a]) * odzt[1] * vit[A + a];
        const double w2 = wkc[(km - 2) * A + a] * (atbn[(km - 1) * A + a] - atbn[km * A + a]) * odzt[km - 1] *
                          vit[(km - 1) * A + a];
        tf[a] = tf[a] - odzp[0] * w1 * 0.5;
        tf[(km - 1) * A + a] = tf[(km - 1) * A + a] + odzp[km - 1] * w2 * (1.0 - aidif);
        if (dg) {
          dzd[n * F + a] = -odzp[0] * w1 * 0.5;
          dzd[n * F + (km - 1) * A + a] = odzp[km - 1] * w2 * 0.5;
        }
      }
    if (n == 1) {
      const double* atbS_top = atb + FB + A;   // S at the surface, previous time level
      for (int j = 0; j < jmt; ++j)
        for (int i = 0; i < imt; ++i) {
          const long a = Q(j, i);
          if (kmt[a] > 0) {
            stf[a] = fresh[a] * 34.7 * p.od0 / 1000.0 + p.gamma * (sss[a] - atbS_top[a]) * seaice[a] / odzp[0] +
                     p.gamma * 30.0 / 365.0 / 4.0 * 50.0 * (sss[a] - atbS_top[a]) / odzp[0] * (1.0 - seaice[a]);
            tf[a] = tf[a] + stf[a] * (1.0 - aidif) * odzp[0];
            net[A + a] = stf[a] * odzp[0];
          }
          temp11[a] = tarea[a] * net[A + a] * vit[a];
        }
    }
    // SSS normalisation: global salt flux removed uniformly (mpi3.F90:26)
    double err_norm2 = 0.0;
    if (n == 1) {
      double err_norm1 = 0.0;
      if (o.tree_sum) {
        std::vector<double> terms;
        terms.reserve((size_t)(jmt - 4) * (imt - 4));
        for (int j = 2; j < jmt - 2; ++j)
          for (int i = 2; i < imt - 2; ++i) terms.push_back(temp11[Q(j, i)]);
        err_norm1 = device_tree_sum(terms);
      } else {
        for (int j = 2; j < jmt - 2; ++j)
          for (int i = 2; i < imt - 2; ++i) err_norm1 = err_norm1 + temp11[Q(j, i)];
      }
      err_norm2 = -err_norm1 / p.area_t;
      o.fw_norm2 = err_norm2;
    }
    // tracer_6: SSS norm (S); heat flux, its half-step tendency and net (T)
    for (int j = 0; j < jmt; ++j)
      for (int i = 0; i < imt; ++i) {
        const long a = Q(j, i);
        if (n == 1) {
          tf[a] = tf[a] + err_norm2 * vit[a];
        } else if (kmt[a] > 0) {
          stf[a] = ((swv[a] + nswv[a]) * p.od0cp + seaice[a] * p.gamma * (sst[a] - atb[A + a]) / odzp[0]);
          tf[a] = tf[a] + stf[a] * odzp[0] * 0.5;
          net[a] = stf[a] * odzp[0];
        }
      }
    halo_r8(net, 2, imt, jmt, o.ew_cyclic, o.tripole);
    // tracer_7: nudging (simple_assm) and restoring (boundary_restore)
    tracer7(p, n, imt, jmt, km, tf, vit, atb + n * FB, restore, restore_at, dt_restore);
    // tracer_8: explicit update into vtl (used as scratch), copy to ori
#pragma omp parallel for
    for (int k = 0; k < km; ++k)
      for (int j = 0; j < jmt; ++j)
        for (int i = 0; i < imt; ++i) {
          const long c = C(k, j, i);
          if (j >= 2 && j < jmt - 2 && i >= 2 && i < imt - 2) vtl[c] = atn[c] + dts * tf[c];
          ori[c] = vtl[c];
        }
    // invtrit: implicit half of vertical diffusion, Thomas sweep per column
#pragma omp parallel for
    for (int j = 2; j < jmt - 2; ++j) {
      std::vector<double> a8(km), b8(km), c8(km), d8(km), e8(km + 1), f8(km + 1);
      for (int i = 2; i < imt - 2; ++i) {
        const long a = Q(j, i);
        const int kz = kmt[a];
        if (kz <= 0) continue;
        for (int k = 1; k < kz; ++k) {
          a8[k] = wkc[(k - 1) * A + a] * odzt[k] * odzp[k] * dts * 0.5;
          d8[k] = vtl[k * A + a];
        }
        for (int k = 1; k < kz - 1; ++k) {
          c8[k] = wkc[k * A + a] * odzt[k + 1] * odzp[k] * dts * 0.5;
          b8[k] = 1.0 + a8[k] + c8[k];
          e8[k] = 0.0;
          f8[k] = 0.0;
        }
        a8[0] = odzp[0] * dts * 0.5;
        c8[0] = wkc[a] * odzt[1] * odzp[0] * dts * 0.5;
        b8[0] = 1.0 + c8[0];
        d8[0] = vtl[a];
        e8[0] = 0.0;
        f8[0] = 0.0;
        b8[kz - 1] = 1.0 + a8[kz - 1];
        c8[kz - 1] = odzp[kz - 1] * dts * 0.5;
        e8[kz] = 0.0;
        f8[kz] = 0.0;
        for (int k = kz - 1; k >= 0; --k) {
          const double g0 = 1.0 / (b8[k] - c8[k] * e8[k + 1]);
          e8[k] = a8[k] * g0;
          f8[k] = (d8[k] + c8[k] * f8[k + 1]) * g0;
        }
        vtl[a] = (e8[0] * stf[a] + f8[0]) * vit[a];
        for (int k = 1; k < kz; ++k) vtl[k * A + a] = (e8[k] * vtl[(k - 1) * A + a] + f8[k]) * vit[k * A + a];
      }
    }
    halo_r8(vtl, km, imt, jmt, o.ew_cyclic, o.tripole);
    // tracer_9: diagnostics and state update (all points incl. ghosts)
#pragma omp parallel for
    for (int k = 0; k < km; ++k)
      for (int j = 0; j < jmt; ++j)
        for (int i = 0; i < imt; ++i) {
          const long c = C(k, j, i), a = Q(j, i);
          if (dg) {
            if (k == 0) dt_diff[n * F + c] = (vtl[c] - ori[c]) / dts * vit[c] - stf[a] * 0.5 * odzp[0];
            else dt_diff[n * F + c] = (vtl[c] - ori[c]) / dts * vit[c];
            tend[n * F + c] = (vtl[c] - at[n * F + c]) / dts * vit[c];
          }
          at[n * F + c] = vtl[c];
          atbn[c + A] = at[n * F + c];
        }
  }
}

// convadj_cu: per-column convective adjustment (convadj.cpp:29-288)
void convadj_call(Oracle& o) {
  o.ensure_all();
  const int km = o.km, imt = o.imt, jmt = o.jmt;
  const long A = o.A, F = o.F, FB = o.FB;
  double* at = o.fd[LT_F_AT].data();
  double* atb = o.fd[LT_F_ATB].data();
  double* tend = o.fd[LT_F_TEND].data();
  double* dt_conv = o.fd[LT_F_DT_CONV].data();
  const double* to = o.fd[LT_F_TO].data();
  const double* so = o.fd[LT_F_SO].data();
  const double* cc = o.fd[LT_F_C].data();
  const double* dzp = o.fd[LT_F_DZP].data();
  const int* kmt = o.fi[LT_F_KMT].data();
  const double c2dtts = o.p.dts;
  auto rho = [&](double t, double s, int l) {  // l: 0-based level of the coefficients
    return (cc[l] + (cc[3 * km + l] + cc[6 * km + l] * s) * s + (cc[2 * km + l] + cc[7 * km + l] * s + cc[5 * km + l] * t) * t) * t +
           (cc[1 * km + l] + (cc[4 * km + l] + cc[8 * km + l] * s) * s) * s;
  };
#pragma omp parallel for
  for (int j = 0; j < jmt; ++j) {
    std::vector<double> rhoup(km, 0.0), rholo(km, 0.0);
    for (int i = 0; i < imt; ++i) {
      const long a = (long)j * imt + i;
      auto T = [&](int l) -> double& { return at[(long)l * A + a]; };       // l 0-based level
      auto S = [&](int l) -> double& { return at[F + (long)l * A + a]; };
      const int kcon = kmt[a];
      std::fill(rhoup.begin(), rhoup.end(), 0.0);
      std::fill(rholo.begin(), rholo.end(), 0.0);
      if (kcon != 0) {
        int lcon = 0;
        for (int l = 0; l < km - 1; ++l) {
          const int l1 = l + 1;
          rhoup[l1] = rho(T(l1) - to[l1], S(l1) - so[l1], l1);
          rholo[l] = rho(T(l) - to[l1], S(l) - so[l1], l1);
        }
        for (int k = kcon - 1; k >= 1; --k)
          if (rholo[k - 1] > rhoup[k]) lcon = k;
        if (lcon != 0) {
          // levels below are 1-based as in the reference's mixing loops
          for (;;) {
            int lcona = lcon, lconb = lcon + 1;
            double dztsum = dzp[lcona - 1] + dzp[lconb - 1];
            double trasum[2];
            for (int n = 0; n < 2; ++n) {
              double* X = at + n * F;
              trasum[n] = X[(long)(lcona - 1) * A + a] * dzp[lcona - 1] + X[(long)(lconb - 1) * A + a] * dzp[lconb - 1];
              const double tramix = trasum[n] / dztsum;
              X[(long)(lcona - 1) * A + a] = tramix;
              X[(long)(lconb - 1) * A + a] = tramix;
            }
            for (;;) {  // grow the mixed layer down or up while unstable
              if (lconb != kcon) {
                const int l1 = lconb + 1;
                rholo[lconb - 1] = rho(T(lconb - 1) - to[l1 - 1], S(lconb - 1) - so[l1 - 1], l1 - 1);
                if (rholo[lconb - 1] > rhoup[l1 - 1]) {
                  lconb = lconb + 1;
                  dztsum = dztsum + dzp[lconb - 1];
                  for (int n = 0; n < 2; ++n) {
                    double* X = at + n * F;
                    trasum[n] = trasum[n] + X[(long)(lconb - 1) * A + a] * dzp[lconb - 1];
                    const double tramix = trasum[n] / dztsum;
                    for (int lm = lcona - 1; lm < lconb; ++lm) X[(long)lm * A + a] = tramix;
                  }
                  continue;
                }
              }
              if (lcona > 1) {
                const int l1 = lcona - 1;
                rholo[l1 - 1] = rho(T(l1 - 1) - to[lcona - 1], S(l1 - 1) - so[lcona - 1], lcona - 1);
                rhoup[lcona - 1] = rho(T(lcona - 1) - to[lcona - 1], S(lcona - 1) - so[lcona - 1], lcona - 1);
                if (rholo[lcona - 2] > rhoup[lcona - 1]) {
                  lcona = lcona - 1;
                  dztsum = dztsum + dzp[lcona - 1];
                  for (int n = 0; n < 2; ++n) {
                    double* X = at + n * F;
                    trasum[n] = trasum[n] + X[(long)(lcona - 1) * A + a] * dzp[lcona - 1];
                    const double tramix = trasum[n] / dztsum;
                    for (int lm = lcona; lm <= lconb; ++lm) X[(long)(lm - 1) * A + a] = tramix;
                  }
                  continue;
                }
              }
              break;
            }
            if (lconb == kcon) break;
            lcon = lconb;
            bool done = false;
            for (;;) {  // search deeper for the next unstable interface
              lcon = lcon + 1;
              if (lcon == kcon) { done = true; break; }
              if (rholo[lcon - 1] <= rhoup[lcon]) continue;
              break;
            }
            if (done) break;
          }
        }
      }
      // (convadj.cpp:258-276) tendency diagnostics and atb = at, for every column
      for (int n = 0; n < 2; ++n)
        for (int k = 0; k < km; ++k) {
          const long c = n * F + (long)k * A + a;
          const double vitk = (k < kmt[a]) ? 1.0 : 0.0;
          dt_conv[c] = (at[c] - atb[n * FB + (long)(k + 1) * A + a]) / c2dtts * vitk;
          tend[c] += dt_conv[c];
          atb[n * FB + (long)(k + 1) * A + a] = at[c];
        }
    }
  }
}

// icesnow_cu over every point of the domain, halo included, with the
// FRC_CORE reset of licomqice first when reset is set (icesnow.cpp:15-85)
void icesnow_call(Oracle& o, const lt_icesnow_params& p) {
  o.ensure_all();
  double* at = o.fd[LT_F_AT].data();
  double* qice = o.fd[LT_F_QICE].data();
  const int* kmt = o.fi[LT_F_KMT].data();
  const double* dzp = o.fd[LT_F_DZP].data();
  const double sal_ocn = 34.7e0, sal_ice = 4.0e0;
  if (p.reset_qice) std::fill(o.fd[LT_F_QICE].begin(), o.fd[LT_F_QICE].end(), 0.0);
  for (long c = 0; c < o.A; ++c) {
    double& t = at[c];
    double& s = at[o.F + c];
    if (t < p.tbice && kmt[c] > 0) {
      const double tdiff = p.tbice - t;
      qice[c] += tdiff * dzp[0] / dzp[0];
      s += tdiff * (sal_ocn - sal_ice) * p.cp / p.latice * 0.001e0;
      t = p.tbice;
    }
    if (qice[c] > 0 && t > p.tbice) {
      const double tdiff = std::fmin(t - p.tbice, qice[c]);
      qice[c] -= tdiff;
      t -= tdiff;
      s -= tdiff * (sal_ocn - sal_ice) * p.cp / p.latice * 0.001e0;
    }
    for (int k = 0; k < o.km; ++k)
      if (at[(long)k * o.A + c] < p.tbice) at[(long)k * o.A + c] = p.tbice;
  }
}


// ---- Canuto turbulence closure (readyc.cpp:880-1612), TIDEMIX configuration.
// Table sizes of canuto_mod.h; constants of pconst_mod.h:242-247.
namespace turb {
constexpr int mt = LT_TURB_MT, mt0 = LT_TURB_MT0, nth = LT_TURB_NTHETA;
constexpr double back_tidalmixing = 1.0e-6, max_tidalmixing = 1.0e-2, mixing_ef = 0.20,
                 local_mixing_fraction = 0.33;
constexpr double epson2__ = 0.288e0, eplatidependmin = 7.0e-2, s2min = 1.0e-14;

inline double sgn(double x, double y) { return y >= 0.0e0 ? std::fabs(x) : -std::fabs(x); }
inline int sgn_i(int x, int y) { return y >= 0 ? std::abs(x) : -std::abs(x); }

// eplatidepend_fun with wavelat (readyc.cpp:880-896)
double eplat(double f, double an) {
  const double an0 = 5.24e-3;
  const double f_30 = 4.0e0 * std::atan(1.0e0) / 43082.0e0;
  const double den = f_30 * std::acosh(an0 / f_30);
  const double anum = f * std::acosh(an / f);
  return anum / den;
}

// formld (readyc.cpp:902-913)
void formld(int n, const double* z, const double* t, double* amld) {
  for (int k = 0; k < n; k++) {
    if (std::fabs(t[k] - t[0]) > 0.1) {
      const double tm = t[0] - sgn(0.1e0, t[0] - t[k]);
      *amld = z[k] + (z[k - 1] - z[k]) * (tm - t[k]) / (t[k - 1] - t[k] + 1.0e-20);
      return;
    }
  }
  *amld = z[n - 1];
}

// interp1d_expabs (readyc.cpp:915-973)
void interp1d(double x, const double* x_1, const double* slq2_1, const double* sm_1, const double* sh_1,
              const double* ss_1, double* slq2, double* sm, double* sh, double* ss, double delta, double rat) {
  int lx0, lx1;
  if (x > x_1[2 * mt]) x = x_1[2 * mt];
  else if (x < x_1[0]) x = x_1[0];
  if (std::fabs(x) >= x_1[mt + mt0] && std::fabs(x) >= x_1[2 * mt]) {
    lx0 = (int)sgn((double)mt, x);
    lx1 = lx0;
  } else {
    if (std::fabs(x) < x_1[mt + mt0]) {
      lx1 = (int)(x / delta) + (int)sgn(1.0, x);
    } else {
      const double tabindx = sgn((double)mt0 + ((std::log(std::fabs(x)) - std::log(x_1[mt + mt0])) / std::log(rat)), x);
      lx1 = (int)tabindx + (int)sgn(1.0, x);
    }
    lx1 = std::max(-mt, std::min(mt, lx1));   // the reference reads past its table here
    if (std::fabs(x_1[mt + lx1]) < std::fabs(x)) lx1 += sgn_i(1, lx1);
    else if (std::fabs(x_1[mt + lx1 - sgn_i(1, lx1)]) > std::fabs(x)) lx1 += -sgn_i(1, lx1);
    lx0 = lx1 - (int)sgn(1.0, x);
    if (std::fabs(x) <= 0.0e0) lx1 = 1;
  }
  if ((x > 0.0e0 && (x < x_1[mt + lx0] || x > x_1[mt + lx1])) ||
      (x < 0.0e0 && (x > x_1[mt + lx0] || x < x_1[mt + lx1])))
    return;
  const double deltaxta = x_1[mt + lx1] - x_1[mt + lx0];
  const double deltax = x - x_1[mt + lx0];
  double dslq2_x, dsm_x, dsh_x, dss_x;
  if (lx1 == lx0) {
    dslq2_x = dsm_x = dsh_x = dss_x = 0.0e0;
  } else {
    dslq2_x = (slq2_1[mt + lx1] - slq2_1[mt + lx0]) / deltaxta;
    dsm_x = (sm_1[mt + lx1] - sm_1[mt + lx0]) / deltaxta;
    dsh_x = (sh_1[mt + lx1] - sh_1[mt + lx0]) / deltaxta;
    dss_x = (ss_1[mt + lx1] - ss_1[mt + lx0]) / deltaxta;
  }
  *slq2 = slq2_1[mt + lx0] + dslq2_x * deltax;
  *sm = sm_1[mt + lx0] + dsm_x * deltax;
  *sh = sh_1[mt + lx0] + dsh_x * deltax;
  *ss = ss_1[mt + lx0] + dss_x * deltax;
}

// index search of interp2d_expabs for one coordinate; false if x is not
// bracketed (the reference returns)
bool index2d(double x, const lt_turb_tables& T, int* l0, int* l1) {
  const double* rib = T.rib;
  const double tmp = rib[mt + mt0], tmp1 = rib[2 * mt];
  if (std::fabs(x) >= tmp && std::fabs(x) >= tmp1) {
    *l0 = (int)sgn((double)mt, x);
    *l1 = *l0;
  } else {
    if (std::fabs(x) < tmp) {
      *l1 = (int)(x / T.dri) + (int)sgn(1.0, x);
    } else {
      const double ti = sgn((double)mt0 + ((std::log(std::fabs(x)) - std::log(tmp)) / std::log(T.rri)), x);
      *l1 = (int)ti + (int)sgn(1.0, x);
    }
    *l1 = std::max(-mt, std::min(mt, *l1));   // the reference reads past its table here
    if (std::fabs(rib[mt + *l1]) < std::fabs(x)) *l1 += sgn_i(1, *l1);
    else if (std::fabs(rib[mt + *l1 - sgn_i(1, *l1)]) > std::fabs(x)) *l1 += -sgn_i(1, *l1);
    *l0 = *l1 - (int)sgn(1.0, x);
    if (x == 0.0e0) *l1 = 1;
  }
  return !((x > 0.0e0 && (x < rib[mt + *l0] || x > rib[mt + *l1])) ||
           (x < 0.0e0 && (x > rib[mt + *l0] || x < rib[mt + *l1])));
}

// interp2d_expabs (readyc.cpp:975-1114)
void interp2d(double* ri, double* rid, double* slq2, double* sm, double* sh, double* ss, const lt_turb_tables& T) {
  const double* rib = T.rib;
  if (*ri > rib[2 * mt]) {
    if (std::fabs(*rid) <= *ri) { *rid = rib[2 * mt] * (*rid / *ri); *ri = rib[2 * mt]; }
    else if (*rid > *ri) { *ri = rib[2 * mt] * (*ri / *rid); *rid = rib[2 * mt]; }
    else if (*rid < -*ri) { *ri = rib[0] * (*ri / *rid); *rid = rib[0]; }
  } else if (*ri < rib[0]) {
    if (std::fabs(*rid) <= -*ri) { *rid = rib[0] * (*rid / *ri); *ri = rib[0]; }
    else if (*rid > -*ri) { *ri = rib[2 * mt] * (*ri / *rid); *rid = rib[2 * mt]; }
    else if (*rid < *ri) { *ri = rib[0] * (*ri / *rid); *rid = rib[0]; }
  } else if (*rid > rib[2 * mt]) {
    *ri = rib[2 * mt] * (*ri / *rid);
    *rid = rib[2 * mt];
  } else if (*rid < rib[0]) {
    *ri = rib[0] * (*ri / *rid);
    *rid = rib[0];
  }
  const double ri_tmp = *ri, rid_tmp = *rid;
  int lrid0, lrid1, lri0, lri1;
  if (!index2d(rid_tmp, T, &lrid0, &lrid1)) return;
  if (ri_tmp > std::fmin(rib[mt + T.irimax[mt + lrid0]], rib[mt + T.irimax[mt + lrid1]])) {
    *slq2 = 0.0e0; *sm = 0.0e0; *sh = 0.0e0; *ss = 0.0e0;
    return;
  }
  if (!index2d(ri_tmp, T, &lri0, &lri1)) return;
  const long w = 2 * mt + 1;
  const long c00 = w * (lrid0 + mt) + lri0 + mt, c10 = w * (lrid1 + mt) + lri0 + mt, c01 = w * (lrid0 + mt) + lri1 + mt;
  const double deltaridta = rib[mt + lrid1] - rib[mt + lrid0];
  const double deltarita = rib[mt + lri1] - rib[mt + lri0];
  const double deltarid = rid_tmp - rib[mt + lrid0];
  const double deltari = ri_tmp - rib[mt + lri0];
  const double* tb[4] = {T.slq2b, T.smb, T.shb, T.ssb};
  double* out[4] = {slq2, sm, sh, ss};
  for (int m = 0; m < 4; ++m) {
    double d_rid = 0.0e0, d_ri = 0.0e0;
    if (lrid1 != lrid0) {
      d_rid = (tb[m][c10] - tb[m][c00]) / deltaridta;
      d_ri = (tb[m][c01] - tb[m][c00]) / deltarita;
    }
    *out[m] = tb[m][c00] + d_ri * deltari + d_rid * deltarid;
  }
}

// turb_device (readyc.cpp:1116-1455) on one column's work arrays; the two
// locals the reference can read unset start at zero
void turb_device(const double* z, const double* t, const double* rh, const double* ri, const double* rid, double* s2,
                 double fricmx, double wndmix, const double* an2, double buoytur, double buoysol, double coriol,
                 double* amld, double* akm, double* akh, double* aks, int n, int nmax, const lt_turb_tables& T) {
  const double b1 = T.b1;
  double v_back, t_back, s_back;
  double al2, tmp = 0.0, slq2 = 0.0, sm = 0.0, ss = 0.0, sh = 0.0;
  double amtaun2 = 0.0;
  double back_ri1 = 0.0e0;
  double sh_back = 0.0, slq2_back = 0.0, sm_back = 0.0, ss_back = 0.0;
  double epson2;
  const int nb = n > 0 ? n : 0;
  const double buoytot = buoytur + buoysol;
  if (n > 0) formld(n, z, t, amld);
  else if (n == 0) *amld = z[0];
  else *amld = 0.0e0;
  const double al0 = 0.17 * *amld;
  double ifbelow = 0;
  double an = 0.0;
  for (int k = 0; k < n; k++) {
    double ifnofsmall = 0;
    if (an2[k] >= 0.0e0) an = std::sqrt(an2[k]);
    if (an < std::fabs(coriol)) ifnofsmall = 1;
    double ri1 = ri[k];
    double rid1 = rid[k];
    const double and2 = rid[k] / (ri[k] + 1.0e-25) * an2[k];
    const double and2on2 = and2 / (an2[k] + 1.0e-25);
    const int ifpureshear = (an2[k] < T.rib[0] * s2[k]) ? 1 : 0;
    if (ifpureshear == 1) {
      interp1d(and2on2, T.and2on2a1, T.amtaun2a1, T.sma1, T.sha1, T.ssa1, &amtaun2, &sm, &sh, &ss, T.dand2on2,
               T.rnd2on2);
      slq2 = (-amtaun2) / ((b1 * b1) * ri[k] + 1.0e-25);
    } else {
      interp2d(&ri1, &rid1, &slq2, &sm, &sh, &ss, T);
      if (slq2 < 0.0e0) return;
      if (slq2 == 0.0e0) ifbelow = 1;
    }
    const bool lifupper = ((ifbelow == 0 || ifnofsmall == 1 || ((ri1 < 0.0e0) && (k <= 1))) && (slq2 > 0.0e0));
    double epsy = 0.0e0;
    bool lifepsy = false;
    if (n > 0) {
      if (slq2 == 0.0e0) epsy = 0.0e0;
      else epsy = -buoytot / ((1.0e0 / ((b1 * b1) * (slq2))) - 0.5e0 * sm);
      lifepsy = ((epsy >= 0.0e0) && lifupper);
    }
    const double akz = 0.4 * z[k];
    const double al = akz * al0 / (al0 + akz);
    al2 = al * al;
    if (ifbelow != 1 && !lifepsy) {
      if (ri1 > 0.0e0) {
        const double anlq2 = slq2 * ri1;
        if (anlq2 > 0.281e0) {
          al2 *= 0.281e0 / anlq2;
          slq2 = 0.281e0 / (ri1 + 1.0e-20);
        }
      }
    }
    if (an2[k] < 0.0e0) {
      epson2 = epson2__;
    } else {
      double eplatidepend = (ifnofsmall == 1) ? 0.0e0 : eplat(std::fabs(coriol), an);
      eplatidepend = std::fmax(eplatidepend, eplatidependmin);
      epson2 = epson2__ * eplatidepend;
    }
    if (ri[k] > 0.0e0) {
      const double rit = (ri[k] + rid[k]) / 2.0e0;
      const double ric = (ri[k] - rid[k]) / 2.0e0;
      const double ra_r = std::sqrt((rit * rit) + (ric * ric));
      double theta_r;
      if (std::fabs(rit) <= 0.0e0) theta_r = (std::fabs(ric) <= 0.0e0) ? std::atan(1.0e0) : 2.0e0 * std::atan(1.0e0);
      else theta_r = std::atan(ric / rit);
      if (std::fabs(theta_r) > 2.0e0 * std::atan(1.0e0)) return;
      if (theta_r < -std::atan(1.0e0)) theta_r += 4.0e0 * std::atan(1.0e0);
      const int jtheta_r0 = (int)((theta_r + std::atan(1.0e0)) / T.deltheta_r);
      int itheta_r0 = jtheta_r0 - nth;
      int itheta_r1 = itheta_r0 + 1;
      double theta_r0 = itheta_r0 * T.deltheta_r;
      double theta_r1 = itheta_r1 * T.deltheta_r;
      if ((theta_r0 <= T.theta_rcrp) && (theta_r > T.theta_rcrp)) {
        theta_r = theta_r1; theta_r0 = theta_r1; itheta_r0 = itheta_r1; ++itheta_r1; theta_r1 += T.deltheta_r;
      } else if ((theta_r1 >= T.theta_rcrn) && (theta_r < T.theta_rcrn)) {
        theta_r = theta_r0; theta_r1 = theta_r0; itheta_r1 = itheta_r0; --itheta_r0; theta_r0 += -T.deltheta_r;
      }
      if ((itheta_r1 > 3 * nth) || (itheta_r0 < -nth)) return;
      double deltheta_r_1 = theta_r - theta_r0;
      const double delback_ra_r = T.back_ra_r[nth + itheta_r1] - T.back_ra_r[nth + itheta_r0];
      const double dback_ra_r_o_dtheta = delback_ra_r / T.deltheta_r;
      double back_ra_r1 = T.back_ra_r[nth + itheta_r0] + deltheta_r_1 * dback_ra_r_o_dtheta;
      int ifrafglt = 0;
      if ((theta_r <= T.theta_rcrp) || (theta_r >= T.theta_rcrn)) {
        if (back_ra_r1 > ra_r) { ifrafglt = 1; back_ra_r1 = ra_r; }
      }
      if (back_ra_r1 < 0.0e0) return;
      const double back_rit1 = std::cos(theta_r) * back_ra_r1;
      const double back_ric1 = std::sin(theta_r) * back_ra_r1;
      back_ri1 = back_rit1 + back_ric1;
      double back_rid1 = back_rit1 - back_ric1;
      if (ifrafglt == 1) {
        interp2d(&back_ri1, &back_rid1, &slq2_back, &sm_back, &sh_back, &ss_back, T);
      } else {
        deltheta_r_1 = theta_r - itheta_r0 * T.deltheta_r;
        sm_back = T.sm_r1[nth + itheta_r0] + deltheta_r_1 * ((T.sm_r1[nth + itheta_r1] - T.sm_r1[nth + itheta_r0]) / T.deltheta_r);
        sh_back = T.sh_r1[nth + itheta_r0] + deltheta_r_1 * ((T.sh_r1[nth + itheta_r1] - T.sh_r1[nth + itheta_r0]) / T.deltheta_r);
        ss_back = T.ss_r1[nth + itheta_r0] + deltheta_r_1 * ((T.ss_r1[nth + itheta_r1] - T.ss_r1[nth + itheta_r0]) / T.deltheta_r);
        slq2_back = T.slq2_r1[nth + itheta_r0] +
                    deltheta_r_1 * ((T.slq2_r1[nth + itheta_r1] - T.slq2_r1[nth + itheta_r0]) / T.deltheta_r);
      }
      if (slq2_back < 0.0e0) return;
    }
    if (ri[k] <= 0.0e0) back_ri1 = 0.0e0;
    if (ri1 <= 0.0e0) { sm_back = 0.0e0; sh_back = 0.0e0; ss_back = 0.0e0; }
    if ((sm_back < 0.0e0) || (sh_back < 0.0e0) || (ss_back < 0.0e0)) return;
    const double tmp_back = 0.5e0 * b1 * b1 * back_ri1 * slq2_back * epson2;
    v_back = tmp_back * sm_back;
    t_back = tmp_back * sh_back;
    s_back = tmp_back * ss_back;
    if ((v_back < 0.0e0) || (t_back < 0.0e0) || (s_back < 0.0e0)) return;
    if ((ri[k] > 0.0e0) && ((std::fabs(v_back) <= 0.0e0) || (std::fabs(t_back) <= 0.0e0) || (std::fabs(s_back) < 0.0e0)))
      return;
    if (ifbelow == 1) {
      if (ri1 >= 0.0e0) {
        tmp = 0.5e0 * b1 * b1 * ri1 * slq2 * epson2;
      } else if (k >= 2) {
        double delz, delrh, del2rh;
        if (k == n - 1) {
          delz = z[k] - z[k - 1]; delrh = rh[k] - rh[k - 1]; del2rh = rh[k] - 2.0e0 * rh[k - 1] + rh[k - 2];
        } else {
          delz = z[k + 1] - z[k - 1]; delrh = rh[k + 1] - rh[k - 1]; del2rh = rh[k + 1] - 2.0e0 * rh[k] + rh[k - 1];
        }
        const double dzrh = delrh / delz;
        const double d2zrh = 4.0e0 * del2rh / (delz * delz);
        const double rdzlndzrh = dzrh / d2zrh;
        const double al0deep = 0.17e0 * std::fabs(rdzlndzrh);
        const double akz2 = 0.4e0 * z[k];
        const double aldeep = akz2 * al0deep / (al0deep + akz2);
        al2 = aldeep * aldeep;
        if (ifpureshear != 1) {
          s2[k] = std::fmax(s2[k], s2min);
          tmp = 0.5e0 * b1 * al2 * std::sqrt(s2[k] / (slq2 + 1.0e-40));
        }
      } else if (ifpureshear != 1) {
        s2[k] = std::fmax(s2[k], s2min);
        if (lifepsy) tmp = 0.5e0 * epsy / (s2[k] + 1.0e-40);
        else tmp = 0.5e0 * b1 * al2 * std::sqrt(s2[k] / (slq2 + 1.0e-40));
      }
    } else if (ifpureshear != 1) {
      s2[k] = std::fmax(s2[k], s2min);
      if (lifepsy) tmp = 0.5e0 * epsy / (s2[k] + 1.0e-40);
      else tmp = 0.5e0 * b1 * al2 * std::sqrt(s2[k] / (slq2 + 1.0e-40));
    }
    if (ifpureshear == 1) tmp = 0.5e0 * (b1 * b1) * al2 * std::sqrt(-an2[k] / amtaun2);
    akm[k] = std::fmin(tmp * sm + v_back, fricmx);
    akh[k] = std::fmin(tmp * sh + t_back, fricmx);
    aks[k] = std::fmin(tmp * ss + s_back, fricmx);
  }
  for (int k = nb; k < nmax; k++) { akm[k] = 0.0e0; akh[k] = 0.0e0; aks[k] = 0.0e0; }
  if (n > 0) {
    if (akm[0] < wndmix) akm[0] = wndmix;
    if (akh[0] < wndmix) akh[0] = wndmix;
    if (aks[0] < wndmix) aks[0] = wndmix;
  }
}
}  // namespace turb

// turb_cu (readyc.cpp:1456-1612) with the memsets of readyc_ before it
// (readyc.cpp:1642, 1647, 1668-1671): every column of the interior ring
// (1 .. imt-2, 1 .. jmt-2) that has a wet top level
void turb_call(Oracle& o, const lt_turb_tables& T, int ncc, double dfricmx) {
  o.ensure_all();
  const int km = o.km, imt = o.imt, jmt = o.jmt;
  const long A = o.A, F = o.F;
  double* akmt = o.fd[LT_F_AKMT].data();
  double* akt = o.fd[LT_F_AKT].data();
  double* ak_tide = o.fd[LT_F_AK_TIDE].data();
  double* amld = o.fd[LT_F_AMLD].data();
  std::fill(o.fd[LT_F_AKMT].begin(), o.fd[LT_F_AKMT].end(), 0.0);
  std::fill(o.fd[LT_F_AK_TIDE].begin(), o.fd[LT_F_AK_TIDE].end(), 0.0);
  std::fill(o.fd[LT_F_AMLD].begin(), o.fd[LT_F_AMLD].end(), 0.0);
  const double* at = o.fd[LT_F_AT].data();
  const double* dzp = o.fd[LT_F_DZP].data();
  const double* zkp = o.fd[LT_F_ZKP].data();
  const double* pdensity = o.fd[LT_F_PDENSITY].data();
  const double* rit = o.fd[LT_F_RIT].data();
  const double* ricdttms = o.fd[LT_F_RICDTTMS].data();
  const double* s2t = o.fd[LT_F_S2T].data();
  const double* rict = o.fd[LT_F_RICT].data();
  const double* fz_tide = o.fd[LT_F_FZ_TIDE].data();
  const int* kmt = o.fi[LT_F_KMT].data();
  const int d_ncc = ncc;
  const double dwndmix = o.p.dwndmix;
#pragma omp parallel for schedule(dynamic, 4)
  for (int j = 1; j < jmt - 1; ++j) {
    std::vector<double> wp1(km), wp3(km), wp7(km), wp8(km), wp4(km), wp5(km), wp6(km), wk1(km), wk2(km), wk3(km);
    for (int i = 1; i < imt - 1; ++i) {
      const long tid = (long)j * imt + i;
      auto vit = [&](int k) { return k < kmt[tid] ? 1.0 : 0.0; };
      if (!(vit(0) > 0.5)) continue;
      const int iwk = kmt[tid] - 1;
      for (int k = 0; k < km; k++) {
        wp1[k] = wp3[k] = wp7[k] = wp8[k] = 0.0e0;
        wp4[k] = wp5[k] = wp6[k] = 0.0e0;
        wk1[k] = wk2[k] = wk3[k] = 0.0e0;
      }
      for (int k = 0; k < iwk; k++) {
        wp8[k] = -vit(k + 1) * zkp[k + 1] * 1.0e+2;
        wp1[k] = vit(k + 1) * (at[k * A + tid] - (at[k * A + tid] - at[(k + 1) * A + tid]) * dzp[k] / (dzp[k] + dzp[k + 1]));
      }
      for (int k = 0; k < iwk; k++) {
        wp4[k] = vit(k + 1) * rit[k * A + tid];
        wp5[k] = vit(k + 1) * ricdttms[k * A + tid];
        wp6[k] = vit(k + 1) * s2t[k * A + tid];
        wp7[k] = vit(k + 1) * rict[k * A + tid];
        wp3[k] = vit(k + 1) * (pdensity[k * A + tid] + (pdensity[(k + 1) * A + tid] - pdensity[k * A + tid]) * dzp[k] /
                                                          (dzp[k] + dzp[k + 1])) * 1.0e-3;
      }
      const double wp10 = vit(0) * o.fd[LT_F_BUOYTUR][tid] * 1.0e+4;
      const double wp11 = vit(0) * o.fd[LT_F_BUOYSOL][tid] * 1.0e+4;
      double mldtmp = 0.0;
      turb::turb_device(wp8.data(), wp1.data(), wp3.data(), wp4.data(), wp5.data(), wp6.data(), dfricmx * 1.0e+4,
                        dwndmix * 1.0e+4, wp7.data(), wp10, wp11, o.fd[LT_F_FCORT][tid], &mldtmp, wk1.data(),
                        wk2.data(), wk3.data(), iwk, km - 1, T);
      amld[tid] = mldtmp * 1.0e-2;
      for (int k = 0; k < iwk; k++) {
        ak_tide[k * A + tid] = turb::back_tidalmixing + turb::mixing_ef * turb::local_mixing_fraction *
                                                            o.fd[LT_F_WAVE_DIS][tid] * fz_tide[k * A + tid] /
                                                            (std::fmax(rict[k * A + tid], 1.0e-8) * (wp3[k] * 1000.0));
        if (ak_tide[k * A + tid] > turb::max_tidalmixing) ak_tide[k * A + tid] = turb::max_tidalmixing;
        o.fd[LT_F_RICHARDSON][k * A + tid] = rict[k * A + tid];
        o.fd[LT_F_FZTIDAL][k * A + tid] = fz_tide[k * A + tid];
        o.fd[LT_F_WP3_TIDAL][k * A + tid] = wp3[k];
      }
      for (int k = iwk - 2; k >= 0; k--) ak_tide[k * A + tid] = std::fmin(ak_tide[k * A + tid], ak_tide[(k + 1) * A + tid]);
      for (int k = 0; k < km - 1; k++) {
        akmt[k * A + tid] = wk1[k] * 1.0e-4 + ak_tide[k * A + tid] * 5.0;
        akt[k * A + tid] = (wk2[k] * 1.0e-4 + ak_tide[k * A + tid]) / (float)d_ncc;
        akt[F + k * A + tid] = (wk3[k] * 1.0e-4 + ak_tide[k * A + tid]) / (float)d_ncc;
      }
    }
  }
}

// readyc_'s BIHAR sequence (readyc.cpp:1754-1775) kernel by kernel over the
// whole domain, one block (ib = jb = 3, ie = imt-2, je = jmt-2)
void del4u_call(Oracle& o, double am, double c0f) {
  o.ensure_all();
  const int km = o.km, imt = o.imt, jmt = o.jmt;
  const long A = o.A, F = o.F;
  const int ib = 3, jb = 3, ie = imt - 2, je = jmt - 2;
  const double p5 = 0.5;
  const double* up = o.fd[LT_F_UP].data();
  const double* vp = o.fd[LT_F_VP].data();
  double* dlu = o.fd[LT_F_DLU].data();
  double* dlv = o.fd[LT_F_DLV].data();
  double* wkad = o.fd[LT_F_WKA_DRAG].data();
  const int* kmt = o.fi[LT_F_KMT].data();
  const int* kmu = o.fi[LT_F_KMU].data();
  const double *htw = o.fd[LT_F_HTW].data(), *hts = o.fd[LT_F_HTS].data(), *tarea_r = o.fd[LT_F_TAREA_R].data();
  const double *dxu = o.fd[LT_F_DXU].data(), *dyu = o.fd[LT_F_DYU].data();
  const double *dxur = o.fd[LT_F_DXUR].data(), *dyur = o.fd[LT_F_DYUR].data(), *uarea_r = o.fd[LT_F_UAREA_R].data();
  const double *duc = o.fd[LT_F_DUC].data(), *dum = o.fd[LT_F_DUM].data(), *dun = o.fd[LT_F_DUN].data();
  const double *dus = o.fd[LT_F_DUS].data(), *due = o.fd[LT_F_DUE].data(), *duw = o.fd[LT_F_DUW].data();
  const double *dmc = o.fd[LT_F_DMC].data(), *dmn = o.fd[LT_F_DMN].data(), *dms = o.fd[LT_F_DMS].data();
  const double *dme = o.fd[LT_F_DME].data(), *dmw = o.fd[LT_F_DMW].data(), *amf = o.fd[LT_F_AMF].data();
  std::vector<double> wka(F), am_factor(F, 0.0), hduk2(F), hdvk2(F), d2uk(F), d2vk(F);
  auto grad = [&]() {   // hdel4_grad (readyc.cpp:405-442)
    for (int k = 0; k < km; ++k)
      for (int j = 0; j < jmt; ++j)
        for (int i = 0; i < imt; ++i) {
          double gradx = 0.0, grady = 0.0;
          const long c = k * A + (long)j * imt + i;
          if ((1 <= i) && (j < jmt - 1) && k <= kmu[j * imt + i] - 1) {
            gradx = dxur[j * imt + i] * p5 * (wka[c + imt] - wka[c - 1] - wka[c + imt - 1] + wka[c]);
            grady = dyur[j * imt + i] * p5 * (wka[c + imt] - wka[c - 1] + wka[c + imt - 1] - wka[c]);
          }
          am_factor[c] += gradx * gradx + grady * grady;
        }
  };
  // hdel4_div (readyc.cpp:372-403)
  for (int k = 0; k < km; ++k)
    for (int j = 0; j < jmt; ++j)
      for (int i = 0; i < imt; ++i) {
        const long t = (long)j * imt + i, c = k * A + t;
        wka[c] = 0.0e0;
        if (i < imt - 1 && j >= 1 && k <= kmt[t] - 1)
          wka[c] = 0.5 * ((up[c + 1] + up[c - imt + 1]) * htw[t + 1] - (up[c] + up[c - imt]) * htw[t] +
                          (vp[c + 1] + vp[c]) * hts[t] - (vp[c - imt + 1] + vp[c - imt]) * hts[t - imt]) *
                   tarea_r[t];
      }
  grad();
  // hdel4_zcurl (readyc.cpp:343-370)
  for (int k = 0; k < km; ++k)
    for (int j = 0; j < jmt; ++j)
      for (int i = 0; i < imt; ++i) {
        const long t = (long)j * imt + i, c = k * A + t;
        wka[c] = 0.0e0;
        if (i >= 1 && j >= 1 && k <= kmt[t] - 1)
          wka[c] = 0.5 * ((vp[c] * dyu[t] + vp[c - imt] * dyu[t - imt] - vp[c - 1] * dyu[t - 1] -
                           vp[c - imt - 1] * dyu[t - imt - 1] - up[c] * dxu[t] - up[c - 1] * dxu[t - 1] +
                           up[c - imt] * dxu[t - imt] + up[c - imt - 1] * dxu[t - imt - 1]));
      }
  grad();
  // hdiffu_del4_0 (readyc.cpp:444-507)
  for (int k = 0; k < km; ++k)
    for (int j = 0; j < jmt; ++j)
      for (int i = 0; i < imt; ++i) {
        const long t = (long)j * imt + i, c = k * A + t;
        double am_f = 1.0e0;
        hduk2[c] = 0.0;
        hdvk2[c] = 0.0;
        if (j >= jb - 2 && j <= je && i >= ib - 2 && i <= ie && k <= kmu[t] - 1) {
          const double t_area = std::sqrt(1.0e0 / uarea_r[t]);
          const double dxdy = t_area * t_area * t_area * t_area * t_area * 45.0e0;
          am_f = std::sqrt(am_factor[c]) * dxdy / std::fabs(am * amf[t]);
          am_f = std::fmin(40.0e0, am_f);
          am_f = std::fmax(1.0e0, am_f);
          hduk2[c] = (((duc[t] + dum[t]) * up[c] + dun[t] * up[c - imt] + dus[t] * up[c + imt] + due[t] * up[c + 1] +
                       duw[t] * up[c - 1]) +
                      (dmc[t] * vp[c] + dmn[t] * vp[c - imt] + dms[t] * vp[c + imt] + dme[t] * vp[c + 1] +
                       dmw[t] * vp[c - 1]));
          hdvk2[c] = (((duc[t] + dum[t]) * vp[c] + dun[t] * vp[c - imt] + dus[t] * vp[c + imt] + due[t] * vp[c + 1] +
                       duw[t] * vp[c - 1]) -
                      (dmc[t] * up[c] + dmn[t] * up[c - imt] + dms[t] * up[c + imt] + dme[t] * up[c + 1] +
                       dmw[t] * up[c - 1]));
        }
        d2uk[c] = am_f * amf[t] * hduk2[c];
        d2vk[c] = am_f * amf[t] * hdvk2[c];
      }
  // hdiffu_del4_1 (readyc.cpp:509-577)
  for (int k = 0; k < km; ++k)
    for (int j = 0; j < jmt; ++j)
      for (int i = 0; i < imt; ++i) {
        const long t = (long)j * imt + i, c = k * A + t;
        hduk2[c] = 0.0;
        hdvk2[c] = 0.0;
        if (j >= jb - 1 && j < je && i >= ib - 1 && i < ie) {
          hduk2[c] = am * (((duc[t] + dum[t]) * d2uk[c] + dun[t] * d2uk[c - imt] + dus[t] * d2uk[c + imt] +
                            due[t] * d2uk[c + 1] + duw[t] * d2uk[c - 1]) +
                           (dmc[t] * d2vk[c] + dmn[t] * d2vk[c - imt] + dms[t] * d2vk[c + imt] + dme[t] * d2vk[c + 1] +
                            dmw[t] * d2vk[c - 1]));
          hdvk2[c] = am * (((duc[t] + dum[t]) * d2vk[c] + dun[t] * d2vk[c - imt] + dus[t] * d2vk[c + imt] +
                            due[t] * d2vk[c + 1] + duw[t] * d2vk[c - 1]) -
                           (dmc[t] * d2uk[c] + dmn[t] * d2uk[c - imt] + dms[t] * d2uk[c + imt] + dme[t] * d2uk[c + 1] +
                            dmw[t] * d2uk[c - 1]));
        }
        if (k > kmu[t] - 1) {
          hduk2[c] = 0.0;
          hdvk2[c] = 0.0;
        }
        if (1 <= j && j < jmt - 1 && 1 <= i && i < imt - 1) {
          dlv[c] = dlv[c] + hdvk2[c];
          dlu[c] = dlu[c] + hduk2[c];
        }
        wkad[c] = c0f * std::sqrt(up[c] * up[c] + vp[c] * vp[c]);
      }
}
}  // namespace

namespace {
void copy_par(std::vector<double>& dst, const std::vector<double>& src) {
  dst.resize(src.size());
  const long n = (long)src.size();
  double* d = dst.data();
  const double* q = src.data();
#pragma omp parallel for schedule(static)
  for (long c = 0; c < n; ++c) d[c] = q[c];
}
// nsteps steps with frozen dynamics; *t_tracer (if given) receives the
// seconds spent inside the tracer_ calls alone, without the copies that
// restore the dynamics between them.
int step_frozen(Oracle& o, int nsteps, double* t_tracer) {
  const int dyn[5] = {LT_F_UTF, LT_F_VTF, LT_F_UTL, LT_F_VTL, LT_F_H0F};
  for (int m = 0; m < 5; ++m) copy_par(o.dyn0[m], o.fd[dyn[m]]);
  double t = 0.0;
  for (int s = 0; s < nsteps; ++s) {
    for (int m = 0; m < 5; ++m) copy_par(o.fd[dyn[m]], o.dyn0[m]);
#ifdef _OPENMP
    const double t0 = omp_get_wtime();
    tracer_call(o);
    t += omp_get_wtime() - t0;
#else
    tracer_call(o);
#endif
  }
  copy_par(o.fd[LT_F_UTF_OUT], o.fd[LT_F_UTF]);
  copy_par(o.fd[LT_F_VTF_OUT], o.fd[LT_F_VTF]);
  copy_par(o.fd[LT_F_H0F_OUT], o.fd[LT_F_H0F]);
  for (int m : {0, 1, 3, 4}) copy_par(o.fd[dyn[m]], o.dyn0[m]);
  if (t_tracer) *t_tracer = t;
  return 0;
}
}  // namespace

extern "C" {

void* or_create(int nx, int ny, int km) {
  if (nx < 4 || ny < 4 || km < 3) return nullptr;
  return new Oracle(nx, ny, km);
}
void or_destroy(void* h) { delete static_cast<Oracle*>(h); }
int or_set_params(void* h, const lt_params* p, int ew_cyclic, int tripole) {
  Oracle& o = *static_cast<Oracle*>(h);
  o.p = *p; o.ew_cyclic = ew_cyclic; o.tripole = tripole;
  return 0;
}
long or_field_count(void* h, int f) {
  if (f < 0 || f >= LT_F_COUNT) return -1;
  return static_cast<Oracle*>(h)->count(f);
}
int or_set_field(void* h, int f, const void* src, size_t nbytes) {
  Oracle& o = *static_cast<Oracle*>(h);
  if (f < 0 || f >= LT_F_COUNT) return LT_E_INVALID;
  o.ensure(f);
  const bool isint = field_info(f).is_int;
  const size_t need = (size_t)o.count(f) * (isint ? sizeof(int) : sizeof(double));
  if (nbytes != need) return LT_E_INVALID;
  if (isint) std::memcpy(o.fi[f].data(), src, nbytes);
  else std::memcpy(o.fd[f].data(), src, nbytes);
  return 0;
}
int or_get_field(void* h, int f, void* dst, size_t nbytes) {
  Oracle& o = *static_cast<Oracle*>(h);
  if (f < 0 || f >= LT_F_COUNT) return LT_E_INVALID;
  o.ensure(f);
  const bool isint = field_info(f).is_int;
  const size_t need = (size_t)o.count(f) * (isint ? sizeof(int) : sizeof(double));
  if (nbytes != need) return LT_E_INVALID;
  if (isint) std::memcpy(dst, o.fi[f].data(), nbytes);
  else std::memcpy(dst, o.fd[f].data(), nbytes);
  return 0;
}
// One literal tracer_ call: utf/vtf/h0f are scaled in place and vtl is left
// holding S, as in the reference.
int or_tracer_call(void* h) {
  tracer_call(*static_cast<Oracle*>(h));
  return 0;
}
// nsteps steps with frozen dynamics: before each step utf, vtf, utl, vtl, h0f
// are restored from the given copies (the model's bclinc/barotr would supply
// fresh ones), then one tracer_ call runs; afterwards UTF/VTF/H0F hold the
// scaled values of the last step, copied to the *_OUT fields.

// nsteps steps with frozen dynamics: before each step utf, vtf, utl, vtl, h0f
// are restored from copies taken at entry (the model's bclinc/barotr would
// supply fresh ones), then one tracer_ call runs; afterwards UTF/VTF/H0F hold
// the scaled values of the last step, copied to the *_OUT fields.
int or_step(void* h, int nsteps) {
  return step_frozen(*static_cast<Oracle*>(h), nsteps, nullptr);
}
// or_step that also reports the seconds spent in the tracer_ calls.
int or_step_timed(void* h, int nsteps, double* t_tracer) {
  return step_frozen(*static_cast<Oracle*>(h), nsteps, t_tracer);
}
// 1: write the diagnostics ax, ay, az, dz, penetrate, tend, dt_diff (the
// reference always does); 0: skip them (the state is the same).
int or_set_diagnostics(void* h, int on) {
  static_cast<Oracle*>(h)->set_diagnostics(on != 0);
  return 0;
}
// Address of a field's storage (allocated on first use), for filling it in place.
void* or_field_ptr(void* h, int f) {
  Oracle& o = *static_cast<Oracle*>(h);
  if (f < 0 || f >= LT_F_COUNT) return nullptr;
  o.ensure(f);
  return field_info(f).is_int ? (void*)o.fi[f].data() : (void*)o.fd[f].data();
}
int or_convadj(void* h) {
  convadj_call(*static_cast<Oracle*>(h));
  return 0;
}
int or_turb(void* h, const lt_turb_tables* t, int ncc, double dfricmx) {
  if (!t || ncc < 1) return LT_E_INVALID;
  turb_call(*static_cast<Oracle*>(h), *t, ncc, dfricmx);
  return 0;
}
int or_hdiffu_del4(void* h, double am, double c0f) {
  del4u_call(*static_cast<Oracle*>(h), am, c0f);
  return 0;
}
int or_icesnow(void* h, const lt_icesnow_params* p) {
  if (!p) return LT_E_INVALID;
  icesnow_call(*static_cast<Oracle*>(h), *p);
  return 0;
}
double or_fw_norm2(void* h) { return static_cast<Oracle*>(h)->fw_norm2; }
// sum(tarea*dzp*vit*tracer) over the interior, sequential order
int or_tracer_content(void* h, double* out2) {
  Oracle& o = *static_cast<Oracle*>(h);
  const double* at = o.fd[LT_F_AT].data();
  for (int n = 0; n < 2; ++n) {
    double s = 0.0;
    for (int k = 0; k < o.km; ++k)
      for (int j = 2; j < o.jmt - 2; ++j)
        for (int i = 2; i < o.imt - 2; ++i) {
          const long a = (long)j * o.imt + i;
          if (k < o.fi[LT_F_KMT][a]) s += o.fd[LT_F_TAREA][a] * o.fd[LT_F_DZP][k] * at[n * o.F + (long)k * o.A + a];
        }
    out2[n] = s;
  }
  return 0;
}
// standalone halo (tests): nz levels of [jmt][imt]
int or_halo(double* a, int nz, int imt, int jmt, int ew_cyclic, int tripole) {
  halo_r8(a, nz, imt, jmt, ew_cyclic, tripole);
  return 0;
}
int or_set_sum_order(void* h, int tree) {
  static_cast<Oracle*>(h)->tree_sum = tree != 0;
  return 0;
}
// tracer_7 alone on caller arrays (the nudging branch is pinned with it
// against the reference's own tracer_7, which the reference's tracer_ never
// runs with simple_assm on)
int or_tracer7(const lt_params* p, int n, int imt, int jmt, int km, double* tf, const double* vit,
               const double* atb, const double* restore, const double* restore_at, double* dt_restore) {
  tracer7(*p, n, imt, jmt, km, tf, vit, atb + (long)n * imt * jmt * (km + 1), restore, restore_at, dt_restore);
  return 0;
}
int or_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
#else
  (void)n;
  return 1;
#endif
}

}  // extern "C"
