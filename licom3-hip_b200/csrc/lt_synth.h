// lt_synth.h - seeded synthetic LICOM tracer domains (grid, masks, state,
// velocities, mixing, forcing) for tests and benchmarks.
//
// Everything a LICOM3 tracer step reads is produced here from a seed:
//   * the horizontal grid metrics of a global lat-lon mesh, LICOM order
//     (j = 0 is the northernmost row, i runs east), halo width 2;
//   * land/ocean depth index KMT from seeded smoothed noise, with the masks
//     LICOM derives from it (KMU, KMTN/S/E/W, VIT, VIV, OHBT, OHBU) and the
//     del4 stencil weights DTN/S/E/W and AHF (hmix_del4.F90:295-405);
//   * stretched vertical levels (ZKP, DZP, ODZP, ODZT as grid.F90:1097-1106);
//   * T/S state, velocities from a per-level streamfunction (so that the
//     horizontal divergence operator of tracer.cpp:980-1006 is zero to
//     round-off), Canuto-like AKT, surface forcing.
//
// 3-D cell values are pure functions of (seed, field, index) built from an
// integer hash and +,-,*,/ only (no transcendental calls), so a host build
// (-ffp-contract=off) and a device build (-fmad=false) give identical bits.
// 2-D and 1-D fields (which need smoothing, trig and pow) are built on the
// host only and uploaded.
#pragma once
#include <stdint.h>
#include <cmath>
#include <vector>
#include <algorithm>
#include <numeric>
#include <cstring>
#include <type_traits>

#if defined(__CUDACC__)
#define LT_HD __host__ __device__ __forceinline__
#else
#define LT_HD inline
#endif

namespace lt {

// ---------------------------------------------------------------- hashing
LT_HD uint64_t mix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
LT_HD uint64_t cell_hash(uint64_t seed, uint32_t tag, uint64_t idx) {
  return mix64(seed ^ mix64(((uint64_t)tag << 56) ^ idx));
}
LT_HD double hash_u01(uint64_t h) { return (double)(h >> 11) * (1.0 / 9007199254740992.0); }
// Approximately standard normal: Irwin-Hall sum of four uniforms, rescaled.
LT_HD double hash_gauss(uint64_t seed, uint32_t tag, uint64_t idx) {
  uint64_t h = cell_hash(seed, tag, idx);
  double s = 0.0;
  for (int r = 0; r < 4; ++r) { s = s + hash_u01(h); h = mix64(h); }
  return (s - 2.0) * 1.7320508075688772;
}

enum SynthTag : uint32_t {
  TAG_LAND = 1, TAG_PSI = 2, TAG_SALT2D = 3, TAG_T3D = 4, TAG_S3D = 5,
  TAG_AKT = 6, TAG_FORC = 7, TAG_H0 = 8, TAG_TPERT = 9
};

// ------------------------------------------------------------- 3-D cells
// All per-cell generators take the dense [k][j][i] index of the cell and the
// per-domain tables built on the host.
struct CellTables {
  int imt, jmt, km;
  uint64_t seed;
  const double* tprof;    // [km]   reference T profile (degC)
  const double* ssurf;    // [jmt*imt] salinity (model units) at each column
  const int* kmt;         // [jmt*imt]
  const int* dmin;        // [jmt*imt] 3x3 minimum of KMT
  const double* psi;      // [jmt*imt] streamfunction (m^3/s per unit profile)
  const double* uprof;    // [km] vertical velocity profile
  const double* rdyu;     // [jmt*imt] 1/DYU
  const double* rdxu;     // [jmt*imt] 1/DXU
  const double* akt_tab;  // [4096] log-uniform mixing table
  double tnoise;          // K
  double snoise;          // model units
  uint32_t member;        // ensemble member id (0 = unperturbed)
  double tpert;           // K, std of member perturbation
};

LT_HD double cell_T(const CellTables& t, int k, int j, int i) {
  const long a = (long)j * t.imt + i;
  if (k >= t.kmt[a]) return 0.0;
  const uint64_t idx = ((uint64_t)k * t.jmt + j) * t.imt + i;
  double v = t.tprof[k] + t.tnoise * hash_gauss(t.seed, TAG_T3D, idx);
  if (t.member != 0) v = v + t.tpert * hash_gauss(t.seed + t.member, TAG_TPERT, idx);
  return v;
}
LT_HD double cell_S(const CellTables& t, int k, int j, int i) {
  const long a = (long)j * t.imt + i;
  if (k >= t.kmt[a]) return 0.0;
  const uint64_t idx = ((uint64_t)k * t.jmt + j) * t.imt + i;
  return t.ssurf[a] + t.snoise * hash_gauss(t.seed, TAG_S3D, idx);
}
// level-k streamfunction at T point (j,i): zero within one cell of any column
// shallower than k+1, so every U point that touches land at level k is at rest.
LT_HD double cell_psi(const CellTables& t, int k, int j, int i) {
  const long a = (long)j * t.imt + i;
  return (k < t.dmin[a]) ? t.psi[a] * t.uprof[k] : 0.0;
}
// U-point velocities (B grid). U(i,j) sits between T(i-1..i, j..j+1).
LT_HD double cell_U(const CellTables& t, int k, int j, int i) {
  if (i < 1 || j >= t.jmt - 1) return 0.0;
  const double px0 = 0.5 * (cell_psi(t, k, j, i - 1) + cell_psi(t, k, j, i));
  const double px1 = 0.5 * (cell_psi(t, k, j + 1, i - 1) + cell_psi(t, k, j + 1, i));
  return (px1 - px0) * t.rdyu[(long)j * t.imt + i];
}
LT_HD double cell_V(const CellTables& t, int k, int j, int i) {
  if (i < 1 || j >= t.jmt - 1) return 0.0;
  const double py1 = 0.5 * (cell_psi(t, k, j, i) + cell_psi(t, k, j + 1, i));
  const double py0 = 0.5 * (cell_psi(t, k, j, i - 1) + cell_psi(t, k, j + 1, i - 1));
  return (py0 - py1) * t.rdxu[(long)j * t.imt + i];
}
LT_HD double cell_akt(const CellTables& t, int n, int k, int j, int i) {
  const uint64_t idx = (((uint64_t)n * t.km + k) * t.jmt + j) * t.imt + i;
  return t.akt_tab[cell_hash(t.seed, TAG_AKT, idx) & 4095u];
}

// ------------------------------------------------------------- host side
// host-only builders below (parsed by every pass, called from host code only)

enum HaloLoc { HALO_CENTER = 0, HALO_SWCORNER = 1 };

// Ghost-cell fill of one horizontal level with LICOM/POP semantics for a
// single block that covers the whole global domain (POP_HaloMod.F90:2716-3139,
// addresses POP_HaloMod.F90:5602-5680, ghost indices POP_BlocksMod.F90:284-375):
//   east-west cyclic copies for the physical rows, then the tripole fold which
//   rewrites the two northern ghost rows and (for cell centres) the top
//   physical row after averaging it with its mirror image; a closed side is
//   left untouched.  Integer fields average with nint().
template <class T>
void halo_level(T* a, int imt, int jmt, bool ew_cyclic, bool tripole, HaloLoc loc) {
  const int nx = imt - 4;
  if (ew_cyclic) {
    for (int j = 2; j < jmt - 2; ++j) {
      T* r = a + (long)j * imt;
      r[0] = r[nx]; r[1] = r[nx + 1];
      r[nx + 2] = r[2]; r[nx + 3] = r[3];
    }
  }
  if (!tripole) return;
  // buffer rows 0..2 = physical rows 2..4, global column g = 1..nx
  std::vector<T> buf(3 * (nx + 1));
  for (int r = 0; r < 3; ++r)
    for (int g = 1; g <= nx; ++g) buf[r * (nx + 1) + g] = a[(long)(2 + r) * imt + g + 1];
  int ioff, joff;
  if (loc == HALO_CENTER) {
    ioff = 1; joff = 1;
    for (int g = 1; g <= nx / 2 - 1; ++g) {
      const T x1 = buf[g], x2 = buf[nx - g];
      T avg;
      if constexpr (std::is_integral<T>::value) {
        avg = (T)std::llround(0.5 * (double)(x1 + x2));
      } else {
        avg = 0.5 * (x1 + x2);
      }
      buf[g] = avg; buf[nx - g] = avg;
    }
  } else {
    ioff = 0; joff = 2;
  }
  auto iglobal = [&](int i0) -> int {  // POP global index of local column i0
    int g = i0 - 1;
    if (g < 1) g = ew_cyclic ? g + nx : 0;
    else if (g > nx) g = ew_cyclic ? g - nx : 0;
    return g;
  };
  for (int jf = 1; jf <= 3; ++jf) {
    const int jsrc = (2 + 3 - jf) - joff;
    if (jsrc <= 0) continue;
    for (int i0 = 0; i0 < imt; ++i0) {
      int isrc = nx - iglobal(i0) + 1 - ioff;
      if (isrc == 0) isrc = nx;
      a[(long)(jf - 1) * imt + i0] = buf[(jsrc - 1) * (nx + 1) + isrc];
    }
  }
}

template <class T>
void halo_fill(T* a, int nz, int imt, int jmt, bool ew_cyclic, bool tripole, HaloLoc loc = HALO_CENTER) {
  for (int z = 0; z < nz; ++z) halo_level(a + (long)z * imt * jmt, imt, jmt, ew_cyclic, tripole, loc);
}

struct SynthConfig {
  int nx = 360, ny = 196, km = 30;
  double lat_s = -78.0, lat_n = 66.0;   // centre latitudes of the outer physical rows
  double dz_top = 10.0, dz_bot = 250.0, depth = 5000.0;
  double umax = 0.1;                    // m/s
  uint64_t seed = 20240611ull;
  int forced = 0;                       // seeded surface forcing and SSH
  int cap_north = 3, cap_south = 3;     // land rows forced at the physical edges
  double land_frac = 0.30;
  int ew_cyclic = 1, tripole = 1;
  double smooth_cells_1deg = 8.0;       // smoothing radius at 1 degree
  int ncc = 1, nbb = 60;
  double dts = 1800.0;
  // Biharmonic tracer diffusivity (m^4/s).  0 selects the configured
  // -1e17, capped at half of this grid's explicit stability limit (see
  // build_domain).
  double ah_bihar = 0.0;
  // Ocean depth map: 0 = KMT linear in the land field above its threshold
  // (3 .. km levels); 1 = depths by the rank of the land field among the
  // ocean cells on the global ocean's area-depth curve (hypsometry), so the
  // shallow cells sit next to the coast and most of the ocean is abyssal.
  int hypsometry = 0;
  double dwndmix = 1.0e-3;
  double gamma_days = 30.0;
  double tnoise = 0.1, snoise_psu = 0.01;
  uint32_t member = 0;
  double tpert = 0.0;
};

// Host-side description of one domain: every 2-D/1-D input of the tracer step
// plus the scalar parameters; 3-D fields are produced on demand.
struct Domain {
  SynthConfig cfg;
  int nx, ny, km, imt, jmt;
  // 1-D
  std::vector<double> zkp, dzp, odzp, odzt, zkt, pen, tprof, uprof, to, so, c9;  // c9 = [9][km]
  // 2-D double
  std::vector<double> tarea, tarea_r, htw, hts, hun, hue, dxu, dyu, ahf;
  std::vector<double> dtn, dts_, dte, dtw, ohbt, ohbu, au0, aus, auw, ausw;
  std::vector<double> h0f, h0l, swv, nswv, sst, sss, fresh, seaice;
  std::vector<double> ssurf, psi, rdyu, rdxu;
  // 2-D int
  std::vector<int> kmt, kmu, kmtn, kmts, kmte, kmtw, dmin;
  // tables
  std::vector<double> akt_tab;
  // scalars
  double dts, oncc, onbc, dwndmix, gamma, od0, od0cp, ah, area_t;
  int nss;

  CellTables tables() const {
    CellTables t;
    t.imt = imt; t.jmt = jmt; t.km = km; t.seed = cfg.seed;
    t.tprof = tprof.data(); t.ssurf = ssurf.data(); t.kmt = kmt.data();
    t.dmin = dmin.data(); t.psi = psi.data(); t.uprof = uprof.data();
    t.rdyu = rdyu.data(); t.rdxu = rdxu.data(); t.akt_tab = akt_tab.data();
    t.tnoise = cfg.tnoise; t.snoise = cfg.snoise_psu * 1.0e-3;
    t.member = cfg.member; t.tpert = cfg.tpert;
    return t;
  }
};

// Separable box smoothing (three passes approximate a Gaussian) of an integer
// field on the physical domain, periodic in i and clamped in j.  Integer
// running sums keep the result exact and platform independent.
inline void box_smooth(std::vector<int64_t>& f, int nx, int ny, int r, bool periodic_i) {
  if (r < 1) return;
  std::vector<int64_t> tmp(f.size());
  const int64_t w = 2 * r + 1;
  for (int pass = 0; pass < 3; ++pass) {
    for (int j = 0; j < ny; ++j) {
      const int64_t* row = &f[(long)j * nx];
      int64_t* out = &tmp[(long)j * nx];
      auto at = [&](int i) -> int64_t {
        if (periodic_i) { i %= nx; if (i < 0) i += nx; return row[i]; }
        return row[std::min(std::max(i, 0), nx - 1)];
      };
      int64_t s = 0;
      for (int d = -r; d <= r; ++d) s += at(d);
      for (int i = 0; i < nx; ++i) { out[i] = s / w; s += at(i + r + 1) - at(i - r); }
    }
    for (int i = 0; i < nx; ++i) {
      auto at = [&](int j) -> int64_t { return tmp[(long)std::min(std::max(j, 0), ny - 1) * nx + i]; };
      int64_t s = 0;
      for (int d = -r; d <= r; ++d) s += at(d);
      for (int j = 0; j < ny; ++j) { f[(long)j * nx + i] = s / w; s += at(j + r + 1) - at(j - r); }
    }
  }
}

inline std::vector<int64_t> smooth_noise(uint64_t seed, uint32_t tag, int nx, int ny, int r) {
  std::vector<int64_t> f((size_t)nx * ny);
  for (size_t a = 0; a < f.size(); ++a) f[a] = (int64_t)(cell_hash(seed, tag, a) >> 44);  // 20-bit
  box_smooth(f, nx, ny, r, true);
  return f;
}

inline Domain build_domain(const SynthConfig& c) {
  Domain d;
  d.cfg = c;
  d.nx = c.nx; d.ny = c.ny; d.km = c.km;
  d.imt = c.nx + 4; d.jmt = c.ny + 4;
  const int imt = d.imt, jmt = d.jmt, km = d.km, nx = c.nx, ny = c.ny;
  const size_t A = (size_t)imt * jmt;
  const double PI = 3.14159265358979323846, R = 6371000.0;

  // ---- vertical levels: dz_k = top + (bot-top)*(k/(km-1))^p, sum = depth
  {
    auto total = [&](double p) {
      double s = 0.0;
      for (int k = 0; k < km; ++k) s += c.dz_top + (c.dz_bot - c.dz_top) * std::pow((double)k / (km - 1), p);
      return s;
    };
    double lo = 0.05, hi = 20.0;
    for (int it = 0; it < 200; ++it) {
      const double mid = 0.5 * (lo + hi);
      if (total(mid) > c.depth) lo = mid; else hi = mid;
    }
    const double p = 0.5 * (lo + hi);
    d.zkp.assign(km + 1, 0.0);
    for (int k = 0; k < km; ++k)
      d.zkp[k + 1] = d.zkp[k] - (c.dz_top + (c.dz_bot - c.dz_top) * std::pow((double)k / (km - 1), p));
    d.dzp.resize(km); d.zkt.resize(km); d.odzp.resize(km); d.odzt.resize(km);
    for (int k = 0; k < km; ++k) {
      d.dzp[k] = d.zkp[k] - d.zkp[k + 1];
      d.zkt[k] = (d.zkp[k] + d.zkp[k + 1]) * 0.5;
      d.odzp[k] = 1.0 / d.dzp[k];
    }
    d.odzt[0] = 2.0 * d.odzp[0];
    for (int k = 1; k < km; ++k) d.odzt[k] = 1.0 / (d.zkt[k - 1] - d.zkt[k]);
    // two-band shortwave penetration times 1/(rho0*cp) (grids.F90:44-59)
    d.pen.assign(km, 0.0);
    const double od0cp = 1.0 / (1026.0 * 3996.0);
    for (int k = 0; k < km - 1; ++k) {
      const double s1 = std::max(d.zkp[k + 1] * (1.0 / 0.35), -70.0);
      const double s2 = std::max(d.zkp[k + 1] * (1.0 / 23.0), -70.0);
      d.pen[k] = (0.58 * std::exp(s1) + (1.0 - 0.58) * std::exp(s2)) * od0cp;
    }
    d.tprof.resize(km); d.uprof.resize(km);
    for (int k = 0; k < km; ++k) {
      d.tprof[k] = 2.0 + 26.0 * std::exp(d.zkt[k] / 700.0);
      d.uprof[k] = std::exp(d.zkt[k] / 1000.0);
    }
    // reference state and density-polynomial coefficients per level (the
    // model reads these from a data file; a smooth synthetic fit is used)
    d.to.resize(km); d.so.resize(km); d.c9.assign(9 * km, 0.0);
    for (int k = 0; k < km; ++k) {
      const double z = -d.zkt[k];
      d.to[k] = d.tprof[k];
      d.so[k] = -0.3e-3;
      const double p_bar = z * 0.1;  // rough pressure in bar
      const double cc[9] = {-2.0e-4 - 1.0e-8 * p_bar * 100.0, 0.77 - 1.0e-5 * p_bar, -5.0e-6,
                            -2.0e-3, -0.5, 2.0e-8, 2.0e-6, 5.0e-4, 0.1};
      for (int m = 0; m < 9; ++m) d.c9[m * km + k] = cc[m] * 1000.0;
    }
  }

  // ---- horizontal metrics on a lat-lon mesh, LICOM row order (north first)
  const double dlat = (c.lat_n - c.lat_s) / (ny - 1) * PI / 180.0;
  const double dlon = 2.0 * PI / nx;
  auto lat_row = [&](int j) { return c.lat_n * PI / 180.0 - (j - 2) * dlat; };  // T row centre
  d.tarea.resize(A); d.tarea_r.resize(A); d.htw.resize(A); d.hts.resize(A);
  d.hun.resize(A); d.hue.resize(A); d.dxu.resize(A); d.dyu.resize(A);
  for (int j = 0; j < jmt; ++j) {
    const double phit = lat_row(j);
    const double phiu = phit - 0.5 * dlat;  // U row sits between T rows j and j+1
    const double dxt = R * std::cos(phit) * dlon, dy = R * dlat;
    const double dxuv = R * std::cos(phiu) * dlon;
    for (int i = 0; i < imt; ++i) {
      const long a = (long)j * imt + i;
      d.tarea[a] = dxt * dy;
      d.tarea_r[a] = 1.0 / d.tarea[a];
      d.htw[a] = dy; d.dyu[a] = dy; d.hue[a] = dy;
      d.hts[a] = dxuv; d.dxu[a] = dxuv;
      d.hun[a] = dxt;
    }
  }
  d.ahf.resize(A);
  const double dxeq = 2.0 * R * PI / (double)nx;
  for (size_t a = 0; a < A; ++a) d.ahf[a] = std::pow(d.tarea[a] / std::pow(dxeq, 2.0), 1.5);

  // ---- land mask and depth index
  const int rad = std::max(1, (int)std::lround(c.smooth_cells_1deg * nx / 360.0 / 1.73));
  {
    std::vector<int64_t> f = smooth_noise(c.seed, TAG_LAND, nx, ny, rad);
    std::vector<int64_t> sorted(f);
    const size_t q = (size_t)(c.land_frac * (double)(sorted.size() - 1));
    std::nth_element(sorted.begin(), sorted.begin() + q, sorted.end());
    const int64_t thr = sorted[q];
    int64_t fmax = *std::max_element(f.begin(), f.end());
    // hypsometry 1: the ocean cells' rank in the land field (ties by
    // position) read as the fraction q of the ocean shallower than the cell,
    // mapped through the global ocean's area-depth curve (piecewise linear
    // between these published fractions: 7.5 % shallower than 200 m, 12 %
    // than 1 km, 16.5 % than 2 km, 25 % than 3 km, 46 % than 4 km, 78 % than
    // 5 km, 99 % than 6 km), depth clipped to the grid's; KMT = the levels
    // whose centre lies above that depth, at least 3
    std::vector<int> hyps_k;
    if (c.hypsometry == 1) {
      std::vector<std::pair<int64_t, long>> ocean;
      for (long q = 0; q < (long)f.size(); ++q)
        if (f[q] > thr) ocean.push_back({f[q], q});
      std::sort(ocean.begin(), ocean.end());
      static const double zq[][2] = {{0.0, 0.0},       {200.0, 0.075},  {1000.0, 0.12}, {2000.0, 0.165},
                                     {3000.0, 0.25},   {4000.0, 0.46},  {5000.0, 0.78}, {6000.0, 0.99},
                                     {11000.0, 1.0}};
      hyps_k.assign(f.size(), 0);
      const long n = (long)ocean.size();
      for (long r = 0; r < n; ++r) {
        const double q = (r + 0.5) / (double)n;
        int s = 1;
        while (s < 8 && zq[s][1] < q) ++s;
        const double z = zq[s - 1][0] + (zq[s][0] - zq[s - 1][0]) * (q - zq[s - 1][1]) / (zq[s][1] - zq[s - 1][1]);
        int k = 0;
        while (k < km && -0.5 * (d.zkp[k] + d.zkp[k + 1]) < z) ++k;
        hyps_k[ocean[r].second] = std::max(3, k);
      }
    }
    d.kmt.assign(A, 0);
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        const int64_t v = f[(long)j * nx + i];
        int k = 0;
        if (v > thr && c.hypsometry == 1) {
          k = hyps_k[(long)j * nx + i];
        } else if (v > thr) {
          const int64_t span = std::max<int64_t>(fmax - thr, 1);
          k = 3 + (int)(((v - thr) * (int64_t)(km - 3)) / span);
          if (k > km) k = km;
        }
        if (j < c.cap_north || j >= ny - c.cap_south) k = 0;
        d.kmt[(long)(j + 2) * imt + i + 2] = k;
      }
    halo_fill(d.kmt.data(), 1, imt, jmt, c.ew_cyclic, c.tripole, HALO_CENTER);
  }
  // derived integer masks (boundary.F90:24-52, grid.F90:1343-1346)
  d.kmu.assign(A, 0);
  for (int j = 0; j < jmt - 1; ++j)
    for (int i = 1; i < imt; ++i) {
      const long a = (long)j * imt + i;
      d.kmu[a] = std::min(std::min(d.kmt[a - 1], d.kmt[a]), std::min(d.kmt[a + imt - 1], d.kmt[a + imt]));
    }
  halo_fill(d.kmu.data(), 1, imt, jmt, c.ew_cyclic, c.tripole, HALO_SWCORNER);
  d.kmtn.assign(A, 0); d.kmts.assign(A, 0); d.kmte.assign(A, 0); d.kmtw.assign(A, 0);
  for (int j = 0; j < jmt; ++j)
    for (int i = 0; i < imt; ++i) {
      const long a = (long)j * imt + i;
      d.kmtn[a] = j > 0 ? d.kmt[a - imt] : 0;
      d.kmts[a] = j < jmt - 1 ? d.kmt[a + imt] : 0;
      d.kmte[a] = i < imt - 1 ? d.kmt[a + 1] : 0;
      d.kmtw[a] = i > 0 ? d.kmt[a - 1] : 0;
    }
  d.dmin.assign(A, 0);
  for (int j = 0; j < jmt; ++j)
    for (int i = 0; i < imt; ++i) {
      int m = km + 1;
      for (int dj = -1; dj <= 1; ++dj)
        for (int di = -1; di <= 1; ++di) {
          const int jj = j + dj;
          int ii = i + di;
          // beyond the outer ghost columns the cyclic domain continues
          if (c.ew_cyclic && ii < 0) ii += nx;
          if (c.ew_cyclic && ii >= imt) ii -= nx;
          const int v = (jj < 0 || jj >= jmt || ii < 0 || ii >= imt) ? 0 : d.kmt[(long)jj * imt + ii];
          m = std::min(m, v);
        }
      d.dmin[(long)j * imt + i] = m;
    }
  // OHBT/OHBU (grid.F90:2030-2051): inverse column depth, sequential k sum
  d.ohbt.assign(A, 0.0); d.ohbu.assign(A, 0.0);
  for (size_t a = 0; a < A; ++a) {
    double s = 0.0;
    for (int k = 0; k < km; ++k) s = s + (k < d.kmt[a] ? 1.0 : 0.0) * d.dzp[k];
    d.ohbt[a] = s > 0.0 ? 1.0 / s : 0.0;
    s = 0.0;
    for (int k = 0; k < km; ++k) s = s + (k < d.kmu[a] ? 1.0 : 0.0) * d.dzp[k];
    d.ohbu[a] = s > 0.0 ? 1.0 / s : 0.0;
  }
  // del4 tracer stencil weights (hmix_del4.F90:368-385), eoshift with zero fill
  d.dtn.assign(A, 0.0); d.dts_.assign(A, 0.0); d.dte.assign(A, 0.0); d.dtw.assign(A, 0.0);
  for (int j = 0; j < jmt; ++j)
    for (int i = 0; i < imt; ++i) {
      const long a = (long)j * imt + i;
      const double wns = d.hts[a] / d.hue[a];
      d.dts_[a] = wns * d.tarea_r[a];
      d.dtn[a] = (j > 0 ? d.hts[a - imt] / d.hue[a - imt] : 0.0) * d.tarea_r[a];
      const double wew = d.htw[a] / d.hun[a];
      d.dtw[a] = wew * d.tarea_r[a];
      d.dte[a] = (i < imt - 1 ? d.htw[a + 1] / d.hun[a + 1] : 0.0) * d.tarea_r[a];
    }
  d.au0.assign(A, 0.25); d.aus.assign(A, 0.25); d.auw.assign(A, 0.25); d.ausw.assign(A, 0.25);
  d.rdyu.resize(A); d.rdxu.resize(A);
  for (size_t a = 0; a < A; ++a) { d.rdyu[a] = 1.0 / d.dyu[a]; d.rdxu[a] = 1.0 / d.dxu[a]; }

  // ---- surface salinity (model units) and streamfunction
  {
    std::vector<int64_t> s = smooth_noise(c.seed, TAG_SALT2D, nx, ny, rad);
    const int64_t smin = *std::min_element(s.begin(), s.end());
    const int64_t smax = *std::max_element(s.begin(), s.end());
    d.ssurf.assign(A, 0.0);
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        const double f01 = (double)(s[(long)j * nx + i] - smin) / (double)std::max<int64_t>(smax - smin, 1);
        d.ssurf[(long)(j + 2) * imt + i + 2] = ((34.0 + 1.5 * f01) - 35.0) * 1.0e-3;
      }
    halo_fill(d.ssurf.data(), 1, imt, jmt, c.ew_cyclic, c.tripole, HALO_CENTER);

    std::vector<int64_t> p = smooth_noise(c.seed, TAG_PSI, nx, ny, std::max(1, rad / 2));
    double mean = 0.0;
    for (auto v : p) mean += (double)v;
    mean /= (double)p.size();
    d.psi.assign(A, 0.0);
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i)
        d.psi[(long)(j + 2) * imt + i + 2] = (double)p[(long)j * nx + i] - mean;
    halo_fill(d.psi.data(), 1, imt, jmt, c.ew_cyclic, c.tripole, HALO_CENTER);
    // scale so that the largest surface speed is umax
    std::vector<double> one(1, 1.0);
    CellTables t = d.tables();
    std::vector<double> unit(km, 1.0);
    t.uprof = unit.data();
    double vmax = 0.0;
    for (int j = 0; j < jmt; ++j)
      for (int i = 0; i < imt; ++i) {
        vmax = std::max(vmax, std::fabs(cell_U(t, 0, j, i)));
        vmax = std::max(vmax, std::fabs(cell_V(t, 0, j, i)));
      }
    const double scale = vmax > 0.0 ? c.umax / vmax : 0.0;
    for (auto& v : d.psi) v *= scale;
  }

  // ---- log-uniform mixing table, 1e-5 .. 1e-1 m^2/s
  d.akt_tab.resize(4096);
  for (int q = 0; q < 4096; ++q) d.akt_tab[q] = std::pow(10.0, -5.0 + 4.0 * (q + 0.5) / 4096.0);

  // ---- scalars (constant_mod.F90:290-324 conventions)
  d.dts = c.dts;
  d.oncc = 1.0 / (double)(c.ncc + 1);
  d.onbc = 1.0 / (double)(c.nbb * c.ncc + 1);
  d.dwndmix = c.dwndmix;
  d.gamma = 1.0 / (c.gamma_days * 86400.0);
  d.od0 = 1.0 / 1026.0;
  d.od0cp = 1.0 / (1026.0 * 3996.0);
  if (c.ah_bihar != 0.0) {
    d.ah = c.ah_bihar;
  } else {
    // The configured -1e17 m^4/s, capped at half the explicit stability limit
    // of this grid.  The step applies ah * L(AHF * L(atb)) with forward time
    // stepping (hmix_del4.F90:626-757), stable while dts * |ah| * rho <= 2 with
    // rho the spectral radius of L AHF L.  Gershgorin bounds |eig(L)| by
    // 2 (dtn+dts+dte+dtw) per cell, so rho <= max AHF (2 sum d)^2 over the
    // interior.  -1e17 is below the cap on the reference's 36 x 40 block and
    // far above it on 1 and 0.1 degree grids (a 360 x 196 oracle run with
    // -1e17 grows T to 1e51 within 20 steps).
    double rho = 0.0;
    for (int j = 2; j < jmt - 2; ++j)
      for (int i = 2; i < imt - 2; ++i) {
        const long a = (long)j * imt + i;
        const double s2 = 2.0 * (d.dtn[a] + d.dts_[a] + d.dte[a] + d.dtw[a]);
        rho = std::max(rho, d.ahf[a] * s2 * s2);
      }
    const double cap = rho > 0.0 ? 0.5 * (2.0 / (c.dts * rho)) : 1.0e17;
    d.ah = -std::min(1.0e17, cap);
  }
  d.nss = (int)std::lround(86400.0 / c.dts);
  d.area_t = 0.0;
  for (int j = 2; j < jmt - 2; ++j)
    for (int i = 2; i < imt - 2; ++i)
      if (d.kmt[(long)j * imt + i] > 0) d.area_t += d.tarea[(long)j * imt + i];

  // ---- surface forcing and sea-surface height
  d.h0f.assign(A, 0.0); d.h0l.assign(A, 0.0);
  d.swv.assign(A, 0.0); d.nswv.assign(A, 0.0); d.fresh.assign(A, 0.0); d.seaice.assign(A, 0.0);
  d.sst.assign(A, 0.0); d.sss.assign(A, 0.0);
  CellTables t = d.tables();
  for (int j = 0; j < jmt; ++j)
    for (int i = 0; i < imt; ++i) {
      const long a = (long)j * imt + i;
      d.sst[a] = cell_T(t, 0, j, i);
      d.sss[a] = cell_S(t, 0, j, i);
      if (c.forced) {
        const uint64_t b = (uint64_t)a * 8;
        d.swv[a] = 100.0 + 100.0 * hash_u01(cell_hash(c.seed, TAG_FORC, b + 0));
        d.nswv[a] = -60.0 + 50.0 * hash_gauss(c.seed, TAG_FORC, b + 1);
        d.sst[a] += 0.5 * hash_gauss(c.seed, TAG_FORC, b + 2);
        d.sss[a] += 2.0e-4 * hash_gauss(c.seed, TAG_FORC, b + 3);
        d.fresh[a] = 1.0e-5 * hash_gauss(c.seed, TAG_FORC, b + 4);
        d.seaice[a] = hash_u01(cell_hash(c.seed, TAG_FORC, b + 5)) < 0.1 ? 1.0 : 0.0;
        d.h0f[a] = 0.3 * hash_gauss(c.seed, TAG_H0, b + 6);
        d.h0l[a] = 0.3 * hash_gauss(c.seed, TAG_H0, b + 7);
      }
    }
  return d;
}

// Fill the dense 3-D inputs of a domain on the host.  at/atb: [2][km(+1)][rows][imt];
// velocities: [km][rows][imt]; akt: [2][km][rows][imt], with rows the number of
// leading rows produced (the whole domain when rows == jmt; fewer give the
// northern band j < rows of the same fields, with its own ghost cells).
// Ghost cells of the tracers are filled with the same halo rule the model
// applies.
inline void fill_state(const Domain& d, double* at, double* atb, int rows = -1) {
  if (rows < 0) rows = d.jmt;
  const CellTables t = d.tables();
  const long A = (long)d.imt * rows, F = A * d.km;
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < d.km; ++k)
    for (int j = 0; j < rows; ++j)
      for (int i = 0; i < d.imt; ++i) {
        const long c = (long)k * A + (long)j * d.imt + i;
        at[c] = cell_T(t, k, j, i);
        at[F + c] = cell_S(t, k, j, i);
      }
  halo_fill(at, 2 * d.km, d.imt, rows, d.cfg.ew_cyclic, d.cfg.tripole);
  const long FB = A * (d.km + 1);
  for (int n = 0; n < 2; ++n) {
    std::memset(atb + n * FB, 0, sizeof(double) * A);
    std::memcpy(atb + n * FB + A, at + n * F, sizeof(double) * F);
  }
}

// One velocity component: which = 0 utf, 1 vtf, 2 utl, 3 vtl.
inline void fill_velocity_one(const Domain& d, int which, double* dst, int rows = -1) {
  if (rows < 0) rows = d.jmt;
  const CellTables t = d.tables();
  const long A = (long)d.imt * rows;
  const double ncc1 = (double)(d.cfg.ncc + 1);
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < d.km; ++k)
    for (int j = 0; j < rows; ++j)
      for (int i = 0; i < d.imt; ++i) {
        const double u = (which & 1) ? cell_V(t, k, j, i) : cell_U(t, k, j, i);
        dst[(long)k * A + (long)j * d.imt + i] = (which < 2) ? ncc1 * u : u;
      }
}

inline void fill_velocity(const Domain& d, double* utf, double* vtf, double* utl, double* vtl, int rows = -1) {
  fill_velocity_one(d, 0, utf, rows);
  fill_velocity_one(d, 1, vtf, rows);
  fill_velocity_one(d, 2, utl, rows);
  fill_velocity_one(d, 3, vtl, rows);
}

inline void fill_akt(const Domain& d, double* akt, int rows = -1) {
  if (rows < 0) rows = d.jmt;
  const CellTables t = d.tables();
  const long A = (long)d.imt * rows, F = A * d.km;
#pragma omp parallel for collapse(3) schedule(static)
  for (int n = 0; n < 2; ++n)
    for (int k = 0; k < d.km; ++k)
      for (int j = 0; j < rows; ++j)
        for (int i = 0; i < d.imt; ++i)
          akt[n * F + (long)k * A + (long)j * d.imt + i] = cell_akt(t, n, k, j, i);
}

}  // namespace lt
