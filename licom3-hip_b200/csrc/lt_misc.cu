// lt_misc.cu - convective adjustment, sea-ice adjustment, mask derivation,
// global sums, numeric scan and the device side of the synthetic-domain
// upload.  Compiled with -fmad=false (operation order kept as written).
#include <cstring>
#include <vector>
#include "lt_common.cuh"
#include "lt_halo.cuh"
#include "lt_synth.h"
#include "../../include/licom_synth.h"

const lt::Domain* lt_synth_domain(const lt_synth* s);

namespace lt {
namespace {

constexpr int KMAX_CONV = 128;

// density departure of the convadj polynomial at coefficient level l
// (convadj.cpp:57-77)
__device__ __forceinline__ double conv_rho(const double* cc, int km, double t, double s, int l) {
  return (cc[l] + (cc[3 * km + l] + cc[6 * km + l] * s) * s +
          (cc[2 * km + l] + cc[7 * km + l] * s + cc[5 * km + l] * t) * t) * t +
         (cc[1 * km + l] + (cc[4 * km + l] + cc[8 * km + l] * s) * s) * s;
}

// convadj_cu (convadj.cpp:29-288): one thread per column; finds the shallowest
// statically unstable interface, mixes T and S thickness-weighted over the
// unstable stretch and grows it up and down while unstable, then continues
// below; finally the tendency diagnostics and atb = at.
__global__ void k_convadj(Arena a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= a.imt || j >= a.jmt) return;
  const int km = a.km;
  const long A = a.A, F = a.F, FB = a.FB;
  const long q = (long)j * a.imt + i;
  double* at = a.at[a.cur];
  double* atb = a.atb[a.cur];
  const double* to = a.to;
  const double* so = a.so;
  const double* cc = a.cc;
  const double* dzp = a.dzp;
  double rhoup[KMAX_CONV], rholo[KMAX_CONV];
  for (int l = 0; l < km; ++l) { rhoup[l] = 0.0; rholo[l] = 0.0; }
  auto T = [&](int l) -> double& { return at[(long)l * A + q]; };
  auto S = [&](int l) -> double& { return at[F + (long)l * A + q]; };
  const int kcon = a.kmt[q];
  if (kcon != 0) {
    int lcon = 0;
    for (int l = 0; l < km - 1; ++l) {
      const int l1 = l + 1;
      rhoup[l1] = conv_rho(cc, km, T(l1) - to[l1], S(l1) - so[l1], l1);
      rholo[l] = conv_rho(cc, km, T(l) - to[l1], S(l) - so[l1], l1);
    }
    for (int k = kcon - 1; k >= 1; --k)
      if (rholo[k - 1] > rhoup[k]) lcon = k;
    if (lcon != 0) {
      for (;;) {
        int lcona = lcon, lconb = lcon + 1;
        double dztsum = dzp[lcona - 1] + dzp[lconb - 1];
        double trasum[2];
        for (int n = 0; n < 2; ++n) {
          double* X = at + n * F;
          trasum[n] = X[(long)(lcona - 1) * A + q] * dzp[lcona - 1] + X[(long)(lconb - 1) * A + q] * dzp[lconb - 1];
          const double tramix = trasum[n] / dztsum;
          X[(long)(lcona - 1) * A + q] = tramix;
          X[(long)(lconb - 1) * A + q] = tramix;
        }
        for (;;) {
          if (lconb != kcon) {
            const int l1 = lconb + 1;
            rholo[lconb - 1] = conv_rho(cc, km, T(lconb - 1) - to[l1 - 1], S(lconb - 1) - so[l1 - 1], l1 - 1);
            if (rholo[lconb - 1] > rhoup[l1 - 1]) {
              lconb = lconb + 1;
              dztsum = dztsum + dzp[lconb - 1];
              for (int n = 0; n < 2; ++n) {
                double* X = at + n * F;
                trasum[n] = trasum[n] + X[(long)(lconb - 1) * A + q] * dzp[lconb - 1];
                const double tramix = trasum[n] / dztsum;
                for (int lm = lcona - 1; lm < lconb; ++lm) X[(long)lm * A + q] = tramix;
              }
              continue;
            }
          }
          if (lcona > 1) {
            const int l1 = lcona - 1;
            rholo[l1 - 1] = conv_rho(cc, km, T(l1 - 1) - to[lcona - 1], S(l1 - 1) - so[lcona - 1], lcona - 1);
            rhoup[lcona - 1] = conv_rho(cc, km, T(lcona - 1) - to[lcona - 1], S(lcona - 1) - so[lcona - 1], lcona - 1);
            if (rholo[lcona - 2] > rhoup[lcona - 1]) {
              lcona = lcona - 1;
              dztsum = dztsum + dzp[lcona - 1];
              for (int n = 0; n < 2; ++n) {
                double* X = at + n * F;
                trasum[n] = trasum[n] + X[(long)(lcona - 1) * A + q] * dzp[lcona - 1];
                const double tramix = trasum[n] / dztsum;
                for (int lm = lcona; lm <= lconb; ++lm) X[(long)(lm - 1) * A + q] = tramix;
              }
              continue;
            }
          }
          break;
        }
        if (lconb == kcon) break;
        lcon = lconb;
        bool done = false;
        for (;;) {
          lcon = lcon + 1;
          if (lcon == kcon) { done = true; break; }
          if (rholo[lcon - 1] <= rhoup[lcon]) continue;
          break;
        }
        if (done) break;
      }
    }
  }
  const double c2dtts = a.p.dts;
  for (int n = 0; n < 2; ++n)
    for (int k = 0; k < km; ++k) {
      const long c = n * F + (long)k * A + q;
      const double vit = (k < kcon) ? 1.0 : 0.0;
      const double d = (at[c] - atb[n * FB + (long)(k + 1) * A + q]) / c2dtts * vit;
      a.dt_conv[c] = d;
      a.tend[c] += d;
      atb[n * FB + (long)(k + 1) * A + q] = at[c];
    }
}

// ---------------------------------------------------------------- icesnow
// icesnow_cu (icesnow.cpp:15-68): one thread per point of the domain, halo
// included, i fastest across a warp.  Surface freezing of ocean columns into
// QICE with the brine term on S, melting of QICE where the surface is above
// the freezing point, then T raised to tbice at every level (land included).
// Operation order is the reference's, so the results are bit-identical; the
// FRC_CORE reset of QICE is folded in (0 + x == x exactly).  HBM-bound: T is
// read at every level and written only where it changes.
__global__ void k_icesnow(Arena a, double tbice, double cp, double latice, int reset) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= a.imt || j >= a.jmt) return;
  const long q = (long)j * a.imt + i;
  const long A = a.A;
  double* T = a.at[a.cur] + q;
  double* S = T + a.F;
  const double sal_ocn = 34.7e0, sal_ice = 4.0e0;
  double qi = reset ? 0.0 : a.qice[q];
  double t0 = T[0];
  if (t0 < tbice && a.kmt[q] > 0) {
    const double tdiff = tbice - t0;
    qi += tdiff * a.dzp[0] / a.dzp[0];
    S[0] += tdiff * (sal_ocn - sal_ice) * cp / latice * 0.001e0;
    t0 = tbice;
    T[0] = t0;
  }
  if (qi > 0.0 && t0 > tbice) {
    const double tdiff = fmin(t0 - tbice, qi);
    qi -= tdiff;
    t0 -= tdiff;
    T[0] = t0;
    S[0] -= tdiff * (sal_ocn - sal_ice) * cp / latice * 0.001e0;
  }
  if (t0 < tbice) T[0] = tbice;
  a.qice[q] = qi;
  // the levels below in groups of 8: all loads of a group issued before any
  // store, so that a warp keeps 8 rows in flight
  for (int k0 = 1; k0 < a.km; k0 += 8) {
    double v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) v[u] = (k0 + u < a.km) ? T[(k0 + u) * A] : 0.0;
#pragma unroll
    for (int u = 0; u < 8; ++u)
      if (k0 + u < a.km && v[u] < tbice) T[(k0 + u) * A] = tbice;
  }
}

// ---------------------------------------------------------------- masks
// boundary.F90:24-52, grid.F90:1343-1346, grid.F90:2030-2051
__global__ void k_masks(Arena a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int imt = a.imt, jmt = a.jmt;
  if (i >= imt || j >= jmt) return;
  const long q = (long)j * imt + i;
  const int* kmt = a.kmt;
  int ku = 0;
  if (j < jmt - 1 && i >= 1) ku = min(min(kmt[q - 1], kmt[q]), min(kmt[q + imt - 1], kmt[q + imt]));
  a.kmu[q] = ku;
  a.kmtn[q] = j > 0 ? kmt[q - imt] : 0;
  a.kmts[q] = j < jmt - 1 ? kmt[q + imt] : 0;
  a.kmte[q] = i < imt - 1 ? kmt[q + 1] : 0;
  a.kmtw[q] = i > 0 ? kmt[q - 1] : 0;
}

// KMU ghost fill, SW-corner location (no averaging, top physical row kept)
__global__ void k_kmu_halo(Arena a) {
  const int imt = a.imt, jmt = a.jmt, nx = imt - 4;
  int* f = a.kmu;
  // ghost rows from the fold first read only physical rows 2,3; E-W copies
  // touch only ghost columns of physical rows - disjoint, so one pass is safe
  for (long m = threadIdx.x; m < (long)imt * jmt; m += blockDim.x) {
    const int j = (int)(m / imt), i = (int)(m % imt);
    if (j >= 2 && j < jmt - 2 && a.ew_cyclic) {
      if (i < 2) f[m] = f[(long)j * imt + nx + i];
      else if (i >= imt - 2) f[m] = f[(long)j * imt + i - nx];
    }
  }
  __syncthreads();
  if (!a.tripole) return;
  for (int i = threadIdx.x; i < imt; i += blockDim.x) {
    int g = halo_iglobal(i, nx, a.ew_cyclic);
    int isrc = nx - g + 1;
    if (isrc == 0) isrc = nx;
    if (isrc > nx) isrc = isrc - nx;  // g == 0 on a closed side maps to nx+1; keep it in range
    f[i] = f[3L * imt + isrc + 1];          // row 0 <- physical row 3
    f[imt + i] = f[2L * imt + isrc + 1];    // row 1 <- physical row 2
  }
}

__global__ void k_inv_depth(Arena a) {
  const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= a.A) return;
  double s = 0.0;
  for (int k = 0; k < a.km; ++k) s = s + (k < a.kmt[q] ? 1.0 : 0.0) * a.dzp[k];
  a.ohbt[q] = s > 0.0 ? 1.0 / s : 0.0;
  s = 0.0;
  for (int k = 0; k < a.km; ++k) s = s + (k < a.kmu[q] ? 1.0 : 0.0) * a.dzp[k];
  a.ohbu[q] = s > 0.0 ? 1.0 / s : 0.0;
  if (q < a.km) a.odzp[q] = 1.0 / a.dzp[q];
}

// ------------------------------------------------------------- reductions
constexpr int RB2 = 1024;
__global__ void k_content_first(const double* at, const double* tarea, const double* dzp, const int* kmt,
                                 int nx, int ny, int imt, long A, long n, double* part) {
  __shared__ double s[2 * RB2];
  const long base = (long)blockIdx.x * 2 * RB2;
  auto term = [&](long m) -> double {
    if (m >= n) return 0.0;
    const long per = (long)nx * ny;
    const int k = (int)(m / per);
    const long r = m % per;
    const int j = 2 + (int)(r / nx), i = 2 + (int)(r % nx);
    const long q = (long)j * imt + i;
    return (k < kmt[q]) ? tarea[q] * dzp[k] * at[(long)k * A + q] : 0.0;
  };
  const int t = threadIdx.x;
  s[t] = term(base + t);
  s[t + RB2] = term(base + t + RB2);
  for (int stride = RB2; stride > 0; stride >>= 1) {
    __syncthreads();
    if (t < stride) s[t] = s[t] + s[t + stride];
  }
  if (t == 0) part[blockIdx.x] = s[0];
}

__global__ void k_count_bad(const double* x, long n, int* count) {
  long m = (long)blockIdx.x * blockDim.x + threadIdx.x;
  int bad = 0;
  for (; m < n; m += (long)gridDim.x * blockDim.x) bad += !isfinite(x[m]);
  if (bad) atomicAdd(count, bad);
}

// ------------------------------------------------------- synthetic upload
__global__ void k_synth_state(CellTables t, double* at, double* atb, double* restore) {
  const long m = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long A = (long)t.imt * t.jmt, F = A * t.km;
  if (m >= F) return;
  const int k = (int)(m / A);
  const long r = m % A;
  const int j = (int)(r / t.imt), i = (int)(r % t.imt);
  const double T = cell_T(t, k, j, i), S = cell_S(t, k, j, i);
  at[m] = T;
  at[F + m] = S;
  if (restore) { restore[m] = T; restore[F + m] = S; }
  (void)atb;
}

__global__ void k_synth_vel(CellTables t, double ncc1, double* utf, double* vtf, double* utl, double* vtl,
                            double* akt) {
  const long m = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long A = (long)t.imt * t.jmt, F = A * t.km;
  if (m >= F) return;
  const int k = (int)(m / A);
  const long r = m % A;
  const int j = (int)(r / t.imt), i = (int)(r % t.imt);
  const double u = cell_U(t, k, j, i), v = cell_V(t, k, j, i);
  utl[m] = u; vtl[m] = v;
  utf[m] = ncc1 * u; vtf[m] = ncc1 * v;
  akt[m] = cell_akt(t, 0, k, j, i);
  akt[F + m] = cell_akt(t, 1, k, j, i);
}

}  // namespace

int launch_convadj(const Arena& a, cudaStream_t s) {
  if (a.km > KMAX_CONV) { set_error("convadj: km > %d", KMAX_CONV); return LT_E_INVALID; }
  dim3 b(8, 16), g((a.imt + 7) / 8, (a.jmt + 15) / 16);
  k_convadj<<<g, b, 0, s>>>(a);
  LT_LAUNCHED();
  return LT_OK;
}

int launch_icesnow(const Arena& a, const lt_icesnow_params& p, cudaStream_t s) {
  dim3 b(32, 8), g((a.imt + 31) / 32, (a.jmt + 7) / 8);
  k_icesnow<<<g, b, 0, s>>>(a, p.tbice, p.cp, p.latice, p.reset_qice != 0);
  LT_LAUNCHED();
  return LT_OK;
}

int launch_derive_masks(const Arena& a, cudaStream_t s) {
  dim3 b(32, 8), g((a.imt + 31) / 32, (a.jmt + 7) / 8);
  k_masks<<<g, b, 0, s>>>(a);
  LT_LAUNCHED();
  k_kmu_halo<<<1, 1024, 0, s>>>(a);
  LT_LAUNCHED();
  k_inv_depth<<<(unsigned)((a.A + 255) / 256), 256, 0, s>>>(a);
  LT_LAUNCHED();
  return LT_OK;
}

int launch_tracer_content(const Arena& a, cudaStream_t s) {
  const long n = (long)a.nx * a.ny * a.km;
  for (int tr = 0; tr < 2; ++tr) {
    long nb = (n + 2 * RB2 - 1) / (2 * RB2);
    k_content_first<<<(unsigned)nb, RB2, 0, s>>>(a.at[a.cur] + tr * a.F, a.tarea, a.dzp, a.kmt, a.nx, a.ny, a.imt,
                                                  a.A, n, a.red_part);
    LT_LAUNCHED();
    int rc = launch_tree_sum(a.red_part, nb, a.red_part + nb, a.scalars + 1 + tr, s);
    if (rc) return rc;
  }
  return LT_OK;
}

int launch_check_numeric(const Arena& a, cudaStream_t s) {
  LT_CUDA_OK(cudaMemsetAsync(a.status, 0, sizeof(int), s));
  k_count_bad<<<1184, 256, 0, s>>>(a.at[a.cur], 2 * a.F, a.status);
  LT_LAUNCHED();
  return LT_OK;
}

}  // namespace lt

using namespace lt;

extern "C" int lt_synth_upload(const lt_synth* syn, lt_domain* dom);

namespace {
template <class T>
int up(cudaStream_t s, T** dst, const std::vector<T>& v, std::vector<void*>& owned) {
  void* p = nullptr;
  if (cudaMalloc(&p, v.size() * sizeof(T)) != cudaSuccess) return LT_E_OOM;
  owned.push_back(p);
  cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s);
  *dst = static_cast<T*>(p);
  return LT_OK;
}
}  // namespace

extern "C" int lt_get_field_device(lt_domain* d, int f, void* dst, size_t nbytes);
extern "C" int lt_set_field_device(lt_domain* d, int f, const void* src, size_t nbytes);

// Device-generated 3-D inputs, host-built 2-D/1-D inputs.
extern "C" int lt_synth_upload(const lt_synth* syn, lt_domain* dom) {
  const Domain* d = lt_synth_domain(syn);
  if (!d || !dom) return LT_E_INVALID;
  lt_grid g;
  lt_synth_grid(syn, &g);
  // 2-D / 1-D from the host builder
  const int two_d[] = {LT_F_H0F, LT_F_H0L, LT_F_SWV, LT_F_NSWV, LT_F_SST, LT_F_SSS, LT_F_FRESH, LT_F_SEAICE,
                       LT_F_TAREA, LT_F_TAREA_R, LT_F_HTW, LT_F_HTS, LT_F_HUN, LT_F_HUE, LT_F_DXU, LT_F_DYU,
                       LT_F_AHF, LT_F_DTN, LT_F_DTS, LT_F_DTE, LT_F_DTW, LT_F_OHBT, LT_F_OHBU, LT_F_AU0,
                       LT_F_AUS, LT_F_AUW, LT_F_AUSW, LT_F_KMT, LT_F_KMU, LT_F_KMTN, LT_F_KMTS, LT_F_KMTE,
                       LT_F_KMTW, LT_F_DZP, LT_F_ODZP, LT_F_ODZT, LT_F_PEN, LT_F_TO, LT_F_SO, LT_F_C};
  for (int f : two_d) {
    const size_t nb = field_bytes(f, d->imt, d->jmt, d->km);
    std::vector<char> buf(nb);
    int rc = lt_synth_field(syn, f, buf.data(), nb);
    if (!rc) rc = lt_set_field(dom, f, buf.data(), nb);
    if (rc) return rc;
  }
  // tables for the device expansion
  cudaStream_t s = nullptr;
  std::vector<void*> owned;
  CellTables t = d->tables();
  int rc = LT_OK;
  double *tprof, *ssurf, *psi, *uprof, *rdyu, *rdxu, *akt_tab;
  int *kmt, *dmin;
  rc |= up(s, &tprof, d->tprof, owned);
  rc |= up(s, &ssurf, d->ssurf, owned);
  rc |= up(s, &psi, d->psi, owned);
  rc |= up(s, &uprof, d->uprof, owned);
  rc |= up(s, &rdyu, d->rdyu, owned);
  rc |= up(s, &rdxu, d->rdxu, owned);
  rc |= up(s, &akt_tab, d->akt_tab, owned);
  rc |= up(s, &kmt, d->kmt, owned);
  rc |= up(s, &dmin, d->dmin, owned);
  if (rc) { for (void* p : owned) cudaFree(p); return LT_E_OOM; }
  t.tprof = tprof; t.ssurf = ssurf; t.psi = psi; t.uprof = uprof; t.rdyu = rdyu; t.rdxu = rdxu;
  t.akt_tab = akt_tab; t.kmt = kmt; t.dmin = dmin;
  const long A = (long)d->imt * d->jmt, F = A * d->km, FB = A * (d->km + 1);
  double *at = nullptr, *atb = nullptr, *vel = nullptr;
  if (cudaMalloc(&at, 2 * F * sizeof(double)) != cudaSuccess || cudaMalloc(&atb, 2 * FB * sizeof(double)) != cudaSuccess) {
    for (void* p : owned) cudaFree(p);
    if (at) cudaFree(at);
    return LT_E_OOM;
  }
  const unsigned nb = (unsigned)((F + 255) / 256);
  k_synth_state<<<nb, 256, 0, s>>>(t, at, atb, nullptr);
  launch_halo_r8(at, 2 * d->km, d->imt, d->jmt, d->cfg.ew_cyclic, d->cfg.tripole, s);
  for (int n = 0; n < 2; ++n) {
    cudaMemsetAsync(atb + n * FB, 0, A * sizeof(double), s);
    cudaMemcpyAsync(atb + n * FB + A, at + n * F, F * sizeof(double), cudaMemcpyDeviceToDevice, s);
  }
  cudaStreamSynchronize(s);
  rc = lt_set_field_device(dom, LT_F_AT, at, 2 * F * sizeof(double));
  if (!rc) rc = lt_set_field_device(dom, LT_F_ATB, atb, 2 * FB * sizeof(double));
  cudaFree(atb);
  if (!rc) {
    if (cudaMalloc(&vel, 6 * F * sizeof(double)) != cudaSuccess) rc = LT_E_OOM;
  }
  if (!rc) {
    k_synth_vel<<<nb, 256, 0, s>>>(t, (double)(d->cfg.ncc + 1), vel, vel + F, vel + 2 * F, vel + 3 * F, vel + 4 * F);
    cudaStreamSynchronize(s);
    rc = lt_set_field_device(dom, LT_F_UTF, vel, F * sizeof(double));
    if (!rc) rc = lt_set_field_device(dom, LT_F_VTF, vel + F, F * sizeof(double));
    if (!rc) rc = lt_set_field_device(dom, LT_F_UTL, vel + 2 * F, F * sizeof(double));
    if (!rc) rc = lt_set_field_device(dom, LT_F_VTL, vel + 3 * F, F * sizeof(double));
    if (!rc) rc = lt_set_field_device(dom, LT_F_AKT, vel + 4 * F, 2 * F * sizeof(double));
    cudaFree(vel);
  }
  cudaFree(at);
  for (void* p : owned) cudaFree(p);
  if (cudaGetLastError() != cudaSuccess && !rc) rc = LT_E_CUDA;
  return rc;
}
