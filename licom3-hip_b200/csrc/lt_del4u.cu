// lt_del4u.cu - biharmonic friction of the momentum equations with its
// flow-dependent factor: readyc_'s BIHAR sequence (readyc.cpp:1754-1775) of
// hdel4_div, hdel4_grad, hdel4_zcurl, hdel4_grad, hdiffu_del4_0 and
// hdiffu_del4_1 (readyc.cpp:343-577) as ONE kernel.  Compiled with
// -fmad=false; every expression keeps the reference's operation order, so the
// results are bit-identical to it.
//
// One CTA per 32x8 tile of U points and level.  The reference passes the
// level through HBM six times (divergence and curl at T points, the squared
// gradients of both into am_factor, the first Laplacian d2uk/d2vk, the
// second); here the tile's velocities with a 3-point halo come into shared
// memory once and each stage works on the halo region the next one needs:
//   T points (11x35): divergence and curl,
//   U points with a 1-point halo (10x34): am_factor, then d2uk and d2vk,
//   the tile's own U points: the second Laplacian into dlu/dlv and the drag
//   speed c0f*|u| the reference leaves in wka.
// The domain is one block: ib = jb = 3, ie = imt-2, je = jmt-2 (the
// reference's 1-based block bounds).
#include "lt_common.cuh"
#include "lt_domain.h"

namespace lt {
namespace {

constexpr int DX = 32, DY = 8, DT = DX * DY;
constexpr int UW = DX + 5, UH = DY + 4;   // velocities: columns x0-3 .. x0+DX+1, rows y0-2 .. y0+DY+1
constexpr int TW = DX + 3, TH = DY + 3;   // divergence, curl: columns x0-2 .. x0+DX, rows y0-1 .. y0+DY+1
constexpr int HW = DX + 2, HH = DY + 2;   // 1-halo U points: columns x0-1 .. x0+DX, rows y0-1 .. y0+DY

struct Del4Smem {
  double u[UH][UW], v[UH][UW];
  double dv[TH][TW], cu[TH][TW];
  double amfac[HH][HW];
  double d2u[HH][HW], d2v[HH][HW];
};

__global__ void __launch_bounds__(DT) k_del4u(Arena a, double am, double c0f) {
  __shared__ Del4Smem S;
  const int imt = a.imt, jmt = a.jmt;
  const int k = blockIdx.z;
  const long A = a.A;
  const long lvl = (long)k * A;
  const int x0 = blockIdx.x * DX, y0 = blockIdx.y * DY;
  const int tid = threadIdx.y * DX + threadIdx.x;
  const int ib = 3, jb = 3, ie = imt - 2, je = jmt - 2;   // one block
  const double p5 = 0.5;

  // ---- velocities of the tile and its halo (0 outside the domain, never used there)
  for (int m = tid; m < UH * UW; m += DT) {
    const int r = m / UW, c = m % UW;
    const int j = y0 - 2 + r, i = x0 - 3 + c;
    const bool in = j >= 0 && j < jmt && i >= 0 && i < imt;
    const long q = lvl + (long)j * imt + i;
    S.u[r][c] = in ? a.up[q] : 0.0;
    S.v[r][c] = in ? a.vp[q] : 0.0;
  }
  __syncthreads();
  // U-point value at global (j, i) from the staged box
  auto U = [&](int j, int i) -> double { return S.u[j - (y0 - 2)][i - (x0 - 3)]; };
  auto V = [&](int j, int i) -> double { return S.v[j - (y0 - 2)][i - (x0 - 3)]; };

  // ---- divergence (hdel4_div, readyc.cpp:372-403) and curl (hdel4_zcurl,
  // readyc.cpp:343-370) at T points
  for (int m = tid; m < TH * TW; m += DT) {
    const int r = m / TW, c = m % TW;
    const int j = y0 - 1 + r, i = x0 - 2 + c;
    double dv = 0.0, cu = 0.0;
    if (j >= 0 && j < jmt && i >= 0 && i < imt) {
      const long t = (long)j * imt + i;
      const bool wet = k <= a.kmt[t] - 1;
      if (i < imt - 1 && j >= 1 && wet) {
        dv = 0.5 *
             ((U(j, i + 1) + U(j - 1, i + 1)) * __ldg(a.htw + t + 1) - (U(j, i) + U(j - 1, i)) * __ldg(a.htw + t) +
              (V(j, i + 1) + V(j, i)) * __ldg(a.hts + t) - (V(j - 1, i + 1) + V(j - 1, i)) * __ldg(a.hts + t - imt)) *
             __ldg(a.tarea_r + t);
      }
      if (i >= 1 && j >= 1 && wet) {
        cu = 0.5 * ((V(j, i) * __ldg(a.dyu + t) + V(j - 1, i) * __ldg(a.dyu + t - imt) -
                     V(j, i - 1) * __ldg(a.dyu + t - 1) - V(j - 1, i - 1) * __ldg(a.dyu + t - imt - 1) -
                     U(j, i) * __ldg(a.dxu + t) - U(j, i - 1) * __ldg(a.dxu + t - 1) +
                     U(j - 1, i) * __ldg(a.dxu + t - imt) + U(j - 1, i - 1) * __ldg(a.dxu + t - imt - 1)));
      }
    }
    S.dv[r][c] = dv;
    S.cu[r][c] = cu;
  }
  __syncthreads();
  auto Dv = [&](int j, int i) -> double { return S.dv[j - (y0 - 1)][i - (x0 - 2)]; };
  auto Cu = [&](int j, int i) -> double { return S.cu[j - (y0 - 1)][i - (x0 - 2)]; };

  // ---- am_factor (hdel4_grad twice, readyc.cpp:405-442, on a zeroed array)
  // and the first Laplacian d2uk, d2vk (hdiffu_del4_0, readyc.cpp:444-507)
  // on the tile's U points and their 1-point halo
  for (int m = tid; m < HH * HW; m += DT) {
    const int r = m / HW, c = m % HW;
    const int j = y0 - 1 + r, i = x0 - 1 + c;
    double d2u = 0.0, d2v = 0.0;
    if (j >= 0 && j < jmt && i >= 0 && i < imt) {
      const long q = (long)j * imt + i;
      const int kmu = a.kmu[q];
      double amfac = 0.0;
      if (1 <= i && j < jmt - 1 && k <= kmu - 1) {
        const double dxr = __ldg(a.dxur + q), dyr = __ldg(a.dyur + q);
        const double gxd = dxr * p5 * (Dv(j + 1, i) - Dv(j, i - 1) - Dv(j + 1, i - 1) + Dv(j, i));
        const double gyd = dyr * p5 * (Dv(j + 1, i) - Dv(j, i - 1) + Dv(j + 1, i - 1) - Dv(j, i));
        amfac = 0.0 + (gxd * gxd + gyd * gyd);
        const double gxc = dxr * p5 * (Cu(j + 1, i) - Cu(j, i - 1) - Cu(j + 1, i - 1) + Cu(j, i));
        const double gyc = dyr * p5 * (Cu(j + 1, i) - Cu(j, i - 1) + Cu(j + 1, i - 1) - Cu(j, i));
        amfac = amfac + (gxc * gxc + gyc * gyc);
      }
      double am_f = 1.0e0, hu = 0.0, hv = 0.0;
      const double amf = __ldg(a.amf + q);
      if (j >= jb - 2 && j <= je && i >= ib - 2 && i <= ie && k <= kmu - 1) {
        const double t_area = sqrt(1.0e0 / __ldg(a.uarea_r + q));
        const double dxdy = t_area * t_area * t_area * t_area * t_area * 45.0e0;
        am_f = sqrt(amfac) * dxdy / fabs(am * amf);
        am_f = fmin(40.0e0, am_f);
        am_f = fmax(1.0e0, am_f);
        const double duc = __ldg(a.duc + q), dum = __ldg(a.dum + q), dun = __ldg(a.dun + q), dus = __ldg(a.dus + q);
        const double due = __ldg(a.due + q), duw = __ldg(a.duw + q), dmc = __ldg(a.dmc + q), dmn = __ldg(a.dmn + q);
        const double dms = __ldg(a.dms + q), dme = __ldg(a.dme + q), dmw = __ldg(a.dmw + q);
        hu = (((duc + dum) * U(j, i) + dun * U(j - 1, i) + dus * U(j + 1, i) + due * U(j, i + 1) +
               duw * U(j, i - 1)) +
              (dmc * V(j, i) + dmn * V(j - 1, i) + dms * V(j + 1, i) + dme * V(j, i + 1) + dmw * V(j, i - 1)));
        hv = (((duc + dum) * V(j, i) + dun * V(j - 1, i) + dus * V(j + 1, i) + due * V(j, i + 1) +
               duw * V(j, i - 1)) -
              (dmc * U(j, i) + dmn * U(j - 1, i) + dms * U(j + 1, i) + dme * U(j, i + 1) + dmw * U(j, i - 1)));
      }
      d2u = am_f * amf * hu;
      d2v = am_f * amf * hv;
    }
    S.d2u[r][c] = d2u;
    S.d2v[r][c] = d2v;
  }
  __syncthreads();

  // ---- second Laplacian into dlu, dlv and the drag speed (hdiffu_del4_1,
  // readyc.cpp:509-577) on the tile's own U points
  const int j = y0 + threadIdx.y, i = x0 + threadIdx.x;
  if (j >= jmt || i >= imt) return;
  const long q = (long)j * imt + i;
  const int r = threadIdx.y + 1, c = threadIdx.x + 1;   // in the 1-halo arrays
  double hu = 0.0, hv = 0.0;
  if (j >= jb - 1 && j < je && i >= ib - 1 && i < ie) {
    const double duc = __ldg(a.duc + q), dum = __ldg(a.dum + q), dun = __ldg(a.dun + q), dus = __ldg(a.dus + q);
    const double due = __ldg(a.due + q), duw = __ldg(a.duw + q), dmc = __ldg(a.dmc + q), dmn = __ldg(a.dmn + q);
    const double dms = __ldg(a.dms + q), dme = __ldg(a.dme + q), dmw = __ldg(a.dmw + q);
    hu = am * (((duc + dum) * S.d2u[r][c] + dun * S.d2u[r - 1][c] + dus * S.d2u[r + 1][c] +
                due * S.d2u[r][c + 1] + duw * S.d2u[r][c - 1]) +
               (dmc * S.d2v[r][c] + dmn * S.d2v[r - 1][c] + dms * S.d2v[r + 1][c] + dme * S.d2v[r][c + 1] +
                dmw * S.d2v[r][c - 1]));
    hv = am * (((duc + dum) * S.d2v[r][c] + dun * S.d2v[r - 1][c] + dus * S.d2v[r + 1][c] +
                due * S.d2v[r][c + 1] + duw * S.d2v[r][c - 1]) -
               (dmc * S.d2u[r][c] + dmn * S.d2u[r - 1][c] + dms * S.d2u[r + 1][c] + dme * S.d2u[r][c + 1] +
                dmw * S.d2u[r][c - 1]));
  }
  if (k > a.kmu[q] - 1) {
    hu = 0.0;
    hv = 0.0;
  }
  const long g = lvl + q;
  if (1 <= j && j < jmt - 1 && 1 <= i && i < imt - 1) {
    a.dlv[g] = a.dlv[g] + hv;
    a.dlu[g] = a.dlu[g] + hu;
  }
  const double uu = S.u[threadIdx.y + 2][threadIdx.x + 3], vv = S.v[threadIdx.y + 2][threadIdx.x + 3];
  a.wka_drag[g] = c0f * sqrt(uu * uu + vv * vv);
}

}  // namespace

int launch_del4u(const Arena& a, double am, double c0f, cudaStream_t s) {
  dim3 b(DX, DY), g((a.imt + DX - 1) / DX, (a.jmt + DY - 1) / DY, a.km);
  k_del4u<<<g, b, 0, s>>>(a, am, c0f);
  LT_LAUNCHED();
  return LT_OK;
}

}  // namespace lt

using namespace lt;

extern "C" int lt_hdiffu_del4(lt_domain* d, const lt_del4u_params* p) {
  if (!d || !p) {
    set_error("lt_hdiffu_del4: invalid arguments");
    return LT_E_INVALID;
  }
  int rc = ensure_mom(d);
  if (rc) return rc;
  return launch_del4u(d->a, p->am, p->c0f, d->stream);
}
