// lt_del4u.cu - biharmonic friction of the momentum equations with its
// flow-dependent factor: readyc_'s BIHAR sequence (readyc.cpp:1754-1775) of
// hdel4_div, hdel4_grad, hdel4_zcurl, hdel4_grad, hdiffu_del4_0 and
// hdiffu_del4_1 (readyc.cpp:343-577) as ONE kernel.  Compiled with
// -fmad=false; every expression keeps the reference's operation order, so the
// results are bit-identical to it.
//
// One CTA per 32x8 tile of U points marches the levels.  The reference passes
// each level through HBM six times (divergence and curl at T points, the
// squared gradients of both into am_factor, the first Laplacian d2uk/d2vk,
// the second) and reads the 2-D stencil coefficients and metrics again in
// every one of those passes.  Here the coefficients and metrics of the tile
// and its halo come into shared memory once per tile (with the level-free
// parts of the flow-dependent factor, sqrt(1/uarea_r)^5 * 45 and |am*amf|,
// formed there by the same expressions); per level the tile's velocities with
// a 3-point halo arrive once (the next level's are loaded into registers while
// this one is computed) and each stage works on the halo region the next needs:
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
constexpr int UW = DX + 5, UH = DY + 4;   // velocities, T metrics: columns x0-3 .. x0+DX+1, rows y0-2 .. y0+DY+1
constexpr int TW = DX + 3, TH = DY + 3;   // divergence, curl: columns x0-2 .. x0+DX, rows y0-1 .. y0+DY+1
constexpr int HW = DX + 2, HH = DY + 2;   // 1-halo U points: columns x0-1 .. x0+DX, rows y0-1 .. y0+DY
constexpr int UPT = (UH * UW + DT - 1) / DT;   // velocity points per thread

// stencil coefficients on the 1-halo U points
enum { C_DUCM = 0, C_DUN, C_DUS, C_DUE, C_DUW, C_DMC, C_DMN, C_DMS, C_DME, C_DMW, C_AMF, C_DXDY, C_AMAMF, NC };
// metrics on the velocity box
enum { M_HTW = 0, M_HTS, M_TAR, M_DXU, M_DYU, NM };

struct Del4Smem {
  double cf[NC][HH][HW];
  double dxr[HH][HW], dyr[HH][HW];
  double met[NM][UH][UW];
  int kmu[HH][HW];
  int kmt[TH][TW];
  double u[UH][UW], v[UH][UW];
  double dv[TH][TW], cu[TH][TW];
  double d2u[HH][HW], d2v[HH][HW];
};

__global__ void __launch_bounds__(DT, 2) k_del4u(Arena a, double am, double c0f) {
  extern __shared__ __align__(16) unsigned char smem_d4[];
  Del4Smem& S = *reinterpret_cast<Del4Smem*>(smem_d4);
  const int imt = a.imt, jmt = a.jmt, km = a.km;
  const long A = a.A;
  const int x0 = blockIdx.x * DX, y0 = blockIdx.y * DY;
  const int tid = threadIdx.y * DX + threadIdx.x;
  const int ib = 3, jb = 3, ie = imt - 2, je = jmt - 2;   // one block
  const double p5 = 0.5;

  // ---- level-free data of the tile
  for (int m = tid; m < HH * HW; m += DT) {
    const int r = m / HW, c = m % HW;
    const int j = y0 - 1 + r, i = x0 - 1 + c;
    const bool in = j >= 0 && j < jmt && i >= 0 && i < imt;
    const long q = in ? (long)j * imt + i : 0;
    S.kmu[r][c] = in ? a.kmu[q] : 0;
    S.dxr[r][c] = in ? a.dxur[q] : 0.0;
    S.dyr[r][c] = in ? a.dyur[q] : 0.0;
    S.cf[C_DUCM][r][c] = in ? a.duc[q] + a.dum[q] : 0.0;
    S.cf[C_DUN][r][c] = in ? a.dun[q] : 0.0;
    S.cf[C_DUS][r][c] = in ? a.dus[q] : 0.0;
    S.cf[C_DUE][r][c] = in ? a.due[q] : 0.0;
    S.cf[C_DUW][r][c] = in ? a.duw[q] : 0.0;
    S.cf[C_DMC][r][c] = in ? a.dmc[q] : 0.0;
    S.cf[C_DMN][r][c] = in ? a.dmn[q] : 0.0;
    S.cf[C_DMS][r][c] = in ? a.dms[q] : 0.0;
    S.cf[C_DME][r][c] = in ? a.dme[q] : 0.0;
    S.cf[C_DMW][r][c] = in ? a.dmw[q] : 0.0;
    const double amf = in ? a.amf[q] : 0.0;
    S.cf[C_AMF][r][c] = amf;
    double dxdy = 0.0;
    if (in) {
      const double t_area = sqrt(1.0e0 / a.uarea_r[q]);
      dxdy = t_area * t_area * t_area * t_area * t_area * 45.0e0;
    }
    S.cf[C_DXDY][r][c] = dxdy;
    S.cf[C_AMAMF][r][c] = fabs(am * amf);
  }
  for (int m = tid; m < UH * UW; m += DT) {
    const int r = m / UW, c = m % UW;
    const int j = y0 - 2 + r, i = x0 - 3 + c;
    const bool in = j >= 0 && j < jmt && i >= 0 && i < imt;
    const long q = in ? (long)j * imt + i : 0;
    S.met[M_HTW][r][c] = in ? a.htw[q] : 0.0;
    S.met[M_HTS][r][c] = in ? a.hts[q] : 0.0;
    S.met[M_TAR][r][c] = in ? a.tarea_r[q] : 0.0;
    S.met[M_DXU][r][c] = in ? a.dxu[q] : 0.0;
    S.met[M_DYU][r][c] = in ? a.dyu[q] : 0.0;
  }
  for (int m = tid; m < TH * TW; m += DT) {
    const int r = m / TW, c = m % TW;
    const int j = y0 - 1 + r, i = x0 - 2 + c;
    S.kmt[r][c] = (j >= 0 && j < jmt && i >= 0 && i < imt) ? a.kmt[(long)j * imt + i] : 0;
  }

  // the velocity box points of this thread and the first level's values
  long vq[UPT];
  bool vin[UPT];
  double ru[UPT], rv[UPT];
#pragma unroll
  for (int p = 0; p < UPT; ++p) {
    const int m = tid + p * DT;
    const int j = y0 - 2 + m / UW, i = x0 - 3 + m % UW;
    vin[p] = m < UH * UW && j >= 0 && j < jmt && i >= 0 && i < imt;
    vq[p] = vin[p] ? (long)j * imt + i : 0;
    ru[p] = vin[p] ? a.up[vq[p]] : 0.0;
    rv[p] = vin[p] ? a.vp[vq[p]] : 0.0;
  }
  // the own point's tendencies, loaded a level ahead like the velocities
  const int oj = y0 + threadIdx.y, oi = x0 + threadIdx.x;
  const bool own_upd = oj < jmt && oi < imt && 1 <= oj && oj < jmt - 1 && 1 <= oi && oi < imt - 1;
  const long oq = own_upd ? (long)oj * imt + oi : 0;
  double rdlu = own_upd ? a.dlu[oq] : 0.0, rdlv = own_upd ? a.dlv[oq] : 0.0;
  // global (j, i) -> staged box
  auto U = [&](int j, int i) -> double { return S.u[j - (y0 - 2)][i - (x0 - 3)]; };
  auto V = [&](int j, int i) -> double { return S.v[j - (y0 - 2)][i - (x0 - 3)]; };
  auto Mt = [&](int w, int j, int i) -> double { return S.met[w][j - (y0 - 2)][i - (x0 - 3)]; };
  auto Dv = [&](int j, int i) -> double { return S.dv[j - (y0 - 1)][i - (x0 - 2)]; };
  auto Cu = [&](int j, int i) -> double { return S.cu[j - (y0 - 1)][i - (x0 - 2)]; };

  for (int k = 0; k < km; ++k) {
    const long lvl = (long)k * A;
    // the previous level is done with the box (barrier at the end of the loop)
#pragma unroll
    for (int p = 0; p < UPT; ++p) {
      const int m = tid + p * DT;
      if (m < UH * UW) {
        S.u[m / UW][m % UW] = ru[p];
        S.v[m / UW][m % UW] = rv[p];
      }
    }
    __syncthreads();
    const double dlu_k = rdlu, dlv_k = rdlv;
    // next level's velocities and tendencies in flight during this level's stages
    if (k + 1 < km) {
#pragma unroll
      for (int p = 0; p < UPT; ++p) {
        ru[p] = vin[p] ? a.up[lvl + A + vq[p]] : 0.0;
        rv[p] = vin[p] ? a.vp[lvl + A + vq[p]] : 0.0;
      }
      rdlu = own_upd ? a.dlu[lvl + A + oq] : 0.0;
      rdlv = own_upd ? a.dlv[lvl + A + oq] : 0.0;
    }

    // ---- divergence (hdel4_div, readyc.cpp:372-403) and curl (hdel4_zcurl,
    // readyc.cpp:343-370) at T points
    for (int m = tid; m < TH * TW; m += DT) {
      const int r = m / TW, c = m % TW;
      const int j = y0 - 1 + r, i = x0 - 2 + c;
      double dv = 0.0, cu = 0.0;
      if (j >= 0 && j < jmt && i >= 0 && i < imt) {
        const bool wet = k <= S.kmt[r][c] - 1;
        if (i < imt - 1 && j >= 1 && wet) {
          dv = 0.5 *
               ((U(j, i + 1) + U(j - 1, i + 1)) * Mt(M_HTW, j, i + 1) - (U(j, i) + U(j - 1, i)) * Mt(M_HTW, j, i) +
                (V(j, i + 1) + V(j, i)) * Mt(M_HTS, j, i) - (V(j - 1, i + 1) + V(j - 1, i)) * Mt(M_HTS, j - 1, i)) *
               Mt(M_TAR, j, i);
        }
        if (i >= 1 && j >= 1 && wet) {
          cu = 0.5 * ((V(j, i) * Mt(M_DYU, j, i) + V(j - 1, i) * Mt(M_DYU, j - 1, i) -
                       V(j, i - 1) * Mt(M_DYU, j, i - 1) - V(j - 1, i - 1) * Mt(M_DYU, j - 1, i - 1) -
                       U(j, i) * Mt(M_DXU, j, i) - U(j, i - 1) * Mt(M_DXU, j, i - 1) +
                       U(j - 1, i) * Mt(M_DXU, j - 1, i) + U(j - 1, i - 1) * Mt(M_DXU, j - 1, i - 1)));
        }
      }
      S.dv[r][c] = dv;
      S.cu[r][c] = cu;
    }
    __syncthreads();

    // ---- am_factor (hdel4_grad twice, readyc.cpp:405-442, on a zeroed array)
    // and the first Laplacian d2uk, d2vk (hdiffu_del4_0, readyc.cpp:444-507)
    // on the tile's U points and their 1-point halo
    for (int m = tid; m < HH * HW; m += DT) {
      const int r = m / HW, c = m % HW;
      const int j = y0 - 1 + r, i = x0 - 1 + c;
      double d2u = 0.0, d2v = 0.0;
      if (j >= 0 && j < jmt && i >= 0 && i < imt) {
        const int kmu = S.kmu[r][c];
        double amfac = 0.0;
        if (1 <= i && j < jmt - 1 && k <= kmu - 1) {
          const double dxr = S.dxr[r][c], dyr = S.dyr[r][c];
          const double gxd = dxr * p5 * (Dv(j + 1, i) - Dv(j, i - 1) - Dv(j + 1, i - 1) + Dv(j, i));
          const double gyd = dyr * p5 * (Dv(j + 1, i) - Dv(j, i - 1) + Dv(j + 1, i - 1) - Dv(j, i));
          amfac = 0.0 + (gxd * gxd + gyd * gyd);
          const double gxc = dxr * p5 * (Cu(j + 1, i) - Cu(j, i - 1) - Cu(j + 1, i - 1) + Cu(j, i));
          const double gyc = dyr * p5 * (Cu(j + 1, i) - Cu(j, i - 1) + Cu(j + 1, i - 1) - Cu(j, i));
          amfac = amfac + (gxc * gxc + gyc * gyc);
        }
        double am_f = 1.0e0, hu = 0.0, hv = 0.0;
        const double amf = S.cf[C_AMF][r][c];
        if (j >= jb - 2 && j <= je && i >= ib - 2 && i <= ie && k <= kmu - 1) {
          am_f = sqrt(amfac) * S.cf[C_DXDY][r][c] / S.cf[C_AMAMF][r][c];
          am_f = fmin(40.0e0, am_f);
          am_f = fmax(1.0e0, am_f);
          const double ducm = S.cf[C_DUCM][r][c], dun = S.cf[C_DUN][r][c], dus = S.cf[C_DUS][r][c];
          const double due = S.cf[C_DUE][r][c], duw = S.cf[C_DUW][r][c], dmc = S.cf[C_DMC][r][c];
          const double dmn = S.cf[C_DMN][r][c], dms = S.cf[C_DMS][r][c], dme = S.cf[C_DME][r][c];
          const double dmw = S.cf[C_DMW][r][c];
          hu = ((ducm * U(j, i) + dun * U(j - 1, i) + dus * U(j + 1, i) + due * U(j, i + 1) + duw * U(j, i - 1)) +
                (dmc * V(j, i) + dmn * V(j - 1, i) + dms * V(j + 1, i) + dme * V(j, i + 1) + dmw * V(j, i - 1)));
          hv = ((ducm * V(j, i) + dun * V(j - 1, i) + dus * V(j + 1, i) + due * V(j, i + 1) + duw * V(j, i - 1)) -
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
    {
      const int j = y0 + threadIdx.y, i = x0 + threadIdx.x;
      if (j < jmt && i < imt) {
        const long q = (long)j * imt + i;
        const int r = threadIdx.y + 1, c = threadIdx.x + 1;   // in the 1-halo arrays
        double hu = 0.0, hv = 0.0;
        if (j >= jb - 1 && j < je && i >= ib - 1 && i < ie) {
          const double ducm = S.cf[C_DUCM][r][c], dun = S.cf[C_DUN][r][c], dus = S.cf[C_DUS][r][c];
          const double due = S.cf[C_DUE][r][c], duw = S.cf[C_DUW][r][c], dmc = S.cf[C_DMC][r][c];
          const double dmn = S.cf[C_DMN][r][c], dms = S.cf[C_DMS][r][c], dme = S.cf[C_DME][r][c];
          const double dmw = S.cf[C_DMW][r][c];
          hu = am * ((ducm * S.d2u[r][c] + dun * S.d2u[r - 1][c] + dus * S.d2u[r + 1][c] + due * S.d2u[r][c + 1] +
                      duw * S.d2u[r][c - 1]) +
                     (dmc * S.d2v[r][c] + dmn * S.d2v[r - 1][c] + dms * S.d2v[r + 1][c] + dme * S.d2v[r][c + 1] +
                      dmw * S.d2v[r][c - 1]));
          hv = am * ((ducm * S.d2v[r][c] + dun * S.d2v[r - 1][c] + dus * S.d2v[r + 1][c] + due * S.d2v[r][c + 1] +
                      duw * S.d2v[r][c - 1]) -
                     (dmc * S.d2u[r][c] + dmn * S.d2u[r - 1][c] + dms * S.d2u[r + 1][c] + dme * S.d2u[r][c + 1] +
                      dmw * S.d2u[r][c - 1]));
        }
        if (k > S.kmu[r][c] - 1) {
          hu = 0.0;
          hv = 0.0;
        }
        const long g = lvl + q;
        if (own_upd) {
          a.dlv[g] = dlv_k + hv;
          a.dlu[g] = dlu_k + hu;
        }
        const double uu = S.u[threadIdx.y + 2][threadIdx.x + 3], vv = S.v[threadIdx.y + 2][threadIdx.x + 3];
        a.wka_drag[g] = c0f * sqrt(uu * uu + vv * vv);
      }
    }
    __syncthreads();
  }
}

}  // namespace

int launch_del4u(const Arena& a, double am, double c0f, cudaStream_t s) {
  static bool attr = false;
  if (!attr) {
    LT_CUDA_OK(cudaFuncSetAttribute(k_del4u, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(Del4Smem)));
    attr = true;
  }
  dim3 b(DX, DY), g((a.imt + DX - 1) / DX, (a.jmt + DY - 1) / DY);
  k_del4u<<<g, b, sizeof(Del4Smem), s>>>(a, am, c0f);
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
