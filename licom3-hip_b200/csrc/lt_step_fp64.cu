// lt_step_fp64.cu - the plain FP64 tracer step (the drop-in form).
//
// Compiled with -fmad=false: every floating-point expression keeps the
// operation order of the reference kernels it replaces (cited per kernel), so
// results match the FP64 CPU oracle bit for bit.
//
// Launch sequence of one step (replacing tracer.cpp:1701-1903):
//   k_ssh           SSH mean (h0f*onbc, stf)                    (tracer_1_0)
//   k_cont_march64  uk/vk, divergence, w by upward integration,
//                   face transports, scaled utf/vtf             (tracer_1, upwell_2..4, advection_tracer_1_0)
//   k_surface_fluxes surface fluxes of both tracers, net, the
//                   surface mixing floor, SSS-norm terms       (tracer_5/6 surface parts)
//   tree sum        deterministic SSS-normalisation sum         (tracer.cpp:1849-1868)
//   halo(net)       in-GPU ghost fill                           (pop_haloupdate_tracer1)
//   k_tracer_tma64  per column tile (its level boxes by per-thread copies
//                   where the layout does not allow TMA boxes; k_tracer64
//                   for the centred and flux schemes), both tracers:
//                   tspas predictor/limiter,
//                   biharmonic diffusion, shortwave, explicit and implicit
//                   vertical diffusion, surface terms, update   (advection_tracer_2/3, tracer_del4_1/2,
//                                                                tracer_5..9, invtrit)
//   k_halo_state    ghost fill + fold of the new state          (pop_haloupdate_tracer2, tracer_9 for ghosts)
#include <cstdio>
#include "lt_common.cuh"
#include "lt_halo.cuh"
#include "lt_tracer_tma.cuh"

namespace lt {

namespace {

__device__ __forceinline__ long q2(int j, int i, int imt) { return (long)j * imt + i; }

// ------------------------------------------------------------------ surface
// One thread per column.  tracer_1_0 (tracer.cpp:1081-1093): h0f*onbc and the
// SSH mean stf; tracer_del4_2's surface floor on akt(T) (tracer.cpp:1315-1317);
// salt flux of tracer_5 (tracer.cpp:1480-1520) and heat flux of tracer_6
// (tracer.cpp:1545-1565) from the previous time level; net (both tracers).
// The SSH part (h0f_out, stf_ssh), which the continuity needs, and the flux
// part, which needs the surface forcing, are separate so that a step can
// run the continuity while its forcing is being copied in.
__device__ __forceinline__ double ssh_col(const Arena& a, long q) {
  const lt_params& p = a.p;
  const double h0 = a.h0f[q] * p.onbc;
  a.h0f_out[q] = h0;
  const double ssh = 0.5 * h0 + 0.5 * a.h0l[q];
  a.stf_ssh[q] = ssh;
  return ssh;
}

__device__ __forceinline__ void flux_col(const Arena& a, int i, int j, long q, double ssh) {
  const lt_params& p = a.p;
  if (i >= 1 && i < a.imt - 1 && j >= 1 && j < a.jmt - 1) {
    if (a.akt) {
      if (a.akt[q] < p.dwndmix) a.akt[q] = p.dwndmix;
    } else if (a.akt32[q] < (float)p.dwndmix) {
      a.akt32[q] = (float)p.dwndmix;
    }
  }
  double sT = ssh, sS = ssh;
  if (a.kmt[q] > 0) {
    const double* atb = a.atb[a.cur];
    const double odzp0 = a.odzp[0];
    const double s_top = atb[a.FB + a.A + q];
    sS = a.fresh[q] * 34.7 * p.od0 / 1000.0 + p.gamma * (a.sss[q] - s_top) * a.seaice[q] / odzp0 +
         p.gamma * 30.0 / 365.0 / 4.0 * 50.0 * (a.sss[q] - s_top) / odzp0 * (1.0 - a.seaice[q]);
    a.net[a.A + q] = sS * odzp0;
    const double t_top = atb[a.A + q];
    sT = ((a.swv[q] + a.nswv[q]) * p.od0cp + a.seaice[q] * p.gamma * (a.sst[q] - t_top) / odzp0);
    a.net[q] = sT * odzp0;
  }
  a.stf_n[q] = sT;
  a.stf_n[a.A + q] = sS;
}

__device__ __forceinline__ void surface_col(const Arena& a, int i, int j) {
  if (i >= a.imt || j >= a.jmt) return;
  const long q = q2(j, i, a.imt);
  flux_col(a, i, j, q, ssh_col(a, q));
}

// tracer_7's nudging toward restore_at (simple_assm; tracer.cpp:1587-1611):
// the rate of level k, 1/(5 days) down to level 45 and smaller by
// ((k+1)/5)^2 below, in the reference's operation order
__device__ __forceinline__ double assm_rate(int k) {
  return k < 45 ? 1.0e0 / (5.e0 * 86400.e0) : 1.0e0 / (5.e0 * 86400.e0) / ((k + 1) * (k + 1) / 5.0 / 5.0);
}

// The nudging term of every inner cell of the levels k < ktv, written to
// dt_restore as tracer_7 writes it (land and below-bottom cells included:
// their vit of 0 makes it a signed zero).  It reads only the step's inputs
// (restore_at, the previous time level atb, kmt), so it runs beside the
// column kernel, which adds the same term to the wet cells' tendencies.
// Grid: x over the cells of a level, y the level, z the tracer.
__global__ void k_assm_dt_restore(Arena a) {
  const int k = blockIdx.y, n = blockIdx.z;
  const int imt = a.imt, jmt = a.jmt;
  const long A = a.A, F = a.F, FB = a.FB;
  const double rate = assm_rate(k);
  const double* atb = a.atb[a.cur] + n * FB + (long)(k + 1) * A;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < A; q += (long)gridDim.x * blockDim.x) {
    const int j = (int)(q / imt), i = (int)(q % imt);
    if (j < 2 || j >= jmt - 2 || i < 2 || i >= imt - 2) continue;
    const double vit = k < a.kmt[q] ? 1.0 : 0.0;
    const long c = n * F + (long)k * A + q;
    a.dt_restore[c] = vit * (a.restore_at[c] - atb[q]) * rate;
  }
}

int launch_assm_dt_restore(const Arena& a, cudaStream_t s) {
  const int levels = a.p.ktv < a.km ? a.p.ktv : a.km;
  if (!a.p.simple_assm || levels <= 0) return LT_OK;
  const int bx = (int)((a.A + 255) / 256 < 64 ? (a.A + 255) / 256 : 64);
  k_assm_dt_restore<<<dim3(bx, levels, 2), 256, 0, s>>>(a);
  LT_LAUNCHED();
  return LT_OK;
}

__global__ void k_ssh(Arena a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= a.imt || j >= a.jmt) return;
  ssh_col(a, q2(j, i, a.imt));
}

__global__ void k_surface_fluxes(Arena a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= a.imt || j >= a.jmt) return;
  const long q = q2(j, i, a.imt);
  flux_col(a, i, j, q, a.stf_ssh[q]);
}

// every member's columns in one launch: blockIdx.z is the member
__global__ void k_surface_batch(const MemberDesc* __restrict__ mem) {
  surface_col(mem[blockIdx.z].a, blockIdx.x * blockDim.x + threadIdx.x, blockIdx.y * blockDim.y + threadIdx.y);
}

// --------------------------------------------------------- deterministic sum
// Fixed binary tree: blocks of 2048 consecutive terms, pairs (t, t+stride) for
// stride = 1024..1, zero padding; repeated on the block sums until one value.
constexpr int RB = 1024;

template <class Term>
__device__ __forceinline__ void tree_block(const Term& term, long n, double* part, long blk) {
  __shared__ double s[2 * RB];
  const long base = blk * 2 * RB;
  const int t = threadIdx.x;
  s[t] = (base + t < n) ? term(base + t) : 0.0;
  s[t + RB] = (base + t + RB < n) ? term(base + t + RB) : 0.0;
  for (int stride = RB; stride > 0; stride >>= 1) {
    __syncthreads();
    if (t < stride) s[t] = s[t] + s[t + stride];
  }
  if (t == 0) part[blk] = s[0];
}

template <class Term>
__global__ void k_tree_first(Term term, long n, double* part) {
  tree_block(term, n, part, blockIdx.x);
}

struct ArrayTerm {
  const double* x;
  __device__ double operator()(long m) const { return x[m]; }
};

// SSS-norm term of interior column m (row-major over j=2..jmt-3, i=2..imt-3):
// tarea*net(S)*vit(k=0) (tracer.cpp:1522-1525)
struct SssTerm {
  const double* tarea;
  const double* net_s;
  const int* kmt;
  int nx, imt;
  __device__ double operator()(long m) const {
    const int j = 2 + (int)(m / nx), i = 2 + (int)(m % nx);
    const long q = (long)j * imt + i;
    return tarea[q] * net_s[q] * (kmt[q] > 0 ? 1.0 : 0.0);
  }
};

__global__ void k_finish_sss(double* scalars, const double* sum, double area_t) {
  scalars[0] = -sum[0] / area_t;
}

// The same tree for every member of a batch, pass by pass: pass 0 sums the
// member's SSS terms into its red_part, pass p > 0 the block sums of pass
// p-1; blockIdx.y is the member, blocks beyond a member's count at this pass
// (or members whose tree ended) leave at once.
__device__ __forceinline__ long tree_blocks(long n) {
  const long nb = (n + 2 * RB - 1) / (2 * RB);
  return nb < 1 ? 1 : nb;
}

__global__ void k_sss_tree_batch(const MemberDesc* __restrict__ mem, int pass) {
  const Arena& a = mem[blockIdx.y].a;
  long n = (long)a.nx * a.ny, nb = tree_blocks(n), off = 0;
  for (int q = 0; q < pass; ++q) {
    if (nb <= 1) return;
    off += nb;
    n = nb;
    nb = tree_blocks(n);
  }
  if ((long)blockIdx.x >= nb) return;
  if (pass == 0) tree_block(SssTerm{a.tarea, a.net + a.A, a.kmt, a.nx, a.imt}, n, a.red_part, blockIdx.x);
  else tree_block(ArrayTerm{a.red_part + off - n}, n, a.red_part + off, blockIdx.x);
}

// the member's total (the last pass's single block sum) and fw_norm2
__global__ void k_finish_sss_batch(const MemberDesc* __restrict__ mem, int nmem) {
  const int z = blockIdx.x * blockDim.x + threadIdx.x;
  if (z >= nmem) return;
  const Arena& a = mem[z].a;
  long nb = tree_blocks((long)a.nx * a.ny), off = 0;
  while (nb > 1) { off += nb; nb = tree_blocks(nb); }
  const double sum = a.red_part[off];
  a.scalars[4] = sum;
  a.scalars[0] = -sum / a.p.area_t;
}

template <class Term>
int tree_sum(Term term, long n, double* part, double* out, cudaStream_t s) {
  long nb = (n + 2 * RB - 1) / (2 * RB);
  if (nb < 1) nb = 1;
  k_tree_first<<<(unsigned)nb, RB, 0, s>>>(term, n, part);
  LT_LAUNCHED();
  double* cur = part;
  double* nxt = part + nb;
  while (nb > 1) {
    const long nb2 = (nb + 2 * RB - 1) / (2 * RB);
    k_tree_first<<<(unsigned)nb2, RB, 0, s>>>(ArrayTerm{cur}, nb, nxt);
    LT_LAUNCHED();
    cur = nxt;
    nxt = nxt + nb2;
    nb = nb2;
  }
  LT_CUDA_OK(cudaMemcpyAsync(out, cur, sizeof(double), cudaMemcpyDeviceToDevice, s));
  return LT_OK;
}

// ------------------------------------------------------------------ halo
// In-place ghost fill of nz levels (e.g. net), one block per level.
__device__ __forceinline__ void halo_r8_level(double* lvl, int imt, int jmt, int ew_cyclic, int tripole) {
  extern __shared__ double top[];
  for (int i = threadIdx.x; i < imt; i += blockDim.x) top[i] = lvl[2L * imt + i];
  __syncthreads();
  HaloCells hc{imt, jmt, tripole};
  const long nc = hc.count();
  for (long m = threadIdx.x; m < nc; m += blockDim.x) {
    int j, i;
    hc.cell(m, j, i);
    double v;
    if (halo_cell_value(lvl, top, j, i, imt, jmt, ew_cyclic, tripole, v)) lvl[(long)j * imt + i] = v;
  }
}

// A level's ghost cells spread over kHaloParts blocks (one block per level
// left most SMs idle: 55 blocks per tracer, each thread walking ~120 cells
// in turn).  With the fold, part 0 takes rows 0..2 (the only cells that read
// the staged top row, and the only ones that rewrite it; rows 0 and 1 read
// interior columns of rows 3 and 4, which no part rewrites) and the other
// parts share the rest; without it the parts share all cells.
constexpr int kHaloParts = 8;
__device__ __forceinline__ bool halo_part(long nc, int imt, int tripole, int part, long& m0, long& m1) {
  long base = 0, parts = kHaloParts;
  if (tripole) {
    if (part == 0) { m0 = 0; m1 = 3L * imt; return true; }
    base = 3L * imt;
    parts = kHaloParts - 1;
    part -= 1;
  }
  const long per = (nc - base + parts - 1) / parts;
  m0 = base + part * per;
  m1 = m0 + per < nc ? m0 + per : nc;
  return m0 < m1;
}

// part blockIdx.x of level blockIdx.y
__global__ void k_halo_r8(double* f, int imt, int jmt, int ew_cyclic, int tripole) {
  double* lvl = f + (long)blockIdx.y * imt * jmt;
  HaloCells hc{imt, jmt, tripole};
  long m0, m1;
  if (!halo_part(hc.count(), imt, tripole, blockIdx.x, m0, m1)) return;
  extern __shared__ double top[];
  const bool fold = tripole && blockIdx.x == 0;
  if (fold) {
    for (int i = threadIdx.x; i < imt; i += blockDim.x) top[i] = lvl[2L * imt + i];
    __syncthreads();
  }
  for (long m = m0 + threadIdx.x; m < m1; m += blockDim.x) {
    int j, i;
    hc.cell(m, j, i);
    double v;
    if (halo_cell_value(lvl, top, j, i, imt, jmt, ew_cyclic, tripole, v)) lvl[(long)j * imt + i] = v;
  }
}

// net (both tracers) of every member: blockIdx.x the level, blockIdx.y the member
__global__ void k_halo_net_batch(const MemberDesc* __restrict__ mem) {
  const Arena& a = mem[blockIdx.y].a;
  halo_r8_level(a.net + (long)blockIdx.x * a.A, a.imt, a.jmt, a.ew_cyclic, a.tripole);
}

// ------------------------------------------------------------- continuity
constexpr int kCont64TileY = 8;   // tile height of the FP64 continuity march (4: slower)

// Continuity as one level march per 32 x BY tile (tracer_1, upwell_2,
// operators_div, advection_tracer_1_0 and upwell_3/4 with the same
// expressions in the same order).  The U-point velocities of the tile and a
// one-point halo north and east go through a three-level staging ring filled
// by per-thread asynchronous copies, so three levels are in flight while one
// is computed; each thread converts the points it copied itself (mean
// velocities wkd, wkb and the free-surface scaled uk, vk, whose level-free
// factor it keeps in registers) into a double-buffered level, read by all
// after the step's one barrier.  Each thread's first copy is its own cell's
// point, so the scaled utf, vtf it writes come from its own staged copies
// (a global re-read of them per level cost 9.00 -> 7.67 ms per 0.1-degree
// step).  The column divergence W accumulates in level order during the
// march; w is integrated upward afterwards from the wka the march wrote.
template <int BY>
__global__ void __launch_bounds__(32 * BY) k_cont_march64(Arena a) {
  constexpr int BX = 32, UX = BX + 1, UY = BY + 1, UN = UX * UY, NT = BX * BY;
  constexpr int NPT = (UN + NT - 1) / NT, NST = 3;
  __shared__ double s_st[NST][4][UN];   // staged utf, utl, vtf, vtl of three levels
  __shared__ double s_wkd[2][UN], s_wkb[2][UN], s_uk[2][UN], s_vk[2][UN];
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * BX + tx;
  const int x0 = blockIdx.x * BX, y0 = blockIdx.y * BY;
  const int imt = a.imt, jmt = a.jmt, km = a.km;
  const long A = a.A;
  const lt_params& p = a.p;
  static_assert(NPT == 2 && UN - NT == UX + BY, "own point plus one of the row above or the column east");
  // region point of this thread's copy pt: its own cell's U point first (so
  // that the own point's raw velocities are this thread's own copies, read
  // without a barrier), then one point of the row above the tile (threads
  // 0 .. UX-1) or of the column east of it (threads UX .. UX+BY-1)
  auto point_of = [&](int pt) {
    if (pt == 0) return (ty + 1) * UX + tx;
    return tid < UX ? tid : (tid - UX + 1) * UX + BX;
  };
  const bool has_extra = tid < UX + BY;
  long rq[NPT];
  bool rin[NPT], rok[NPT];
  double rfac[NPT];
#pragma unroll
  for (int pt = 0; pt < NPT; ++pt) {
    const int m = point_of(pt);
    const int uj = y0 - 1 + m / UX, ui = x0 + m % UX;
    rin[pt] = (pt == 0 || has_extra) && uj >= 0 && uj < jmt && ui < imt;
    rq[pt] = rin[pt] ? q2(uj, ui, imt) : 0;
    rok[pt] = rin[pt] && uj < jmt - 1 && ui >= 1;
    rfac[pt] = 0.0;
    if (rok[pt]) {
      const long q = rq[pt];
      const double work = a.au0[q] * a.stf_ssh[q] + a.aus[q] * a.stf_ssh[q + imt] +
                          a.auw[q] * a.stf_ssh[q - 1] + a.ausw[q] * a.stf_ssh[q + imt - 1];
      rfac[pt] = 1.0 + work * a.ohbu[q];
    }
  }
  auto issue = [&](int L) {
    if (L < km) {
      const long lvl = (long)L * A;
#pragma unroll
      for (int pt = 0; pt < NPT; ++pt) {
        if (!rin[pt]) continue;
        const int m = point_of(pt);
        const long c = lvl + rq[pt];
        double(*st)[UN] = s_st[L % NST];
        cp_async8(&st[0][m], a.utf + c);
        cp_async8(&st[1][m], a.utl + c);
        cp_async8(&st[2][m], a.vtf + c);
        cp_async8(&st[3][m], a.vtl + c);
      }
    }
    cp_async_commit();
  };
  // the points this thread copied, level L, into buffer b; the own point's
  // raw utf, vtf of level L into own_utf, own_vtf
  double own_utf = 0.0, own_vtf = 0.0;
  auto park = [&](int L, int b) {
    const double(*st)[UN] = s_st[L % NST];
#pragma unroll
    for (int pt = 0; pt < NPT; ++pt) {
      if (pt > 0 && !has_extra) continue;
      const int m = point_of(pt);
      if (pt == 0) {
        own_utf = rin[0] ? st[0][m] : 0.0;
        own_vtf = rin[0] ? st[2][m] : 0.0;
      }
      double wkd = 0.0, wkb = 0.0, uk = 0.0, vk = 0.0;
      if (rin[pt]) {
        wkd = 0.5 * (st[0][m] * p.oncc) + 0.5 * st[1][m];
        wkb = 0.5 * (st[2][m] * p.oncc) + 0.5 * st[3][m];
        if (rok[pt]) {
          uk = rfac[pt] * wkd;
          vk = rfac[pt] * wkb;
        }
      }
      s_wkd[b][m] = wkd; s_wkb[b][m] = wkb; s_uk[b][m] = uk; s_vk[b][m] = vk;
    }
  };
  issue(0);
  issue(1);
  issue(2);
  cp_async_wait<2>();
  park(0, 0);
  const int i = x0 + tx, j = y0 + ty;
  const bool own = i < imt && j < jmt;
  const bool col = own && j >= 1 && j < jmt - 1 && i >= 1 && i < imt - 1;
  const long qo = own ? q2(j, i, imt) : 0;
  const int kz = own ? a.kmt[qo] : 0;
  const double htw_o = own ? a.htw[qo] : 0.0, hts_o = own ? a.hts[qo] : 0.0;
  const double htw_e = (own && i < imt - 1) ? a.htw[qo + 1] : 0.0;
  const double hts_n = (own && j >= 1) ? a.hts[qo - imt] : 0.0;
  // flux scheme: each U-point mean weighted by its own dyu (west face) or
  // dxu (south face) before the face mean (advection_tracer_1_0, Str 1)
  const bool flux = p.adv_tracer == LT_ADV_FLUX;
  const double dyu_o = (flux && own) ? a.dyu[qo] : 0.0, dyu_n = (flux && own && j >= 1) ? a.dyu[qo - imt] : 0.0;
  const double dxu_o = (flux && own) ? a.dxu[qo] : 0.0, dxu_e = (flux && own && i < imt - 1) ? a.dxu[qo + 1] : 0.0;
  const double trr = own ? a.tarea_r[qo] : 0.0;
  const int m0 = (ty + 1) * UX + tx, mn = ty * UX + tx;
  double W = 0.0;
  double dzp_k = a.dzp[0];
  int kf = 0;   // one past the deepest level with a nonzero west/south face transport or w here
  for (int k = 0; k < km; ++k) {
    const int b = k & 1;
    const double dzp_c = dzp_k;
    if (k + 1 < km) dzp_k = a.dzp[k + 1];
    // level k parked by every thread; buffer b^1 and the staging slot of
    // level k are no longer read
    __syncthreads();
    issue(k + 3);
    if (own) {
      const double* wd = s_wkd[b];
      const double* wb = s_wkb[b];
      const double* uk = s_uk[b];
      const double* vk = s_vk[b];
      const long c = (long)k * A + qo;
      __stcs(a.utf_out + c, own_utf * p.oncc);
      __stcs(a.vtf_out + c, own_vtf * p.oncc);
      double uwv = 0.0, vsv = 0.0;   // the faces outside these ranges stay zero
      if (flux) {
        if (j >= 1 && j < jmt - 1) __stcs(a.uwf + c, uwv = (wd[mn] * dyu_n + wd[m0] * dyu_o) * 0.25);
        if (i >= 1 && i < imt - 1) __stcs(a.vsf + c, vsv = (wb[m0] * dxu_o + wb[m0 + 1] * dxu_e) * 0.25);
      } else {
        if (j >= 1 && j < jmt - 1) __stcs(a.uwf + c, uwv = (wd[mn] + wd[m0]) * htw_o * 0.25);
        if (i >= 1 && i < imt - 1) __stcs(a.vsf + c, vsv = (wb[m0] + wb[m0 + 1]) * hts_o * 0.25);
      }
      if (uwv != 0.0 || vsv != 0.0) kf = k + 1;
      double wka = 0.0;
      if (j >= 1 && i < imt - 1 && k <= kz - 1) {
        const double east = (uk[m0 + 1] + uk[mn + 1]) * htw_e;
        const double west = (uk[m0] + uk[mn]) * htw_o;
        const double south = (vk[m0 + 1] + vk[m0]) * hts_o;
        const double north = (vk[mn + 1] + vk[mn]) * hts_n;
        wka = 0.5 * (east - west + south - north) * trr;
      }
      st_l2(a.wka + c, wka, l2_evict_last());
      if (col) W = W - dzp_c * wka * (k < kz ? 1.0 : 0.0);
    }
    if (k + 1 < km) {
      cp_async_wait<2>();   // this thread's copies of level k+1 have landed
      park(k + 1, b ^ 1);
    }
  }
  cp_async_wait<0>();
  if (!col) {
    if (a.kfz && own) a.kfz[qo] = kf;
    return;
  }
  const double ohbt = a.ohbt[qo];
  const double fac = 1.0 / (1.0 + a.stf_ssh[qo] * ohbt);
  double wsp = a.ws[qo];
  // upward integration; the wka of CH levels are loaded together ahead of
  // their stores (one round trip per CH levels).  The march wrote wka with
  // an L2 evict-last policy (the tile's levels stay in L2 until read here,
  // then leave it); the outputs go out as streaming stores.
  constexpr int CH = 8;
  for (int k0 = 1; k0 < km; k0 += CH) {
    double wk[CH];
#pragma unroll
    for (int c = 0; c < CH; ++c) wk[c] = k0 + c < km ? ld_l2(a.wka + (long)(k0 + c - 1) * A + qo, l2_evict_first()) : 0.0;
#pragma unroll
    for (int c = 0; c < CH; ++c) {
      const int k = k0 + c;
      if (k >= km) break;
      const double raw = (k < kz ? 1.0 : 0.0) * (wsp + a.dzp[k - 1] * (W * ohbt + wk[c]));
      const double wv = raw * fac;
      __stcs(a.ws + (long)k * A + qo, wv);
      if (wv != 0.0) kf = max(kf, k + 1);
      wsp = raw;
    }
  }
  if (a.kfz) a.kfz[qo] = kf;
}

// ------------------------------------------- plain-load march (centred, flux)
// The column march of the centred and flux advection schemes (no predictor
// or limiter), with each level's region loaded by plain loads.
// Shared-memory regions of a TX x TY column tile:
//   H2: rows y0-2..y0+TY+1, cols x0-2..x0+TX+1   (RY x RX)   tracer, atb, kmt
//   H1: rows y0-1..y0+TY,   cols x0-1..x0+TX     (QY x QX)   w, d2tk
constexpr int RX = TX + 4, RY = TY + 4, QX = TX + 2, QY = TY + 2;
constexpr int UWN = QY * RX;          // u_wface: H1 rows, cols x0-2..x0+TX+1
constexpr int VSN = (QY + 1) * QX;    // v_sface: rows y0-2..y0+TY, H1 cols

struct TSmem {
  double at[4][RY * RX];
  double ws[3][QY * QX];
  double uw[2][UWN], vs[2][VSN];
  double atb[RY * RX];
  double d2[QY * QX];
  double tr[QY * QX];
  double dtn[QY * QX], dts[QY * QX], dte[QY * QX], dtw[QY * QX], ahf[QY * QX];
  int kmt[RY * RX];
};

__device__ __forceinline__ int slot4(int k) { return k & 3; }
__device__ __forceinline__ int slot3(int k) { return k % 3; }

// load one level of a [km][jmt][imt] field over region rows r0.., cols c0..
// (ny x nxr), zero outside the domain
__device__ __forceinline__ void load_region(double* dst, const double* lvl, int r0, int c0, int nyr, int nxr,
                                            int imt, int jmt) {
  for (int m = threadIdx.x; m < nyr * nxr; m += TTHREADS) {
    const int gj = r0 + m / nxr, gi = c0 + m % nxr;
    dst[m] = (gj >= 0 && gj < jmt && gi >= 0 && gi < imt) ? lvl[(long)gj * imt + gi] : 0.0;
  }
}

// first masked Laplacian of atb at level kk on H1 (tracer_del4_1, tracer.cpp:1238-1293)
__device__ void del4_first(TSmem& S, const Arena& a, int kk, int x0, int y0) {
  for (int m = threadIdx.x; m < QY * QX; m += TTHREADS) {
    const int hj = m / QX, hi = m % QX;
    const int gj = y0 - 1 + hj, gi = x0 - 1 + hi;
    if (!(gi >= 1 && gi < a.imt - 1 && gj >= 1 && gj < a.jmt - 1)) { S.d2[m] = 0.0; continue; }
    const int r = (hj + 1) * RX + (hi + 1);
    double h = 0.0, cc = 0.0;
    if (kk <= S.kmt[r] - 1) {
      if (kk <= S.kmt[r - RX] - 1) { h += S.dtn[m] * S.atb[r - RX]; cc -= S.dtn[m]; }
      if (kk <= S.kmt[r + RX] - 1) { h += S.dts[m] * S.atb[r + RX]; cc -= S.dts[m]; }
      if (kk <= S.kmt[r + 1] - 1) { h += S.dte[m] * S.atb[r + 1]; cc -= S.dte[m]; }
      if (kk <= S.kmt[r - 1] - 1) { h += S.dtw[m] * S.atb[r - 1]; cc -= S.dtw[m]; }
    }
    S.d2[m] = S.ahf[m] * (cc * S.atb[r] + h);
  }
}

// advection_tracer_1 for the centred (Str 0) and flux (Str 1) schemes at one
// inner cell of level k (tracer.cpp:120-289), from the tile's level slots.
// The centred form accumulates ax, ay, az with weight 1/nss, once per level
// (the reference repeats its top- and bottom-level statements in every
// level thread of its launch, so there those two levels' accumulations race).
template <int ADV, bool DIAG>
__device__ __forceinline__ double simple_adv(const TSmem& S, const Arena& a, int k, int n, long cg, int rc, int hc,
                                             int uc, int vc, const double* at_c, const double* at_u,
                                             const double* at_d) {
  const int km = a.km;
  const double* odzp = a.odzp;
  const double tr = S.tr[hc];
  const double c = at_c[rc], e = at_c[rc + 1], w = at_c[rc - 1], s = at_c[rc + RX], nn = at_c[rc - RX];
  const double* uw = S.uw[k & 1];
  const double* vs = S.vs[k & 1];
  const double ue = uw[uc + 1], uwc = uw[uc], vsc = vs[vc], vn = vs[vc - QX];
  const double wk = S.ws[slot3(k)][hc];
  const double w1 = k < km - 1 ? S.ws[slot3(k + 1)][hc] : 0.0;
  if (ADV == LT_ADV_CENTERED) {
    const double h = (-uwc * (c - w) - ue * (e - c) - vsc * (s - c) - vn * (c - nn)) * tr;
    double z;
    if (k == 0) z = 0.5 * odzp[0] * (w1 * (c - at_d[rc]));
    else if (k == km - 1) z = 0.5 * odzp[km - 1] * (wk * (at_u[rc] - c));
    else z = 0.5 * odzp[k] * (wk * (at_u[rc] - c) + w1 * (c - at_d[rc]));
    if (DIAG) {
      const long q = (long)n * a.F + cg;
      const double nss = (double)a.p.nss;
      a.ax[q] = a.ax[q] + (-uwc * (c - w) - ue * (e - c)) * tr / nss;
      a.ay[q] = a.ay[q] + (-vsc * (s - c) - vn * (c - nn)) * tr / nss;
      a.az[q] = a.az[q] - z / nss;
    }
    return h - z;
  } else {
    const double h = (-uwc * (c + w) + ue * (e + c) - vn * (c + nn) + vsc * (s + c)) * tr;
    const double z1 = k == 0 ? 0.0 : wk * (at_u[rc] + c) * 0.5;
    const double z2 = k == km - 1 ? 0.0 : w1 * (c + at_d[rc]) * 0.5;
    return h - odzp[k] * (z2 - z1);
  }
}

template <bool DIAG, int ADV>
__global__ void __launch_bounds__(TTHREADS) k_tracer64(Arena a, int ntx, long ntiles) {
  static_assert(ADV == LT_ADV_CENTERED || ADV == LT_ADV_FLUX, "the tspas scheme runs in k_tracer_tma64");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TSmem& S = *reinterpret_cast<TSmem*>(smem_raw);
  const int tid = threadIdx.x, tx = tid % TX, ty = tid / TX;
  const int imt = a.imt, jmt = a.jmt, km = a.km;
  const long A = a.A, F = a.F, FB = a.FB;
  const lt_params& p = a.p;
  const double dts = p.dts;
  const double aidif = 0.5;
  const double* __restrict__ odzp = a.odzp;
  const double* __restrict__ odzt = a.odzt;
  const int NV = a.nv_scratch;
  double* scr = a.col_scratch + (long)blockIdx.x * km * NV * TTHREADS;

  for (long w = blockIdx.x; w < 2 * ntiles; w += gridDim.x) {
    const long tile = w >> 1;
    const int n = (int)(w & 1);
    const int x0 = (int)(tile % ntx) * TX, y0 = (int)(tile / ntx) * TY;
    const int i = x0 + tx, j = y0 + ty;
    const double* at_in = a.at[a.cur] + n * F;
    const double* atb_in = a.atb[a.cur] + n * FB;
    double* at_out = a.at[a.cur ^ 1] + n * F;
    double* atb_out = a.atb[a.cur ^ 1] + n * FB;
    const double* akt = a.akt + n * F;

    __syncthreads();  // previous tile finished with shared memory
    // ---- per-tile 2-D statics
    for (int m = tid; m < RY * RX; m += TTHREADS) {
      const int gj = y0 - 2 + m / RX, gi = x0 - 2 + m % RX;
      S.kmt[m] = (gj >= 0 && gj < jmt && gi >= 0 && gi < imt) ? a.kmt[q2(gj, gi, imt)] : 0;
    }
    for (int m = tid; m < QY * QX; m += TTHREADS) {
      const int gj = y0 - 1 + m / QX, gi = x0 - 1 + m % QX;
      const bool in = (gj >= 0 && gj < jmt && gi >= 0 && gi < imt);
      const long q = in ? q2(gj, gi, imt) : 0;
      S.tr[m] = in ? a.tarea_r[q] : 0.0;
      S.dtn[m] = in ? a.dtn[q] : 0.0;
      S.dts[m] = in ? a.dts[q] : 0.0;
      S.dte[m] = in ? a.dte[q] : 0.0;
      S.dtw[m] = in ? a.dtw[q] : 0.0;
      S.ahf[m] = in ? a.ahf[q] : 0.0;
    }
    // ---- prologue: levels km-1 and km-2 of the tracer, w and faces at km-1
    load_region(S.at[slot4(km - 1)], at_in + (long)(km - 1) * A, y0 - 2, x0 - 2, RY, RX, imt, jmt);
    load_region(S.at[slot4(km - 2)], at_in + (long)(km - 2) * A, y0 - 2, x0 - 2, RY, RX, imt, jmt);
    load_region(S.ws[slot3(km - 1)], a.ws + (long)(km - 1) * A, y0 - 1, x0 - 1, QY, QX, imt, jmt);
    load_region(S.uw[(km - 1) & 1], a.uwf + (long)(km - 1) * A, y0 - 1, x0 - 2, QY, RX, imt, jmt);
    load_region(S.vs[(km - 1) & 1], a.vsf + (long)(km - 1) * A, y0 - 2, x0 - 1, QY + 1, QX, imt, jmt);

    const bool own = (i < imt && j < jmt);
    const bool inner = own && i >= 2 && i < imt - 2 && j >= 2 && j < jmt - 2;
    const long qo = own ? q2(j, i, imt) : 0;
    const int kz = own ? a.kmt[qo] : 0;
    const int rc = (ty + 2) * RX + (tx + 2);     // own cell in H2
    const int hc = (ty + 1) * QX + (tx + 1);     // own cell in H1
    const int uc = (ty + 1) * RX + (tx + 2);     // own column in uw
    const int vc = (ty + 2) * QX + (tx + 1);     // own row in vs
    const double swv = (inner && n == 0) ? a.swv[qo] : 0.0;
    const double stf = own ? a.stf_n[n * A + qo] : 0.0;
    double atb_kp1 = 0.0;                                       // tracer level k+1 of atb
    double atb_k = own ? atb_in[(long)km * A + qo] : 0.0;       // level km-1
    double wkc_k = 0.0;
    double e_prev = 0.0, f_prev = 0.0;

    for (int k = km - 1; k >= 0; --k) {
      // ---- phase A: loads for this level
      __syncthreads();
      if (k >= 2) load_region(S.at[slot4(k - 2)], at_in + (long)(k - 2) * A, y0 - 2, x0 - 2, RY, RX, imt, jmt);
      if (k >= 1) {
        load_region(S.ws[slot3(k - 1)], a.ws + (long)(k - 1) * A, y0 - 1, x0 - 1, QY, QX, imt, jmt);
        load_region(S.uw[(k - 1) & 1], a.uwf + (long)(k - 1) * A, y0 - 1, x0 - 2, QY, RX, imt, jmt);
        load_region(S.vs[(k - 1) & 1], a.vsf + (long)(k - 1) * A, y0 - 2, x0 - 1, QY + 1, QX, imt, jmt);
      }
      load_region(S.atb, atb_in + (long)(k + 1) * A, y0 - 2, x0 - 2, RY, RX, imt, jmt);
      const double atb_km1 = (own && k >= 1) ? atb_in[(long)k * A + qo] : 0.0;  // tracer level k-1
      const double wkc_km1 = (own && k >= 1) ? akt[(long)(k - 1) * A + qo] : 0.0;
      if (k == km - 1) wkc_k = 0.0;
      __syncthreads();
      // ---- phase B: first Laplacian at this level
      del4_first(S, a, k, x0, y0);
      __syncthreads();
      // ---- phase C: own column
      if (inner) {
        const double* at_c = S.at[slot4(k)];
        const double* at_u = k > 0 ? S.at[slot4(k - 1)] : nullptr;
        const double* at_d = k < km - 1 ? S.at[slot4(k + 1)] : nullptr;
        const long cg = (long)k * A + qo;
        const double adv = simple_adv<ADV, DIAG>(S, a, k, n, cg, rc, hc, uc, vc, at_c, at_u, at_d);
        if (inner) {
          const double vit_k = k < kz ? 1.0 : 0.0;
          const double vit_kp1 = (k + 1 < kz) ? 1.0 : 0.0;
          double tf = adv * vit_k;
          // second Laplacian (tracer_del4_2)
          {
            const int r = rc;
            double h = 0.0, cc = 0.0;
            if (k <= S.kmt[r] - 1) {
              if (k <= S.kmt[r - RX] - 1) { h += S.dtn[hc] * S.d2[hc - QX]; cc -= S.dtn[hc]; }
              if (k <= S.kmt[r + RX] - 1) { h += S.dts[hc] * S.d2[hc + QX]; cc -= S.dts[hc]; }
              if (k <= S.kmt[r + 1] - 1) { h += S.dte[hc] * S.d2[hc + 1]; cc -= S.dte[hc]; }
              if (k <= S.kmt[r - 1] - 1) { h += S.dtw[hc] * S.d2[hc - 1]; cc -= S.dtw[hc]; }
            }
            tf += p.ah * (cc * S.d2[hc] + h);
          }
          // shortwave penetration, temperature only (tracer_5)
          if (n == 0) {
            if (k >= 1 && k < km - 1) {
              const double w1 = swv * a.pen[k - 1] * vit_k;
              const double w2 = swv * a.pen[k] * vit_kp1;
              tf = tf + (w1 - w2) * odzp[k];
              if (DIAG) a.penetrate[cg] = (w1 - w2) * odzp[k];
            } else if (k == 0) {
              const double w1 = swv * a.pen[0] * ((1 < kz) ? 1.0 : 0.0);
              tf = tf - odzp[0] * w1;
              if (DIAG) a.penetrate[cg] = -w1 * odzp[0];
            } else {
              const double w2 = swv * a.pen[km - 2] * vit_k;
              tf = tf + odzp[km - 1] * w2;
              if (DIAG) a.penetrate[cg] = w2 * odzp[km - 1];
            }
          }
          // explicit half of the vertical diffusion (tracer_5)
          if (k >= 1 && k < km - 1) {
            const double w1 = wkc_km1 * (atb_km1 - atb_k) * odzt[k] * vit_k;
            const double w2 = wkc_k * (atb_k - atb_kp1) * odzt[k + 1] * vit_kp1;
            tf = tf + odzp[k] * (w1 - w2) * 0.5;
            if (DIAG) a.dzd[n * F + cg] = odzp[k] * (w1 - w2) * 0.5;
          } else if (k == 0) {
            const double w1 = wkc_k * (atb_k - atb_kp1) * odzt[1] * vit_kp1;
            tf = tf - odzp[0] * w1 * 0.5;
            if (DIAG) a.dzd[n * F + cg] = -odzp[0] * w1 * 0.5;
          } else {
            const double w2 = wkc_km1 * (atb_km1 - atb_k) * odzt[km - 1] * vit_k;
            tf = tf + odzp[km - 1] * w2 * (1.0 - aidif);
            if (DIAG) a.dzd[n * F + cg] = odzp[km - 1] * w2 * 0.5;
          }
          // surface fluxes (tracer_5 salt, tracer_6 SSS norm / heat)
          if (k == 0) {
            if (n == 1) {
              if (kz > 0) tf = tf + stf * (1.0 - aidif) * odzp[0];
              tf = tf + a.scalars[0] * vit_k;
            } else if (kz > 0) {
              tf = tf + stf * odzp[0] * 0.5;
            }
          }
          // nudging (tracer_7, simple_assm), then restoring (boundary_restore == 1)
          if (p.simple_assm && k < p.ktv) tf = tf + vit_k * (a.restore_at[n * F + cg] - atb_k) * assm_rate(k);
          if (p.boundary_restore == 1 && k >= 1) {
            const double lamda = 1.0 / (15.0 * 86400.0);
            tf = tf + vit_k * (a.restore[n * F + cg] - atb_k) * lamda;
          }
          // explicit update (tracer_8) and one elimination step of the
          // implicit sweep (invtrit, tracer.cpp:923-978)
          const double d8 = at_c[rc] + dts * tf;
          double ev = 0.0, fv = d8;
          if (k < kz) {
            double a8, c8, b8;
            if (k >= 1) a8 = wkc_km1 * odzt[k] * odzp[k] * dts * 0.5;
            else a8 = odzp[0] * dts * 0.5;
            if (k == kz - 1) {
              c8 = odzp[kz - 1] * dts * 0.5;
              b8 = 1.0 + a8;
            } else if (k >= 1) {
              c8 = wkc_k * odzt[k + 1] * odzp[k] * dts * 0.5;
              b8 = 1.0 + a8 + c8;
            } else {
              c8 = wkc_k * odzt[k + 1] * odzp[k] * dts * 0.5;
              b8 = 1.0 + c8;
            }
            if (k == kz - 1) { e_prev = 0.0; f_prev = 0.0; }
            const double g0 = 1.0 / (b8 - c8 * e_prev);
            ev = a8 * g0;
            fv = (d8 + c8 * f_prev) * g0;
            e_prev = ev;
            f_prev = fv;
          }
          double* sl = scr + (long)k * NV * TTHREADS;
          sl[tid] = ev;
          sl[TTHREADS + tid] = fv;
          if (DIAG) sl[2 * TTHREADS + tid] = d8;
        }
      }
      atb_kp1 = atb_k;
      atb_k = atb_km1;
      wkc_k = wkc_km1;
    }
    // ---- substitution, top down, and the new state of the inner cells
    if (inner) {
      double x = 0.0;
      const double stf_c = stf;
      for (int k = 0; k < km; ++k) {
        const double* sl = scr + (long)k * NV * TTHREADS;
        const double ev = sl[tid], fv = sl[TTHREADS + tid];
        const long cg = (long)k * A + qo;
        double v;
        if (k < kz) {
          const double vit_k = 1.0;
          v = (k == 0) ? (ev * stf_c + fv) * vit_k : (ev * x + fv) * vit_k;
          x = v;
        } else {
          v = fv;
        }
        if (DIAG) {
          const double d8 = sl[2 * TTHREADS + tid];
          const double vit_k = k < kz ? 1.0 : 0.0;
          const double at_old = at_in[cg];
          a.tend[n * F + cg] = (v - at_old) / dts * vit_k;
          if (k == 0) a.dt_diff[n * F + cg] = (v - d8) / dts * vit_k - stf_c * 0.5 * odzp[0];
          else a.dt_diff[n * F + cg] = (v - d8) / dts * vit_k;
          if (j == 2 && a.tripole) a.fold_save[((long)(n * km + k)) * imt + i] = d8;
        }
        at_out[cg] = v;
        atb_out[(long)(k + 1) * A + qo] = v;
      }
    }
  }
}

// -------------------------------------------- tracer march, TMA pipeline
// The tspas column march (advection_tracer_2/3 with tracer_del4_1/2,
// tracer_5..9 and invtrit, each expression in the reference's order), its
// level data staged by TMA boxes (or, where the row pitch does not allow
// TMA, by per-thread asynchronous copies into the same slots).
// Three level slots: step k reads levels k-2 .. k from shared memory; the
// own cell's at, ws and atb of level k+1 that the column phase also needs are
// carried in registers from step k+1, so the slot of level k takes level k-3
// at the end of step k.  Predictor ring and first Laplacian in shared memory;
// the 2-D metric terms are read through L1 (the same 2-D values serve every
// level), so kFp64CtasPerSm CTAs fit on an SM.
constexpr int NSX = 3;
constexpr bool kStageDel4 = kFp64CtasPerSm <= 2;
// the own cell's unlimited horizontal fluxes and centred transports of a
// level, as its predictor formed them one step before the column phase
// needs them (same expressions, same inputs), kept per level parity where
// the room is
constexpr bool kCacheXY = kFp64CtasPerSm <= 2;
struct ExSmem {
  LevelSlot<double> slot[NSX];
  unsigned char flag[3][HN];   // limiter flag (a00 > amax || a00 < amin) per level parity of three
  double d2[HN];
  // level-free metric terms of the 1-halo region: tarea_r per cell, htw*hun
  // at its x faces (west face of column x0-1+fi), hts*hue at its y faces
  // (south face of row y0-2+fj)
  double tr[HN];
  double hw[HQY * (HQX + 1)];
  double hs[(HQY + 1) * HQX];
  // the biharmonic coefficients dtn, dts, dte, dtw, ahf of the 1-halo region
  // where two CTAs per SM leave the room (read through L1 otherwise)
  double dt5[kStageDel4 ? 5 : 1][kStageDel4 ? HN : 1];
  double xyc[kCacheXY ? 2 : 1][6][kCacheXY ? TTHREADS : 1];
  int kmt[(TY + 4) * SW];
  int wmax[TTHREADS / 32];       // per-warp maxima of the region's bottom level
  uint64_t bar[NSX];
};

// Predictor, masked extrema and limiter flag of one cell (hj, hi) of the
// 1-halo region at level kk; returns the flag (a00 > amax || a00 < amin).
// sc, su, sd: the slots (and flag sets) of levels kk, kk-1, kk+1
// dry_out: the flag of a land cell whose four horizontal faces carry no
// transport is left 0 without computing its predictor: a flag only chooses
// between the upwind and Lax-Wendroff forms of its faces' fluxes, which are
// the same zero for a zero transport, and the vertical faces below a
// column's bottom carry w = 0.  The column phase forms such a cell's
// cached terms (xy_out) itself.  (Model velocities vanish on land faces; the
// reference's literal tracer_ sequence, which leaves vtl holding S, does not
// keep them zero, hence the test.)
__device__ __forceinline__ bool pred_one64(ExSmem& S, const Arena& a, int kk, int sc, int su, int sd, int hj, int hi,
                                           int x0, int y0, double* xy_out = nullptr, bool dry_out = false) {
  const int km = a.km, imt = a.imt, jmt = a.jmt;
  const double dts = a.p.dts;
  const double* odzp = a.odzp;
  const double* odzt = a.odzt;
  const LevelSlot<double>& Lc = S.slot[sc];
  const double* at_c = Lc.at;
  const double* at_u = kk > 0 ? S.slot[su].at : nullptr;
  const double* at_d = kk < km - 1 ? S.slot[sd].at : nullptr;
  const double* ws_c = Lc.ws;
  const double* ws_d = kk < km - 1 ? S.slot[sd].ws : nullptr;
  const double* uw = Lc.uw;
  const double* vs = Lc.vs;
  unsigned char* fl = S.flag[sc];
  {
    const int m = hj * HQX + hi;
    const int gj = y0 - 1 + hj, gi = x0 - 1 + hi;
    if (!(gi >= 1 && gi < imt - 1 && gj >= 1 && gj < jmt - 1)) {
      fl[m] = 0;   // a00 = amax = amin = 0
      return false;
    }
    const int r = r2(hj, hi), u = ru(hj, hi), v = rv(hj, hi);
    if (dry_out && kk >= S.kmt[r] && uw[u] == 0.0 && uw[u + 1] == 0.0 && vs[v] == 0.0 && vs[v - SW] == 0.0) {
      fl[m] = 0;
      return false;
    }
    const double tr = S.tr[m];
    const double hwe = S.hw[hj * (HQX + 1) + hi + 1], hww = S.hw[hj * (HQX + 1) + hi];
    const double hss = S.hs[(hj + 1) * HQX + hi], hsn = S.hs[hj * HQX + hi];
    const double c = at_c[r], e = at_c[r + 1], w = at_c[r - 1], s = at_c[r + SW], n = at_c[r - SW];
    const double ue = uw[u + 1], uwc = uw[u];
    const double vsc = vs[v], vn = vs[v - SW];
    const double x0v = (e + c) * ue * tr - (c + w) * uwc * tr;
    const double y0v = ((s + c) * vsc - (c + n) * vn) * tr;
    const double xy1 = -dts * (e - c) * 2.0 * tr * ue * ue / hwe;
    const double xy2 = dts * (c - w) * 2.0 * tr * uwc * uwc / hww;
    const double xy3 = -dts * (s - c) * 2.0 * tr * vsc * vsc / hss;
    const double xy4 = dts * (c - n) * 2.0 * tr * vn * vn / hsn;
    if (kCacheXY && xy_out) {
      xy_out[0] = xy1;
      xy_out[TTHREADS] = xy2;
      xy_out[2 * TTHREADS] = xy3;
      xy_out[3 * TTHREADS] = xy4;
      xy_out[4 * TTHREADS] = x0v;
      xy_out[5 * TTHREADS] = y0v;
    }
    const double cx = -c * (ue - uwc) * tr * 2.0;
    const double cy = -c * (vsc - vn) * tr * 2.0;
    double za, zb1, zb2, zc;
    const double wk = ws_c[u];
    if (kk == 0) {
      const double w1 = ws_d[u], ad = at_d[r];
      za = -0.5 * odzp[0] * w1 * (ad + c);
      zb1 = 0.0;
      zb2 = 0.5 * odzp[0] * w1 * w1 * odzt[1] * (c - ad) * dts;
      zc = odzp[0] * c * w1;
    } else if (kk == km - 1) {
      const double au = at_u[r];
      za = 0.5 * odzp[km - 1] * wk * (c + au);
      zb1 = -0.5 * odzp[km - 1] * wk * wk * odzt[km - 1] * (au - c) * dts;
      zb2 = 0.0;
      zc = -odzp[km - 1] * c * wk;
    } else {
      const double au = at_u[r], ad = at_d[r], w1 = ws_d[u];
      za = 0.5 * odzp[kk] * wk * (c + au) - 0.5 * odzp[kk] * w1 * (c + ad);
      zb1 = -0.5 * odzp[kk] * wk * wk * odzt[kk] * (au - c) * dts;
      zb2 = 0.5 * odzp[kk] * w1 * w1 * odzt[kk + 1] * (c - ad) * dts;
      zc = -odzp[kk] * c * (wk - w1);
    }
    const double xx = -(x0v + xy1 + xy2 + cx);
    const double yy = -(y0v + xy3 + xy4 + cy);
    const double zz = -(zb1 + zb2 + za + zc);
    const double a00 = c + (xx + yy + zz) * dts;
    auto vitk = [&](int kl, int rr) { return (kl < S.kmt[rr]) ? 1.0 : 0.0; };
    auto mxv = [&](double t, double vt) { return t * vt + (1.0 - vt) * -1.0e10; };
    auto mnv = [&](double t, double vt) { return t * vt + (1.0 - vt) * 1.0e10; };
    const double vc = vitk(kk, r), vn_ = vitk(kk, r - SW), vs_ = vitk(kk, r + SW), vw = vitk(kk, r - 1),
                 ve = vitk(kk, r + 1);
    double hi_ = mxv(c, vc), lo_ = mnv(c, vc), t;
    t = mxv(n, vn_); if (hi_ < t) hi_ = t;
    t = mxv(s, vs_); if (hi_ < t) hi_ = t;
    t = mxv(w, vw); if (hi_ < t) hi_ = t;
    t = mxv(e, ve); if (hi_ < t) hi_ = t;
    t = mnv(n, vn_); if (lo_ > t) lo_ = t;
    t = mnv(s, vs_); if (lo_ > t) lo_ = t;
    t = mnv(w, vw); if (lo_ > t) lo_ = t;
    t = mnv(e, ve); if (lo_ > t) lo_ = t;
    if (kk > 0) {
      const double au = at_u[r], vu = vitk(kk - 1, r);
      t = mxv(au, vu); if (hi_ < t) hi_ = t;
      t = mnv(au, vu); if (lo_ > t) lo_ = t;
    }
    if (kk < km - 1) {
      const double ad = at_d[r], vd = vitk(kk + 1, r);
      t = mxv(ad, vd); if (hi_ < t) hi_ = t;
      t = mnv(ad, vd); if (lo_ > t) lo_ = t;
    }
    const bool f = a00 > hi_ || a00 < lo_;
    fl[m] = f ? 1 : 0;
    return f;
  }
}

// biharmonic coefficient c (dtn, dts, dte, dtw, ahf) of region cell m at q
__device__ __forceinline__ double del4c(const ExSmem& S, const Arena& a, int c, int m, long q) {
  if (kStageDel4) return S.dt5[c][m];
  const double* f = c == 0 ? a.dtn : c == 1 ? a.dts : c == 2 ? a.dte : c == 3 ? a.dtw : a.ahf;
  return __ldg(f + q);
}

// First Laplacian of atb at level kk for one cell (hj, hi) of the 1-halo region.
__device__ __forceinline__ void del4_one64(ExSmem& S, const Arena& a, int kk, int sk, int hj, int hi, int x0,
                                           int y0) {
  const double* atb = S.slot[sk].atb;
  {
    const int m = hj * HQX + hi;
    const int gj = y0 - 1 + hj, gi = x0 - 1 + hi;
    if (!(gi >= 1 && gi < a.imt - 1 && gj >= 1 && gj < a.jmt - 1)) { S.d2[m] = 0.0; return; }
    const int r = r2(hj, hi);
    const long q = (long)gj * a.imt + gi;
    double h = 0.0, cc = 0.0;
    if (kk <= S.kmt[r] - 1) {
      if (kk <= S.kmt[r - SW] - 1) { const double cf = del4c(S, a, 0, m, q); h += cf * atb[r - SW]; cc -= cf; }
      if (kk <= S.kmt[r + SW] - 1) { const double cf = del4c(S, a, 1, m, q); h += cf * atb[r + SW]; cc -= cf; }
      if (kk <= S.kmt[r + 1] - 1) { const double cf = del4c(S, a, 2, m, q); h += cf * atb[r + 1]; cc -= cf; }
      if (kk <= S.kmt[r - 1] - 1) { const double cf = del4c(S, a, 3, m, q); h += cf * atb[r - 1]; cc -= cf; }
    }
    S.d2[m] = del4c(S, a, 4, m, q) * (cc * atb[r] + h);
  }
}

// Every thread handles the interior cell above its column; the RING64 ring
// cells of the 1-halo region go to threads 0 .. RING64-1.
constexpr int RING64 = HN - TTHREADS;
__device__ __forceinline__ void ring_cell64(int q, int& hj, int& hi) {
  if (q < HQX) { hj = 0; hi = q; }
  else if (q < 2 * HQX) { hj = HQY - 1; hi = q - HQX; }
  else if (q < 2 * HQX + TY) { hj = q - 2 * HQX + 1; hi = 0; }
  else { hj = q - 2 * HQX - TY + 1; hi = HQX - 1; }
}

// kFp64CtasPerSm CTAs per SM: 228 KB of shared memory, 1 KB reserved per CTA
static_assert(kFp64CtasPerSm * (sizeof(ExSmem) + 1024) <= 228 * 1024,
              "FP64 tracer tile no longer fits kFp64CtasPerSm CTAs per SM");

// The six boxes of level L of tracer n by per-thread asynchronous copies, for
// grids whose row pitch TMA cannot take (not a multiple of 16 bytes): every
// thread copies its share of the boxes' elements (zeros outside the domain,
// as TMA fills them) and the slot's mbarrier counts one arrival per thread
// once its copies have landed.  The slot layout and the waits are the TMA
// path's (issue_level).
__device__ __forceinline__ void copy_level64(LevelSlot<double>& sl, uint64_t* bar, const Arena& a, int n, int L,
                                             int x0, int y0) {
  const int imt = a.imt, jmt = a.jmt;
  const long A = a.A, F = a.F, FB = a.FB;
  constexpr int NAT = (TY + 4) * SW, NWS = (TY + 2) * SW, NUW = (TY + 2) * SW, NVS = (TY + 3) * SW, NAK = TY * TX;
  constexpr int TOT = 2 * NAT + NWS + NUW + NVS + NAK;
  for (int e = threadIdx.x; e < TOT; e += TTHREADS) {
    const double* base;
    double* dst;
    int r, w, gj0, gi0;
    if (e < 2 * NAT) {
      const int b = e / NAT;
      r = e % NAT; w = SW; gj0 = y0 - 2; gi0 = x0 - 4;
      base = b == 0 ? a.at[a.cur] + n * F + (long)L * A : a.atb[a.cur] + n * FB + (long)(L + 1) * A;
      dst = b == 0 ? sl.at : sl.atb;
    } else if (e < 2 * NAT + NWS) {
      r = e - 2 * NAT; w = SW; gj0 = y0 - 1; gi0 = x0 - 4;
      base = a.ws + (long)L * A; dst = sl.ws;
    } else if (e < 2 * NAT + NWS + NUW) {
      r = e - 2 * NAT - NWS; w = SW; gj0 = y0 - 1; gi0 = x0 - 4;
      base = a.uwf + (long)L * A; dst = sl.uw;
    } else if (e < 2 * NAT + NWS + NUW + NVS) {
      r = e - 2 * NAT - NWS - NUW; w = SW; gj0 = y0 - 2; gi0 = x0 - 4;
      base = a.vsf + (long)L * A; dst = sl.vs;
    } else {
      r = e - 2 * NAT - NWS - NUW - NVS; w = TX; gj0 = y0; gi0 = x0;
      base = a.akt + n * F + (long)L * A; dst = sl.akt;
    }
    const int gj = gj0 + r / w, gi = gi0 + r % w;
    const bool in = gj >= 0 && gj < jmt && gi >= 0 && gi < imt;
    cp_async8z(dst + r, base + (in ? (long)gj * imt + gi : 0), in);
  }
  cp_async_mbar_arrive(bar);
}

// With diagnostics: the level from which a ring cell (where diagnostics are
// written) is below its bottom and carries no transport through its four
// faces or w (kfz of its own column covers its west and south faces and
// w, its east and north neighbours' cover the other two faces).  From there
// down its diagnostics need no limiter flag: a zero transport gives the same
// signed zero in the upwind and Lax-Wendroff form of every face flux.
__device__ __forceinline__ int deep_start_cell(const Arena& a, int i, int j) {
  if (!(i >= 1 && i < a.imt - 1 && j >= 1 && j < a.jmt - 1)) return 0;
  const long q = (long)j * a.imt + i;
  return max(max(a.kmt[q], a.kfz[q]), max(a.kfz[q + 1], a.kfz[q - a.imt]));
}

template <bool DIAG>
__global__ void __launch_bounds__(TTHREADS, kFp64CtasPerSm)
    k_tracer_tma64(Arena a, const __grid_constant__ TracerMaps maps, int ntx, long ntiles, int tma) {
  extern __shared__ __align__(128) unsigned char smem_tma[];
  ExSmem& S = *reinterpret_cast<ExSmem*>(smem_tma);
  const int tid = threadIdx.x, tx = tid % TX, ty = tid / TX;
  const int imt = a.imt, jmt = a.jmt, km = a.km;
  const long A = a.A, F = a.F, FB = a.FB;
  const lt_params& p = a.p;
  const double dts = p.dts;
  const double aidif = 0.5;
  const double* __restrict__ odzp = a.odzp;
  const double* __restrict__ odzt = a.odzt;
  const int NV = a.nv_scratch;
  double* scr = a.col_scratch + (long)blockIdx.x * km * NV * TTHREADS;
  if (tid == 0) {
    for (int s = 0; s < NSX; ++s) mbar_init(&S.bar[s], TTHREADS);   // one arrival per thread and level
    mbar_fence_init();
  }
  __syncthreads();
  uint32_t par = 0, outstanding = 0;
  const bool has_ring = tid < RING64;
  int ring_hj = 0, ring_hi = 0;
  if (has_ring) ring_cell64(tid, ring_hj, ring_hi);

  for (long w = blockIdx.x; w < 2 * ntiles; w += gridDim.x) {
    const long tile = w >> 1;
    const int n = (int)(w & 1);
    const int x0 = (int)(tile % ntx) * TX, y0 = (int)(tile / ntx) * TY;
    const int i = x0 + tx, j = y0 + ty;
    const double* at_in = a.at[a.cur] + n * F;
    double* at_out = a.at[a.cur ^ 1] + n * F;
    double* atb_out = a.atb[a.cur ^ 1] + n * FB;

    __syncthreads();  // the previous item is done with every slot
    // level L goes to slot s = L % NSX
    auto issue = [&](int L, int s) {
      if (tma) {
        if (tid == 0) issue_level(S.slot[s], &S.bar[s], maps, a.cur, n, km, L, x0, y0);
        else mbar_arrive(&S.bar[s]);
      } else {
        copy_level64(S.slot[s], &S.bar[s], a, n, L, x0, y0);
      }
      outstanding |= 1u << s;
    };
    auto wait = [&](int s) -> bool {
      const bool ok = mbar_wait(&S.bar[s], (par >> s) & 1u, a.wait_limit);
      if (ok) { par ^= 1u << s; outstanding &= ~(1u << s); }
      return ok;
    };
    for (int m = tid; m < (TY + 4) * SW; m += TTHREADS) {
      const int gj = y0 - 2 + m / SW, gi = x0 - 4 + m % SW;
      S.kmt[m] = (gj >= 0 && gj < jmt && gi >= 0 && gi < imt) ? a.kmt[(long)gj * imt + gi] : 0;
    }
    // Without diagnostics, levels at and below the deepest bottom of the
    // tile's own columns are land for every cell the march updates there:
    // the reference's arithmetic leaves them as they are (every term is
    // masked, the new value is at + dts * 0), so the march starts at the
    // first of them and the inner cells' values below it are copied.  (At
    // that level a wetter cell of the halo may form its limiter flag from the
    // level below, which is not loaded; the flag only meets the tile's cells
    // through faces and a w that carry no transport there, where every form
    // of the flux gives the same bits.)  With diagnostics the march starts at
    // the deepest deep_start_cell of the tile and k_diag_deep writes the
    // levels below it.
    int ks = km - 1;
    if (DIAG) {
      int kmax = deep_start_cell(a, i, j);
      kmax = __reduce_max_sync(0xffffffffu, kmax);
      if (tx == 0) S.wmax[ty] = kmax;
      __syncthreads();
#pragma unroll
      for (int q = 0; q < TTHREADS / 32; ++q) kmax = max(kmax, S.wmax[q]);
      ks = min(km - 1, kmax);
    } else {
      __syncthreads();
      int kmax = (int)S.kmt[r2(ty + 1, tx + 1)];
      kmax = __reduce_max_sync(0xffffffffu, kmax);
      if (tx == 0) S.wmax[ty] = kmax;
      __syncthreads();
#pragma unroll
      for (int q = 0; q < TTHREADS / 32; ++q) kmax = max(kmax, S.wmax[q]);
      ks = min(km - 1, kmax);
    }
    const int lowest_pro = ks - NSX + 1 > 0 ? ks - NSX + 1 : 0;
    for (int L = ks; L >= lowest_pro; --L) issue(L, L % NSX);
    // the level-free metric terms (products formed once, as the reference
    // forms them at every use)
    for (int m = tid; m < HN; m += TTHREADS) {
      const int gj = y0 - 1 + m / HQX, gi = x0 - 1 + m % HQX;
      const bool in = gj >= 0 && gj < jmt && gi >= 0 && gi < imt;
      const long q = in ? (long)gj * imt + gi : 0;
      S.tr[m] = in ? a.tarea_r[q] : 0.0;
      if (kStageDel4) {
        S.dt5[0][m] = in ? a.dtn[q] : 0.0;
        S.dt5[1][m] = in ? a.dts[q] : 0.0;
        S.dt5[2][m] = in ? a.dte[q] : 0.0;
        S.dt5[3][m] = in ? a.dtw[q] : 0.0;
        S.dt5[4][m] = in ? a.ahf[q] : 0.0;
      }
    }
    for (int m = tid; m < HQY * (HQX + 1); m += TTHREADS) {
      const int gj = y0 - 1 + m / (HQX + 1), gi = x0 - 1 + m % (HQX + 1);
      const long q = (long)gj * imt + gi;
      S.hw[m] = (gj >= 0 && gj < jmt && gi >= 0 && gi < imt) ? a.htw[q] * a.hun[q] : 0.0;
    }
    for (int m = tid; m < (HQY + 1) * HQX; m += TTHREADS) {
      const int gj = y0 - 2 + m / HQX, gi = x0 - 1 + m % HQX;
      const long q = (long)gj * imt + gi;
      S.hs[m] = (gj >= 0 && gj < jmt && gi >= 0 && gi < imt) ? a.hts[q] * a.hue[q] : 0.0;
    }

    const bool own = (i < imt && j < jmt);
    const bool ring = own && i >= 1 && i < imt - 1 && j >= 1 && j < jmt - 1;
    const bool inner = own && i >= 2 && i < imt - 2 && j >= 2 && j < jmt - 2;
    const long qo = own ? (long)j * imt + i : 0;
    const int kz = own ? a.kmt[qo] : 0;
    if (!DIAG && inner) {
      // eight levels' loads in flight ahead of their stores
      const double* __restrict__ src = at_in;
      double* __restrict__ d1 = at_out;
      double* __restrict__ d2 = atb_out;
      for (int k0 = ks + 1; k0 < km; k0 += 8) {
        double v[8];
#pragma unroll
        for (int c = 0; c < 8; ++c) v[c] = k0 + c < km ? src[(long)(k0 + c) * A + qo] : 0.0;
#pragma unroll
        for (int c = 0; c < 8; ++c)
          if (k0 + c < km) {
            __stcs(d1 + (long)(k0 + c) * A + qo, v[c]);
            __stcs(d2 + (long)(k0 + c + 1) * A + qo, v[c]);
          }
      }
    }
    const int hc = (ty + 1) * HQX + (tx + 1);
    const int rc = r2(ty + 1, tx + 1), uc = ru(ty + 1, tx + 1), vc = rv(ty + 1, tx + 1), ac = ty * TX + tx;
    const double swv = (inner && n == 0) ? a.swv[qo] : 0.0;
    const double stf = own ? a.stf_n[n * A + qo] : 0.0;
    const double err_norm2 = a.scalars[0];
    double e_prev = 0.0, f_prev = 0.0;
    // own cell's at, ws and atb of level k+1, kept from step k+1 (with
    // diagnostics, those of the level below the first marched one)
    double at_dn = 0.0, ws_dn = 0.0, atb_dn = 0.0;
    if (DIAG && own && ks < km - 1) {
      at_dn = at_in[(long)(ks + 1) * A + qo];
      ws_dn = a.ws[(long)(ks + 1) * A + qo];
      atb_dn = a.atb[a.cur][n * FB + (long)(ks + 2) * A + qo];
    }

    // slots of levels k, k-1, k+1 (NSX == 3: level k-2 shares k+1's), carried
    // through the level loop
    static_assert(NSX == 3, "slot rotation below assumes three slots");
    // (below ks the slot of level ks+1 holds level ks-2: the first
    // predictor's limiter flags of level ks meet the tile's cells only
    // through zero transports.)  Every level the prologue issued is waited
    // before any of them is used: with the third one still in flight the
    // results came out different at a cell's bottom wet level in some runs,
    // in the cells of the threads that also carry a ring cell.
    int sk = ks % NSX;
    int sm1 = sk == 0 ? 2 : sk - 1, sp1 = sk == 2 ? 0 : sk + 1;
    {
      const bool ok = wait(sk) && (ks == 0 || wait(sm1)) && (ks < 2 || wait(sp1));
      // a wait that ran out anywhere in the CTA sends every thread out together
      if (__syncthreads_or(!ok)) { tma_bail(S, a, par, outstanding); return; }
    }
    // limiter flags of the own cell at levels k+1, k (earlier steps) and k-1
    bool out_kp1 = false,
         out_k = pred_one64(S, a, ks, sk, sm1, sp1, ty + 1, tx + 1, x0, y0,
                            &S.xyc[0][0][0] + tid + (kCacheXY ? (ks & 1) * 6 * TTHREADS : 0), true),
         out_km1 = false;
    if (has_ring) pred_one64(S, a, ks, sk, sm1, sp1, ring_hj, ring_hi, x0, y0, nullptr, true);

    for (int k = ks; k >= 0; --k) {
      // ---- phase B1: first Laplacian at level k (arrived in an earlier step)
      del4_one64(S, a, k, sk, ty + 1, tx + 1, x0, y0);
      if (has_ring) del4_one64(S, a, k, sk, ring_hj, ring_hi, x0, y0);
      const bool ok = (k >= 2 && k != ks) ? wait(sp1) : true;   // level k-2 (the prologue waited ks-2)
      if (__syncthreads_or(!ok)) { tma_bail(S, a, par, outstanding); return; }
      // ---- phase B2: predictor one level up.  The column phase below reads
      // the flags of level k of the neighbours (written in the previous step)
      // and only its own cell's flags of the levels k-1 and k+1, which this
      // thread computed: no barrier between the two phases.
      if (k >= 1) {
        out_km1 = pred_one64(S, a, k - 1, sm1, sp1, sk, ty + 1, tx + 1, x0, y0,
                             &S.xyc[0][0][0] + tid + (kCacheXY ? ((k - 1) & 1) * 6 * TTHREADS : 0), true);
        if (has_ring) pred_one64(S, a, k - 1, sm1, sp1, sk, ring_hj, ring_hi, x0, y0, nullptr, true);
      }
      // ---- phase C.  Without diagnostics an inner cell below its column's
      // bottom keeps its value (every term of the step is masked) and only
      // hands its level's values up to the level above.
      if (!DIAG && inner && k >= kz) {
        const LevelSlot<double>& Lk = S.slot[sk];
        const double c = Lk.at[rc];
        __stcs(at_out + (long)k * A + qo, c);
        __stcs(atb_out + (long)(k + 1) * A + qo, c);
        at_dn = c;
        ws_dn = Lk.ws[uc];
        atb_dn = Lk.atb[rc];
      } else if (ring) {
        const LevelSlot<double>& Lk = S.slot[sk];
        const double* at_c = Lk.at;
        const double* at_u = k > 0 ? S.slot[sm1].at : nullptr;
        const unsigned char* fl = S.flag[sk];
        const double tr = S.tr[hc];
        const double hwe = S.hw[(ty + 1) * (HQX + 1) + tx + 2], hww = S.hw[(ty + 1) * (HQX + 1) + tx + 1];
        const double hss = S.hs[(ty + 2) * HQX + tx + 1], hsn = S.hs[(ty + 1) * HQX + tx + 1];
        const double c = at_c[rc], e = at_c[rc + 1], w = at_c[rc - 1], s = at_c[rc + SW], nn = at_c[rc - SW];
        const double ue = Lk.uw[uc + 1], uwc = Lk.uw[uc], vsc = Lk.vs[vc], vn = Lk.vs[vc - SW];
        const bool self = out_k;
        const bool edge_k = (k == 0 || k == km - 1);
        auto lim = [&](int m, bool guard) {
          const bool nb = fl[m] != 0;
          return edge_k ? (self || (nb && guard)) : ((self || nb) && guard);
        };
        double xy1, xy2, xy3, xy4, zb1, zb2, za, zc;
        const double* xc = &S.xyc[0][0][0] + tid + (kCacheXY ? (k & 1) * 6 * TTHREADS : 0);
        // the predictor of a dry cell whose faces carry no transport was
        // skipped (pred_one64's dry_out), so its cached terms are stale:
        // with diagnostics they are formed here from the same expressions
        // (without, such a cell is inner and copied above, or on the ring,
        // where its tendency is not used)
        const bool cached =
            kCacheXY && !(DIAG && k >= kz && ue == 0.0 && uwc == 0.0 && vsc == 0.0 && vn == 0.0);
        if (lim(hc + 1, i <= imt - 3)) xy1 = -(e - c) * fabs(ue) * tr;
        else xy1 = cached ? xc[0] : -dts * (e - c) * 2.0 * tr * ue * ue / hwe;
        if (lim(hc - 1, i >= 2)) xy2 = (c - w) * fabs(uwc) * tr;
        else xy2 = cached ? xc[TTHREADS] : dts * (c - w) * 2.0 * tr * uwc * uwc / hww;
        if (lim(hc + HQX, j <= jmt - 3)) xy3 = -(s - c) * fabs(vsc) * tr;
        else xy3 = cached ? xc[2 * TTHREADS] : -dts * (s - c) * 2.0 * tr * vsc * vsc / hss;
        if (lim(hc - HQX, j >= 2)) xy4 = (c - nn) * fabs(vn) * tr;
        else xy4 = cached ? xc[3 * TTHREADS] : dts * (c - nn) * 2.0 * tr * vn * vn / hsn;
        const double wk = Lk.ws[uc];
        if (k == 0) {
          const double w1 = ws_dn, ad = at_dn;
          zb1 = 0.0;
          if (self || (out_kp1 && k <= km - 2))
            zb2 = 0.5 * fabs(w1) * odzp[k] * (c - ad);
          else
            zb2 = 0.5 * odzp[0] * w1 * w1 * odzt[1] * (c - ad) * dts;
          za = -0.5 * odzp[0] * w1 * (ad + c);
          zc = odzp[0] * c * w1;
        } else if (k == km - 1) {
          const double au = at_u[rc];
          if (self || out_km1)
            zb1 = -0.5 * fabs(wk) * odzp[k] * (au - c);
          else
            zb1 = -0.5 * odzp[k] * wk * wk * odzt[k] * (au - c) * dts;
          zb2 = 0.0;
          za = 0.5 * odzp[km - 1] * wk * (c + au);
          zc = -odzp[km - 1] * c * wk;
        } else {
          const double au = at_u[rc], ad = at_dn, w1 = ws_dn;
          if ((self || out_km1) && k >= 1)
            zb1 = -0.5 * fabs(wk) * odzp[k] * (au - c);
          else
            zb1 = -0.5 * odzp[k] * wk * wk * odzt[k] * (au - c) * dts;
          if ((self || out_kp1) && k <= km - 2)
            zb2 = 0.5 * fabs(w1) * odzp[k] * (c - ad);
          else
            zb2 = 0.5 * odzp[k] * w1 * w1 * odzt[k + 1] * (c - ad) * dts;
          za = 0.5 * odzp[k] * wk * (c + au) - 0.5 * odzp[k] * w1 * (c + ad);
          zc = -odzp[k] * c * (wk - w1);
        }
        const double cx = -c * (ue - uwc) * tr * 2.0;
        const double cy = -c * (vsc - vn) * tr * 2.0;
        const double x0v = cached ? xc[4 * TTHREADS] : (e + c) * ue * tr - (c + w) * uwc * tr;
        const double y0v = cached ? xc[5 * TTHREADS] : ((s + c) * vsc - (c + nn) * vn) * tr;
        const double xx = -(x0v + xy1 + xy2 + cx);
        const double yy = -(y0v + xy3 + xy4 + cy);
        const double zz = -(za + zb1 + zb2 + zc);
        const double adv = xx + yy + zz;
        const long cg = (long)k * A + qo;
        if (DIAG) {
          a.ax[n * F + cg] = xx;
          a.ay[n * F + cg] = yy;
          a.az[n * F + cg] = zz;
        }
        if (inner) {
          const double vit_k = k < kz ? 1.0 : 0.0;
          const double vit_kp1 = (k + 1 < kz) ? 1.0 : 0.0;
          const double atb_k = Lk.atb[rc];
          const double atb_km1 = k >= 1 ? S.slot[sm1].atb[rc] : 0.0;
          const double atb_kp1 = k < km - 1 ? atb_dn : 0.0;
          const double wkc_k = Lk.akt[ac];
          const double wkc_km1 = k >= 1 ? S.slot[sm1].akt[ac] : 0.0;
          // below the column's bottom every term of the step is masked (its
          // new value is at + dts*0 = at): with diagnostics only they are
          // formed there, and the state is copied (without diagnostics such
          // cells take the copy path above)
          const bool dry = DIAG && k >= kz;
          double tf = adv * vit_k;
          if (!dry) {
            const int r = rc;
            double h = 0.0, cc = 0.0;
            if (k <= S.kmt[r] - 1) {
              if (k <= S.kmt[r - SW] - 1) { const double cf = del4c(S, a, 0, hc, qo); h += cf * S.d2[hc - HQX]; cc -= cf; }
              if (k <= S.kmt[r + SW] - 1) { const double cf = del4c(S, a, 1, hc, qo); h += cf * S.d2[hc + HQX]; cc -= cf; }
              if (k <= S.kmt[r + 1] - 1) { const double cf = del4c(S, a, 2, hc, qo); h += cf * S.d2[hc + 1]; cc -= cf; }
              if (k <= S.kmt[r - 1] - 1) { const double cf = del4c(S, a, 3, hc, qo); h += cf * S.d2[hc - 1]; cc -= cf; }
            }
            tf += p.ah * (cc * S.d2[hc] + h);
          }
          if (n == 0) {
            if (k >= 1 && k < km - 1) {
              const double w1 = swv * a.pen[k - 1] * vit_k;
              const double w2 = swv * a.pen[k] * vit_kp1;
              tf = tf + (w1 - w2) * odzp[k];
              if (DIAG) a.penetrate[cg] = (w1 - w2) * odzp[k];
            } else if (k == 0) {
              const double w1 = swv * a.pen[0] * ((1 < kz) ? 1.0 : 0.0);
              tf = tf - odzp[0] * w1;
              if (DIAG) a.penetrate[cg] = -w1 * odzp[0];
            } else {
              const double w2 = swv * a.pen[km - 2] * vit_k;
              tf = tf + odzp[km - 1] * w2;
              if (DIAG) a.penetrate[cg] = w2 * odzp[km - 1];
            }
          }
          if (k >= 1 && k < km - 1) {
            const double w1 = wkc_km1 * (atb_km1 - atb_k) * odzt[k] * vit_k;
            const double w2 = wkc_k * (atb_k - atb_kp1) * odzt[k + 1] * vit_kp1;
            tf = tf + odzp[k] * (w1 - w2) * 0.5;
            if (DIAG) a.dzd[n * F + cg] = odzp[k] * (w1 - w2) * 0.5;
          } else if (k == 0) {
            const double w1 = wkc_k * (atb_k - atb_kp1) * odzt[1] * vit_kp1;
            tf = tf - odzp[0] * w1 * 0.5;
            if (DIAG) a.dzd[n * F + cg] = -odzp[0] * w1 * 0.5;
          } else {
            const double w2 = wkc_km1 * (atb_km1 - atb_k) * odzt[km - 1] * vit_k;
            tf = tf + odzp[km - 1] * w2 * (1.0 - aidif);
            if (DIAG) a.dzd[n * F + cg] = odzp[km - 1] * w2 * 0.5;
          }
          if (dry) {
            // tracer_9's diagnostics of the unchanged cell, formed as for
            // any cell: v = d8 = at
            const double v = c;
            a.tend[n * F + cg] = (v - c) / dts * vit_k;
            if (k == 0) a.dt_diff[n * F + cg] = (v - v) / dts * vit_k - stf * 0.5 * odzp[0];
            else a.dt_diff[n * F + cg] = (v - v) / dts * vit_k;
            if (j == 2 && a.tripole) a.fold_save[((long)(n * km + k)) * imt + i] = v;
            at_out[cg] = v;
            atb_out[(long)(k + 1) * A + qo] = v;
          } else {
          if (k == 0) {
            if (n == 1) {
              if (kz > 0) tf = tf + stf * (1.0 - aidif) * odzp[0];
              tf = tf + err_norm2 * vit_k;
            } else if (kz > 0) {
              tf = tf + stf * odzp[0] * 0.5;
            }
          }
          if (p.simple_assm && k < p.ktv) tf = tf + vit_k * (a.restore_at[n * F + cg] - atb_k) * assm_rate(k);
          if (p.boundary_restore == 1 && k >= 1) {
            const double lamda = 1.0 / (15.0 * 86400.0);
            tf = tf + vit_k * (a.restore[n * F + cg] - atb_k) * lamda;
          }
          const double d8 = c + dts * tf;
          double ev = 0.0, fv = d8;
          if (k < kz) {
            double a8, c8, b8;
            if (k >= 1) a8 = wkc_km1 * odzt[k] * odzp[k] * dts * 0.5;
            else a8 = odzp[0] * dts * 0.5;
            if (k == kz - 1) {
              c8 = odzp[kz - 1] * dts * 0.5;
              b8 = 1.0 + a8;
            } else if (k >= 1) {
              c8 = wkc_k * odzt[k + 1] * odzp[k] * dts * 0.5;
              b8 = 1.0 + a8 + c8;
            } else {
              c8 = wkc_k * odzt[k + 1] * odzp[k] * dts * 0.5;
              b8 = 1.0 + c8;
            }
            if (k == kz - 1) { e_prev = 0.0; f_prev = 0.0; }
            const double g0 = 1.0 / (b8 - c8 * e_prev);
            ev = a8 * g0;
            fv = (d8 + c8 * f_prev) * g0;
            e_prev = ev;
            f_prev = fv;
          }
          double* sl = scr + (long)k * NV * TTHREADS;
          const uint64_t pl = l2_evict_last();
          st_l2(sl + tid, ev, pl);
          st_l2(sl + TTHREADS + tid, fv, pl);
          if (DIAG) st_l2(sl + 2 * TTHREADS + tid, d8, pl);
          }  // wet
          atb_dn = atb_k;
        }
        at_dn = c;
        ws_dn = wk;
      }
      out_kp1 = out_k;
      out_k = out_km1;
      __syncthreads();  // level k is no longer read: its slot takes level k-NSX
      if (k - NSX >= 0) issue(k - NSX, sk);
      // one level down: the slots of k-1, k-2, k
      sp1 = sk;
      sk = sm1;
      sm1 = sk == 0 ? 2 : sk - 1;
    }
    // ---- substitution, top down: the elimination coefficients of SUB levels
    // are loaded together ahead of their stores (the scratch round trip is
    // paid once per SUB levels, not once per level)
    if (inner) {
      double x = 0.0;
      constexpr int SUB = 8;
      const int kend = min(kz, ks + 1);   // the levels the march left in the scratch (the wet ones)
      const uint64_t pf = l2_evict_first();
      for (int k0 = 0; k0 < kend; k0 += SUB) {
        double evs[SUB], fvs[SUB];
#pragma unroll
        for (int c = 0; c < SUB; ++c) {
          const double* sl = scr + (long)(k0 + c) * NV * TTHREADS;
          evs[c] = k0 + c < kend ? ld_l2(sl + tid, pf) : 0.0;
          fvs[c] = k0 + c < kend ? ld_l2(sl + TTHREADS + tid, pf) : 0.0;
        }
#pragma unroll
      for (int c = 0; c < SUB; ++c) {
        const int k = k0 + c;
        if (k >= kend) break;
        const double* sl = scr + (long)k * NV * TTHREADS;
        const double ev = evs[c], fv = fvs[c];
        const long cg = (long)k * A + qo;
        double v;
        if (k < kz) {
          const double vit_k = 1.0;
          v = (k == 0) ? (ev * stf + fv) * vit_k : (ev * x + fv) * vit_k;
          x = v;
        } else {
          v = fv;
        }
        if (DIAG) {
          const double d8 = ld_l2(sl + 2 * TTHREADS + tid, pf);
          const double vit_k = k < kz ? 1.0 : 0.0;
          const double at_old = at_in[cg];
          a.tend[n * F + cg] = (v - at_old) / dts * vit_k;
          if (k == 0) a.dt_diff[n * F + cg] = (v - d8) / dts * vit_k - stf * 0.5 * odzp[0];
          else a.dt_diff[n * F + cg] = (v - d8) / dts * vit_k;
          if (j == 2 && a.tripole) a.fold_save[((long)(n * km + k)) * imt + i] = d8;
        }
        __stcs(at_out + cg, v);
        __stcs(atb_out + (long)(k + 1) * A + qo, v);
      }
      }
    }
  }
}

// ------------------------------------------------- deep levels (diagnostics)
// The levels k_tracer_tma64<true> leaves to this kernel: below the deepest
// deep_start_cell of a tile every ring cell of the tile is below its bottom
// and carries no transport, so per cell and level it writes the diagnostics
// of advection_tracer_3 (the upwind forms of the face fluxes, the same bits
// as any form at a zero transport), of tracer_5 (penetrate, dz) and of
// tracer_9 (tend, dt_diff, with the state unchanged: every term is masked),
// reading the level fields directly.  Block = one tile (the column kernel's
// decomposition), blockIdx.y = tracer.
__global__ void __launch_bounds__(TTHREADS) k_diag_deep(Arena a, int ntx) {
  __shared__ int wmax[TTHREADS / 32];
  const int n = blockIdx.y, tid = threadIdx.x, tx = tid % TX, ty = tid / TX;
  const int x0 = (int)(blockIdx.x % ntx) * TX, y0 = (int)(blockIdx.x / ntx) * TY;
  const int i = x0 + tx, j = y0 + ty;
  const int imt = a.imt, jmt = a.jmt, km = a.km;
  const long A = a.A, F = a.F, FB = a.FB;
  int kmax = deep_start_cell(a, i, j);
  kmax = __reduce_max_sync(0xffffffffu, kmax);
  if (tx == 0) wmax[ty] = kmax;
  __syncthreads();
#pragma unroll
  for (int q = 0; q < TTHREADS / 32; ++q) kmax = max(kmax, wmax[q]);
  const int ks = min(km - 1, kmax);
  const bool own = i < imt && j < jmt;
  const bool ring = own && i >= 1 && i < imt - 1 && j >= 1 && j < jmt - 1;
  const bool inner = own && i >= 2 && i < imt - 2 && j >= 2 && j < jmt - 2;
  if (!ring || ks >= km - 1) return;
  const long qo = (long)j * imt + i;
  const double dts = a.p.dts;
  const double* __restrict__ at = a.at[a.cur] + n * F;
  const double* __restrict__ atb = a.atb[a.cur] + n * FB;
  const double* __restrict__ akt = a.akt + n * F;
  const double* __restrict__ uwf = a.uwf;
  const double* __restrict__ vsf = a.vsf;
  const double* __restrict__ ws = a.ws;
  const double* __restrict__ odzp = a.odzp;
  const double* __restrict__ odzt = a.odzt;
  const double tr = __ldg(a.tarea_r + qo);
  const double swv = (inner && n == 0) ? __ldg(a.swv + qo) : 0.0;
  const double vit_k = 0.0, vit_kp1 = 0.0;   // below the bottom
  for (int k = ks + 1; k < km; ++k) {
    const long cg = (long)k * A + qo;
    const double c = __ldg(at + cg), e = __ldg(at + cg + 1), w = __ldg(at + cg - 1);
    const double s = __ldg(at + cg + imt), nn = __ldg(at + cg - imt);
    const double au = __ldg(at + cg - A);
    const double ue = __ldg(uwf + cg + 1), uwc = __ldg(uwf + cg), vsc = __ldg(vsf + cg), vn = __ldg(vsf + cg - imt);
    const double wk = __ldg(ws + cg);
    const double xy1 = -(e - c) * fabs(ue) * tr;
    const double xy2 = (c - w) * fabs(uwc) * tr;
    const double xy3 = -(s - c) * fabs(vsc) * tr;
    const double xy4 = (c - nn) * fabs(vn) * tr;
    double zb1, zb2, za, zc;
    if (k == km - 1) {
      zb1 = -0.5 * fabs(wk) * odzp[k] * (au - c);
      zb2 = 0.0;
      za = 0.5 * odzp[km - 1] * wk * (c + au);
      zc = -odzp[km - 1] * c * wk;
    } else {
      const double ad = __ldg(at + cg + A), w1 = __ldg(ws + cg + A);
      zb1 = -0.5 * fabs(wk) * odzp[k] * (au - c);
      zb2 = 0.5 * fabs(w1) * odzp[k] * (c - ad);
      za = 0.5 * odzp[k] * wk * (c + au) - 0.5 * odzp[k] * w1 * (c + ad);
      zc = -odzp[k] * c * (wk - w1);
    }
    const double cx = -c * (ue - uwc) * tr * 2.0;
    const double cy = -c * (vsc - vn) * tr * 2.0;
    const double x0v = (e + c) * ue * tr - (c + w) * uwc * tr;
    const double y0v = ((s + c) * vsc - (c + nn) * vn) * tr;
    a.ax[n * F + cg] = -(x0v + xy1 + xy2 + cx);
    a.ay[n * F + cg] = -(y0v + xy3 + xy4 + cy);
    a.az[n * F + cg] = -(za + zb1 + zb2 + zc);
    if (!inner) continue;
    const double atb_k = __ldg(atb + cg + A), atb_km1 = __ldg(atb + cg);
    const double wkc_km1 = __ldg(akt + cg - A);
    if (k < km - 1) {
      if (n == 0) {
        const double w1p = swv * a.pen[k - 1] * vit_k;
        const double w2p = swv * a.pen[k] * vit_kp1;
        a.penetrate[cg] = (w1p - w2p) * odzp[k];
      }
      const double atb_kp1 = __ldg(atb + cg + 2 * A), wkc_k = __ldg(akt + cg);
      const double w1 = wkc_km1 * (atb_km1 - atb_k) * odzt[k] * vit_k;
      const double w2 = wkc_k * (atb_k - atb_kp1) * odzt[k + 1] * vit_kp1;
      a.dzd[n * F + cg] = odzp[k] * (w1 - w2) * 0.5;
    } else {
      if (n == 0) {
        const double w2p = swv * a.pen[km - 2] * vit_k;
        a.penetrate[cg] = w2p * odzp[km - 1];
      }
      const double w2 = wkc_km1 * (atb_km1 - atb_k) * odzt[km - 1] * vit_k;
      a.dzd[n * F + cg] = odzp[km - 1] * w2 * 0.5;
    }
    // tracer_8, invtrit and tracer_9 of a masked cell: v = d8 = at
    const double v = c;
    a.tend[n * F + cg] = (v - c) / dts * vit_k;
    a.dt_diff[n * F + cg] = (v - v) / dts * vit_k;
    if (j == 2 && a.tripole) a.fold_save[((long)(n * km + k)) * imt + i] = v;
    a.at[a.cur ^ 1][n * F + cg] = v;
    a.atb[a.cur ^ 1][n * FB + (long)(k + 1) * A + qo] = v;
  }
}

// ------------------------------------------------------------- state halo
// One block per (level, tracer): ghost cells of the new state take the halo
// values (pop_haloupdate_tracer2 then tracer_9 for every point); cells the
// halo does not reach take the vtl input, which is what the reference's
// scratch use of vtl leaves there (tracer.cpp:1629-1653, 1895).
// Launched once per tracer (temperature first), so the salinity pass can read
// the temperature's final ghost values, which is what vtl holds in the
// reference between the two passes.
template <bool DIAG>
__device__ __forceinline__ void halo_state_level(const Arena& a, int n, int k) {
  extern __shared__ double top[];
  const int imt = a.imt, jmt = a.jmt;
  const long A = a.A, F = a.F, FB = a.FB;
  double* lvl = a.at[a.cur ^ 1] + n * F + (long)k * A;
  double* lvlb = a.atb[a.cur ^ 1] + n * FB + (long)(k + 1) * A;
  const double* old = a.at[a.cur] + n * F + (long)k * A;
  const double* vin = a.vtl ? a.vtl + (long)k * A : nullptr;
  const float* vin32 = a.vtl32 ? a.vtl32 + (long)k * A : nullptr;
  const double* tnew = a.at[a.cur ^ 1] + (long)k * A;  // temperature after its halo (n == 1 only)
  for (int i = threadIdx.x; i < imt; i += blockDim.x) top[i] = lvl[2L * imt + i];
  __syncthreads();
  HaloCells hc{imt, jmt, a.tripole};
  const long nc = hc.count();
  const double dts = a.p.dts;
  for (long m = threadIdx.x; m < nc; m += blockDim.x) {
    int j, i;
    hc.cell(m, j, i);
    const long q = (long)j * imt + i;
    double v;
    const bool filled = halo_cell_value(lvl, top, j, i, imt, jmt, a.ew_cyclic, a.tripole, v);
    if (!filled) v = vin ? vin[q] : (double)vin32[q];
    if (DIAG) {
      const double vit = k < a.kmt[q] ? 1.0 : 0.0;
      const bool inner = (i >= 2 && i < imt - 2 && j >= 2 && j < jmt - 2);
      double ori;
      if (inner) ori = a.fold_save[((long)(n * a.km + k)) * imt + i];
      else if (n == 0 || !filled) ori = vin ? vin[q] : (double)vin32[q];
      else ori = tnew[q];
      a.tend[n * F + (long)k * A + q] = (v - old[q]) / dts * vit;
      if (k == 0)
        a.dt_diff[n * F + q] = (v - ori) / dts * vit - a.stf_n[n * A + q] * 0.5 * a.odzp[0];
      else
        a.dt_diff[n * F + (long)k * A + q] = (v - ori) / dts * vit;
    }
    lvl[q] = v;
    lvlb[q] = v;
  }
}

template <bool DIAG>
__global__ void k_halo_state(Arena a, int n) {
  halo_state_level<DIAG>(a, n, blockIdx.x);
}

// Without diagnostics the two tracers' ghost fills are independent: one
// launch, part blockIdx.x (as k_halo_r8) of level blockIdx.y of tracer
// blockIdx.z, the same values as halo_state_level<false>.
__global__ void k_halo_state_parts(Arena a) {
  const int n = blockIdx.z, k = blockIdx.y;
  const int imt = a.imt, jmt = a.jmt;
  HaloCells hc{imt, jmt, a.tripole};
  long m0, m1;
  if (!halo_part(hc.count(), imt, a.tripole, blockIdx.x, m0, m1)) return;
  const long A = a.A, F = a.F, FB = a.FB;
  double* lvl = a.at[a.cur ^ 1] + n * F + (long)k * A;
  double* lvlb = a.atb[a.cur ^ 1] + n * FB + (long)(k + 1) * A;
  const double* vin = a.vtl ? a.vtl + (long)k * A : nullptr;
  const float* vin32 = a.vtl32 ? a.vtl32 + (long)k * A : nullptr;
  extern __shared__ double top[];
  if (a.tripole && blockIdx.x == 0) {
    for (int i = threadIdx.x; i < imt; i += blockDim.x) top[i] = lvl[2L * imt + i];
    __syncthreads();
  }
  for (long m = m0 + threadIdx.x; m < m1; m += blockDim.x) {
    int j, i;
    hc.cell(m, j, i);
    const long q = (long)j * imt + i;
    double v;
    if (!halo_cell_value(lvl, top, j, i, imt, jmt, a.ew_cyclic, a.tripole, v)) v = vin ? vin[q] : (double)vin32[q];
    lvl[q] = v;
    lvlb[q] = v;
  }
}

// tracer n of every member: blockIdx.x the level, blockIdx.y the member
__global__ void k_halo_state_batch(const MemberDesc* __restrict__ mem, int n) {
  const Arena& a = mem[blockIdx.y].a;
  if ((int)blockIdx.x >= a.km) return;
  if (a.diagnostics) halo_state_level<true>(a, n, blockIdx.x);
  else halo_state_level<false>(a, n, blockIdx.x);
}

__global__ void k_vtl_clobber(Arena a) {
  // tracer_ leaves vtl holding S with its halo (tracer.cpp:1891-1893)
  const long m = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= a.F) return;
  a.vtl[m] = a.at[a.cur][a.F + m];
}

}  // namespace

// ---------------------------------------------------------------- launchers
int launch_ssh(const Arena& a, cudaStream_t s) {
  dim3 b(32, 8), g((a.imt + 31) / 32, (a.jmt + 7) / 8);
  k_ssh<<<g, b, 0, s>>>(a);
  LT_LAUNCHED();
  return LT_OK;
}

int launch_surface_fluxes(const Arena& a, cudaStream_t s) {
  dim3 b(32, 8), g((a.imt + 31) / 32, (a.jmt + 7) / 8);
  k_surface_fluxes<<<g, b, 0, s>>>(a);
  LT_LAUNCHED();
  return LT_OK;
}

size_t tree_sum_part_elems(long n) {
  size_t tot = 0;
  long nb = (n + 2 * RB - 1) / (2 * RB);
  if (nb < 1) nb = 1;
  tot += nb;
  while (nb > 1) { nb = (nb + 2 * RB - 1) / (2 * RB); tot += nb; }
  return tot + 4;
}

int launch_interior_sum_sss(const Arena& a, cudaStream_t s) {
  SssTerm t{a.tarea, a.net + a.A, a.kmt, a.nx, a.imt};
  int rc = tree_sum(t, (long)a.nx * a.ny, a.red_part, a.scalars + 4, s);
  if (rc) return rc;
  k_finish_sss<<<1, 1, 0, s>>>(a.scalars, a.scalars + 4, a.p.area_t);
  LT_LAUNCHED();
  return LT_OK;
}

int launch_tree_sum(const double* x, long n, double* part, double* out, cudaStream_t s) {
  return tree_sum(ArrayTerm{x}, n, part, out, s);
}

int launch_halo_r8(double* f, int nz, int imt, int jmt, int ew_cyclic, int tripole, cudaStream_t s) {
  k_halo_r8<<<dim3(kHaloParts, nz), 256, imt * sizeof(double), s>>>(f, imt, jmt, ew_cyclic, tripole);
  LT_LAUNCHED();
  return LT_OK;
}

int launch_continuity_fp64(const Arena& a, cudaStream_t s) {
  constexpr int BY = kCont64TileY;
  dim3 b(32, BY), g((a.imt + 31) / 32, (a.jmt + BY - 1) / BY);
  k_cont_march64<BY><<<g, b, 0, s>>>(a);
  LT_LAUNCHED();
  return LT_OK;
}

int tracer_slots(const Arena& a) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long ntiles = (long)((a.imt + TX - 1) / TX) * ((a.jmt + TY - 1) / TY);
  long slots = (long)sms * 4;
  if (slots > 2 * ntiles) slots = 2 * ntiles;
  return (int)slots;
}

int launch_tracer_fp64(const Arena& a, cudaStream_t s, int slots) {
  const int ntx = (a.imt + TX - 1) / TX;
  const long ntiles = (long)ntx * ((a.jmt + TY - 1) / TY);
  const size_t sm = sizeof(TSmem);
  // [scheme - 1][diagnostics]: the centred and flux schemes (lt_adv_scheme order)
  using Kern = void (*)(Arena, int, long);
  static const Kern kern[2][2] = {
      {k_tracer64<false, LT_ADV_CENTERED>, k_tracer64<true, LT_ADV_CENTERED>},
      {k_tracer64<false, LT_ADV_FLUX>, k_tracer64<true, LT_ADV_FLUX>}};
  static bool attr = false;
  if (!attr) {
    for (auto& row : kern)
      for (Kern k : row) LT_CUDA_OK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    attr = true;
  }
  const int adv = a.p.adv_tracer;
  if (adv != LT_ADV_CENTERED && adv != LT_ADV_FLUX) return LT_E_INVALID;
  if (int rc = launch_assm_dt_restore(a, s)) return rc;
  kern[adv - 1][a.diagnostics ? 1 : 0]<<<slots, TTHREADS, sm, s>>>(a, ntx, ntiles);
  LT_LAUNCHED();
  return LT_OK;
}

int launch_tracer_tma64(const Arena& a, const TracerMaps& maps, cudaStream_t s, int grid, bool tma) {
  const int ntx = (a.imt + TX - 1) / TX;
  const long ntiles = (long)ntx * ((a.jmt + TY - 1) / TY);
  const size_t sm = sizeof(ExSmem);
  static bool attr = false;
  if (!attr) {
    LT_CUDA_OK(cudaFuncSetAttribute(k_tracer_tma64<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    LT_CUDA_OK(cudaFuncSetAttribute(k_tracer_tma64<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    attr = true;
  }
  if (int rc = launch_assm_dt_restore(a, s)) return rc;
  if (a.diagnostics) {
    k_tracer_tma64<true><<<grid, TTHREADS, sm, s>>>(a, maps, ntx, ntiles, tma ? 1 : 0);
    LT_LAUNCHED();
    // the levels below each tile's march
    k_diag_deep<<<dim3((unsigned)ntiles, 2), TTHREADS, 0, s>>>(a, ntx);
  } else {
    k_tracer_tma64<false><<<grid, TTHREADS, sm, s>>>(a, maps, ntx, ntiles, tma ? 1 : 0);
  }
  LT_LAUNCHED();
  return LT_OK;
}

int launch_halo_state(const Arena& a, cudaStream_t s) {
  if (!a.diagnostics) {
    k_halo_state_parts<<<dim3(kHaloParts, a.km, 2), 256, a.imt * sizeof(double), s>>>(a);
    LT_LAUNCHED();
    return LT_OK;
  }
  // with diagnostics, salinity's dt_diff reads temperature's new ghost values
  for (int n = 0; n < 2; ++n) {
    if (a.diagnostics) k_halo_state<true><<<a.km, 256, a.imt * sizeof(double), s>>>(a, n);
    else k_halo_state<false><<<a.km, 256, a.imt * sizeof(double), s>>>(a, n);
    LT_LAUNCHED();
  }
  return LT_OK;
}

// The small kernels of a batch step over every member at once (member
// descriptors in device memory; the largest member's sizes set the grids).
int launch_small_batch_pre(const MemberDesc* mem, int nmem, int max_imt, int max_jmt, long max_cols,
                           cudaStream_t s) {
  {
    dim3 b(32, 8), g((max_imt + 31) / 32, (max_jmt + 7) / 8, nmem);
    k_surface_batch<<<g, b, 0, s>>>(mem);
    LT_LAUNCHED();
  }
  long nb = (max_cols + 2 * RB - 1) / (2 * RB);
  if (nb < 1) nb = 1;
  for (int pass = 0;; ++pass) {
    k_sss_tree_batch<<<dim3((unsigned)nb, nmem), RB, 0, s>>>(mem, pass);
    LT_LAUNCHED();
    if (nb <= 1) break;
    nb = (nb + 2 * RB - 1) / (2 * RB);
  }
  k_finish_sss_batch<<<(nmem + 127) / 128, 128, 0, s>>>(mem, nmem);
  LT_LAUNCHED();
  k_halo_net_batch<<<dim3(2, nmem), 256, max_imt * sizeof(double), s>>>(mem);
  LT_LAUNCHED();
  return LT_OK;
}

int launch_halo_state_batch(const MemberDesc* mem, int nmem, int max_imt, int km_max, cudaStream_t s) {
  for (int n = 0; n < 2; ++n) {
    k_halo_state_batch<<<dim3(km_max, nmem), 256, max_imt * sizeof(double), s>>>(mem, n);
    LT_LAUNCHED();
  }
  return LT_OK;
}

int launch_vtl_clobber(const Arena& a, cudaStream_t s) {
  const long nb = (a.F + 255) / 256;
  k_vtl_clobber<<<(unsigned)nb, 256, 0, s>>>(a);
  LT_LAUNCHED();
  return LT_OK;
}

}  // namespace lt
