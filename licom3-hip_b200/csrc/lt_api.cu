// lt_api.cu - C ABI of the tracer step: per-domain device arena (replacing the
// reference's global d_* state, cuda_data.h / cuda_init.cpp:372-707), field
// transfer, the step sequence and the reference-named shims.
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <atomic>
#include <mutex>
#include <new>
#include <vector>
#include "lt_common.cuh"
#include "lt_tracer_tma.cuh"
#include <cudaTypedefs.h>

#include "lt_domain.h"

namespace lt {

static thread_local char g_err[512] = "";

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

static std::atomic<long long> g_launches{0};
long long launch_counter() { return g_launches.load(); }
void count_launches(int n) { g_launches += n; }

int cuda_fail(cudaError_t e, const char* what) {
  set_error("CUDA error %d (%s) in %s", (int)e, cudaGetErrorString(e), what);
  return e == cudaErrorMemoryAllocation ? LT_E_OOM : LT_E_CUDA;
}

namespace {

lt_domain* g_shim = nullptr;

// f32 device storage of a field in a mixed-precision domain, else null
float* field_ptr32(lt_domain* d, int f) {
  Arena& a = d->a;
  switch (f) {
    case LT_F_UTF: return a.utf32;
    case LT_F_VTF: return a.vtf32;
    case LT_F_UTL: return a.utl32;
    case LT_F_VTL: return a.vtl32;
    case LT_F_AKT: return a.akt32;
    case LT_F_WS: return a.ws32;
    case LT_F_UTF_OUT: return a.utf_out32;
    case LT_F_VTF_OUT: return a.vtf_out32;
  }
  return nullptr;
}

// device pointer of a field in the arena (current state buffer for AT/ATB)
void* field_ptr(lt_domain* d, int f, int which_state) {
  Arena& a = d->a;
  if (float* p = field_ptr32(d, f)) return p;
  switch (f) {
    case LT_F_AT: return a.at[which_state];
    case LT_F_ATB: return a.atb[which_state];
    case LT_F_UTF: return a.utf;
    case LT_F_VTF: return a.vtf;
    case LT_F_UTL: return a.utl;
    case LT_F_VTL: return a.vtl;
    case LT_F_H0F: return a.h0f;
    case LT_F_H0L: return a.h0l;
    case LT_F_AKT: return a.akt;
    case LT_F_WS: return a.ws;
    case LT_F_NET: return a.net;
    case LT_F_UTF_OUT: return a.utf_out;
    case LT_F_VTF_OUT: return a.vtf_out;
    case LT_F_H0F_OUT: return a.h0f_out;
    case LT_F_SWV: return a.swv;
    case LT_F_NSWV: return a.nswv;
    case LT_F_SST: return a.sst;
    case LT_F_SSS: return a.sss;
    case LT_F_FRESH: return a.fresh;
    case LT_F_SEAICE: return a.seaice;
    case LT_F_TAREA: return a.tarea;
    case LT_F_TAREA_R: return a.tarea_r;
    case LT_F_HTW: return a.htw;
    case LT_F_HTS: return a.hts;
    case LT_F_HUN: return a.hun;
    case LT_F_HUE: return a.hue;
    case LT_F_DXU: return a.dxu;
    case LT_F_DYU: return a.dyu;
    case LT_F_AHF: return a.ahf;
    case LT_F_DTN: return a.dtn;
    case LT_F_DTS: return a.dts;
    case LT_F_DTE: return a.dte;
    case LT_F_DTW: return a.dtw;
    case LT_F_OHBT: return a.ohbt;
    case LT_F_OHBU: return a.ohbu;
    case LT_F_AU0: return a.au0;
    case LT_F_AUS: return a.aus;
    case LT_F_AUW: return a.auw;
    case LT_F_AUSW: return a.ausw;
    case LT_F_KMT: return a.kmt;
    case LT_F_KMU: return a.kmu;
    case LT_F_KMTN: return a.kmtn;
    case LT_F_KMTS: return a.kmts;
    case LT_F_KMTE: return a.kmte;
    case LT_F_KMTW: return a.kmtw;
    case LT_F_DZP: return a.dzp;
    case LT_F_ODZP: return a.odzp;
    case LT_F_ODZT: return a.odzt;
    case LT_F_PEN: return a.pen;
    case LT_F_TO: return a.to;
    case LT_F_SO: return a.so;
    case LT_F_C: return a.cc;
    case LT_F_RESTORE: return a.restore;
    case LT_F_RESTORE_AT: return a.restore_at;
    case LT_F_DT_RESTORE: return a.dt_restore;
    case LT_F_AX: return a.ax;
    case LT_F_AY: return a.ay;
    case LT_F_AZ: return a.az;
    case LT_F_DZ: return a.dzd;
    case LT_F_TEND: return a.tend;
    case LT_F_DT_DIFF: return a.dt_diff;
    case LT_F_DT_CONV: return a.dt_conv;
    case LT_F_PENETRATE: return a.penetrate;
    case LT_F_QICE: return a.qice;
    case LT_F_RIT: return a.rit;
    case LT_F_RICDTTMS: return a.ricdttms;
    case LT_F_S2T: return a.s2t;
    case LT_F_RICT: return a.rict;
    case LT_F_PDENSITY: return a.pdensity;
    case LT_F_FZ_TIDE: return a.fz_tide;
    case LT_F_BUOYTUR: return a.buoytur;
    case LT_F_BUOYSOL: return a.buoysol;
    case LT_F_FCORT: return a.fcort;
    case LT_F_WAVE_DIS: return a.wave_dis;
    case LT_F_ZKP: return a.zkp;
    case LT_F_AKMT: return a.akmt;
    case LT_F_AK_TIDE: return a.ak_tide;
    case LT_F_AMLD: return a.amld;
    case LT_F_RICHARDSON: return a.richardson;
    case LT_F_FZTIDAL: return a.fztidal;
    case LT_F_WP3_TIDAL: return a.wp3_tidal;
    case LT_F_UP: return a.up;
    case LT_F_VP: return a.vp;
    case LT_F_DLU: return a.dlu;
    case LT_F_DLV: return a.dlv;
    case LT_F_WKA_DRAG: return a.wka_drag;
    case LT_F_DUC: return a.duc;
    case LT_F_DUM: return a.dum;
    case LT_F_DUN: return a.dun;
    case LT_F_DUS: return a.dus;
    case LT_F_DUE: return a.due;
    case LT_F_DUW: return a.duw;
    case LT_F_DMC: return a.dmc;
    case LT_F_DMN: return a.dmn;
    case LT_F_DMS: return a.dms;
    case LT_F_DME: return a.dme;
    case LT_F_DMW: return a.dmw;
    case LT_F_AMF: return a.amf;
    case LT_F_UAREA_R: return a.uarea_r;
    case LT_F_DXUR: return a.dxur;
    case LT_F_DYUR: return a.dyur;
  }
  return nullptr;
}

bool grid_ok(const lt_grid* g) {
  if (!g) return false;
  if (g->nx < 8 || g->ny < 8 || g->km < 3 || g->km > 256) return false;
  if (g->tripole && (g->nx % 2)) return false;
  if (g->precision != LT_PREC_FP64 && g->precision != LT_PREC_MIXED) return false;
  // the mixed kernel's per-level constants live in shared memory: at most 128 levels
  if (g->precision == LT_PREC_MIXED && g->km > kMixedMaxLevels) return false;
  return true;
}

struct Plan {
  size_t off = 0;
  std::vector<std::pair<void**, size_t>> items;
  void add(void** p, size_t bytes) { items.push_back({p, bytes}); off += (bytes + 255) / 256 * 256; }
};

void plan_arena(Arena& a, Plan& pl) {
  const size_t A = a.A, F = a.F, FB = a.FB, km = a.km;
  auto D = [&](double** p, size_t n) { pl.add(reinterpret_cast<void**>(p), n * sizeof(double)); };
  auto I = [&](int** p, size_t n) { pl.add(reinterpret_cast<void**>(p), n * sizeof(int)); };
  auto S = [&](float** p, size_t n) { pl.add(reinterpret_cast<void**>(p), n * sizeof(float)); };
  D(&a.at[0], 2 * F); D(&a.at[1], 2 * F); D(&a.atb[0], 2 * FB); D(&a.atb[1], 2 * FB);
  if (a.precision == LT_PREC_MIXED) {
    S(&a.utf32, F); S(&a.vtf32, F); S(&a.utl32, F); S(&a.vtl32, F); S(&a.akt32, 2 * F);
    S(&a.utf_out32, F); S(&a.vtf_out32, F); S(&a.ws32, FB); S(&a.wkd32, F); S(&a.wkb32, F);
  } else {
    D(&a.utf, F); D(&a.vtf, F); D(&a.utl, F); D(&a.vtl, F); D(&a.akt, 2 * F);
    D(&a.utf_out, F); D(&a.vtf_out, F); D(&a.ws, FB); D(&a.uwf, F); D(&a.vsf, F); D(&a.wka, F);
  }
  D(&a.h0f, A); D(&a.h0l, A); D(&a.h0f_out, A); D(&a.net, 2 * A);
  double** two_d[] = {&a.swv, &a.nswv, &a.sst, &a.sss, &a.fresh, &a.seaice, &a.tarea, &a.tarea_r, &a.htw,
                      &a.hts, &a.hun, &a.hue, &a.dxu, &a.dyu, &a.ahf, &a.dtn, &a.dts, &a.dte, &a.dtw,
                      &a.ohbt, &a.ohbu, &a.au0, &a.aus, &a.auw, &a.ausw, &a.stf_ssh};
  for (auto p : two_d) D(p, A);
  D(&a.stf_n, 2 * A);
  D(&a.qice, A);
  int** masks[] = {&a.kmt, &a.kmu, &a.kmtn, &a.kmts, &a.kmte, &a.kmtw};
  for (auto p : masks) I(p, A);
  D(&a.dzp, km); D(&a.odzp, km); D(&a.odzt, km); D(&a.pen, km); D(&a.to, km); D(&a.so, km); D(&a.cc, 9 * km);
  D(&a.red_part, tree_sum_part_elems((long)a.A * a.km) + 16);
  D(&a.scalars, 16);
  I(&a.status, 16);
  if (a.p.boundary_restore == 1) D(&a.restore, 2 * F);
  if (a.p.simple_assm) { D(&a.restore_at, 2 * F); D(&a.dt_restore, 2 * F); }
  if (a.diagnostics) {
    D(&a.ax, 2 * F); D(&a.ay, 2 * F); D(&a.az, 2 * F); D(&a.dzd, 2 * F);
    D(&a.tend, 2 * F); D(&a.dt_diff, 2 * F); D(&a.dt_conv, 2 * F); D(&a.penetrate, F);
    D(&a.fold_save, 2 * km * (size_t)a.imt);
    I(&a.kfz, A);
  } else {
    D(&a.dt_conv, 2 * F);  // convadj writes it
    D(&a.tend, 2 * F);     // convadj accumulates into it
  }
  // the Thomas sweep's per-level coefficients of each resident CTA
  const size_t cta_threads = a.precision == LT_PREC_MIXED ? kMixedThreads : TTHREADS;
  D(&a.col_scratch, (size_t)a.col_scratch_slots * km * a.nv_scratch * cta_threads);
}

void init_arena_dims(Arena& a, const lt_grid* g, const lt_params* p) {
  std::memset(&a, 0, sizeof(a));
  a.nx = g->nx; a.ny = g->ny; a.km = g->km;
  a.imt = g->nx + 4; a.jmt = g->ny + 4;
  a.A = (long)a.imt * a.jmt; a.F = a.A * a.km; a.FB = a.A * (a.km + 1);
  a.ew_cyclic = g->ew_cyclic; a.tripole = g->tripole;
  a.diagnostics = g->diagnostics; a.precision = g->precision;
  if (p) a.p = *p;
  a.nv_scratch = a.precision == LT_PREC_MIXED ? kMixedScratchPerLevel : (a.diagnostics ? 3 : 2);
  a.wait_limit = 1u << 24;
}

long slots_for(const Arena& a, int sms) {
  const int ty = a.precision == LT_PREC_MIXED ? kMixedTileY : TY;
  const long ntiles = (long)((a.imt + TX - 1) / TX) * ((a.jmt + ty - 1) / ty);
  long s = (long)sms * (a.precision == LT_PREC_MIXED ? kMixedCtasPerSm : kFp64CtasPerSm);
  // work items: (tile, tracer) pairs in FP64, tiles (both tracers) in mixed
  const long items = a.precision == LT_PREC_MIXED ? ntiles : 2 * ntiles;
  if (s > items) s = items;
  return s;
}

}  // namespace

bool make_tensor_map_3d(CUtensorMap* map, const void* base, int esize, long nx, long ny, long nz, int bx, int by) {
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  if (!encode) {
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", reinterpret_cast<void**>(&encode), cudaEnableDefault,
                                &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !encode)
      return false;
  }
  if ((nx * esize) % 16 != 0 || (reinterpret_cast<uintptr_t>(base) % 16) != 0 || (bx * esize) % 16 != 0) return false;
  const cuuint64_t dims[3] = {(cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)nz};
  const cuuint64_t strides[2] = {(cuuint64_t)(nx * esize), (cuuint64_t)(nx * ny * esize)};
  const cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  const CUresult r = encode(map, esize == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3,
                            const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

bool build_tracer_maps(const Arena& a, TracerMaps* m) {
  const long imt = a.imt, jmt = a.jmt, km = a.km;
  const bool mx = a.precision == LT_PREC_MIXED;
  const int ty = mx ? kMixedTileY : TY;   // tile rows of the column kernel
  bool ok = true;
  const int bw64 = mx ? kMixedBoxW64 : SW;   // state box width
  for (int b = 0; b < 2; ++b) {
    ok = ok && make_tensor_map_3d(&m->at[b], a.at[b], 8, imt, jmt, 2 * km, bw64, ty + 4);
    ok = ok && make_tensor_map_3d(&m->atb[b], a.atb[b], 8, imt, jmt, 2 * (km + 1), bw64, ty + 4);
  }
  const int es = mx ? 4 : 8;
  ok = ok && make_tensor_map_3d(&m->ws, mx ? (const void*)a.ws32 : a.ws, es, imt, jmt, km + 1, SW, ty + 2);
  // f64: face transports u_wface (rows y0-1..) and v_sface (rows y0-2..);
  // mixed: the U-point means wkd, wkb (rows y0-2..), faces formed in the kernel
  ok = ok && make_tensor_map_3d(&m->uw, mx ? (const void*)a.wkd32 : a.uwf, es, imt, jmt, km, SW, mx ? ty + 3 : ty + 2);
  ok = ok && make_tensor_map_3d(&m->vs, mx ? (const void*)a.wkb32 : a.vsf, es, imt, jmt, km, SW, ty + 3);
  ok = ok && make_tensor_map_3d(&m->akt, mx ? (const void*)a.akt32 : a.akt, es, imt, jmt, 2 * km, TX, ty);
  if (mx) {
    const float* vel[4] = {a.utf32, a.vtf32, a.utl32, a.vtl32};
    for (int v = 0; v < 4; ++v)
      ok = ok && make_tensor_map_3d(&m->vel[v], vel[v], 4, imt, jmt, km, kMixedContBoxW, kMixedContTileY + 1);
  }
  return ok;
}

int run_step(lt_domain* d, cudaEvent_t forcing_ready) {
  Arena& a = d->a;
  cudaStream_t s = d->stream;
  int rc;
  cudaEvent_t* ev = nullptr;
  if (d->profile && d->prof_steps < LT_PROF_STEPS) {
    ev = &d->prof_ev[(size_t)d->prof_steps * (LT_NPHASE + 1)];
    d->prof_steps++;
  }
  // events bound the phases in launch order (LT_PHASE_ORDER)
  auto mark = [&](int ph) { if (ev) cudaEventRecord(ev[ph], s); };
  mark(0);
  // continuity first: it reads the SSH mean and the velocities, not the
  // surface forcing
  if ((rc = launch_ssh(a, s))) return rc;
  if (a.precision == LT_PREC_MIXED) rc = launch_continuity_mixed(a, d->maps, d->use_tma, s);
  else rc = launch_continuity_fp64(a, s);
  if (rc) return rc;
  mark(1);
  if (forcing_ready) LT_CUDA_OK(cudaStreamWaitEvent(s, forcing_ready, 0));
  if ((rc = launch_surface_fluxes(a, s))) return rc;
  mark(2);
  if ((rc = launch_interior_sum_sss(a, s))) return rc;
  mark(3);
  if ((rc = launch_halo_r8(a.net, 2, a.imt, a.jmt, a.ew_cyclic, a.tripole, s))) return rc;
  mark(4);
  if (a.precision == LT_PREC_MIXED) {
    if ((rc = launch_tracer_tma_mixed(a, d->maps, d->use_tma, s, d->tma_grid))) return rc;
  } else if (a.p.adv_tracer == LT_ADV_TSPAS) {
    // the TMA-slot column kernel is the tspas scheme's (its level boxes by
    // per-thread copies where the row pitch does not allow TMA); the centred
    // and flux schemes run in the plain-load kernel
    if ((rc = launch_tracer_tma64(a, d->maps, s, d->tma_grid, d->use_tma))) return rc;
  } else {
    if ((rc = launch_tracer_fp64(a, s, d->slots))) return rc;
  }
  mark(5);
  if ((rc = launch_halo_state(a, s))) return rc;
  mark(6);
  a.cur ^= 1;
  d->steps_done++;
  return LT_OK;
}

// After the stream has drained: a column kernel whose bounded wait for its
// TMA boxes ran out set status[1] and returned early; report it once.
int timeout_status(lt_domain* d) {
  int h = 0;
  LT_CUDA_OK(cudaMemcpy(&h, d->a.status + 1, sizeof(int), cudaMemcpyDeviceToHost));
  if (!h) return LT_OK;
  LT_CUDA_OK(cudaMemset(d->a.status + 1, 0, sizeof(int)));
  set_error("a tracer column kernel gave up waiting for its level data; the state of that step is not valid");
  return LT_E_TIMEOUT;
}

}  // namespace lt

namespace lt {
// The turbulence closure's fields: one zeroed allocation, taken the first time
// the domain uses any of them (a domain that only steps tracers never pays
// for them).
int ensure_turb(lt_domain* d) {
  Arena& a = d->a;
  if (a.rit) return LT_OK;
  double** f3m1[] = {&a.rit, &a.ricdttms, &a.s2t, &a.rict};
  double** f3[] = {&a.fz_tide, &a.akmt, &a.ak_tide, &a.richardson, &a.fztidal, &a.wp3_tidal};
  double** f2[] = {&a.buoytur, &a.buoysol, &a.fcort, &a.wave_dis, &a.amld};
  Plan pl;
  for (auto p : f3m1) pl.add(reinterpret_cast<void**>(p), sizeof(double) * a.A * (a.km - 1));
  for (auto p : f3) pl.add(reinterpret_cast<void**>(p), sizeof(double) * a.F);
  for (auto p : f2) pl.add(reinterpret_cast<void**>(p), sizeof(double) * a.A);
  pl.add(reinterpret_cast<void**>(&a.pdensity), sizeof(double) * a.FB);
  pl.add(reinterpret_cast<void**>(&a.zkp), sizeof(double) * (a.km + 1));
  char* base = nullptr;
  cudaError_t e = cudaMalloc(&base, pl.off);
  if (e != cudaSuccess) {
    set_error("turbulence fields: cudaMalloc(%zu) failed: %s", pl.off, cudaGetErrorString(e));
    return LT_E_OOM;
  }
  d->allocations.push_back(base);
  size_t off = 0;
  for (auto& it : pl.items) {
    *it.first = base + off;
    off += (it.second + 255) / 256 * 256;
  }
  LT_CUDA_OK(cudaMemsetAsync(base, 0, pl.off, d->stream));
  return LT_OK;
}
// The momentum friction's fields: one zeroed allocation on first use.
int ensure_mom(lt_domain* d) {
  Arena& a = d->a;
  if (a.up) return LT_OK;
  double** f3[] = {&a.up, &a.vp, &a.dlu, &a.dlv, &a.wka_drag};
  double** f2[] = {&a.duc, &a.dum, &a.dun, &a.dus, &a.due, &a.duw, &a.dmc, &a.dmn,
                   &a.dms, &a.dme, &a.dmw, &a.amf, &a.uarea_r, &a.dxur, &a.dyur};
  Plan pl;
  for (auto p : f3) pl.add(reinterpret_cast<void**>(p), sizeof(double) * a.F);
  for (auto p : f2) pl.add(reinterpret_cast<void**>(p), sizeof(double) * a.A);
  char* base = nullptr;
  cudaError_t e = cudaMalloc(&base, pl.off);
  if (e != cudaSuccess) {
    set_error("momentum fields: cudaMalloc(%zu) failed: %s", pl.off, cudaGetErrorString(e));
    return LT_E_OOM;
  }
  d->allocations.push_back(base);
  size_t off = 0;
  for (auto& it : pl.items) {
    *it.first = base + off;
    off += (it.second + 255) / 256 * 256;
  }
  LT_CUDA_OK(cudaMemsetAsync(base, 0, pl.off, d->stream));
  return LT_OK;
}
}  // namespace lt

using namespace lt;

extern "C" {

const char* lt_last_error(void) { return lt::g_err; }

static const char* const k_field_names[LT_F_COUNT] = {
    "AT", "ATB", "UTF", "VTF", "UTL", "VTL", "H0F", "H0L", "AKT", "WS", "NET", "UTF_OUT", "VTF_OUT", "H0F_OUT",
    "SWV", "NSWV", "SST", "SSS", "FRESH", "SEAICE", "TAREA", "TAREA_R", "HTW", "HTS", "HUN", "HUE", "DXU", "DYU",
    "AHF", "DTN", "DTS", "DTE", "DTW", "OHBT", "OHBU", "AU0", "AUS", "AUW", "AUSW", "KMT", "KMU", "KMTN", "KMTS",
    "KMTE", "KMTW", "DZP", "ODZP", "ODZT", "PEN", "TO", "SO", "C", "RESTORE", "AX", "AY", "AZ", "DZ", "TEND",
    "DT_DIFF", "DT_CONV", "PENETRATE", "QICE", "RIT", "RICDTTMS", "S2T", "RICT", "PDENSITY", "FZ_TIDE",
    "BUOYTUR", "BUOYSOL", "FCORT", "WAVE_DIS", "ZKP", "AKMT", "AK_TIDE", "AMLD", "RICHARDSON", "FZTIDAL",
    "WP3_TIDAL", "UP", "VP", "DLU", "DLV", "WKA_DRAG", "DUC", "DUM", "DUN", "DUS", "DUE", "DUW", "DMC", "DMN",
    "DMS", "DME", "DMW", "AMF", "UAREA_R", "DXUR", "DYUR", "RESTORE_AT", "DT_RESTORE"};

const char* lt_field_name(int f) { return (f >= 0 && f < LT_F_COUNT) ? k_field_names[f] : nullptr; }
long lt_field_count(int f, int nx, int ny, int km) {
  if (f < 0 || f >= LT_F_COUNT || nx < 1 || ny < 1 || km < 1) return -1;
  return lt::field_count(f, nx + 4, ny + 4, km);
}
int lt_field_is_int(int f) { return (f >= 0 && f < LT_F_COUNT) ? (int)lt::field_is_int(f) : 0; }
int lt_field_on_demand(int f) {
  return (f >= 0 && f < LT_F_COUNT) ? (int)(lt::field_is_turb(f) || lt::field_is_mom(f)) : 0;
}

const char* lt_version(void) { return "licom3-hip_b200 tracer 0.1 (sm_100a)"; }

int lt_set_device(int dev) {
  cudaError_t e = cudaSetDevice(dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
  return LT_OK;
}

long long lt_launch_count(void) { return lt::launch_counter(); }

int lt_profile(lt_domain* d, int on) {
  if (!d) return LT_E_INVALID;
  if (on && d->prof_ev.empty()) {
    d->prof_ev.resize((size_t)LT_PROF_STEPS * (LT_NPHASE + 1));
    for (auto& e : d->prof_ev) LT_CUDA_OK(cudaEventCreate(&e));
  }
  d->profile = on;
  d->prof_steps = 0;
  return LT_OK;
}

int lt_phase_ms(lt_domain* d, float* ms, int nphase) {
  if (!d || !ms || nphase < LT_NPHASE) return LT_E_INVALID;
  for (int p = 0; p < LT_NPHASE; ++p) ms[p] = 0.0f;
  if (d->prof_steps == 0) return LT_OK;
  LT_CUDA_OK(cudaStreamSynchronize(d->stream));
  for (int st = 0; st < d->prof_steps; ++st) {
    cudaEvent_t* ev = &d->prof_ev[(size_t)st * (LT_NPHASE + 1)];
    for (int p = 0; p < LT_NPHASE; ++p) {
      float t = 0.0f;
      LT_CUDA_OK(cudaEventElapsedTime(&t, ev[p], ev[p + 1]));
      ms[LT_PHASE_ORDER[p]] += t;
    }
  }
  return d->prof_steps;
}

int lt_device_count(int* count) {
  if (!count) return LT_E_INVALID;
  cudaError_t e = cudaGetDeviceCount(count);
  if (e != cudaSuccess) { *count = 0; return LT_E_NODEVICE; }
  return LT_OK;
}

size_t lt_domain_bytes(const lt_grid* g) {
  if (!grid_ok(g)) return 0;
  Arena a;
  lt_params p{};
  init_arena_dims(a, g, &p);
  a.col_scratch_slots = slots_for(a, 148);
  Plan pl;
  plan_arena(a, pl);
  return pl.off;
}

// the advection scheme: one of lt_adv_scheme, and tspas in mixed precision
static bool scheme_ok(int precision, const lt_params* p, const char* where) {
  if (p->adv_tracer < LT_ADV_TSPAS || p->adv_tracer > LT_ADV_FLUX) {
    set_error("%s: adv_tracer %d is not an lt_adv_scheme", where, p->adv_tracer);
    return false;
  }
  if (precision == LT_PREC_MIXED && p->adv_tracer != LT_ADV_TSPAS) {
    set_error("%s: the centred and flux advection schemes run in the FP64 form only", where);
    return false;
  }
  if (p->simple_assm != 0 && p->simple_assm != 1) {
    set_error("%s: simple_assm %d is not 0 or 1", where, p->simple_assm);
    return false;
  }
  if (p->simple_assm && precision == LT_PREC_MIXED) {
    set_error("%s: tracer_7's nudging (simple_assm) runs in the FP64 form only", where);
    return false;
  }
  if (p->simple_assm && p->ktv < 0) {
    set_error("%s: ktv %d is negative", where, p->ktv);
    return false;
  }
  return true;
}

int lt_create(const lt_grid* g, const lt_params* p, lt_domain** out) {
  if (!out || !grid_ok(g) || !p) { set_error("lt_create: invalid grid or params"); return LT_E_INVALID; }
  if (g->precision == LT_PREC_MIXED && g->diagnostics) {
    set_error("lt_create: the diagnostics (AX .. PENETRATE, TEND, DT_DIFF) are written by the FP64 form only");
    return LT_E_INVALID;
  }
  if (!scheme_ok(g->precision, p, "lt_create")) return LT_E_INVALID;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    set_error("lt_create: no CUDA device");
    return LT_E_NODEVICE;
  }
  lt_domain* d = new (std::nothrow) lt_domain;
  if (!d) return LT_E_OOM;
  init_arena_dims(d->a, g, p);
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  d->a.col_scratch_slots = slots_for(d->a, sms);
  d->slots = (int)d->a.col_scratch_slots;
  Plan pl;
  plan_arena(d->a, pl);
  size_t free_b = 0, total_b = 0;
  cudaMemGetInfo(&free_b, &total_b);
  if (pl.off + (64u << 20) > free_b) {
    set_error("lt_create: domain needs %zu bytes, %zu free", pl.off, free_b);
    delete d;
    return LT_E_OOM;
  }
  char* base = nullptr;
  cudaError_t e = cudaMalloc(&base, pl.off);
  if (e != cudaSuccess) {
    set_error("lt_create: cudaMalloc(%zu) failed: %s", pl.off, cudaGetErrorString(e));
    delete d;
    return LT_E_OOM;
  }
  d->allocations.push_back(base);
  size_t off = 0;
  for (auto& it : pl.items) {
    *it.first = base + off;
    off += (it.second + 255) / 256 * 256;
  }
  if (cudaStreamCreateWithFlags(&d->stream, cudaStreamNonBlocking) != cudaSuccess) {
    cudaFree(base);
    delete d;
    return LT_E_CUDA;
  }
  d->owns_stream = true;
  // cleared on the domain's own stream, so every later use on that stream is
  // ordered after it without stalling other streams of the device
  cudaMemsetAsync(base, 0, pl.off, d->stream);
  cudaEventCreate(&d->ev0);
  cudaEventCreate(&d->ev1);
  cudaEventCreateWithFlags(&d->ev_free, cudaEventDisableTiming);
  cudaEventCreateWithFlags(&d->ev_forcing, cudaEventDisableTiming);
  cudaStreamCreateWithFlags(&d->copy_stream, cudaStreamNonBlocking);
  // TMA-fed tracer kernel where the row pitch is a multiple of 16 bytes
  d->use_tma = build_tracer_maps(d->a, &d->maps);
  // one persistent CTA per resident slot (kFp64CtasPerSm, kMixedCtasPerSm
  // per SM: the kernels' __launch_bounds__ and shared-memory footprints)
  const long per_sm = d->a.precision == LT_PREC_MIXED ? kMixedCtasPerSm : kFp64CtasPerSm;
  d->tma_grid = (int)std::min<long>(d->a.col_scratch_slots, (long)sms * per_sm);
  if (cudaStreamSynchronize(d->stream) != cudaSuccess) {
    lt_destroy(d);
    return LT_E_CUDA;
  }
  *out = d;
  return LT_OK;
}

int lt_destroy(lt_domain* d) {
  if (!d) return LT_E_INVALID;
  if (g_shim == d) g_shim = nullptr;
  cudaStreamSynchronize(d->stream);
  for (void* p : d->allocations) cudaFree(p);
  if (d->copy_stream) cudaStreamSynchronize(d->copy_stream);
  if (d->ev0) cudaEventDestroy(d->ev0);
  if (d->ev1) cudaEventDestroy(d->ev1);
  if (d->ev_free) cudaEventDestroy(d->ev_free);
  if (d->ev_forcing) cudaEventDestroy(d->ev_forcing);
  for (int k = 0; k < 2; ++k) {
    if (d->ev_set_used[k]) cudaEventDestroy(d->ev_set_used[k]);
    if (d->ev_set_ready[k]) cudaEventDestroy(d->ev_set_ready[k]);
  }
  if (d->copy_stream) cudaStreamDestroy(d->copy_stream);
  for (auto e : d->prof_ev) cudaEventDestroy(e);
  if (d->owns_stream) cudaStreamDestroy(d->stream);
  delete d;
  return LT_OK;
}

int lt_set_params(lt_domain* d, const lt_params* p) {
  if (!d || !p) return LT_E_INVALID;
  if (!scheme_ok(d->a.precision, p, "lt_set_params")) return LT_E_INVALID;
  if (p->boundary_restore == 1 && !d->a.restore) {
    set_error("lt_set_params: boundary_restore needs a domain created with it");
    return LT_E_STATE;
  }
  if (p->simple_assm && !d->a.restore_at) {
    set_error("lt_set_params: simple_assm needs a domain created with it");
    return LT_E_STATE;
  }
  d->a.p = *p;
  return LT_OK;
}


static int xfer(lt_domain* d, int f, void* ptr, size_t nbytes, cudaMemcpyKind kind, bool set) {
  if (!d || !ptr || f < 0 || f >= LT_F_COUNT) { set_error("bad field transfer"); return LT_E_INVALID; }
  if (lt::field_is_turb(f) || lt::field_is_mom(f)) {
    const int rc = lt::field_is_turb(f) ? lt::ensure_turb(d) : lt::ensure_mom(d);
    if (rc) return rc;
  }
  const size_t need = lt::field_bytes(f, d->a.imt, d->a.jmt, d->a.km);
  if (nbytes != need) {
    set_error("field %d: %zu bytes given, %zu expected", f, nbytes, need);
    return LT_E_INVALID;
  }
  void* dev = field_ptr(d, f, d->a.cur);
  if (!dev) { set_error("field %d not held by this domain (diagnostics/restore off)", f); return LT_E_STATE; }
  if (float* d32 = field_ptr32(d, f)) {
    // f32 storage (mixed precision): the boundary stays f64, converted on the device
    const long n = (long)(nbytes / sizeof(double));
    double* tmp = nullptr;
    LT_CUDA_OK(cudaMallocAsync(reinterpret_cast<void**>(&tmp), nbytes, d->stream));
    int rc = LT_OK;
    if (set) {
      if (cudaMemcpyAsync(tmp, ptr, nbytes, kind, d->stream) != cudaSuccess) rc = LT_E_CUDA;
      if (!rc) rc = launch_f64_to_f32(tmp, d32, n, d->stream);
    } else {
      rc = launch_f32_to_f64(d32, tmp, n, d->stream);
      if (!rc && cudaMemcpyAsync(ptr, tmp, nbytes, kind, d->stream) != cudaSuccess) rc = LT_E_CUDA;
    }
    cudaFreeAsync(tmp, d->stream);
    LT_CUDA_OK(cudaStreamSynchronize(d->stream));
    return rc;
  }
  if (set) {
    LT_CUDA_OK(cudaMemcpyAsync(dev, ptr, nbytes, kind, d->stream));
    if (f == LT_F_AT || f == LT_F_ATB) {  // both state buffers start equal
      LT_CUDA_OK(cudaMemcpyAsync(field_ptr(d, f, d->a.cur ^ 1), ptr, nbytes, kind, d->stream));
    }
  } else {
    LT_CUDA_OK(cudaMemcpyAsync(ptr, dev, nbytes, kind, d->stream));
  }
  LT_CUDA_OK(cudaStreamSynchronize(d->stream));
  return LT_OK;
}

int lt_set_field(lt_domain* d, int f, const void* src, size_t nbytes) {
  return xfer(d, f, const_cast<void*>(src), nbytes, cudaMemcpyHostToDevice, true);
}
int lt_get_field(lt_domain* d, int f, void* dst, size_t nbytes) {
  return xfer(d, f, dst, nbytes, cudaMemcpyDeviceToHost, false);
}
int lt_set_field_device(lt_domain* d, int f, const void* src, size_t nbytes) {
  return xfer(d, f, const_cast<void*>(src), nbytes, cudaMemcpyDeviceToDevice, true);
}
int lt_get_field_device(lt_domain* d, int f, void* dst, size_t nbytes) {
  return xfer(d, f, dst, nbytes, cudaMemcpyDeviceToDevice, false);
}

int lt_derive_masks(lt_domain* d) {
  if (!d) return LT_E_INVALID;
  int rc = launch_derive_masks(d->a, d->stream);
  if (rc) return rc;
  LT_CUDA_OK(cudaStreamSynchronize(d->stream));
  return LT_OK;
}

int lt_step(lt_domain* d, int nsteps) {
  if (!d || nsteps < 0) return LT_E_INVALID;
  LT_CUDA_OK(cudaEventRecord(d->ev0, d->stream));
  for (int s = 0; s < nsteps; ++s) {
    int rc = run_step(d);
    if (rc) return rc;
  }
  LT_CUDA_OK(cudaEventRecord(d->ev1, d->stream));
  return LT_OK;
}

int lt_step_host(lt_domain* d, const double* const forcing6[6], double* fw_norm2_out, double* content2_out) {
  if (!d) return LT_E_INVALID;
  Arena& a = d->a;
  double* dst[6] = {a.swv, a.nswv, a.sst, a.sss, a.fresh, a.seaice};
  const size_t bytes = sizeof(double) * a.A;
  // The forcing goes up on the copy stream once the domain's earlier work
  // (which may read the previous forcing) is done, while the step's
  // continuity runs; the surface fluxes wait for it.
  // (without a copy stream or its events the copies go on the domain's
  // stream, in order before the step)
  cudaEvent_t ready = nullptr;
  const bool overlap = d->copy_stream && d->ev_free && d->ev_forcing;
  if (forcing6) {
    cudaStream_t cs = overlap ? d->copy_stream : d->stream;
    if (overlap) {
      LT_CUDA_OK(cudaEventRecord(d->ev_free, d->stream));
      LT_CUDA_OK(cudaStreamWaitEvent(cs, d->ev_free, 0));
    }
    for (int m = 0; m < 6; ++m)
      if (forcing6[m]) LT_CUDA_OK(cudaMemcpyAsync(dst[m], forcing6[m], bytes, cudaMemcpyHostToDevice, cs));
    if (overlap) {
      LT_CUDA_OK(cudaEventRecord(d->ev_forcing, cs));
      ready = d->ev_forcing;
    }
  }
  int rc = run_step(d, ready);
  if (rc) return rc;
  if (content2_out) {
    if ((rc = launch_tracer_content(a, d->stream))) return rc;
    LT_CUDA_OK(cudaMemcpyAsync(content2_out, a.scalars + 1, 2 * sizeof(double), cudaMemcpyDeviceToHost, d->stream));
  }
  if (fw_norm2_out) LT_CUDA_OK(cudaMemcpyAsync(fw_norm2_out, a.scalars, sizeof(double), cudaMemcpyDeviceToHost, d->stream));
  LT_CUDA_OK(cudaStreamSynchronize(d->stream));
  return timeout_status(d);
}

int lt_step_host_async(lt_domain* d, const double* const forcing6[6], double* fw_norm2_out, double* content2_out) {
  if (!d) return LT_E_INVALID;
  Arena& a = d->a;
  double** field[6] = {&a.swv, &a.nswv, &a.sst, &a.sss, &a.fresh, &a.seaice};
  const size_t bytes = sizeof(double) * a.A;
  if (!d->forcing_set[1][0]) {
    // first asynchronous step: the second set and the events
    char* p = nullptr;
    cudaError_t e = cudaMalloc(&p, 6 * bytes);
    if (e != cudaSuccess) {
      set_error("lt_step_host_async: cudaMalloc(%zu) for the second forcing set failed", 6 * bytes);
      return LT_E_OOM;
    }
    d->allocations.push_back(p);
    for (int m = 0; m < 6; ++m) {
      d->forcing_set[0][m] = *field[m];
      d->forcing_set[1][m] = reinterpret_cast<double*>(p) + (size_t)m * a.A;
    }
    for (int s = 0; s < 2; ++s) {
      LT_CUDA_OK(cudaEventCreateWithFlags(&d->ev_set_used[s], cudaEventDisableTiming));
      LT_CUDA_OK(cudaEventCreateWithFlags(&d->ev_set_ready[s], cudaEventDisableTiming));
      LT_CUDA_OK(cudaEventRecord(d->ev_set_used[s], d->stream));
    }
    d->forcing_cur = 0;
  }
  // This step reads the other set: its copies wait only for the last step
  // that read that set (two steps back), so they overlap the previous step.
  const int nb = d->forcing_cur ^ 1;
  cudaStream_t cs = d->copy_stream;
  LT_CUDA_OK(cudaStreamWaitEvent(cs, d->ev_set_used[nb], 0));
  bool keeps = !forcing6;
  for (int m = 0; m < 6 && !keeps; ++m) keeps = !forcing6[m];
  if (keeps) {   // the current set may have been written on the domain's stream (lt_set_field)
    LT_CUDA_OK(cudaEventRecord(d->ev_free, d->stream));
    LT_CUDA_OK(cudaStreamWaitEvent(cs, d->ev_free, 0));
  }
  for (int m = 0; m < 6; ++m) {
    if (forcing6 && forcing6[m])
      LT_CUDA_OK(cudaMemcpyAsync(d->forcing_set[nb][m], forcing6[m], bytes, cudaMemcpyHostToDevice, cs));
    else   // a field kept resident: the current set's copy, once its writers are done
      LT_CUDA_OK(cudaMemcpyAsync(d->forcing_set[nb][m], d->forcing_set[d->forcing_cur][m], bytes,
                                 cudaMemcpyDeviceToDevice, cs));
  }
  LT_CUDA_OK(cudaEventRecord(d->ev_set_ready[nb], cs));
  for (int m = 0; m < 6; ++m) *field[m] = d->forcing_set[nb][m];
  d->forcing_cur = nb;
  int rc = run_step(d, d->ev_set_ready[nb]);
  if (rc) return rc;
  LT_CUDA_OK(cudaEventRecord(d->ev_set_used[nb], d->stream));
  if (content2_out) {
    if ((rc = launch_tracer_content(a, d->stream))) return rc;
    LT_CUDA_OK(cudaMemcpyAsync(content2_out, a.scalars + 1, 2 * sizeof(double), cudaMemcpyDeviceToHost, d->stream));
  }
  if (fw_norm2_out) LT_CUDA_OK(cudaMemcpyAsync(fw_norm2_out, a.scalars, sizeof(double), cudaMemcpyDeviceToHost, d->stream));
  return LT_OK;
}

int lt_convadj(lt_domain* d) {
  if (!d) return LT_E_INVALID;
  int rc = launch_convadj(d->a, d->stream);
  if (rc) return rc;
  return LT_OK;
}

void lt_icesnow_defaults(lt_icesnow_params* p) {
  if (!p) return;
  p->tbice = -1.8;       // constant_mod.F90:168
  p->cp = 3996.0;        // constant_mod.F90:164
  p->latice = 3.337e5;   // shr_const_mod.h:51
  p->reset_qice = 1;     // def-undef.h defines FRC_CORE
}

int lt_icesnow(lt_domain* d, const lt_icesnow_params* p) {
  if (!d) return LT_E_INVALID;
  lt_icesnow_params def;
  lt_icesnow_defaults(&def);
  return launch_icesnow(d->a, p ? *p : def, d->stream);
}

int lt_tracer_content(lt_domain* d, double* out2) {
  if (!d || !out2) return LT_E_INVALID;
  int rc = launch_tracer_content(d->a, d->stream);
  if (rc) return rc;
  LT_CUDA_OK(cudaMemcpyAsync(out2, d->a.scalars + 1, 2 * sizeof(double), cudaMemcpyDeviceToHost, d->stream));
  LT_CUDA_OK(cudaStreamSynchronize(d->stream));
  return LT_OK;
}

int lt_fw_norm2(lt_domain* d, double* out) {
  if (!d || !out) return LT_E_INVALID;
  LT_CUDA_OK(cudaMemcpyAsync(out, d->a.scalars, sizeof(double), cudaMemcpyDeviceToHost, d->stream));
  LT_CUDA_OK(cudaStreamSynchronize(d->stream));
  return LT_OK;
}

int lt_sync(lt_domain* d) {
  if (!d) return LT_E_INVALID;
  LT_CUDA_OK(cudaStreamSynchronize(d->stream));
  return timeout_status(d);
}

int lt_check_numeric(lt_domain* d, long long* bad) {
  if (!d) return LT_E_INVALID;
  int rc = launch_check_numeric(d->a, d->stream);
  if (rc) return rc;
  int h = 0;
  LT_CUDA_OK(cudaMemcpyAsync(&h, d->a.status, sizeof(int), cudaMemcpyDeviceToHost, d->stream));
  LT_CUDA_OK(cudaStreamSynchronize(d->stream));
  if (bad) *bad = h;
  if (h) { set_error("%d non-finite tracer values", h); return LT_E_NUMERIC; }
  return LT_OK;
}

int lt_mark(lt_domain* d, int which) {
  if (!d || (which != 0 && which != 1)) return LT_E_INVALID;
  LT_CUDA_OK(cudaEventRecord(which ? d->ev1 : d->ev0, d->stream));
  return LT_OK;
}

int lt_last_step_ms(lt_domain* d, float* ms) {
  if (!d || !ms) return LT_E_INVALID;
  LT_CUDA_OK(cudaEventSynchronize(d->ev1));
  LT_CUDA_OK(cudaEventElapsedTime(ms, d->ev0, d->ev1));
  return LT_OK;
}

int lt_use_tma(lt_domain* d, int on) {
  if (!d) return LT_E_INVALID;
  if (on && !build_tracer_maps(d->a, &d->maps)) {
    set_error("lt_use_tma: row pitch of this domain does not allow TMA boxes");
    return LT_E_INVALID;
  }
  d->use_tma = on != 0;
  return LT_OK;
}

int lt_set_wait_limit(lt_domain* d, unsigned polls) {
  if (!d) return LT_E_INVALID;
  d->a.wait_limit = polls;
  return LT_OK;
}

int lt_shim_bind(lt_domain* d) {
  g_shim = d;
  return LT_OK;
}

// tracer.cpp:1701 - one step with the reference's visible side effects on the
// bound domain: utf/vtf/h0f scaled in place, vtl left holding S.
void tracer_(int ii) {
  (void)ii;
  set_error("%s", "");   // the shim has no status: an empty lt_last_error() means success
  lt_domain* d = g_shim;
  if (!d) { set_error("tracer_: no domain bound (lt_shim_bind)"); return; }
  Arena& a = d->a;
  if (run_step(d)) return;
  if (a.precision == LT_PREC_MIXED) {
    const size_t fb = sizeof(float) * a.F;
    cudaMemcpyAsync(a.utf32, a.utf_out32, fb, cudaMemcpyDeviceToDevice, d->stream);
    cudaMemcpyAsync(a.vtf32, a.vtf_out32, fb, cudaMemcpyDeviceToDevice, d->stream);
    launch_f64_to_f32(a.at[a.cur] + a.F, a.vtl32, a.F, d->stream);
  } else {
    const size_t fb = sizeof(double) * a.F;
    cudaMemcpyAsync(a.utf, a.utf_out, fb, cudaMemcpyDeviceToDevice, d->stream);
    cudaMemcpyAsync(a.vtf, a.vtf_out, fb, cudaMemcpyDeviceToDevice, d->stream);
    launch_vtl_clobber(a, d->stream);
  }
  cudaMemcpyAsync(a.h0f, a.h0f_out, sizeof(double) * a.A, cudaMemcpyDeviceToDevice, d->stream);
  cudaError_t e = cudaStreamSynchronize(d->stream);
  if (e != cudaSuccess) cuda_fail(e, "tracer_");
  else timeout_status(d);
}

// convadj.cpp:290
void convadj_(void) {
  set_error("%s", "");
  lt_domain* d = g_shim;
  if (!d) { set_error("convadj_: no domain bound (lt_shim_bind)"); return; }
  if (launch_convadj(d->a, d->stream)) return;
  cudaError_t e = cudaStreamSynchronize(d->stream);
  if (e != cudaSuccess) cuda_fail(e, "convadj_");
}

// icesnow.cpp:70
void icesnow_(void) {
  set_error("%s", "");
  lt_domain* d = g_shim;
  if (!d) { set_error("icesnow_: no domain bound (lt_shim_bind)"); return; }
  lt_icesnow_params p;
  lt_icesnow_defaults(&p);
  if (launch_icesnow(d->a, p, d->stream)) return;
  cudaError_t e = cudaStreamSynchronize(d->stream);
  if (e != cudaSuccess) cuda_fail(e, "icesnow_");
}

}  // extern "C"
