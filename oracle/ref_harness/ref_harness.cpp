// ref_harness.cpp - host-side harness that runs the reference's own
// tracer.cpp / convadj.cpp / icesnow.cpp (compiled from their place in the
// reference tree with the CPU HIP stand-in in oracle/ref_harness/hip) on one
// block.  icesnow.cpp is compiled twice: as configured (def-undef.h defines
// FRC_CORE: licomqice is zeroed before each call) and, renamed
// icesnow_nofrc_, with that one define removed (licomqice carries over).
// TEST INFRASTRUCTURE ONLY: builds oracle/_ref/libref_tracer.so, used by tests
// to pin the oracle against the reference's own code.
//
// The reference fixes the block size at compile time (def-undef.h: BLCKX=36,
// BLCKY=40, NKM=55, so imt=40, jmt=44, km=55).  This harness defines the
// device pointers and Fortran module variables tracer_ reads, and supplies the
// three host callbacks it makes: the halo update of net and vtl (a single
// block covering the global domain: east-west cyclic, tripole fold, closed
// south) and the MPI sum (identity on one rank).
#include <pthread.h>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#include "hip/hip_runtime.h"
#include "../../include/licom_tracer.h"
#include "../../licom3-hip_b200/csrc/lt_synth.h"


// sizes of the compiled reference
#include <def-undef.h>
static const int R_IMT = BLCKX + 4, R_JMT = BLCKY + 4, R_KM = NKM;

thread_local dim3 threadIdx, blockIdx, blockDim, gridDim;

extern "C" void tracer_(int ii);
// tracer.cpp's tracer_7 kernel (__global__ is empty in the CPU stand-in)
void tracer_7(int d_imt, int d_jmt, int d_km, int n, double* d_tf, double* d_vit, double* d_atb, double* d_restore,
              double* d_restore_at, double* d_dt_restore, int d_boundary_restore, int d_simple_assm, int d_ktv);
extern "C" void convadj_();
extern "C" void icesnow_();
extern "C" void icesnow_nofrc_();

// ---- device pointers (cuda_data.h) used by tracer.cpp / convadj.cpp
double *d_at00, *d_atmax, *d_atmin, *d_adv_tt, *d_ori, *d_temp11, *d_uk, *d_vk, *d_u_wface, *d_v_sface;
double *d_ohbu, *d_vit, *d_dzp, *d_to, *d_so, *d_c, *d_ohbt, *d_odzp, *d_odzt;
double *d_h0f, *d_h0l, *d_stf, *d_utf, *d_vtf, *d_utl, *d_vtl, *d_work, *d_wka, *d_wkb, *d_wkd, *d_wkc;
double *d_au0, *d_aus, *d_auw, *d_ausw, *d_htw, *d_hts, *d_hun, *d_hue, *d_dxu, *d_dyu, *d_tarea_r, *d_tarea;
double *d_ws, *d_at, *d_atb, *d_ax, *d_ay, *d_az, *d_tf, *d_akt, *d_d2tk, *d_ahf;
double *d_dtn, *d_dts, *d_dte, *d_dtw, *d_swv, *d_pen, *d_penetrate, *d_dz, *d_ssf, *d_sss, *d_ifrac, *d_net;
double *d_dt_restore, *d_fresh, *d_seaice, *d_tsf, *d_nswv, *d_sst, *d_dqdt, *d_restore, *d_restore_at;
double *d_tend, *d_dt_diff, *d_dt_conv, *d_icmon;
double *d_licomqice;
int *d_kmt, *d_kmtn, *d_kmts, *d_kmte, *d_kmtw;
size_t dataSize2d, dataSize3d, dataSize33d, dataSize4d, dataSize44d;

// ---- Fortran module variables read by tracer_
char pconst_mod_mp_adv_tracer_[80];
double pconst_mod_mp_onbc_, pconst_mod_mp_oncc_, pconst_mod_mp_dts_, pconst_mod_mp_dwndmix_;
double pconst_mod_mp_gamma_, pconst_mod_mp_od0_, pconst_mod_mp_od0cp_;
int pconst_mod_mp_nss_, pconst_mod_mp_ist_, pconst_mod_mp_boundary_restore_;
double hmix_del4_mp_ah_, grid_mp_area_t_, tracer_mod_mp_fw_norm2_;
double pconst_mod_mp_tbice_ = -1.8, pconst_mod_mp_cp_ = 3996.0;   // constant_mod.F90:164,168
int param_mod_mp_mytid_ = 0;
double (*tracer_mod_mp_net_)[2][R_JMT][R_IMT];
double (*dyn_mod_mp_vtl_)[R_KM][R_JMT][R_IMT];

static int g_ew_cyclic = 1, g_tripole = 1;

extern "C" void pop_haloupdate_tracer1_(int* err) {
  lt::halo_fill(&tracer_mod_mp_net_[0][0][0][0], 2, R_IMT, R_JMT, g_ew_cyclic, g_tripole);
  *err = 0;
}
extern "C" void pop_haloupdate_tracer2_(int* err) {
  lt::halo_fill(&dyn_mod_mp_vtl_[0][0][0][0], R_KM, R_IMT, R_JMT, g_ew_cyclic, g_tripole);
  *err = 0;
}
extern "C" void mpi3_(double*) {}

namespace {
const long A = (long)R_IMT * R_JMT, F = A * R_KM, FB = A * (R_KM + 1);
std::vector<double> store[LT_F_COUNT];
std::vector<int> istore[LT_F_COUNT];
std::vector<double> scratch_pool;
bool ready = false;

long field_count(int f) {
  switch (f) {
    case LT_F_AT: case LT_F_AKT: case LT_F_RESTORE: case LT_F_RESTORE_AT: case LT_F_DT_RESTORE:
    case LT_F_AX: case LT_F_AY: case LT_F_AZ: case LT_F_DZ:
    case LT_F_TEND: case LT_F_DT_DIFF: case LT_F_DT_CONV: return 2 * F;
    case LT_F_ATB: return 2 * FB;
    case LT_F_UTF: case LT_F_VTF: case LT_F_UTL: case LT_F_VTL: case LT_F_UTF_OUT: case LT_F_VTF_OUT:
    case LT_F_PENETRATE: case LT_F_FZ_TIDE: case LT_F_AKMT: case LT_F_AK_TIDE: case LT_F_RICHARDSON:
    case LT_F_FZTIDAL: case LT_F_WP3_TIDAL: case LT_F_UP: case LT_F_VP: case LT_F_DLU: case LT_F_DLV:
    case LT_F_WKA_DRAG: return F;
    case LT_F_RIT: case LT_F_RICDTTMS: case LT_F_S2T: case LT_F_RICT: return A * (R_KM - 1);
    case LT_F_ZKP: return R_KM + 1;
    case LT_F_WS: case LT_F_PDENSITY: return FB;
    case LT_F_NET: return 2 * A;
    case LT_F_DZP: case LT_F_ODZP: case LT_F_ODZT: case LT_F_PEN: case LT_F_TO: case LT_F_SO: return R_KM;
    case LT_F_C: return 9L * R_KM;
    default: return A;
  }
}
bool field_int(int f) { return f >= LT_F_KMT && f <= LT_F_KMTW; }

std::vector<std::vector<double>> scratch;
double* fresh_scratch(long n) { scratch.emplace_back(n, 0.0); return scratch.back().data(); }

void setup() {
  if (ready) return;
  for (int f = 0; f < LT_F_COUNT; ++f) {
    if (field_int(f)) istore[f].assign(field_count(f), 0);
    else store[f].assign(field_count(f), 0.0);
  }
  d_at = store[LT_F_AT].data(); d_atb = store[LT_F_ATB].data();
  d_utf = store[LT_F_UTF].data(); d_vtf = store[LT_F_VTF].data();
  d_utl = store[LT_F_UTL].data(); d_vtl = store[LT_F_VTL].data();
  d_h0f = store[LT_F_H0F].data(); d_h0l = store[LT_F_H0L].data();
  d_akt = store[LT_F_AKT].data(); d_ws = store[LT_F_WS].data(); d_net = store[LT_F_NET].data();
  d_swv = store[LT_F_SWV].data(); d_nswv = store[LT_F_NSWV].data(); d_sst = store[LT_F_SST].data();
  d_sss = store[LT_F_SSS].data(); d_fresh = store[LT_F_FRESH].data(); d_seaice = store[LT_F_SEAICE].data();
  d_tarea = store[LT_F_TAREA].data(); d_tarea_r = store[LT_F_TAREA_R].data();
  d_htw = store[LT_F_HTW].data(); d_hts = store[LT_F_HTS].data(); d_hun = store[LT_F_HUN].data();
  d_hue = store[LT_F_HUE].data(); d_dxu = store[LT_F_DXU].data(); d_dyu = store[LT_F_DYU].data();
  d_ahf = store[LT_F_AHF].data(); d_dtn = store[LT_F_DTN].data(); d_dts = store[LT_F_DTS].data();
  d_dte = store[LT_F_DTE].data(); d_dtw = store[LT_F_DTW].data(); d_ohbt = store[LT_F_OHBT].data();
  d_ohbu = store[LT_F_OHBU].data(); d_au0 = store[LT_F_AU0].data(); d_aus = store[LT_F_AUS].data();
  d_auw = store[LT_F_AUW].data(); d_ausw = store[LT_F_AUSW].data();
  d_kmt = istore[LT_F_KMT].data(); d_kmtn = istore[LT_F_KMTN].data(); d_kmts = istore[LT_F_KMTS].data();
  d_kmte = istore[LT_F_KMTE].data(); d_kmtw = istore[LT_F_KMTW].data();
  d_dzp = store[LT_F_DZP].data(); d_odzp = store[LT_F_ODZP].data(); d_odzt = store[LT_F_ODZT].data();
  d_pen = store[LT_F_PEN].data(); d_to = store[LT_F_TO].data(); d_so = store[LT_F_SO].data();
  d_c = store[LT_F_C].data(); d_restore = store[LT_F_RESTORE].data();
  d_ax = store[LT_F_AX].data(); d_ay = store[LT_F_AY].data(); d_az = store[LT_F_AZ].data();
  d_dz = store[LT_F_DZ].data(); d_tend = store[LT_F_TEND].data(); d_dt_diff = store[LT_F_DT_DIFF].data();
  d_dt_conv = store[LT_F_DT_CONV].data(); d_penetrate = store[LT_F_PENETRATE].data();
  d_licomqice = store[LT_F_QICE].data();
  // scratch arrays of the reference (sizes from cuda_init.cpp)
  d_at00 = fresh_scratch(F); d_atmax = fresh_scratch(F); d_atmin = fresh_scratch(F);
  d_adv_tt = fresh_scratch(F); d_ori = fresh_scratch(F); d_temp11 = fresh_scratch(A);
  d_uk = fresh_scratch(F); d_vk = fresh_scratch(F); d_u_wface = fresh_scratch(F); d_v_sface = fresh_scratch(F);
  d_stf = fresh_scratch(A); d_work = fresh_scratch(A); d_wka = fresh_scratch(F); d_wkb = fresh_scratch(F);
  d_wkd = fresh_scratch(F); d_wkc = fresh_scratch(F); d_tf = fresh_scratch(F); d_d2tk = fresh_scratch(F);
  d_vit = fresh_scratch(F); d_ssf = fresh_scratch(A); d_ifrac = fresh_scratch(A);
  d_dt_restore = fresh_scratch(2 * F); d_tsf = fresh_scratch(A); d_dqdt = fresh_scratch(A);
  d_restore_at = fresh_scratch(2 * F); d_icmon = fresh_scratch(2 * A);
  tracer_mod_mp_net_ = reinterpret_cast<double(*)[2][R_JMT][R_IMT]>(fresh_scratch(2 * A));
  dyn_mod_mp_vtl_ = reinterpret_cast<double(*)[R_KM][R_JMT][R_IMT]>(fresh_scratch(F));
  dataSize2d = sizeof(double) * A;
  dataSize3d = sizeof(double) * F;
  dataSize33d = sizeof(double) * 2 * A;
  dataSize4d = sizeof(double) * 2 * F;
  dataSize44d = sizeof(double) * 2 * FB;
  std::strncpy(pconst_mod_mp_adv_tracer_, "tspas", sizeof(pconst_mod_mp_adv_tracer_));
  ready = true;
}

void refresh_vit() {
  for (int k = 0; k < R_KM; ++k)
    for (long a = 0; a < A; ++a) d_vit[k * A + a] = (k < d_kmt[a]) ? 1.0 : 0.0;
}

void* run_tracer(void* arg) {
  tracer_(*static_cast<int*>(arg));
  return nullptr;
}
void* run_convadj(void*) {
  convadj_();
  return nullptr;
}
int in_big_stack(void* (*fn)(void*), void* arg) {
  pthread_attr_t attr;
  pthread_attr_init(&attr);
  pthread_attr_setstacksize(&attr, (size_t)1 << 30);
  pthread_t t;
  if (pthread_create(&t, &attr, fn, arg) != 0) return LT_E_STATE;
  pthread_join(t, nullptr);
  pthread_attr_destroy(&attr);
  return 0;
}
}  // namespace

extern "C" {

int ref_dims(int* imt, int* jmt, int* km) {
  *imt = R_IMT; *jmt = R_JMT; *km = R_KM;
  return 0;
}
int ref_set_params(const lt_params* p, int ew_cyclic, int tripole) {
  setup();
  pconst_mod_mp_dts_ = p->dts; pconst_mod_mp_oncc_ = p->oncc; pconst_mod_mp_onbc_ = p->onbc;
  pconst_mod_mp_dwndmix_ = p->dwndmix; pconst_mod_mp_gamma_ = p->gamma; pconst_mod_mp_od0_ = p->od0;
  pconst_mod_mp_od0cp_ = p->od0cp; hmix_del4_mp_ah_ = p->ah; grid_mp_area_t_ = p->area_t;
  pconst_mod_mp_nss_ = p->nss; pconst_mod_mp_boundary_restore_ = p->boundary_restore;
  // the namelist string tracer_ matches (tracer.cpp:1712-1714), blank-padded
  // like a Fortran CHARACTER variable
  const char* scheme = p->adv_tracer == LT_ADV_CENTERED ? "centered" : p->adv_tracer == LT_ADV_FLUX ? "flux" : "tspas";
  std::memset(pconst_mod_mp_adv_tracer_, ' ', sizeof(pconst_mod_mp_adv_tracer_));
  std::memcpy(pconst_mod_mp_adv_tracer_, scheme, std::strlen(scheme));
  g_ew_cyclic = ew_cyclic; g_tripole = tripole;
  return 0;
}
int ref_set_field(int f, const void* src, size_t nbytes) {
  setup();
  if (f < 0 || f >= LT_F_COUNT) return LT_E_INVALID;
  const size_t need = field_count(f) * (field_int(f) ? sizeof(int) : sizeof(double));
  if (nbytes != need) return LT_E_INVALID;
  if (field_int(f)) std::memcpy(istore[f].data(), src, nbytes);
  else std::memcpy(store[f].data(), src, nbytes);
  if (f == LT_F_NET) std::memcpy(&tracer_mod_mp_net_[0][0][0][0], src, nbytes);  // host copy of net
  return 0;
}
int ref_get_field(int f, void* dst, size_t nbytes) {
  setup();
  if (f < 0 || f >= LT_F_COUNT) return LT_E_INVALID;
  const size_t need = field_count(f) * (field_int(f) ? sizeof(int) : sizeof(double));
  if (nbytes != need) return LT_E_INVALID;
  if (f == LT_F_NET) { std::memcpy(dst, &tracer_mod_mp_net_[0][0][0][0], nbytes); return 0; }
  if (field_int(f)) std::memcpy(dst, istore[f].data(), nbytes);
  else std::memcpy(dst, store[f].data(), nbytes);
  return 0;
}
int ref_tracer_call(int ii) {
  setup();
  refresh_vit();
  return in_big_stack(run_tracer, &ii);
}
int ref_convadj_call(void) {
  setup();
  refresh_vit();
  return in_big_stack(run_convadj, nullptr);
}
// icesnow_ with the given tbice and cp (SHR_CONST_LATICE is compiled in);
// frc_core 1 runs the file as configured, 0 the build without FRC_CORE
int ref_icesnow_call(double tbice, double cp, int frc_core) {
  setup();
  pconst_mod_mp_tbice_ = tbice;
  pconst_mod_mp_cp_ = cp;
  if (frc_core) icesnow_();
  else icesnow_nofrc_();
  return 0;
}
double ref_fw_norm2(void) { return tracer_mod_mp_fw_norm2_; }
// tracer_7 alone on the caller's arrays of the reference's block size,
// launched as tracer_ launches it (8x8x4 threads).  tracer_ passes
// simple_assm = 0 (tracer.cpp:1877-1879); this runs the nudging branch too.
int ref_tracer7_call(int n, double* tf, double* vit, double* atb, double* restore, double* restore_at,
                     double* dt_restore, int boundary_restore, int simple_assm, int ktv) {
  setup();
  dim3 threads(8, 8, 4);
  dim3 blocks((R_IMT + threads.x - 1) / threads.x, (R_JMT + threads.y - 1) / threads.y,
              (R_KM + threads.z - 1) / threads.z);
  hipLaunchKernelGGL(tracer_7, dim3(blocks), dim3(threads), 0, 0, R_IMT, R_JMT, R_KM, n, tf, vit, atb, restore,
                     restore_at, dt_restore, boundary_restore, simple_assm, ktv);
  return 0;
}

}  // extern "C"
