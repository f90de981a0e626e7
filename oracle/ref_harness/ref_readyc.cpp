// ref_readyc.cpp - host-side harness that runs kernels of the reference's own
// readyc.cpp (compiled from its place in the reference tree with the CPU HIP
// stand-in in oracle/ref_harness/hip) on one block of the reference's built-in
// size (imt = 40, jmt = 44, km = 55): the turbulence closure turb_cu and the
// momentum biharmonic friction (hdel4_div, hdel4_grad, hdel4_zcurl,
// hdiffu_del4_0, hdiffu_del4_1).  TEST INFRASTRUCTURE ONLY: builds
// oracle/_ref/libref_readyc.so, used by tests to pin the oracle's
// restatements against the reference's own code.
//
// readyc.cpp refers to many device pointers and module variables of the
// model; this file defines every one of them (those the two sequences do not
// read stay null), fills the ones they read from host arrays, does the
// memsets readyc_ does before them (readyc.cpp:1642, 1647, 1668-1671, 1757)
// and launches the kernels with the reference's grids.
#include <cstring>
#include <string>
#include <vector>
#include "hip/hip_runtime.h"
#include "../../include/licom_tracer.h"

#include <def-undef.h>
static const int R_IMT = BLCKX + 4, R_JMT = BLCKY + 4, R_KM = NKM;

thread_local dim3 threadIdx, blockIdx, blockDim, gridDim;

// ---- device pointers (cuda_data.h, canuto_mod.h, turb.h) that readyc.cpp names
double *d_ak_tide, *d_akmt, *d_akmu, *d_akt, *d_am_factor, *d_amf, *d_amld, *d_amtaun2a1, *d_and2on2a1, *d_at;
double *d_at0, *d_ate, *d_atn, *d_atne, *d_au0, *d_aus, *d_ausw, *d_auw, *d_back_ra_r, *d_bbcx, *d_bbcy;
double *d_buoysol, *d_buoytur, *d_d2uk, *d_d2vk, *d_diff_back, *d_dlu, *d_dlub, *d_dlv, *d_dlvb, *d_dmc;
double *d_dme, *d_dmn, *d_dms, *d_dmw, *d_duc, *d_due, *d_dum, *d_dun, *d_dus, *d_duw, *d_dxu, *d_dxur, *d_dyu;
double *d_dyur, *d_dzp, *d_fcort, *d_fz_tide, *d_fztidal, *d_h0, *d_h0bf, *d_h0bl, *d_hduk2, *d_hdvk2, *d_hts;
double *d_htw, *d_hue, *d_hun, *d_odzp, *d_odzt, *d_ohbt, *d_ohbu, *d_pdensity, *d_rib, *d_ric, *d_ricdttms;
double *d_richardson, *d_rict, *d_rit, *d_riu, *d_riv1, *d_riv2, *d_s2t, *d_s2u, *d_sbcx, *d_sbcy, *d_sh_r1;
double *d_sha1, *d_shb, *d_slq2_r1, *d_slq2b, *d_sm_r1, *d_sma1, *d_smb, *d_snlat, *d_ss_r1, *d_ssa1, *d_ssb;
double *d_su, *d_sv, *d_tarea_r, *d_turb_param, *d_u, *d_u_wface, *d_uarea_r, *d_uk, *d_up, *d_v, *d_v_sface;
double *d_vit, *d_viv, *d_vk, *d_vp, *d_wave_dis, *d_wk1, *d_wk2, *d_wk3, *d_wka, *d_work, *d_wp1, *d_wp12;
double *d_wp13, *d_wp3, *d_wp3_tidal, *d_wp7, *d_wp8, *d_ws, *d_zkp;
int *d_kmt, *d_kmu, *d_irimax;
size_t dataSize2d, dataSize3d;
// ---- module variables readyc.cpp names (only readyc_ reads them)
double hmix_del4_mp_am_, pconst_mod_mp_c0f_, pconst_mod_mp_cag_, pconst_mod_mp_od0_, pconst_mod_mp_sag_;
char blocks_mp_all_blocks_[4096];
int domain_mp_blocks_clinic_[8];

void turb_cu(double* d_akmt, double* d_akt, double* d_ak_tide, double* d_amld, double* d_amtaun2a1,
             double* d_and2on2a1, double* d_at, double* d_back_ra_r, double* d_buoysol, double* d_buoytur,
             double* d_dzp, double* d_fcort, double* d_fztidal, double* d_fz_tide, double* d_pdensity, double* d_rib,
             double* d_ricdttms, double* d_richardson, double* d_rict, double* d_rit, double* d_s2t, double* d_sha1,
             double* d_shb, double* d_sh_r1, double* d_slq2b, double* d_slq2_r1, double* d_sma1, double* d_smb,
             double* d_sm_r1, double* d_ssa1, double* d_ssb, double* d_ss_r1, double* d_turb_param, double* d_vit,
             double* d_wave_dis, double* d_wp3_tidal, double* d_zkp, int* d_irimax, int* d_kmt, double* d_diff_back,
             double* d_wk1, double* d_wk2, double* d_wk3, double* d_wp1, double* d_wp3, double* d_wp7, double* d_wp8);
void hdel4_div(double* d_hts, double* d_htw, double* d_tarea_r, double* d_up, double* d_vp, double* d_wka, int* d_kmt);
void hdel4_grad(double* d_wka, double* d_dxur, double* d_dyur, int* d_kmu, double* d_am_factor);
void hdel4_zcurl(double* d_dxu, double* d_dyu, double* d_up, double* d_vp, double* d_wka, int* d_kmt);
void hdiffu_del4_0(double* d_hduk2, double* d_hdvk2, int d_jb, int d_je, int d_ib, int d_ie, double* d_uarea_r,
                   double d_c0f, double* d_up, double* d_vp, double* d_duc, double* d_dum, double* d_dun, double* d_dus,
                   double* d_due, double* d_duw, double* d_dmc, double* d_dmn, double* d_dms, double* d_dme,
                   double* d_dmw, double d_am, double* d_dlu, double* d_dlv, double* d_viv, int* d_kmu,
                   double* d_amf, double* d_am_factor, double* d_d2uk, double* d_d2vk);
void hdiffu_del4_1(double* d_hduk2, double* d_hdvk2, int d_jb, int d_je, int d_ib, int d_ie, double* d_wka,
                   double d_c0f, double* d_up, double* d_vp, double* d_duc, double* d_dum, double* d_dun, double* d_dus,
                   double* d_due, double* d_duw, double* d_dmc, double* d_dmn, double* d_dms, double* d_dme,
                   double* d_dmw, double d_am, double* d_dlu, double* d_dlv, double* d_viv, int* d_kmu,
                   double* d_amf, double* d_am_factor, double* d_d2uk, double* d_d2vk);

namespace {
const long A = (long)R_IMT * R_JMT, F = A * R_KM;
struct Arr { double** p; long n; };
std::vector<std::vector<double>> keep;
std::vector<int> kmt_store, kmu_store;
std::vector<int> irimax_store;
double turb_param[11];
bool ready = false;

long count_of(const std::string& n) {
  if (n == "AT" || n == "AKT") return 2 * F;
  if (n == "RIT" || n == "RICDTTMS" || n == "S2T" || n == "RICT") return A * (R_KM - 1);
  if (n == "PDENSITY") return A * (R_KM + 1);
  if (n == "FZ_TIDE" || n == "AKMT" || n == "AK_TIDE" || n == "RICHARDSON" || n == "FZTIDAL" || n == "WP3_TIDAL")
    return F;
  if (n == "BUOYTUR" || n == "BUOYSOL" || n == "FCORT" || n == "WAVE_DIS" || n == "AMLD") return A;
  if (n == "DZP") return R_KM;
  if (n == "ZKP") return R_KM + 1;
  if (n == "UP" || n == "VP" || n == "DLU" || n == "DLV" || n == "WKA_DRAG") return F;
  if (n == "HTW" || n == "HTS" || n == "TAREA_R" || n == "DXU" || n == "DYU" || n == "DXUR" || n == "DYUR" ||
      n == "UAREA_R" || n == "DUC" || n == "DUM" || n == "DUN" || n == "DUS" || n == "DUE" || n == "DUW" ||
      n == "DMC" || n == "DMN" || n == "DMS" || n == "DME" || n == "DMW" || n == "AMF")
    return A;
  return -1;
}
double** slot_of(const std::string& n) {
  if (n == "AT") return &d_at;
  if (n == "AKT") return &d_akt;
  if (n == "RIT") return &d_rit;
  if (n == "RICDTTMS") return &d_ricdttms;
  if (n == "S2T") return &d_s2t;
  if (n == "RICT") return &d_rict;
  if (n == "PDENSITY") return &d_pdensity;
  if (n == "FZ_TIDE") return &d_fz_tide;
  if (n == "AKMT") return &d_akmt;
  if (n == "AK_TIDE") return &d_ak_tide;
  if (n == "RICHARDSON") return &d_richardson;
  if (n == "FZTIDAL") return &d_fztidal;
  if (n == "WP3_TIDAL") return &d_wp3_tidal;
  if (n == "BUOYTUR") return &d_buoytur;
  if (n == "BUOYSOL") return &d_buoysol;
  if (n == "FCORT") return &d_fcort;
  if (n == "WAVE_DIS") return &d_wave_dis;
  if (n == "AMLD") return &d_amld;
  if (n == "DZP") return &d_dzp;
  if (n == "ZKP") return &d_zkp;
  if (n == "UP") return &d_up;
  if (n == "VP") return &d_vp;
  if (n == "DLU") return &d_dlu;
  if (n == "DLV") return &d_dlv;
  if (n == "WKA_DRAG") return &d_wka;
  if (n == "HTW") return &d_htw;
  if (n == "HTS") return &d_hts;
  if (n == "TAREA_R") return &d_tarea_r;
  if (n == "DXU") return &d_dxu;
  if (n == "DYU") return &d_dyu;
  if (n == "DXUR") return &d_dxur;
  if (n == "DYUR") return &d_dyur;
  if (n == "UAREA_R") return &d_uarea_r;
  if (n == "DUC") return &d_duc;
  if (n == "DUM") return &d_dum;
  if (n == "DUN") return &d_dun;
  if (n == "DUS") return &d_dus;
  if (n == "DUE") return &d_due;
  if (n == "DUW") return &d_duw;
  if (n == "DMC") return &d_dmc;
  if (n == "DMN") return &d_dmn;
  if (n == "DMS") return &d_dms;
  if (n == "DME") return &d_dme;
  if (n == "DMW") return &d_dmw;
  if (n == "AMF") return &d_amf;
  return nullptr;
}
double* fresh(long n) { keep.emplace_back(n, 0.0); return keep.back().data(); }
void setup() {
  if (ready) return;
  const char* names[] = {"AT", "AKT", "RIT", "RICDTTMS", "S2T", "RICT", "PDENSITY", "FZ_TIDE", "AKMT", "AK_TIDE",
                         "RICHARDSON", "FZTIDAL", "WP3_TIDAL", "BUOYTUR", "BUOYSOL", "FCORT", "WAVE_DIS", "AMLD",
                         "DZP", "ZKP", "UP", "VP", "DLU", "DLV", "WKA_DRAG", "HTW", "HTS", "TAREA_R", "DXU",
                         "DYU", "DXUR", "DYUR", "UAREA_R", "DUC", "DUM", "DUN", "DUS", "DUE", "DUW", "DMC", "DMN",
                         "DMS", "DME", "DMW", "AMF"};
  for (const char* n : names) *slot_of(n) = fresh(count_of(n));
  kmt_store.assign(A, 0);
  d_kmt = kmt_store.data();
  kmu_store.assign(A, 0);
  d_kmu = kmu_store.data();
  d_am_factor = fresh(F); d_d2uk = fresh(F); d_d2vk = fresh(F); d_hduk2 = fresh(F); d_hdvk2 = fresh(F);
  d_vit = fresh(F);
  d_wk1 = fresh(F); d_wk2 = fresh(F); d_wk3 = fresh(F);
  d_wp1 = fresh(F); d_wp3 = fresh(F); d_wp7 = fresh(F); d_wp8 = fresh(F);
  d_diff_back = fresh(A);
  d_turb_param = turb_param;
  dataSize2d = sizeof(double) * A;
  dataSize3d = sizeof(double) * F;
  ready = true;
}
}  // namespace

extern "C" {

int ref_turb_dims(int* imt, int* jmt, int* km) {
  *imt = R_IMT; *jmt = R_JMT; *km = R_KM;
  return 0;
}
int ref_turb_set(const char* name, const void* src, size_t nbytes) {
  setup();
  const std::string n(name);
  if (n == "KMT" || n == "KMU") {
    if (nbytes != sizeof(int) * A) return LT_E_INVALID;
    std::memcpy(n == "KMT" ? kmt_store.data() : kmu_store.data(), src, nbytes);
    return 0;
  }
  const long c = count_of(n);
  if (c < 0 || nbytes != sizeof(double) * c) return LT_E_INVALID;
  std::memcpy(*slot_of(n), src, nbytes);
  return 0;
}
int ref_turb_get(const char* name, void* dst, size_t nbytes) {
  setup();
  const std::string n(name);
  const long c = count_of(n);
  if (c < 0 || nbytes != sizeof(double) * c) return LT_E_INVALID;
  std::memcpy(dst, *slot_of(n), nbytes);
  return 0;
}
// the tables are read where they lie (host memory stands in for the device)
int ref_turb_set_tables(const lt_turb_tables* t) {
  setup();
  d_rib = const_cast<double*>(t->rib);
  irimax_store.assign(t->irimax, t->irimax + LT_TURB_N1);
  d_irimax = irimax_store.data();
  d_slq2b = const_cast<double*>(t->slq2b); d_smb = const_cast<double*>(t->smb);
  d_shb = const_cast<double*>(t->shb); d_ssb = const_cast<double*>(t->ssb);
  d_and2on2a1 = const_cast<double*>(t->and2on2a1); d_amtaun2a1 = const_cast<double*>(t->amtaun2a1);
  d_sma1 = const_cast<double*>(t->sma1); d_sha1 = const_cast<double*>(t->sha1); d_ssa1 = const_cast<double*>(t->ssa1);
  d_back_ra_r = const_cast<double*>(t->back_ra_r); d_sm_r1 = const_cast<double*>(t->sm_r1);
  d_sh_r1 = const_cast<double*>(t->sh_r1); d_ss_r1 = const_cast<double*>(t->ss_r1);
  d_slq2_r1 = const_cast<double*>(t->slq2_r1);
  turb_param[0] = t->rri; turb_param[1] = t->rnd2on2; turb_param[2] = t->dri; turb_param[3] = t->deltheta_r;
  turb_param[4] = t->b1; turb_param[5] = t->theta_rcrp; turb_param[6] = t->theta_rcrn; turb_param[10] = t->dand2on2;
  return 0;
}
// turbinit's d_turb_param[7..9] (turb_init.cpp:81), the memsets of readyc_
// and the launch of turb_cu (readyc.cpp:1674-1678)
int ref_turb_call(int ncc, double dfricmx, double dwndmix) {
  setup();
  turb_param[7] = (double)ncc; turb_param[8] = dfricmx; turb_param[9] = dwndmix;
  for (int k = 0; k < R_KM; ++k)
    for (long a = 0; a < A; ++a) d_vit[k * A + a] = (k < d_kmt[a]) ? 1.0 : 0.0;
  hipMemset(d_amld, 0, dataSize2d);
  hipMemset(d_akmt, 0, dataSize3d);
  hipMemset(d_ak_tide, 0, dataSize3d);
  hipMemset(d_wk1, 0, dataSize3d);
  hipMemset(d_wk2, 0, dataSize3d);
  hipMemset(d_wk3, 0, dataSize3d);
  dim3 block(8, 16, 1), grid((R_IMT + 7) / 8, (R_JMT + 15) / 16);
  hipLaunchKernelGGL(turb_cu, grid, block, 0, 0, d_akmt, d_akt, d_ak_tide, d_amld, d_amtaun2a1, d_and2on2a1, d_at,
                     d_back_ra_r, d_buoysol, d_buoytur, d_dzp, d_fcort, d_fztidal, d_fz_tide, d_pdensity, d_rib,
                     d_ricdttms, d_richardson, d_rict, d_rit, d_s2t, d_sha1, d_shb, d_sh_r1, d_slq2b, d_slq2_r1,
                     d_sma1, d_smb, d_sm_r1, d_ssa1, d_ssb, d_ss_r1, d_turb_param, d_vit, d_wave_dis, d_wp3_tidal,
                     d_zkp, d_irimax, d_kmt, d_diff_back, d_wk1, d_wk2, d_wk3, d_wp1, d_wp3, d_wp7, d_wp8);
  return 0;
}

// readyc_'s BIHAR sequence (readyc.cpp:1754-1775) for one block covering the
// domain (Fortran block bounds ib = jb = 3, ie = imt-2, je = jmt-2)
int ref_del4u_call(double am, double c0f) {
  setup();
  const int jb = 3, je = R_JMT - 2, ib = 3, ie = R_IMT - 2;
  dim3 block(8, 16, 4), grid((R_IMT + 7) / 8, (R_JMT + 15) / 16, (R_KM + 3) / 4);
  hipLaunchKernelGGL(hdel4_div, grid, block, 0, 0, d_hts, d_htw, d_tarea_r, d_up, d_vp, d_wka, d_kmt);
  hipMemset(d_am_factor, 0, dataSize3d);
  hipLaunchKernelGGL(hdel4_grad, grid, block, 0, 0, d_wka, d_dxur, d_dyur, d_kmu, d_am_factor);
  hipLaunchKernelGGL(hdel4_zcurl, grid, block, 0, 0, d_dxu, d_dyu, d_up, d_vp, d_wka, d_kmt);
  hipLaunchKernelGGL(hdel4_grad, grid, block, 0, 0, d_wka, d_dxur, d_dyur, d_kmu, d_am_factor);
  hipLaunchKernelGGL(hdiffu_del4_0, grid, block, 0, 0, d_hduk2, d_hdvk2, jb, je, ib, ie, d_uarea_r, c0f, d_up, d_vp,
                     d_duc, d_dum, d_dun, d_dus, d_due, d_duw, d_dmc, d_dmn, d_dms, d_dme, d_dmw, am, d_dlu, d_dlv,
                     d_viv, d_kmu, d_amf, d_am_factor, d_d2uk, d_d2vk);
  hipLaunchKernelGGL(hdiffu_del4_1, grid, block, 0, 0, d_hduk2, d_hdvk2, jb, je, ib, ie, d_wka, c0f, d_up, d_vp,
                     d_duc, d_dum, d_dun, d_dus, d_due, d_duw, d_dmc, d_dmn, d_dms, d_dme, d_dmw, am, d_dlu, d_dlv,
                     d_viv, d_kmu, d_amf, d_am_factor, d_d2uk, d_d2vk);
  return 0;
}

}  // extern "C"
