// lt_common.cuh - device arena and launch parameters shared by the tracer
// step's translation units.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "../../include/licom_tracer.h"
#include "lt_fields.h"

namespace lt {

// Column tile of the fused tracer kernel: TX columns along i (one warp) by TY
// rows along j; one thread per column.
constexpr int TX = 32;
constexpr int TY = 8;
constexpr int TTHREADS = TX * TY;
// Persistent CTAs per SM of the column kernels (their shared-memory footprint
// decides): FP64 2 of 256 threads (its tile's metric and biharmonic
// coefficients staged in shared memory, no register spills), mixed 2 of 256
// (both tracers' level boxes per CTA).
constexpr int kFp64CtasPerSm = 2;
constexpr int kMixedCtasPerSm = 2;
// The mixed column kernel's tile: TX x kMixedTileY columns, one thread each
// (both tracers); its f64 state boxes are kMixedBoxW64 columns wide
// (x0-2 .. x0+TX+1) and its Thomas sweep keeps four values per level and
// column (e, f of T and S).
constexpr int kMixedTileY = 8;
constexpr int kMixedThreads = TX * kMixedTileY;
constexpr int kMixedBoxW64 = TX + 4;
constexpr int kMixedScratchPerLevel = 4;
constexpr int kMixedMaxLevels = 128;
// The mixed continuity march: tiles of 32 x kMixedContTileY columns, each
// level's U-point velocities as boxes kMixedContBoxW wide (x0 .. x0+35: the
// 33 columns the march reads, rounded up to 16 bytes) and kMixedContTileY+1
// rows (y0-1 .. y0+kMixedContTileY-1).
constexpr int kMixedContTileY = 4;
constexpr int kMixedContBoxW = 36;

// Everything the step kernels touch, as raw device pointers (dense
// [n][k][j][i] layout of the reference, i fastest).
struct alignas(16) Arena {   // copied into shared memory as 16-byte words
  int nx, ny, km, imt, jmt;
  long A, F, FB;
  int ew_cyclic, tripole, diagnostics, precision;
  lt_params p;

  // state, ping-pong: index cur holds the state the next step reads
  double* at[2];
  double* atb[2];
  int cur;

  // dynamics inputs (frozen across lt_step calls) and step outputs
  double *utf, *vtf, *utl, *vtl, *h0f, *h0l, *akt;
  double *utf_out, *vtf_out, *h0f_out;
  double *ws, *net;
  // surface forcing and grid
  double *swv, *nswv, *sst, *sss, *fresh, *seaice;
  double *tarea, *tarea_r, *htw, *hts, *hun, *hue, *dxu, *dyu, *ahf, *dtn, *dts, *dte, *dtw, *ohbt, *ohbu;
  double *au0, *aus, *auw, *ausw;
  int *kmt, *kmu, *kmtn, *kmts, *kmte, *kmtw;
  double *dzp, *odzp, *odzt, *pen, *to, *so, *cc, *restore;
  double *restore_at, *dt_restore;   // tracer_7's nudging (simple_assm)
  double *qice;               // [jmt][imt] ice formed by icesnow (tracer_mod licomqice)
  // turbulence closure (lt_turb): inputs and outputs, null until the domain
  // first uses one of them
  double *rit, *ricdttms, *s2t, *rict, *pdensity, *fz_tide, *buoytur, *buoysol, *fcort, *wave_dis, *zkp;
  double *akmt, *ak_tide, *amld, *richardson, *fztidal, *wp3_tidal;
  // momentum biharmonic friction (lt_hdiffu_del4), null until first used
  double *up, *vp, *dlu, *dlv, *wka_drag;
  double *duc, *dum, *dun, *dus, *due, *duw, *dmc, *dmn, *dms, *dme, *dmw, *amf, *uarea_r, *dxur, *dyur;
  // diagnostics (null when off)
  double *ax, *ay, *az, *dzd, *tend, *dt_diff, *dt_conv, *penetrate;
  // [jmt][imt], with diagnostics: one past the deepest level at which the
  // column's west or south face transport or its w is nonzero (written by
  // the continuity; the column kernel's deep-level shortcut reads it)
  int* kfz;

  // step scratch
  double *uwf, *vsf;          // face transports u_wface, v_sface [km][jmt][imt]
  double *wka;                // horizontal divergence [km][jmt][imt]
  // mixed precision: f32 storage of the dynamics inputs, mixing and the
  // derived fields (the f64 pointers above are null for these; the
  // horizontal divergence lives only in registers of the continuity march)
  float *utf32, *vtf32, *utl32, *vtl32, *akt32, *ws32, *utf_out32, *vtf_out32;
  float *wkd32, *wkb32;       // U-point mean velocities wkd, wkb; the tracer kernel forms the faces from them
  double *stf_ssh;            // [jmt][imt] 0.5*(h0f*onbc + h0l)
  double *stf_n;              // [2][jmt][imt] surface flux per tracer (T, S)
  double *red_part;           // partial sums of the deterministic reductions
  double *scalars;            // [0] err_norm2 (fw_norm2), [1..2] tracer content, [3..] spare
  double *col_scratch;        // per-slot Thomas sweep storage
  double *fold_save;          // [2][km][2][imt] pre-fold values of the top physical row (diagnostics)
  int *status;                // [4] device status words
  long col_scratch_slots;
  int nv_scratch;             // values per level per column in col_scratch
  unsigned wait_limit;        // polls of each level wait in the column kernels before giving up
};

// The turbulence closure's tables on the device (lt_turb_tables, copied by
// lt_turb_tables_create).
struct TurbTabDev {
  const double *rib, *slq2b, *smb, *shb, *ssb, *and2on2a1, *amtaun2a1, *sma1, *sha1, *ssa1;
  const double *back_ra_r, *sm_r1, *sh_r1, *ss_r1, *slq2_r1;
  const int* irimax;
  double rri, rnd2on2, dri, deltheta_r, b1, theta_rcrp, theta_rcrn, dand2on2;
};

#define LT_CUDA_OK(call)                                   \
  do {                                                     \
    cudaError_t e_ = (call);                               \
    if (e_ != cudaSuccess) return lt::cuda_fail(e_, #call); \
  } while (0)

// after a kernel launch: check the launch and count it
#define LT_LAUNCHED()                    \
  do {                                   \
    LT_CUDA_OK(cudaGetLastError());      \
    lt::count_launches(1);               \
  } while (0)

int cuda_fail(cudaError_t e, const char* what);
// process-wide count of kernels launched by this library
long long launch_counter();
void count_launches(int n);
void set_error(const char* fmt, ...);

// host launchers (defined in the step translation units)
// the surface kernel in two parts: the SSH mean (h0f_out, stf_ssh), which the
// continuity needs, and the surface fluxes, net and the mixing floor (which
// read stf_ssh and the forcing)
int launch_ssh(const Arena& a, cudaStream_t s);
int launch_surface_fluxes(const Arena& a, cudaStream_t s);
int launch_continuity_fp64(const Arena& a, cudaStream_t s);
int launch_tracer_fp64(const Arena& a, cudaStream_t s, int slots);
int launch_halo_state(const Arena& a, cudaStream_t s);
int launch_halo_r8(double* f, int nz, int imt, int jmt, int ew_cyclic, int tripole, cudaStream_t s);
int launch_tree_sum(const double* x, long n, double* part, double* out, cudaStream_t s);
int launch_interior_sum_sss(const Arena& a, cudaStream_t s);
int launch_tracer_content(const Arena& a, cudaStream_t s);
int launch_convadj(const Arena& a, cudaStream_t s);
int launch_icesnow(const Arena& a, const lt_icesnow_params& p, cudaStream_t s);
int launch_turb(const Arena& a, const TurbTabDev& T, int ncc, double dfricmx, cudaStream_t s);
int launch_del4u(const Arena& a, double am, double c0f, cudaStream_t s);
int launch_check_numeric(const Arena& a, cudaStream_t s);
int launch_derive_masks(const Arena& a, cudaStream_t s);
int launch_vtl_clobber(const Arena& a, cudaStream_t s);

int launch_f64_to_f32(const double* x, float* y, long n, cudaStream_t s);
int launch_f32_to_f64(const float* x, double* y, long n, cudaStream_t s);
int tracer_slots(const Arena& a);
size_t tree_sum_part_elems(long n);

// L2 policies of the column sweeps' scratch.  The elimination coefficients of
// a work item's wet levels are written during its march and read once, in
// reverse order, by its substitution.  Written with evict_last they stay in
// L2 against the streaming level boxes and state stores (on a deep ocean the
// scratch of all resident CTAs is close to the L2's size); read with
// evict_first they leave it once used.  The kernels write the new state with
// streaming stores (__stcs): nothing reads it again within the step.
__device__ __forceinline__ uint64_t l2_evict_last() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint64_t l2_evict_first() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ void st_l2(double* p, double v, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.f64 [%0], %1, %2;" ::"l"(p), "d"(v), "l"(pol) : "memory");
}
__device__ __forceinline__ double ld_l2(const double* p, uint64_t pol) {
  double v;
  asm volatile("ld.global.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ void st_l2(double2* p, double2 v, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.v2.f64 [%0], {%1, %2}, %3;" ::"l"(p), "d"(v.x), "d"(v.y), "l"(pol) : "memory");
}
__device__ __forceinline__ double2 ld_l2(const double2* p, uint64_t pol) {
  double2 v;
  asm volatile("ld.global.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;" : "=d"(v.x), "=d"(v.y) : "l"(p), "l"(pol));
  return v;
}

}  // namespace lt
