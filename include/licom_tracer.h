/*
 * licom_tracer.h - C ABI of the B200 LICOM3 baroclinic tracer step.
 *
 * Drop-in for the tracer path of LICOM3-HIP:
 *   tracer_(int ii)   replaces  tracer.cpp:1701-1903   (extern "C" void tracer_(int))
 *   convadj_(void)    replaces  convadj.cpp:290-298    (extern "C" void convadj_())
 *   icesnow_(void)    replaces  icesnow.cpp:70-85      (extern "C" void icesnow_())
 * and the device state those read, which the reference keeps in global d_*
 * pointers (cuda_data.h:35-345, allocated by cudainit in cuda_init.cpp:372-707).
 * Here the state lives in a per-domain arena created by lt_create; the two
 * reference-named shims act on the domain bound with lt_shim_bind.
 *
 * Array layout is the reference's: C row-major [n][k][j][i] (Fortran
 * (i,j,k,n)), i fastest, halo width 2 on each side (imt = nx+4, jmt = ny+4),
 * j = 0 the northern edge.  ATB carries km+1 levels (Fortran 0:km) and WS km+1
 * levels.  Every entry point returns an lt_status; nothing prints or exits.
 */
#ifndef LICOM_TRACER_H
#define LICOM_TRACER_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  LT_OK = 0,
  LT_E_INVALID = 1,   /* bad argument, size or field id */
  LT_E_OOM = 2,       /* device memory admission failed */
  LT_E_CUDA = 3,      /* a CUDA runtime call failed */
  LT_E_NUMERIC = 4,   /* NaN/Inf found by the step's status scan */
  LT_E_TIMEOUT = 5,   /* a bounded device wait ran out */
  LT_E_STATE = 6,     /* call out of order (e.g. step before inputs) */
  LT_E_NODEVICE = 7   /* no CUDA device visible */
} lt_status;

/* Field identifiers.  Shapes use km, jmt, imt of the domain. */
typedef enum {
  /* prognostic state, f64 */
  LT_F_AT = 0,        /* [2][km][jmt][imt]  T (degC), S ((psu-35)/1000)  tracer_mod at  */
  LT_F_ATB,           /* [2][km+1][jmt][imt] previous tracers, level 0 unused  tracer_mod atb */
  /* dynamics inputs (produced by barotr/bclinc in the model), f64 */
  LT_F_UTF,           /* [km][jmt][imt] */
  LT_F_VTF,
  LT_F_UTL,
  LT_F_VTL,
  LT_F_H0F,           /* [jmt][imt] */
  LT_F_H0L,
  LT_F_AKT,           /* [2][km][jmt][imt] Canuto diffusivity (readyc.cpp:1569-1572) */
  /* outputs / persistent side state */
  LT_F_WS,            /* [km+1][jmt][imt] vertical velocity */
  LT_F_NET,           /* [2][jmt][imt] surface net flux, halo-updated */
  LT_F_UTF_OUT,       /* [km][jmt][imt] utf*oncc (the reference scales utf in place) */
  LT_F_VTF_OUT,
  LT_F_H0F_OUT,       /* [jmt][imt] h0f*onbc */
  /* surface forcing, f64 [jmt][imt] */
  LT_F_SWV, LT_F_NSWV, LT_F_SST, LT_F_SSS, LT_F_FRESH, LT_F_SEAICE,
  /* horizontal grid, f64 [jmt][imt] */
  LT_F_TAREA, LT_F_TAREA_R, LT_F_HTW, LT_F_HTS, LT_F_HUN, LT_F_HUE, LT_F_DXU, LT_F_DYU,
  LT_F_AHF, LT_F_DTN, LT_F_DTS, LT_F_DTE, LT_F_DTW, LT_F_OHBT, LT_F_OHBU,
  LT_F_AU0, LT_F_AUS, LT_F_AUW, LT_F_AUSW,
  /* integer masks, i32 [jmt][imt] */
  LT_F_KMT, LT_F_KMU, LT_F_KMTN, LT_F_KMTS, LT_F_KMTE, LT_F_KMTW,
  /* vertical, f64 */
  LT_F_DZP, LT_F_ODZP, LT_F_ODZT,   /* [km] */
  LT_F_PEN,                         /* [km] shortwave penetration (km-1 used) */
  LT_F_TO, LT_F_SO,                 /* [km] convadj reference T/S */
  LT_F_C,                           /* [9][km] convadj density polynomial */
  LT_F_RESTORE,                     /* [2][km][jmt][imt] restoring target */
  /* diagnostics, f64 (written when the domain was created with diagnostics) */
  LT_F_AX, LT_F_AY, LT_F_AZ, LT_F_DZ, LT_F_TEND, LT_F_DT_DIFF, LT_F_DT_CONV,  /* [2][km][jmt][imt] */
  LT_F_PENETRATE,                   /* [km][jmt][imt] */
  /* sea-ice bookkeeping of icesnow, f64 */
  LT_F_QICE,                        /* [jmt][imt] ice formed, tracer_mod licomqice (d_licomqice) */
  /* Canuto turbulence closure (lt_turb), f64; allocated on first use */
  LT_F_RIT, LT_F_RICDTTMS,          /* [km-1][jmt][imt] Richardson numbers Ri = Ri_T + Ri_C, Ri_d = Ri_T - Ri_C */
  LT_F_S2T,                         /* [km-1][jmt][imt] shear squared at T points (readyc1_2) */
  LT_F_RICT,                        /* [km-1][jmt][imt] buoyancy frequency squared N^2 */
  LT_F_PDENSITY,                    /* [km+1][jmt][imt] potential density (levels 0..km-1 used) */
  LT_F_FZ_TIDE,                     /* [km][jmt][imt] vertical structure of tidal dissipation */
  LT_F_BUOYTUR, LT_F_BUOYSOL,       /* [jmt][imt] turbulent and solar surface buoyancy flux */
  LT_F_FCORT,                       /* [jmt][imt] Coriolis parameter at T points */
  LT_F_WAVE_DIS,                    /* [jmt][imt] tidal wave dissipation */
  LT_F_ZKP,                         /* [km+1] depths of the level interfaces (negative, m) */
  LT_F_AKMT,                        /* [km][jmt][imt] viscosity at T points (output) */
  LT_F_AK_TIDE,                     /* [km][jmt][imt] tidal mixing (output) */
  LT_F_AMLD,                        /* [jmt][imt] mixed-layer depth (output, m) */
  LT_F_RICHARDSON, LT_F_FZTIDAL, LT_F_WP3_TIDAL,  /* [km][jmt][imt] tidal diagnostics (output) */
  /* momentum biharmonic friction (lt_hdiffu_del4), f64; allocated on first use */
  LT_F_UP, LT_F_VP,                 /* [km][jmt][imt] velocities at U points (dyn_mod up, vp) */
  LT_F_DLU, LT_F_DLV,               /* [km][jmt][imt] momentum tendencies, accumulated into */
  LT_F_WKA_DRAG,                    /* [km][jmt][imt] c0f*|u| left in the reference's wka (output) */
  LT_F_DUC, LT_F_DUM, LT_F_DUN, LT_F_DUS, LT_F_DUE, LT_F_DUW,  /* [jmt][imt] del4 stencil (init_del4u) */
  LT_F_DMC, LT_F_DMN, LT_F_DMS, LT_F_DME, LT_F_DMW,
  LT_F_AMF,                         /* [jmt][imt] resolution factor of the viscosity */
  LT_F_UAREA_R, LT_F_DXUR, LT_F_DYUR,  /* [jmt][imt] U-cell metrics */
  /* tracer_7's nudging (simple_assm), f64; held by domains created with it */
  LT_F_RESTORE_AT,                  /* [2][km][jmt][imt] nudging target (d_restore_at) */
  LT_F_DT_RESTORE,                  /* [2][km][jmt][imt] the nudging term of the last step (d_dt_restore) */
  LT_F_COUNT
} lt_field;

/* Precision of the step arithmetic.  The state is always f64.  A mixed
 * domain stores its dynamics inputs and mixing in f32 and takes at most 128
 * levels (its per-level constants stay in shared memory). */
typedef enum {
  LT_PREC_FP64 = 0,   /* plain f64 drop-in: the correctness form */
  LT_PREC_MIXED = 1   /* f32 storage of the dynamics inputs, f32 predictor, f64 state, fluxes and sums */
} lt_precision;

typedef struct {
  int nx, ny, km;        /* physical sizes; imt = nx+4, jmt = ny+4 */
  int precision;         /* lt_precision */
  int diagnostics;       /* nonzero: write AX..PENETRATE, TEND, DT_DIFF (FP64 form only; a mixed
                            domain with diagnostics is refused with LT_E_INVALID) */
  int ew_cyclic;         /* 1 cyclic east-west, 0 closed */
  int tripole;           /* 1 tripole north fold, 0 closed north */
} lt_grid;

/* Tracer advection scheme: pconst_mod adv_tracer, which tracer_ matches as
 * "centered" / "flux" / "tspas" (tracer.cpp:1712-1714) and passes to the
 * advection kernels as Str 0 / 1 / 2.  The centred and flux forms run in the
 * FP64 form only (a mixed domain refuses them with LT_E_INVALID). */
typedef enum {
  LT_ADV_TSPAS = 0,     /* two-step shape-preserving (Str 2, advection_tracer_1_0/2/3), the default */
  LT_ADV_CENTERED = 1,  /* centred differences of the tracer across each face (Str 0, advection_tracer_1) */
  LT_ADV_FLUX = 2       /* face means times dx/dy-weighted transports (Str 1, advection_tracer_1_0/1) */
} lt_adv_scheme;

/* Scalars read by tracer_ from Fortran module variables (tracer.cpp:1712-1896). */
typedef struct {
  double dts;            /* pconst_mod dts */
  double oncc;           /* pconst_mod oncc */
  double onbc;           /* pconst_mod onbc */
  double dwndmix;        /* pconst_mod dwndmix */
  double gamma;          /* pconst_mod gamma (1/s) */
  double od0;            /* pconst_mod od0 */
  double od0cp;          /* pconst_mod od0cp */
  double ah;             /* hmix_del4 ah */
  double area_t;         /* grid area_t (global ocean surface area) */
  int nss;               /* pconst_mod nss */
  int boundary_restore;  /* pconst_mod boundary_restore (1 = 15-day restoring) */
  int adv_tracer;        /* lt_adv_scheme from pconst_mod adv_tracer (0 = tspas) */
  int simple_assm;       /* 1 = tracer_7's nudging toward LT_F_RESTORE_AT in the levels k < ktv
                            (tracer.cpp:1595-1611; 5-day time scale, weaker below level 45), with
                            its term written to LT_F_DT_RESTORE; FP64 form only.  The reference's
                            tracer_ passes 0 (tracer.cpp:1877-1879). */
  int ktv;               /* levels the nudging reaches (the reference's d_ktv) */
} lt_params;

typedef struct lt_domain lt_domain;

/* --- domain lifecycle ---------------------------------------------------- */
/* Allocates the device arena for one domain on the current device.
 * Replaces cudainit (cuda_init.cpp:372-707) for the tracer working set. */
int lt_create(const lt_grid* grid, const lt_params* params, lt_domain** out);
int lt_destroy(lt_domain* dom);
int lt_set_params(lt_domain* dom, const lt_params* params);
/* Bytes one domain of this grid holds on the device (admission control). */
size_t lt_domain_bytes(const lt_grid* grid);

/* --- data movement (host pointers; synchronous on the domain's stream) --- */
int lt_set_field(lt_domain* dom, int field, const void* host_src, size_t nbytes);
int lt_get_field(lt_domain* dom, int field, void* host_dst, size_t nbytes);
/* Device-to-device variants (pointers into the caller's device memory). */
int lt_set_field_device(lt_domain* dom, int field, const void* dev_src, size_t nbytes);
int lt_get_field_device(lt_domain* dom, int field, void* dev_dst, size_t nbytes);
/* Derive KMU, KMTN/S/E/W, OHBT, OHBU, ODZP, ODZT on the device from KMT
 * (ghosts filled) and DZP, as boundary.F90:24-52 and grid.F90:1097-1106,
 * 1343-1346, 2030-2051 do on the host. */
int lt_derive_masks(lt_domain* dom);

/* --- the step ------------------------------------------------------------ */
/* Advance nsteps tracer steps with frozen dynamics inputs: each step reads
 * UTF/VTF/UTL/VTL/H0F/H0L/AKT as given and writes the scaled copies to the
 * *_OUT fields.  Asynchronous on the domain's stream. */
int lt_step(lt_domain* dom, int nsteps);
/* One step taking this step's surface forcing from HOST buffers (swv, nswv,
 * sst, sss, fresh, seaice; each [jmt][imt] f64, any may be NULL to keep the
 * resident field; pinned memory makes the copies asynchronous, on a copy
 * stream of the domain, overlapped with the step's continuity) and returning
 * fw_norm2 (fw_norm2_out) and, if content2_out is not NULL, the two global
 * tracer integrals sum(tarea*dzp*vit*tracer).  Synchronous. */
int lt_step_host(lt_domain* dom, const double* const forcing6[6], double* fw_norm2_out, double* content2_out);
/* The same step, asynchronous: enqueues the forcing copies, the step and the
 * reads of fw_norm2 (and the integrals) into the given host addresses, and
 * returns.  The domain keeps two device sets of the six forcing fields (the
 * second allocated on the first call) and the step reads the set this call
 * filled, so a step's copies overlap the previous step's work.  Host buffers
 * must stay unchanged, and the outputs unread, until lt_sync; pinned memory
 * makes the copies asynchronous.  A NULL field keeps the previous step's
 * values.  A batch holding the domain picks up the swapped set at its next
 * step (its descriptors are rebuilt).  No counterpart in the reference,
 * whose tracer_ copies synchronously (tracer.cpp:1838). */
int lt_step_host_async(lt_domain* dom, const double* const forcing6[6], double* fw_norm2_out, double* content2_out);
/* Convective adjustment of the current state (convadj.cpp:29-288). */
int lt_convadj(lt_domain* dom);

/* Parameters of the sea-ice adjustment (icesnow.cpp:15-85). */
typedef struct {
  double tbice;          /* freezing point of sea water, degC: pconst_mod tbice (constant_mod.F90:168, -1.8) */
  double cp;             /* heat capacity of sea water: pconst_mod cp (constant_mod.F90:164, 3996.0) */
  double latice;         /* latent heat of fusion, J/kg: SHR_CONST_LATICE (shr_const_mod.h:51, 3.337e5) */
  int reset_qice;        /* 1: QICE set to zero first, as the FRC_CORE build does (icesnow.cpp:76-78);
                            0: QICE carries over between calls */
} lt_icesnow_params;
/* The reference's values: tbice -1.8, cp 3996.0, latice 3.337e5, reset_qice 1
 * (its def-undef.h defines FRC_CORE). */
void lt_icesnow_defaults(lt_icesnow_params* p);
/* Sea-ice adjustment of the current state over every point of the domain,
 * halo included (icesnow_cu, icesnow.cpp:15-68): where the surface T of an
 * ocean column is below tbice, the deficit goes to QICE, S(level 0) gains
 * the brine term and T is set to tbice; where QICE is positive and the
 * surface T is above tbice, ice melts back (T and S lowered, QICE reduced);
 * finally T at every level is raised to tbice where below.  p NULL means
 * lt_icesnow_defaults.  Asynchronous on the domain's stream. */
int lt_icesnow(lt_domain* dom, const lt_icesnow_params* p);

/* --- Canuto turbulence closure (turb_cu, readyc.cpp:1456-1612) ------------ */
/* Table sizes of the reference's canuto_mod.h (mt, mt0, n_theta_r_oct). */
#define LT_TURB_MT 1462
#define LT_TURB_MT0 400
#define LT_TURB_NTHETA 75
#define LT_TURB_N1 (2 * LT_TURB_MT + 1)       /* entries of the Ri-type tables */
#define LT_TURB_NB (4 * LT_TURB_NTHETA + 1)   /* entries of the background tables */
/* The closure's tables, as canuto_ini_2002.F90 leaves them in canuto_mod and
 * turbinit (turb_init.cpp:37-88) copies them to the device.  Host pointers. */
typedef struct {
  const double* rib;        /* [N1] Richardson-number grid, linear |i| <= MT0, geometric beyond */
  const int* irimax;        /* [N1] last realizable Ri index for each Ri_d index (-MT .. MT) */
  const double* slq2b;      /* [N1][N1] (S l/q)^2, row = Ri_d index, column = Ri index */
  const double* smb;        /* [N1][N1] S_M */
  const double* shb;        /* [N1][N1] S_H */
  const double* ssb;        /* [N1][N1] S_S */
  const double* and2on2a1;  /* [N1] zero-shear table grid of N_d^2/N^2 */
  const double* amtaun2a1;  /* [N1] -(tau N)^2 of the zero-shear table */
  const double* sma1;       /* [N1] zero-shear S_M, S_H, S_S */
  const double* sha1;
  const double* ssa1;
  const double* back_ra_r;  /* [NB] background radius in the (Ri_T, Ri_C) plane vs angle */
  const double* sm_r1;      /* [NB] background S_M, S_H, S_S, (S l/q)^2 vs angle */
  const double* sh_r1;
  const double* ss_r1;
  const double* slq2_r1;
  double rri;               /* ratio of adjacent Ri in the geometric part (canuto_mod rri) */
  double rnd2on2;           /* the same for the zero-shear table */
  double dri;               /* Ri step of the linear part */
  double deltheta_r;        /* angle step of the background tables */
  double b1;                /* B_1 */
  double theta_rcrp;        /* critical angles */
  double theta_rcrn;
  double dand2on2;          /* N_d^2/N^2 step of the zero-shear table */
} lt_turb_tables;
typedef struct lt_turb_tab lt_turb_tab;
/* Copy the tables to the current device once; a table set serves any number
 * of domains on that device. */
int lt_turb_tables_create(const lt_turb_tables* host, lt_turb_tab** out);
int lt_turb_tables_destroy(lt_turb_tab* tab);
typedef struct {
  int ncc;                  /* pconst_mod ncc (akt is divided by it) */
  double dfricmx;           /* pconst_mod dfricmx: upper bound of the diffusivities (m^2/s) */
} lt_turb_params;
/* The closure over the current state, every column with i in 1..imt-2,
 * j in 1..jmt-2 and kmt >= 1 (turb_cu with TIDEMIX, the reference's
 * configuration): writes AKT (levels 0..km-2; the tracer step's mixing, as f32
 * in a mixed-precision domain), AKMT, AK_TIDE, AMLD and the tidal
 * diagnostics; reads T of AT, DZP, KMT, dwndmix of the domain's parameters and
 * the turbulence inputs (RIT .. ZKP).  AKMT, AK_TIDE and AMLD are zero where
 * no column is computed, as after the reference's memsets (readyc.cpp:1642,
 * 1647, 1668).  Asynchronous on the domain's stream.  The reference leaves two
 * locals unset on some paths (the buoyancy frequency when N^2 < 0 at the top
 * level, the background S l/q where Ri <= 0 before any Ri > 0); they start at
 * zero here. */
int lt_turb(lt_domain* dom, const lt_turb_tab* tab, const lt_turb_params* p);

/* --- momentum biharmonic friction (readyc.cpp:343-577) -------------------- */
typedef struct {
  double am;             /* hmix_del4 am (AM_BIHAR) */
  double c0f;            /* pconst_mod c0f (bottom drag coefficient) */
} lt_del4u_params;
/* The biharmonic friction of UP, VP with the flow-dependent factor (readyc_'s
 * BIHAR sequence, readyc.cpp:1754-1775: hdel4_div, hdel4_grad, hdel4_zcurl,
 * hdel4_grad, hdiffu_del4_0, hdiffu_del4_1) for a domain that is one block
 * (ib = jb = 3, ie = imt-2, je = jmt-2 in the reference's 1-based block
 * bounds): DLU and DLV are increased by it over i in 1..imt-2, j in 1..jmt-2
 * and WKA_DRAG = c0f*sqrt(up^2 + vp^2) everywhere.  Reads DXU, DYU, HTW, HTS,
 * TAREA_R, KMT, KMU of the domain and the momentum fields above.  One fused
 * kernel per 32x8 tile and level; FP64 with the reference's operation order,
 * bit-identical to it.  Asynchronous on the domain's stream. */
int lt_hdiffu_del4(lt_domain* dom, const lt_del4u_params* p);
/* Global tracer integrals sum(tarea*dzp*vit*tracer) over the interior, f64,
 * fixed-order pairwise tree (deterministic). out2[0] = T, out2[1] = S. */
int lt_tracer_content(lt_domain* dom, double* out2);
/* No counterpart in the reference.  The same integrals as lt_tracer_content,
 * bit-identical, for callers that cannot let a library allocate device memory
 * (a host model that owns all of HBM through its own pool or data regions).
 * Every argument is a device pointer the caller owns, in the layouts of
 * lt_set_field: at = AT [2][km][ny+4][nx+4], tarea = TAREA and kmt = KMT
 * [ny+4][nx+4], dzp = DZP [km]; out2[0..1] receives T and S.  stream is a
 * cudaStream_t (NULL = legacy default stream); the call only enqueues work.
 * Partial sums live in a fixed 2 MiB device array inside the library (held on
 * every GPU that loads it until exit), which caps nx*ny*km at about 5.3e8
 * cells; larger sizes return LT_E_INVALID.  All calls share that array, so
 * calls that overlap on the GPU race.  The first call on each device looks up
 * the array's address and should come before any stream capture; later calls
 * outside a capture look it up again (so a call after cudaDeviceReset finds
 * the reloaded array).  Allocates nothing. */
int lt_tracer_content_noalloc(const double* at, const double* tarea, const double* dzp, const int* kmt,
                              int nx, int ny, int km, double* out2, void* stream);
/* fw_norm2 of the last step (tracer.cpp:1862-1865). */
int lt_fw_norm2(lt_domain* dom, double* out);
int lt_sync(lt_domain* dom);
/* Scan AT for NaN/Inf; LT_E_NUMERIC if any. */
int lt_check_numeric(lt_domain* dom, long long* bad_count);
/* Elapsed device time (ms) of the last lt_step call, CUDA events. */
int lt_last_step_ms(lt_domain* dom, float* ms);
/* Record the start (which = 0) or end (which = 1) event that lt_last_step_ms
 * measures, on the domain's stream, around any sequence of calls. */
int lt_mark(lt_domain* dom, int which);
/* Per-phase device timing: lt_profile(dom, 1) records CUDA events around the
 * six launch phases of each step; lt_phase_ms sums them over the recorded
 * steps into ms[0..5] = surface fluxes, SSS-norm sum, net halo, continuity
 * (with the SSH mean it needs), tracer column kernel, state halo, and returns
 * the number of steps.  The continuity is launched first (it needs no
 * forcing); with lt_step_host, the surface-flux phase includes any wait for
 * the forcing copies still in flight after it. */
int lt_profile(lt_domain* dom, int on);
int lt_phase_ms(lt_domain* dom, float* ms, int nphase);
/* How the column kernels' level slots are filled: 1 = TMA boxes (the default
 * where the row pitch allows 16-byte strides; refused with LT_E_INVALID
 * elsewhere), 0 = per-thread asynchronous copies into the same slots (the
 * default where it does not).  The results are the same bits either way. */
int lt_use_tma(lt_domain* dom, int on);
/* Failure-detection hook.  Each level wait of the TMA-fed column kernels polls
 * its mbarrier at most `polls` times (default 2^24) before the CTA records a
 * timeout, drains the boxes it has in flight and returns; lt_sync and
 * lt_step_host then return LT_E_TIMEOUT.  0 makes every wait give up at once,
 * which exercises that path without any fault. */
int lt_set_wait_limit(lt_domain* dom, unsigned polls);
/* Kernels this library has launched in this process (all domains). */
long long lt_launch_count(void);

/* --- reference-named shims ---------------------------------------------- */
/* Bind the domain the shims act on (the reference uses process globals). */
int lt_shim_bind(lt_domain* dom);
/* tracer.cpp:1701: one step with the reference's side effects on the bound
 * domain: UTF/VTF/H0F scaled in place, VTL left holding S with halo. */
void tracer_(int ii);
/* convadj.cpp:290: convective adjustment of the bound domain. */
void convadj_(void);
/* icesnow.cpp:70 (called after tracer_ in stepon.cpp:71): sea-ice adjustment
 * of the bound domain with the reference's parameters (lt_icesnow_defaults). */
void icesnow_(void);

/* --- field metadata ------------------------------------------------------ */
/* Upper-case name of a field id without the LT_F_ prefix ("AT", "ATB", ...). */
const char* lt_field_name(int field);
/* Element count of a field for physical sizes nx, ny, km; -1 if invalid. */
long lt_field_count(int field, int nx, int ny, int km);
/* 1 for the int32 mask fields, 0 for f64 fields. */
int lt_field_is_int(int field);
/* 1 for the turbulence closure's fields (LT_F_RIT .. LT_F_WP3_TIDAL) and the
 * momentum friction's fields (LT_F_UP .. LT_F_DYUR), which a domain allocates
 * on the first use of a field of each group. */
int lt_field_on_demand(int field);

/* --- errors, device ------------------------------------------------------ */
const char* lt_last_error(void);
int lt_device_count(int* count);
/* Make device dev current for this library's CUDA runtime on the calling
 * thread (the library carries its own runtime; other runtimes in the
 * process keep their own current device). */
int lt_set_device(int dev);
/* Library version/build id string. */
const char* lt_version(void);

#ifdef __cplusplus
}
#endif
#endif /* LICOM_TRACER_H */
