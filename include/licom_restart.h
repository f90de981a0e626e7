/*
 * licom_restart.h - the reference's restart file, read and written here, so
 * that states move between LICOM3-HIP and this library.
 *
 * Format (the records ssave-cdf-instant.F90:93-761 writes to fort.22 .. fort.27
 * and inirun.F90:598-679 reads back, in that order, from one file): Fortran
 * unformatted sequential records, each framed by its length in bytes as a
 * 4-byte little-endian integer before and after, each holding one global
 * field buffer(imt_global, jmt_global) of f64 (i fastest, the physical grid
 * without halo, j = 1 the northern row as in the model):
 *   h0;  u(k), k = 1..km;  v(k);  at(k, T);  at(k, S);  ws(k);
 *   su;  sv;  swv;  sshf;  lthf;  fresh;  then one record of two 4-byte
 *   integers (number_month, number_day).
 * The writer zeroes su, sv over land (viv < 0.5, no wet U level) and swv,
 * sshf, lthf, fresh over land (vit < 0.5) before writing them, as the
 * reference does.
 */
#ifndef LICOM_RESTART_H
#define LICOM_RESTART_H

#include "licom_tracer.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int nx, ny, km;                 /* imt_global, jmt_global, km */
  double* h0;                     /* [ny][nx] */
  double *u, *v;                  /* [km][ny][nx] */
  double *t, *s;                  /* [km][ny][nx] tracer_mod at(:,:,k,1), at(:,:,k,2) */
  double* ws;                     /* [km][ny][nx] */
  double *su, *sv, *swv, *sshf, *lthf, *fresh;   /* [ny][nx] */
  int number_month, number_day;
} lt_restart;

/* Write a restart file.  A NULL array is written as zeros.  LT_E_INVALID on
 * bad sizes, LT_E_STATE if the file cannot be written. */
int lt_restart_write(const char* path, const lt_restart* r);
/* Read a restart file written by the reference or by lt_restart_write; the
 * sizes in r must match the file's records.  NULL arrays are skipped.
 * LT_E_INVALID on a record of unexpected length, LT_E_STATE if the file
 * cannot be read. */
int lt_restart_read(const char* path, lt_restart* r);

/* Restart of a domain: save writes the domain's current T and S (AT), the
 * vertical velocity (WS, levels 0..km-1), h0 (H0F), SWV and FRESH, with u, v,
 * su, sv, sshf, lthf and the date from `extra` (NULL arrays as zeros; extra
 * may be NULL).  load sets AT from the file's T and S with the halo and fold
 * of the domain, then, as NEXTSTEP does after the reference reads its restart
 * (nextstep.F90:19-44): ATB levels 1..km = AT, H0F = h0, UTF, VTF = u, v;
 * it also returns u, v and the date in `extra` if given (arrays may be
 * NULL).  Synchronous. */
int lt_domain_save_restart(lt_domain* dom, const char* path, const lt_restart* extra);
int lt_domain_load_restart(lt_domain* dom, const char* path, lt_restart* extra);

#ifdef __cplusplus
}
#endif

#endif
