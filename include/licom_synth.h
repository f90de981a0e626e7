/*
 * licom_synth.h - seeded synthetic LICOM tracer domains (C ABI).
 *
 * Builds every input of the tracer step from a seed: a global lat-lon grid in
 * LICOM order with halo 2, KMT from smoothed noise and the masks derived from
 * it, stretched vertical levels, T/S, velocities from a per-level
 * streamfunction, log-uniform AKT and (optionally) surface forcing.  The
 * reference reads these from NetCDF/binary files (rdriver.F90, inirun.F90,
 * grid.F90); this library stands in for them with synthetic data of the
 * benchmark configurations' shapes.
 */
#ifndef LICOM_SYNTH_H
#define LICOM_SYNTH_H
#include <stddef.h>
#include <stdint.h>
#include "licom_tracer.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int nx, ny, km;
  double lat_s, lat_n;        /* centre latitudes of the southern/northern physical rows (deg) */
  double dz_top, dz_bot, depth;
  double umax;                /* largest surface speed, m/s */
  uint64_t seed;
  int forced;                 /* 1: seeded surface forcing and sea-surface height */
  int cap_north, cap_south;   /* land rows forced at the northern/southern physical edge */
  int ew_cyclic, tripole;
  double land_frac;
  uint32_t member;            /* ensemble member (0 = unperturbed) */
  double tpert;               /* K, std of the member's T perturbation */
  double ah_bihar;            /* m^4/s; 0 = -min(1e17, half the grid's explicit stability limit) */
  int hypsometry;             /* ocean depths: 0 = linear in the land field above its threshold (3 .. km
                                 levels, mostly shallow); 1 = the global ocean's area-depth curve
                                 (mean depth about 3.7 km, 30 % of the ocean deeper than 5 km) */
} lt_synth_config;

typedef struct lt_synth lt_synth;

/* Fill cfg with the defaults of a 1-degree 360 x 196 x 30 domain. */
void lt_synth_defaults(lt_synth_config* cfg);
int lt_synth_build(const lt_synth_config* cfg, lt_synth** out);
int lt_synth_free(lt_synth* s);
int lt_synth_params(const lt_synth* s, lt_params* out);
int lt_synth_grid(const lt_synth* s, lt_grid* out);
/* Host copy of any input field (3-D fields are generated on the host). */
int lt_synth_field(const lt_synth* s, int field, void* dst, size_t nbytes);
/* The same field for the northern band of the domain, rows j < rows (halo
 * included, 5 <= rows <= jmt): 3-D fields are generated for those rows only
 * (cell values identical to lt_synth_field's), 2-D fields are their leading
 * rows, 1-D fields whole.  nbytes is the byte size of the band's field. */
int lt_synth_field_rows(const lt_synth* s, int field, int rows, void* dst, size_t nbytes);
/* Element count of a field for this domain. */
long lt_synth_field_count(const lt_synth* s, int field);
/* Upload every input of a domain: 2-D/1-D fields from the host, 3-D fields
 * generated on the device (bit-identical to lt_synth_field). */
int lt_synth_upload(const lt_synth* s, lt_domain* dom);

#ifdef __cplusplus
}
#endif
#endif /* LICOM_SYNTH_H */
