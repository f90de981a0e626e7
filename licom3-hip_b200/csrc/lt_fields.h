// lt_fields.h - shapes of the lt_field identifiers (host/device agnostic).
#pragma once
#include "../../include/licom_tracer.h"

namespace lt {

enum FieldShape {
  SH_TRACER3 = 0,   // [2][km][jmt][imt]
  SH_TRACERB,       // [2][km+1][jmt][imt]
  SH_LEVEL3,        // [km][jmt][imt]
  SH_W3,            // [km+1][jmt][imt]
  SH_SURF2,         // [jmt][imt]
  SH_SURF2N,        // [2][jmt][imt]
  SH_MASK2,         // [jmt][imt] int32
  SH_COL1,          // [km]
  SH_COEF9,         // [9][km]
  SH_LEVEL3M1,      // [km-1][jmt][imt]
  SH_COL1P          // [km+1]
};

inline int field_shape(int f) {
  switch (f) {
    case LT_F_AT: case LT_F_AKT: case LT_F_RESTORE: case LT_F_AX: case LT_F_AY: case LT_F_AZ:
    case LT_F_DZ: case LT_F_TEND: case LT_F_DT_DIFF: case LT_F_DT_CONV: case LT_F_RESTORE_AT: case LT_F_DT_RESTORE:
      return SH_TRACER3;
    case LT_F_ATB: return SH_TRACERB;
    case LT_F_UTF: case LT_F_VTF: case LT_F_UTL: case LT_F_VTL: case LT_F_UTF_OUT: case LT_F_VTF_OUT:
    case LT_F_PENETRATE: case LT_F_FZ_TIDE: case LT_F_AKMT: case LT_F_AK_TIDE: case LT_F_RICHARDSON:
    case LT_F_FZTIDAL: case LT_F_WP3_TIDAL: case LT_F_UP: case LT_F_VP: case LT_F_DLU: case LT_F_DLV:
    case LT_F_WKA_DRAG:
      return SH_LEVEL3;
    case LT_F_RIT: case LT_F_RICDTTMS: case LT_F_S2T: case LT_F_RICT: return SH_LEVEL3M1;
    case LT_F_ZKP: return SH_COL1P;
    case LT_F_WS: case LT_F_PDENSITY: return SH_W3;
    case LT_F_NET: return SH_SURF2N;
    case LT_F_KMT: case LT_F_KMU: case LT_F_KMTN: case LT_F_KMTS: case LT_F_KMTE: case LT_F_KMTW:
      return SH_MASK2;
    case LT_F_DZP: case LT_F_ODZP: case LT_F_ODZT: case LT_F_PEN: case LT_F_TO: case LT_F_SO:
      return SH_COL1;
    case LT_F_C: return SH_COEF9;
    default: return SH_SURF2;
  }
}

inline bool field_is_int(int f) { return field_shape(f) == SH_MASK2; }

// fields of the turbulence closure and of the momentum friction, each group
// allocated with the domain's first use of any of its fields
inline bool field_is_turb(int f) { return f >= LT_F_RIT && f <= LT_F_WP3_TIDAL; }
inline bool field_is_mom(int f) { return f >= LT_F_UP && f <= LT_F_DYUR; }

inline long field_count(int f, int imt, int jmt, int km) {
  const long A = (long)imt * jmt;
  switch (field_shape(f)) {
    case SH_TRACER3: return 2 * A * km;
    case SH_TRACERB: return 2 * A * (km + 1);
    case SH_LEVEL3: return A * km;
    case SH_W3: return A * (km + 1);
    case SH_SURF2: case SH_MASK2: return A;
    case SH_SURF2N: return 2 * A;
    case SH_COL1: return km;
    case SH_COEF9: return 9L * km;
    case SH_LEVEL3M1: return A * (km - 1);
    case SH_COL1P: return km + 1;
  }
  return 0;
}

inline size_t field_bytes(int f, int imt, int jmt, int km) {
  return (size_t)field_count(f, imt, jmt, km) * (field_is_int(f) ? 4 : 8);
}

}  // namespace lt
