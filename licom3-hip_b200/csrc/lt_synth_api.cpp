// lt_synth_api.cpp - C ABI over the host side of the synthetic domain builder.
#include <cstring>
#include <new>
#include "lt_synth.h"
#include "lt_fields.h"
#include "../../include/licom_synth.h"

struct lt_synth {
  lt::Domain d;
};

namespace {
lt::SynthConfig to_cfg(const lt_synth_config& c) {
  lt::SynthConfig s;
  s.nx = c.nx; s.ny = c.ny; s.km = c.km;
  s.lat_s = c.lat_s; s.lat_n = c.lat_n;
  s.dz_top = c.dz_top; s.dz_bot = c.dz_bot; s.depth = c.depth;
  s.umax = c.umax; s.seed = c.seed; s.forced = c.forced;
  s.cap_north = c.cap_north; s.cap_south = c.cap_south;
  s.ew_cyclic = c.ew_cyclic; s.tripole = c.tripole;
  s.land_frac = c.land_frac; s.member = c.member; s.tpert = c.tpert;
  s.ah_bihar = c.ah_bihar;
  s.hypsometry = c.hypsometry;
  return s;
}
}  // namespace

extern "C" {

void lt_synth_defaults(lt_synth_config* c) {
  lt::SynthConfig s;
  c->nx = s.nx; c->ny = s.ny; c->km = s.km;
  c->lat_s = s.lat_s; c->lat_n = s.lat_n;
  c->dz_top = s.dz_top; c->dz_bot = s.dz_bot; c->depth = s.depth;
  c->umax = s.umax; c->seed = s.seed; c->forced = s.forced;
  c->cap_north = s.cap_north; c->cap_south = s.cap_south;
  c->ew_cyclic = s.ew_cyclic; c->tripole = s.tripole;
  c->land_frac = s.land_frac; c->member = s.member; c->tpert = s.tpert;
  c->ah_bihar = s.ah_bihar;
  c->hypsometry = s.hypsometry;
}

int lt_synth_build(const lt_synth_config* cfg, lt_synth** out) {
  if (!cfg || !out) return LT_E_INVALID;
  if (cfg->nx < 8 || cfg->ny < 8 || cfg->km < 3 || (cfg->tripole && (cfg->nx % 2))) return LT_E_INVALID;
  lt_synth* s = new (std::nothrow) lt_synth;
  if (!s) return LT_E_OOM;
  try {
    s->d = lt::build_domain(to_cfg(*cfg));
  } catch (...) {
    delete s;
    return LT_E_OOM;
  }
  *out = s;
  return LT_OK;
}

int lt_synth_free(lt_synth* s) {
  delete s;
  return LT_OK;
}

int lt_synth_params(const lt_synth* s, lt_params* p) {
  if (!s || !p) return LT_E_INVALID;
  const lt::Domain& d = s->d;
  p->dts = d.dts; p->oncc = d.oncc; p->onbc = d.onbc; p->dwndmix = d.dwndmix; p->gamma = d.gamma;
  p->od0 = d.od0; p->od0cp = d.od0cp; p->ah = d.ah; p->area_t = d.area_t; p->nss = d.nss;
  p->boundary_restore = 0;
  p->adv_tracer = LT_ADV_TSPAS;
  p->simple_assm = 0;
  p->ktv = 0;
  return LT_OK;
}

int lt_synth_grid(const lt_synth* s, lt_grid* g) {
  if (!s || !g) return LT_E_INVALID;
  g->nx = s->d.nx; g->ny = s->d.ny; g->km = s->d.km;
  g->precision = LT_PREC_FP64; g->diagnostics = 0;
  g->ew_cyclic = s->d.cfg.ew_cyclic; g->tripole = s->d.cfg.tripole;
  return LT_OK;
}

long lt_synth_field_count(const lt_synth* s, int f) {
  if (!s || f < 0 || f >= LT_F_COUNT) return -1;
  return lt::field_count(f, s->d.imt, s->d.jmt, s->d.km);
}

int lt_synth_field(const lt_synth* s, int f, void* dst, size_t nbytes) {
  if (!s) return LT_E_INVALID;
  return lt_synth_field_rows(s, f, s->d.jmt, dst, nbytes);
}

int lt_synth_field_rows(const lt_synth* s, int f, int rows, void* dst, size_t nbytes) {
  if (!s || !dst || f < 0 || f >= LT_F_COUNT) return LT_E_INVALID;
  const lt::Domain& d = s->d;
  if (rows < 5 || rows > d.jmt) return LT_E_INVALID;
  const size_t need = lt::field_bytes(f, d.imt, rows, d.km);
  if (nbytes != need) return LT_E_INVALID;
  const long F = (long)d.imt * rows * d.km;
  double* o = static_cast<double*>(dst);
  // 2-D fields [jmt][imt]: the leading rows
  auto copy = [&](const void* src) { std::memcpy(dst, src, nbytes); return LT_OK; };
  switch (f) {
    case LT_F_AT: case LT_F_RESTORE: {
      std::vector<double> atb(2 * (size_t)d.imt * rows * (d.km + 1));
      lt::fill_state(d, o, atb.data(), rows);
      return LT_OK;
    }
    case LT_F_ATB: {
      std::vector<double> at(2 * (size_t)F);
      lt::fill_state(d, at.data(), o, rows);
      return LT_OK;
    }
    case LT_F_UTF: case LT_F_VTF: case LT_F_UTL: case LT_F_VTL:
      lt::fill_velocity_one(d, f - LT_F_UTF, o, rows);
      return LT_OK;
    case LT_F_AKT: lt::fill_akt(d, o, rows); return LT_OK;
    case LT_F_H0F: return copy(d.h0f.data());
    case LT_F_H0L: return copy(d.h0l.data());
    case LT_F_SWV: return copy(d.swv.data());
    case LT_F_NSWV: return copy(d.nswv.data());
    case LT_F_SST: return copy(d.sst.data());
    case LT_F_SSS: return copy(d.sss.data());
    case LT_F_FRESH: return copy(d.fresh.data());
    case LT_F_SEAICE: return copy(d.seaice.data());
    case LT_F_TAREA: return copy(d.tarea.data());
    case LT_F_TAREA_R: return copy(d.tarea_r.data());
    case LT_F_HTW: return copy(d.htw.data());
    case LT_F_HTS: return copy(d.hts.data());
    case LT_F_HUN: return copy(d.hun.data());
    case LT_F_HUE: return copy(d.hue.data());
    case LT_F_DXU: return copy(d.dxu.data());
    case LT_F_DYU: return copy(d.dyu.data());
    case LT_F_AHF: return copy(d.ahf.data());
    case LT_F_DTN: return copy(d.dtn.data());
    case LT_F_DTS: return copy(d.dts_.data());
    case LT_F_DTE: return copy(d.dte.data());
    case LT_F_DTW: return copy(d.dtw.data());
    case LT_F_OHBT: return copy(d.ohbt.data());
    case LT_F_OHBU: return copy(d.ohbu.data());
    case LT_F_AU0: return copy(d.au0.data());
    case LT_F_AUS: return copy(d.aus.data());
    case LT_F_AUW: return copy(d.auw.data());
    case LT_F_AUSW: return copy(d.ausw.data());
    case LT_F_KMT: return copy(d.kmt.data());
    case LT_F_KMU: return copy(d.kmu.data());
    case LT_F_KMTN: return copy(d.kmtn.data());
    case LT_F_KMTS: return copy(d.kmts.data());
    case LT_F_KMTE: return copy(d.kmte.data());
    case LT_F_KMTW: return copy(d.kmtw.data());
    case LT_F_DZP: return copy(d.dzp.data());
    case LT_F_ODZP: return copy(d.odzp.data());
    case LT_F_ODZT: return copy(d.odzt.data());
    case LT_F_PEN: return copy(d.pen.data());
    case LT_F_TO: return copy(d.to.data());
    case LT_F_SO: return copy(d.so.data());
    case LT_F_C: return copy(d.c9.data());
    default:
      std::memset(dst, 0, nbytes);
      return LT_OK;
  }
}

}  // extern "C"

// accessor for the device-side uploader (lt_synth_dev.cu)
const lt::Domain* lt_synth_domain(const lt_synth* s) { return s ? &s->d : nullptr; }
