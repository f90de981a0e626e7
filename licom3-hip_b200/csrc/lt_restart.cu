// lt_restart.cu - the reference's restart file (the records of
// ssave-cdf-instant.F90:93-761, read back by inirun.F90:598-679): Fortran
// unformatted sequential records of global f64 fields, read and written on
// the host, and the moves between such a file and a domain.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>
#include "lt_common.cuh"
#include "lt_domain.h"
#include "../../include/licom_restart.h"

using namespace lt;

namespace {

// one Fortran record: 4-byte length, the data, the length again
bool put_record(FILE* f, const void* data, size_t bytes, bool zeros) {
  const uint32_t n = (uint32_t)bytes;
  if (fwrite(&n, 4, 1, f) != 1) return false;
  if (zeros) {
    static const char z[1 << 16] = {};
    size_t left = bytes;
    while (left) {
      const size_t c = left < sizeof(z) ? left : sizeof(z);
      if (fwrite(z, 1, c, f) != c) return false;
      left -= c;
    }
  } else if (fwrite(data, 1, bytes, f) != bytes) {
    return false;
  }
  return fwrite(&n, 4, 1, f) == 1;
}

// one record of exactly `bytes`; into dst, or skipped when dst is null
int get_record(FILE* f, void* dst, size_t bytes, const char* what) {
  uint32_t n0 = 0, n1 = 0;
  if (fread(&n0, 4, 1, f) != 1) {
    set_error("restart: file ends before the %s record", what);
    return LT_E_STATE;
  }
  if (n0 != bytes) {
    set_error("restart: %s record holds %u bytes, %zu expected", what, n0, bytes);
    return LT_E_INVALID;
  }
  if (dst) {
    if (fread(dst, 1, bytes, f) != bytes) {
      set_error("restart: %s record cut short", what);
      return LT_E_STATE;
    }
  } else if (fseek(f, (long)bytes, SEEK_CUR) != 0) {
    set_error("restart: %s record cut short", what);
    return LT_E_STATE;
  }
  if (fread(&n1, 4, 1, f) != 1 || n1 != n0) {
    set_error("restart: %s record's closing length does not match", what);
    return LT_E_INVALID;
  }
  return LT_OK;
}

bool sizes_ok(const lt_restart* r) {
  if (!r || r->nx < 1 || r->ny < 1 || r->km < 1) return false;
  return (size_t)r->nx * r->ny * sizeof(double) < 0x7fffffffu;   // one record, no subrecords
}

struct FileCloser {
  FILE* f;
  ~FileCloser() { if (f) fclose(f); }
};

}  // namespace

extern "C" {

int lt_restart_write(const char* path, const lt_restart* r) {
  if (!path || !sizes_ok(r)) { set_error("lt_restart_write: bad arguments"); return LT_E_INVALID; }
  FILE* f = fopen(path, "wb");
  if (!f) { set_error("lt_restart_write: cannot open %s", path); return LT_E_STATE; }
  FileCloser fc{f};
  const size_t A = (size_t)r->nx * r->ny, rb = A * sizeof(double);
  bool ok = put_record(f, r->h0, rb, !r->h0);
  const double* lv[5] = {r->u, r->v, r->t, r->s, r->ws};
  for (int m = 0; m < 5 && ok; ++m)
    for (int k = 0; k < r->km && ok; ++k) ok = put_record(f, lv[m] ? lv[m] + k * A : nullptr, rb, !lv[m]);
  const double* sf[6] = {r->su, r->sv, r->swv, r->sshf, r->lthf, r->fresh};
  for (int m = 0; m < 6 && ok; ++m) ok = put_record(f, sf[m], rb, !sf[m]);
  const int32_t date[2] = {r->number_month, r->number_day};
  if (ok) ok = put_record(f, date, sizeof(date), false);
  if (!ok || fflush(f) != 0) { set_error("lt_restart_write: write to %s failed", path); return LT_E_STATE; }
  return LT_OK;
}

int lt_restart_read(const char* path, lt_restart* r) {
  if (!path || !sizes_ok(r)) { set_error("lt_restart_read: bad arguments"); return LT_E_INVALID; }
  FILE* f = fopen(path, "rb");
  if (!f) { set_error("lt_restart_read: cannot open %s", path); return LT_E_STATE; }
  FileCloser fc{f};
  const size_t A = (size_t)r->nx * r->ny, rb = A * sizeof(double);
  int rc = get_record(f, r->h0, rb, "h0");
  double* lv[5] = {r->u, r->v, r->t, r->s, r->ws};
  const char* lname[5] = {"u", "v", "T", "S", "ws"};
  for (int m = 0; m < 5 && !rc; ++m)
    for (int k = 0; k < r->km && !rc; ++k) rc = get_record(f, lv[m] ? lv[m] + k * A : nullptr, rb, lname[m]);
  double* sf[6] = {r->su, r->sv, r->swv, r->sshf, r->lthf, r->fresh};
  const char* sname[6] = {"su", "sv", "swv", "sshf", "lthf", "fresh"};
  for (int m = 0; m < 6 && !rc; ++m) rc = get_record(f, sf[m], rb, sname[m]);
  int32_t date[2] = {0, 0};
  if (!rc) rc = get_record(f, date, sizeof(date), "date");
  if (rc) return rc;
  r->number_month = date[0];
  r->number_day = date[1];
  return LT_OK;
}

int lt_domain_save_restart(lt_domain* d, const char* path, const lt_restart* extra) {
  if (!d || !path) { set_error("lt_domain_save_restart: bad arguments"); return LT_E_INVALID; }
  Arena& a = d->a;
  const int nx = a.nx, ny = a.ny, km = a.km, imt = a.imt;
  if (extra && (extra->nx != nx || extra->ny != ny || extra->km != km)) {
    set_error("lt_domain_save_restart: extra has other sizes than the domain");
    return LT_E_INVALID;
  }
  const size_t A = (size_t)nx * ny;
  std::vector<double> at((size_t)2 * a.F), ws((size_t)a.FB), h0f(a.A), swv(a.A), fresh(a.A);
  std::vector<int> kmt(a.A), kmu(a.A);
  int rc;
  if ((rc = lt_get_field(d, LT_F_AT, at.data(), at.size() * 8)) || (rc = lt_get_field(d, LT_F_WS, ws.data(), ws.size() * 8)) ||
      (rc = lt_get_field(d, LT_F_H0F, h0f.data(), h0f.size() * 8)) ||
      (rc = lt_get_field(d, LT_F_SWV, swv.data(), swv.size() * 8)) ||
      (rc = lt_get_field(d, LT_F_FRESH, fresh.data(), fresh.size() * 8)) ||
      (rc = lt_get_field(d, LT_F_KMT, kmt.data(), kmt.size() * 4)) ||
      (rc = lt_get_field(d, LT_F_KMU, kmu.data(), kmu.size() * 4)))
    return rc;
  // the physical grid without halo
  auto inner2 = [&](const double* src, std::vector<double>& dst) {
    dst.resize(A);
    for (int j = 0; j < ny; ++j) std::memcpy(&dst[(size_t)j * nx], src + (size_t)(j + 2) * imt + 2, nx * 8);
  };
  std::vector<double> t(A * km), s(A * km), w(A * km), h0, sw, fr, tmp;
  for (int k = 0; k < km; ++k) {
    inner2(at.data() + (size_t)k * a.A, tmp);
    std::memcpy(&t[k * A], tmp.data(), A * 8);
    inner2(at.data() + (size_t)a.F + (size_t)k * a.A, tmp);
    std::memcpy(&s[k * A], tmp.data(), A * 8);
    inner2(ws.data() + (size_t)k * a.A, tmp);
    std::memcpy(&w[k * A], tmp.data(), A * 8);
  }
  inner2(h0f.data(), h0);
  inner2(swv.data(), sw);
  inner2(fresh.data(), fr);
  std::vector<char> land_t(A), land_u(A);
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) {
      const size_t q = (size_t)(j + 2) * imt + i + 2;
      land_t[(size_t)j * nx + i] = kmt[q] < 1;   // vit(:,:,1) < 0.5
      land_u[(size_t)j * nx + i] = kmu[q] < 1;   // viv(:,:,1) < 0.5
    }
  // the reference zeroes the surface fields over land before writing them
  auto masked = [&](const double* src, const std::vector<char>& land, std::vector<double>& dst) -> double* {
    if (!src) return nullptr;
    dst.assign(src, src + A);
    for (size_t q = 0; q < A; ++q)
      if (land[q]) dst[q] = 0.0;
    return dst.data();
  };
  std::vector<double> msu, msv, msh, mlt;
  for (size_t q = 0; q < A; ++q)
    if (land_t[q]) { sw[q] = 0.0; fr[q] = 0.0; }
  lt_restart r{};
  r.nx = nx; r.ny = ny; r.km = km;
  r.h0 = h0.data(); r.t = t.data(); r.s = s.data(); r.ws = w.data(); r.swv = sw.data(); r.fresh = fr.data();
  if (extra) {
    r.u = extra->u; r.v = extra->v;
    r.su = masked(extra->su, land_u, msu);
    r.sv = masked(extra->sv, land_u, msv);
    r.sshf = masked(extra->sshf, land_t, msh);
    r.lthf = masked(extra->lthf, land_t, mlt);
    r.number_month = extra->number_month;
    r.number_day = extra->number_day;
  }
  return lt_restart_write(path, &r);
}

int lt_domain_load_restart(lt_domain* d, const char* path, lt_restart* extra) {
  if (!d || !path) { set_error("lt_domain_load_restart: bad arguments"); return LT_E_INVALID; }
  Arena& a = d->a;
  const int nx = a.nx, ny = a.ny, km = a.km, imt = a.imt;
  if (extra && (extra->nx != nx || extra->ny != ny || extra->km != km)) {
    set_error("lt_domain_load_restart: extra has other sizes than the domain");
    return LT_E_INVALID;
  }
  const size_t A = (size_t)nx * ny;
  std::vector<double> t(A * km), s(A * km), h0(A);
  lt_restart r{};
  r.nx = nx; r.ny = ny; r.km = km;
  r.h0 = h0.data(); r.t = t.data(); r.s = s.data();
  if (extra) { r.u = extra->u; r.v = extra->v; }
  int rc = lt_restart_read(path, &r);
  if (rc) return rc;
  if (extra) { extra->number_month = r.number_month; extra->number_day = r.number_day; }
  // interior into the domain's layout, halo and fold on the device
  std::vector<double> at((size_t)2 * a.F, 0.0), h0f(a.A, 0.0);
  for (int n = 0; n < 2; ++n)
    for (int k = 0; k < km; ++k)
      for (int j = 0; j < ny; ++j)
        std::memcpy(&at[(size_t)n * a.F + (size_t)k * a.A + (size_t)(j + 2) * imt + 2],
                    (n ? s.data() : t.data()) + k * A + (size_t)j * nx, nx * 8);
  for (int j = 0; j < ny; ++j) std::memcpy(&h0f[(size_t)(j + 2) * imt + 2], &h0[(size_t)j * nx], nx * 8);
  if ((rc = lt_set_field(d, LT_F_AT, at.data(), at.size() * 8)) ||
      (rc = lt_set_field(d, LT_F_H0F, h0f.data(), h0f.size() * 8)))
    return rc;
  cudaStream_t st = d->stream;
  if ((rc = launch_halo_r8(a.at[a.cur], 2 * km, imt, a.jmt, a.ew_cyclic, a.tripole, st)) ||
      (rc = launch_halo_r8(a.h0f, 1, imt, a.jmt, a.ew_cyclic, a.tripole, st)))
    return rc;
  const size_t fb = sizeof(double) * a.F;
  LT_CUDA_OK(cudaMemcpyAsync(a.at[a.cur ^ 1], a.at[a.cur], 2 * fb, cudaMemcpyDeviceToDevice, st));
  // NEXTSTEP: atb(1..km) = at (nextstep.F90:27-28); level 0 stays as it is
  for (int b = 0; b < 2; ++b)
    for (int n = 0; n < 2; ++n)
      LT_CUDA_OK(cudaMemcpyAsync(a.atb[b] + (size_t)n * a.FB + a.A, a.at[a.cur] + (size_t)n * a.F, fb,
                                 cudaMemcpyDeviceToDevice, st));
  LT_CUDA_OK(cudaStreamSynchronize(st));
  d->have_state = true;
  return LT_OK;
}

}  // extern "C"
