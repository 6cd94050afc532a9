// Restart files in the reference's checkpoint format, MPCNSRST version 1
// (IOModule::WriteRestartBinFile / ReadRestartBinFile,
// src/6_io/IOModule_Bin.cpp:168-420), holding the fields the reference's
// Mercury solver checkpoints: U_H, U_Na, B_xi, B_eta, B_zeta
// (Z4_Mercury/src/MercurySolver.cpp:33-35).  Layout, native little-endian:
//   "MPCNSRST", int32 version = 1, int32 step, double time,
//   int32 blocks, int32 fields,
//   per field: int32 name length + name bytes, int32 location, int32 ncomp,
//     int32 nghost, then per block: int32 lo[3], int32 hi[3] (the FieldBlock
//     range [-nghost, n + stagger + nghost)), int32 active flag and, when
//     active, the doubles in (i, j, k, component) order.
// The reader follows the reference's rules: fields it does not restore are
// skipped, and a restored field must match location, component count,
// nghost, block count and ranges exactly.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>

#include "mercury_mhd.h"
#include "mhd_error.h"
#include "mhd_layout.cuh"

namespace {

struct StateField {
  const char *name;
  int field;
};
// in the reference's restart list order
constexpr StateField kState[MHD_RESTART_FIELDS] = {
    {"U_H", MHD_U_H}, {"U_Na", MHD_U_NA}, {"B_xi", MHD_B_XI}, {"B_eta", MHD_B_ETA}, {"B_zeta", MHD_B_ZETA}};

bool check_image(const mhd_restart_image *img) {
  if (!img || img->n_blocks < 1 || !img->cells || img->nghost < 0) return false;
  for (int b = 0; b < 3 * img->n_blocks; ++b)
    if (img->cells[b] < 1) return false;
  return true;
}

// FieldBlock range of state field f in block b
void field_range(const mhd_restart_image *img, int f, int b, int32_t lo[3], int32_t hi[3]) {
  const int *st = mhd::kStagger[mhd::kFieldSpec[kState[f].field].loc];
  for (int a = 0; a < 3; ++a) {
    lo[a] = -img->nghost;
    hi[a] = img->cells[3 * b + a] + st[a] + img->nghost;
  }
}

int64_t block_values(const mhd_restart_image *img, int f, int b) {
  int32_t lo[3], hi[3];
  field_range(img, f, b, lo, hi);
  return (int64_t)(hi[0] - lo[0]) * (hi[1] - lo[1]) * (hi[2] - lo[2]) * mhd::kFieldSpec[kState[f].field].ncomp;
}

struct File {
  FILE *fp = nullptr;
  ~File() {
    if (fp) std::fclose(fp);
  }
};

}  // namespace

extern "C" {

int64_t mhd_restart_values(const mhd_restart_image *img, int32_t state_field) {
  if (!check_image(img) || state_field < 0 || state_field >= MHD_RESTART_FIELDS) return -1;
  int64_t n = 0;
  for (int b = 0; b < img->n_blocks; ++b) n += block_values(img, state_field, b);
  return n;
}

int mhd_restart_write(const char *path, const mhd_restart_image *img) {
  if (!path || !check_image(img)) return mhd::set_error(MHD_ERR_ARG, "mhd_restart_write: bad arguments");
  for (int f = 0; f < MHD_RESTART_FIELDS; ++f)
    if (!img->data[f]) return mhd::set_error(MHD_ERR_ARG, "mhd_restart_write: no data for %s", kState[f].name);
  File out;
  out.fp = std::fopen(path, "wb");
  if (!out.fp) return mhd::set_error(MHD_ERR_ARG, "mhd_restart_write: cannot open %s", path);
  bool ok = true;
  auto bytes = [&](const void *p, size_t n) { ok = ok && std::fwrite(p, 1, n, out.fp) == n; };
  auto i32 = [&](int32_t v) { bytes(&v, 4); };
  auto f64 = [&](double v) { bytes(&v, 8); };
  bytes("MPCNSRST", 8);
  i32(1);
  i32(img->step);
  f64(img->time);
  i32(img->n_blocks);
  i32(MHD_RESTART_FIELDS);
  for (int f = 0; f < MHD_RESTART_FIELDS; ++f) {
    const int32_t len = (int32_t)std::strlen(kState[f].name);
    i32(len);
    bytes(kState[f].name, (size_t)len);
    i32(mhd::kFieldSpec[kState[f].field].loc);
    i32(mhd::kFieldSpec[kState[f].field].ncomp);
    i32(img->nghost);
    const double *d = img->data[f];
    for (int b = 0; b < img->n_blocks; ++b) {
      int32_t lo[3], hi[3];
      field_range(img, f, b, lo, hi);
      for (int a = 0; a < 3; ++a) i32(lo[a]);
      for (int a = 0; a < 3; ++a) i32(hi[a]);
      i32(1);  // active
      const int64_t n = block_values(img, f, b);
      bytes(d, sizeof(double) * (size_t)n);
      d += n;
    }
  }
  ok = ok && std::fflush(out.fp) == 0;
  if (!ok) return mhd::set_error(MHD_ERR_ARG, "mhd_restart_write: write to %s failed", path);
  return MHD_OK;
}

int mhd_restart_read(const char *path, mhd_restart_image *img) {
  if (!path || !check_image(img)) return mhd::set_error(MHD_ERR_ARG, "mhd_restart_read: bad arguments");
  File in;
  in.fp = std::fopen(path, "rb");
  if (!in.fp) return mhd::set_error(MHD_ERR_ARG, "mhd_restart_read: cannot open %s", path);
  bool ok = true;
  auto bytes = [&](void *p, size_t n) { ok = ok && std::fread(p, 1, n, in.fp) == n; };
  auto i32 = [&]() {
    int32_t v = 0;
    bytes(&v, 4);
    return v;
  };
  auto f64 = [&]() {
    double v = 0.0;
    bytes(&v, 8);
    return v;
  };
  auto bad = [&](const char *what) { return mhd::set_error(MHD_ERR_ARG, "mhd_restart_read: %s (%s)", what, path); };
  char magic[8];
  bytes(magic, 8);
  if (!ok || std::memcmp(magic, "MPCNSRST", 8) != 0) return bad("not an MPCNSRST file");
  const int32_t version = i32();
  if (!ok || version != 1) return bad("unsupported version");
  const int32_t step = i32();
  const double time = f64();
  const int32_t nblock = i32(), nfield = i32();
  if (!ok || nfield < 0) return bad("truncated header");
  if (nblock != img->n_blocks) return bad("block count differs from the solve's");
  uint32_t loaded = 0;
  for (int32_t q = 0; q < nfield; ++q) {
    const int32_t len = i32();
    if (!ok || len < 0 || len > 4096) return bad("bad field name");
    std::string name((size_t)len, '\0');
    if (len) bytes(&name[0], (size_t)len);
    const int32_t loc = i32(), ncomp = i32(), nghost = i32();
    if (!ok) return bad("truncated field header");
    int f = -1;
    for (int c = 0; c < MHD_RESTART_FIELDS; ++c)
      if (name == kState[c].name) f = c;
    if (f >= 0) {
      if (loc != mhd::kFieldSpec[kState[f].field].loc) return bad("location mismatch");
      if (ncomp != mhd::kFieldSpec[kState[f].field].ncomp) return bad("component count mismatch");
      if (nghost != img->nghost) return bad("nghost mismatch");
      if (loaded & (1u << f)) return bad("field stored twice");
    }
    double *d = f >= 0 ? img->data[f] : nullptr;
    if (f >= 0 && !d) return bad("no buffer for a stored field");
    for (int32_t b = 0; b < nblock; ++b) {
      int32_t lo[3], hi[3];
      for (int a = 0; a < 3; ++a) lo[a] = i32();
      for (int a = 0; a < 3; ++a) hi[a] = i32();
      const int32_t active = i32();
      if (!ok) return bad("truncated block header");
      for (int a = 0; a < 3; ++a)
        if (hi[a] < lo[a]) return bad("negative extent");
      const int64_t n = (int64_t)(hi[0] - lo[0]) * (hi[1] - lo[1]) * (hi[2] - lo[2]) * (int64_t)ncomp;
      if (f < 0) {  // a field this library does not restore: skip its values
        if (active == 1 && fseeko(in.fp, (off_t)(n * 8), SEEK_CUR) != 0) return bad("truncated data");
        continue;
      }
      int32_t elo[3], ehi[3];
      field_range(img, f, b, elo, ehi);
      for (int a = 0; a < 3; ++a)
        if (lo[a] != elo[a] || hi[a] != ehi[a]) return bad("block range differs from the solve's");
      if (active != 1) return bad("inactive block for an allocated field");
      bytes(d, sizeof(double) * (size_t)n);
      if (!ok) return bad("truncated data");
      d += n;
    }
    if (f >= 0) loaded |= 1u << f;
  }
  img->step = step;
  img->time = time;
  img->loaded = loaded;
  return MHD_OK;
}

// The run-data file written beside each checkpoint (RunData::WriteBinary,
// include/6_io/RunData.h:96-149, through IOModule::WriteRunDataFile):
// "MPCNSRUN", int32 version = 1, int32 step, double time, double dt,
// int32 nref + nref doubles, double residual_max, then the double and the
// int32 monitor maps, each an int32 count and per entry (in key order, as a
// std::map holds them) int32 key length, key bytes and the value.  The
// Mercury solver's monitors are RuntimeMonitor's (src/6_io/RuntimeMonitor.cpp:
// 28-55): "Perf/CPUInterval_s", "Perf/s_per_MCells_step" and "Perf/Cells".
int mhd_rundata_write(const char *path, int32_t step, double time, double dt, int32_t nref,
                      const double *residual_ref, double residual_max, int32_t n_dmon, const char *const *dkeys,
                      const double *dvals, int32_t n_imon, const char *const *ikeys, const int32_t *ivals) {
  if (!path || nref < 0 || (nref > 0 && !residual_ref) || n_dmon < 0 || n_imon < 0 ||
      (n_dmon > 0 && (!dkeys || !dvals)) || (n_imon > 0 && (!ikeys || !ivals)))
    return mhd::set_error(MHD_ERR_ARG, "mhd_rundata_write: bad arguments");
  std::map<std::string, double> dm;
  std::map<std::string, int32_t> im;
  for (int q = 0; q < n_dmon; ++q) {
    if (!dkeys[q]) return mhd::set_error(MHD_ERR_ARG, "mhd_rundata_write: null key");
    dm[dkeys[q]] = dvals[q];
  }
  for (int q = 0; q < n_imon; ++q) {
    if (!ikeys[q]) return mhd::set_error(MHD_ERR_ARG, "mhd_rundata_write: null key");
    im[ikeys[q]] = ivals[q];
  }
  std::string out("MPCNSRUN");
  auto put = [&](const void *p, size_t n) { out.append((const char *)p, n); };
  auto key = [&](const std::string &k) {
    const int32_t n = (int32_t)k.size();
    put(&n, 4);
    out += k;
  };
  const int32_t version = 1, nd = (int32_t)dm.size(), ni = (int32_t)im.size();
  put(&version, 4);
  put(&step, 4);
  put(&time, 8);
  put(&dt, 8);
  put(&nref, 4);
  if (nref > 0) put(residual_ref, 8 * (size_t)nref);
  put(&residual_max, 8);
  put(&nd, 4);
  for (const auto &e : dm) {
    key(e.first);
    put(&e.second, 8);
  }
  put(&ni, 4);
  for (const auto &e : im) {
    key(e.first);
    put(&e.second, 4);
  }
  File f;
  f.fp = std::fopen(path, "wb");
  if (!f.fp) return mhd::set_error(MHD_ERR_ARG, "mhd_rundata_write: cannot open %s", path);
  bool ok = std::fwrite(out.data(), 1, out.size(), f.fp) == out.size();
  ok = std::fclose(f.fp) == 0 && ok;
  f.fp = nullptr;
  return ok ? MHD_OK : mhd::set_error(MHD_ERR_ARG, "mhd_rundata_write: write failed");
}

// RunData::ReadBinary (include/6_io/RunData.h:151-200): step, time and dt of
// a run-data file (its residuals and monitors are not needed to resume).
int mhd_rundata_read(const char *path, int32_t *step, double *time, double *dt) {
  if (!path || !step || !time || !dt) return mhd::set_error(MHD_ERR_ARG, "mhd_rundata_read: bad arguments");
  File f;
  f.fp = std::fopen(path, "rb");
  if (!f.fp) return mhd::set_error(MHD_ERR_ARG, "mhd_rundata_read: cannot open %s", path);
  char magic[8];
  int32_t version = 0;
  if (std::fread(magic, 1, 8, f.fp) != 8 || std::memcmp(magic, "MPCNSRUN", 8) != 0)
    return mhd::set_error(MHD_ERR_ARG, "mhd_rundata_read: %s is not a run-data file", path);
  if (std::fread(&version, 4, 1, f.fp) != 1 || version != 1)
    return mhd::set_error(MHD_ERR_ARG, "mhd_rundata_read: %s: unsupported version", path);
  if (std::fread(step, 4, 1, f.fp) != 1 || std::fread(time, 8, 1, f.fp) != 1 || std::fread(dt, 8, 1, f.fp) != 1)
    return mhd::set_error(MHD_ERR_ARG, "mhd_rundata_read: %s: truncated", path);
  return MHD_OK;
}

}  // extern "C"
