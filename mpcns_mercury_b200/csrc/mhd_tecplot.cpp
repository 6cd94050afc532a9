// The checkpoint plot file MercurySolver writes beside each restart file:
// IOModule::WriteTecplotBinFile (src/6_io/IOModule_Tecplot.cpp:749-1017) in
// the AllNode mode and with the variables its constructor selects
// (Z4_Mercury/src/MercurySolver.cpp:49-86), written from host arrays in the
// FieldBlock layout (the arrays mhd_download_field returns).  Every value is
// evaluated and every byte is written in the reference's order, so the file
// is the reference's byte for byte (tests/test_tecplot.py).
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "mercury_mhd.h"
#include "mhd_error.h"
#include "mhd_parallel.h"

namespace {

// Components of the cell fields, in the order of MHD_TECPLOT_FIELDS, and the
// variable names SetTecplotFieldComponentNames gives them.
constexpr int kComps[MHD_TECPLOT_FIELDS] = {5, 5, 3, 3, 1, 3};
const char *const kNames[] = {"x",   "y",    "z",    "u_H",    "v_H",    "w_H",    "p_H",  "T_H",
                              "u_Na", "v_Na", "w_Na", "p_Na",  "T_Na",   "Bx",     "By",   "Bz",
                              "bx_ind", "by_ind", "bz_ind", "n_Na", "Jx", "Jy",   "Jz"};
constexpr int kNumVars = 3 + 5 + 5 + 3 + 3 + 1 + 3;
static_assert(sizeof(kNames) / sizeof(kNames[0]) == kNumVars, "a name per variable");

struct Out {
  std::vector<unsigned char> buf;
  void i32(int32_t v) { put(&v, 4); }
  void f32(float v) { put(&v, 4); }
  void f64(double v) { put(&v, 8); }
  // a Tecplot binary string: one int32 per character, then 0 (TecWriteStr_)
  void str(const std::string &s) {
    for (char c : s) i32((int32_t)c);
    i32(0);
  }
  void put(const void *p, size_t n) {
    const auto *c = (const unsigned char *)p;
    buf.insert(buf.end(), c, c + n);
  }
};

// A FieldBlock array over [-g, n + extra + g) per axis with nc components.
struct View {
  const double *p;
  int g, e[3], nc;
  double at(int i, int j, int k, int m) const {
    return p[(((int64_t)(i + g) * e[1] + (j + g)) * e[2] + (k + g)) * nc + m];
  }
  bool in(int i, int j, int k) const {
    return i >= -g && i < e[0] - g && j >= -g && j < e[1] - g && k >= -g && k < e[2] - g;
  }
};

}  // namespace

extern "C" int mhd_tecplot_write(const char *path, const mhd_tecplot_image *img) {
  if (!path || !img || img->n_blocks < 1 || !img->cells || !img->block_names || !img->nodes || !img->jac ||
      img->cell_ghost < 1 || img->jac_ghost < 1)
    return mhd::set_error(MHD_ERR_ARG, "mhd_tecplot_write: bad arguments");
  for (int f = 0; f < MHD_TECPLOT_FIELDS; ++f)
    if (!img->cell[f]) return mhd::set_error(MHD_ERR_ARG, "mhd_tecplot_write: field %d missing", f);
  const int nb = img->n_blocks;
  for (int b = 0; b < nb; ++b) {
    for (int a = 0; a < 3; ++a)
      if (img->cells[3 * b + a] < 1) return mhd::set_error(MHD_ERR_ARG, "mhd_tecplot_write: block %d cells", b);
    if (!img->nodes[b] || !img->jac[b] || !img->block_names[b])
      return mhd::set_error(MHD_ERR_ARG, "mhd_tecplot_write: block %d arrays", b);
    for (int f = 0; f < MHD_TECPLOT_FIELDS; ++f)
      if (!img->cell[f][b]) return mhd::set_error(MHD_ERR_ARG, "mhd_tecplot_write: block %d field %d", b, f);
  }

  Out o;
  // header (plt_write_header_): magic, byte order, file type, title, variables
  o.put("#!TDV112", 8);
  o.i32(1);
  o.i32(0);
  o.str("flow_field");
  o.i32(kNumVars);
  for (const char *name : kNames) o.str(name);
  // zone headers (plt_write_zone_header_): every variable at the nodes
  for (int b = 0; b < nb; ++b) {
    const int *n = img->cells + 3 * b;
    o.f32(299.0f);
    o.str("Zone" + std::to_string(b) + "_" + img->block_names[b]);
    o.i32(-1);
    o.i32(-2);
    o.f64(img->time);
    o.i32(-1);
    o.i32(0);
    o.i32(1);
    for (int v = 0; v < kNumVars; ++v) o.i32(0);
    o.i32(0);
    o.i32(0);
    o.i32(n[0] + 1);
    o.i32(n[1] + 1);
    o.i32(n[2] + 1);
    o.i32(0);
  }
  o.f32(357.0f);

  for (int b = 0; b < nb; ++b) {
    const int *n = img->cells + 3 * b;
    const int N[3] = {n[0] + 1, n[1] + 1, n[2] + 1};
    const int64_t nn = (int64_t)N[0] * N[1] * N[2];
    const View X{img->nodes[b], 0, {N[0], N[1], N[2]}, 3};
    const int gj = img->jac_ghost, gc = img->cell_ghost;
    const View J{img->jac[b], gj, {n[0] + 2 * gj, n[1] + 2 * gj, n[2] + 2 * gj}, 1};
    View C[MHD_TECPLOT_FIELDS];
    for (int f = 0; f < MHD_TECPLOT_FIELDS; ++f)
      C[f] = View{img->cell[f][b], gc, {n[0] + 2 * gc, n[1] + 2 * gc, n[2] + 2 * gc}, kComps[f]};
    // node values of every variable, (k, j, i) order with i fastest
    std::vector<double> val((size_t)kNumVars * nn);
    mhd::parallel_for(N[2], [&](int k) {
      for (int j = 0; j < N[1]; ++j)
        for (int i = 0; i < N[0]; ++i) {
          const int64_t q = ((int64_t)k * N[1] + j) * N[0] + i;
          for (int a = 0; a < 3; ++a) val[(size_t)a * nn + q] = X.at(i, j, k, a);
          // EvalValue_CellToNode_: the |Jac|-weighted average of the eight
          // cells around the node (ghost cells included), in the reference's
          // order; cells outside the arrays or with a non-finite or
          // non-positive weight are left out
          int v = 3;
          for (int f = 0; f < MHD_TECPLOT_FIELDS; ++f)
            for (int m = 0; m < kComps[f]; ++m, ++v) {
              double ws = 0.0, wt = 0.0;
              const int cells[8][3] = {{i - 1, j - 1, k - 1}, {i, j - 1, k - 1}, {i - 1, j, k - 1}, {i, j, k - 1},
                                       {i - 1, j - 1, k},     {i, j - 1, k},     {i - 1, j, k},     {i, j, k}};
              for (const auto &c : cells) {
                if (!C[f].in(c[0], c[1], c[2]) || !J.in(c[0], c[1], c[2])) continue;
                const double w = std::abs(J.at(c[0], c[1], c[2], 0));
                if (!std::isfinite(w) || w <= 0.0) continue;
                ws += w * C[f].at(c[0], c[1], c[2], m);
                wt += w;
              }
              val[(size_t)v * nn + q] = wt > 0.0 ? ws / wt : 0.0;
            }
        }
    });
    // data section header (plt_write_data_section_header_): every variable float
    o.f32(299.0f);
    for (int v = 0; v < kNumVars; ++v) o.i32(1);
    o.i32(0);
    o.i32(0);
    o.i32(-1);
    for (int v = 0; v < kNumVars; ++v) {
      const double *x = val.data() + (size_t)v * nn;
      double lo = x[0], hi = x[0];
      for (int64_t q = 1; q < nn; ++q) {
        if (x[q] < lo) lo = x[q];
        if (x[q] > hi) hi = x[q];
      }
      o.f64(lo);
      o.f64(hi);
    }
    for (int v = 0; v < kNumVars; ++v) {
      const double *x = val.data() + (size_t)v * nn;
      for (int64_t q = 0; q < nn; ++q) o.f32((float)x[q]);
    }
  }

  FILE *fp = std::fopen(path, "wb");
  if (!fp) return mhd::set_error(MHD_ERR_ARG, "mhd_tecplot_write: cannot open %s", path);
  const size_t w = std::fwrite(o.buf.data(), 1, o.buf.size(), fp);
  const int closed = std::fclose(fp);
  if (w != o.buf.size() || closed != 0) return mhd::set_error(MHD_ERR_ARG, "mhd_tecplot_write: write failed");
  return MHD_OK;
}
