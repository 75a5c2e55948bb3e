// host_io.cpp -- format boundary and host precompute of the engine.
//
//  * ASCII .ini reader         (reference src/readwrite.c:975-1082)
//  * binary .out writer        (reference src/readwrite.c:160-366)
//  * grid metric from positions (reference initgrid, src/init.cu:2502-3060)
// These run once per run (set-up and snapshot output), on the host, exactly
// as in the reference; the time advance itself is device-only.
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/smaug_b200.h"
#include "engine_internal.h"

namespace smaug {

// ---- grid metric ---------------------------------------------------------
// Padded copy T of each position field (one extra layer per side), linear
// extrapolation (1+|ixe-ix|) T[ixe] - |ixe-ix| T[ixf] into the outer layers:
// upper side padded indices n-1..n+1 from n-2, n-3; lower side 0..1 from
// 2, 3 along dim 0 and 0..2 from 3, 4 along the other dims (the reference's
// ixmax is 1 for dim 0 and 2 otherwise, src/init.cu:2672,2765).  Ghost
// positions are then rewritten from T and delx = (T[i+1] - T[i-1]) / 2.
int grid_metric(int ndim, const int32_t* nn, double* pos, double* delx) {
  int n[3] = {nn[0], nn[1], ndim == 3 ? nn[2] : 1};
  int m[3] = {n[0] + 2, n[1] + 2, ndim == 3 ? n[2] + 2 : 1};
  long dimp = (long)n[0] * n[1] * n[2];
  long msz = (long)m[0] * m[1] * m[2];
  std::vector<double> T((size_t)ndim * msz, 0.0);
  auto TI = [&](int a, int b, int c, int f) {
    return (((long)c * m[1] + b) * m[0] + a) + (long)f * msz;
  };
  int k3 = (ndim == 3);
  for (int f = 0; f < ndim; f++)
    for (int c = 0; c < n[2]; c++)
      for (int b = 0; b < n[1]; b++)
        for (int a = 0; a < n[0]; a++)
          T[TI(a + 1, b + 1, c + k3, f)] = pos[(long)f * dimp + ((long)c * n[1] + b) * n[0] + a];
  for (int dir = 0; dir < ndim; dir++) {
    for (int side = 0; side < 2; side++) {
      int ixmin, ixmax, ixe, ixf;
      if (side == 0) {
        ixmax = n[dir] + 1; ixmin = n[dir] - 1; ixe = ixmin - 1; ixf = ixe - 1;
      } else {
        ixmin = 0; ixmax = (dir == 0) ? 1 : 2; ixe = ixmax + 1; ixf = ixe + 1;
      }
      for (int f = 0; f < ndim; f++)
        for (int c = 0; c < m[2]; c++)
          for (int b = 0; b < m[1]; b++)
            for (int a = 0; a < m[0]; a++) {
              int ii[3] = {a, b, c};
              int ix = ii[dir];
              if (ix < ixmin || ix > ixmax) continue;
              int i1[3] = {a, b, c}, i2[3] = {a, b, c};
              i1[dir] = ixe;
              i2[dir] = ixf;
              double wgt = (double)std::abs(ixe - ix);
              T[TI(a, b, c, f)] = (1 + wgt) * T[TI(i1[0], i1[1], i1[2], f)] -
                                  wgt * T[TI(i2[0], i2[1], i2[2], f)];
            }
    }
  }
  for (int f = 0; f < ndim; f++)
    for (int c = 0; c < n[2]; c++)
      for (int b = 0; b < n[1]; b++)
        for (int a = 0; a < n[0]; a++)
          pos[(long)f * dimp + ((long)c * n[1] + b) * n[0] + a] = T[TI(a + 1, b + 1, c + k3, f)];
  for (int dir = 0; dir < ndim; dir++)
    for (int c = 0; c < n[2]; c++)
      for (int b = 0; b < n[1]; b++)
        for (int a = 0; a < n[0]; a++) {
          int p[3] = {a + 1, b + 1, c + k3};
          int pp[3] = {p[0], p[1], p[2]}, pm[3] = {p[0], p[1], p[2]};
          pp[dir] += 1;
          pm[dir] -= 1;
          delx[(long)dir * dimp + ((long)c * n[1] + b) * n[0] + a] =
              0.5 * (T[TI(pp[0], pp[1], pp[2], dir)] - T[TI(pm[0], pm[1], pm[2], dir)]);
        }
  return SMAUG_OK;
}

// ---- .ini reader -----------------------------------------------------------
static bool read_line(FILE* f, std::string& out) {
  out.clear();
  int c;
  while ((c = fgetc(f)) != EOF) {
    if (c == '\n') return true;
    out.push_back((char)c);
  }
  return !out.empty();
}

int read_ini(const char* path, int ndim, const int32_t* n, double* w, double* pos,
             int32_t* it, double* t) {
  FILE* f = fopen(path, "r");
  if (!f) return set_error(SMAUG_E_IO, "cannot open %s: %s", path, strerror(errno));
  std::string line;
  // header: name, "it t ndim neqpar nw", grid, eqpar, names
  if (!read_line(f, line)) { fclose(f); return set_error(SMAUG_E_FORMAT, "%s: empty file", path); }
  if (!read_line(f, line)) { fclose(f); return set_error(SMAUG_E_FORMAT, "%s: missing header line 2", path); }
  int fit = 0, fndim = 0, fneq = 0, fnw = 0;
  double ft = 0;
  if (sscanf(line.c_str(), "%d %lg %d %d %d", &fit, &ft, &fndim, &fneq, &fnw) != 5) {
    fclose(f);
    return set_error(SMAUG_E_FORMAT, "%s: bad header line 2", path);
  }
  int nvar = 4 + 3 * ndim;
  if (fndim != ndim || fnw != nvar) {
    fclose(f);
    return set_error(SMAUG_E_FORMAT, "%s: file has ndim=%d nw=%d, expected %d/%d", path, fndim, fnw,
                     ndim, nvar);
  }
  if (!read_line(f, line)) { fclose(f); return set_error(SMAUG_E_FORMAT, "%s: missing grid line", path); }
  {
    int fn[3] = {0, 0, 0};
    int got = sscanf(line.c_str(), "%d %d %d", &fn[0], &fn[1], &fn[2]);
    if (got < ndim) { fclose(f); return set_error(SMAUG_E_FORMAT, "%s: bad grid line", path); }
    for (int d = 0; d < ndim; d++)
      if (fn[d] != n[d]) {
        fclose(f);
        return set_error(SMAUG_E_FORMAT, "%s: grid %d along dim %d, expected %d", path, fn[d], d, n[d]);
      }
  }
  for (int i = 0; i < 2; i++)
    if (!read_line(f, line)) { fclose(f); return set_error(SMAUG_E_FORMAT, "%s: short header", path); }
  long dimp = 1;
  for (int d = 0; d < ndim; d++) dimp *= n[d];
  for (long c = 0; c < dimp; c++) {
    for (int d = 0; d < ndim; d++)
      if (fscanf(f, "%lf", &pos[(long)d * dimp + c]) != 1) {
        fclose(f);
        return set_error(SMAUG_E_FORMAT, "%s: truncated at cell %ld", path, c);
      }
    for (int v = 0; v < nvar; v++)
      if (fscanf(f, "%lf", &w[(long)v * dimp + c]) != 1) {
        fclose(f);
        return set_error(SMAUG_E_FORMAT, "%s: truncated at cell %ld", path, c);
      }
  }
  fclose(f);
  if (it) *it = fit;
  if (t) *t = ft;
  return SMAUG_OK;
}

// ---- .out writer -------------------------------------------------------------
int write_out_host(const char* path, const smaug_params_t* p, const double* w, const double* pos,
                   const char* name, int32_t it, double t) {
  int nd = p->ndim;
  long dimp = 1;
  for (int d = 0; d < nd; d++) dimp *= p->n[d];
  int nvar = 4 + 3 * nd;
  FILE* f = fopen(path, "wb");
  if (!f) return set_error(SMAUG_E_IO, "cannot open %s: %s", path, strerror(errno));
  char nbuf[79];
  memset(nbuf, 0, sizeof(nbuf));
  if (name) strncpy(nbuf, name, sizeof(nbuf));
  fwrite(nbuf, 1, 79, f);
  fwrite(&it, sizeof(int32_t), 1, f);
  fwrite(&t, sizeof(double), 1, f);
  int32_t ib[3] = {nd, nd == 2 ? 6 : 7, nvar};
  fwrite(ib, sizeof(int32_t), 3, f);
  int32_t nb[3] = {p->n[0], p->n[1], p->n[2]};
  fwrite(nb, sizeof(int32_t), nd, f);
  double eq[7] = {p->gamma, p->eta, p->g[0], p->g[1], 0, 0, 0};
  if (nd == 3) { eq[4] = p->g[2]; }
  fwrite(eq, sizeof(double), nd == 2 ? 6 : 7, f);
  char vb[79];
  memset(vb, 0, sizeof(vb));
  snprintf(vb, sizeof(vb), "%s", nd == 2 ? "x y rho mx my e bx by  gamma eta g1 g2"
                                         : "x y z rho mx my mz e bx by bz gamma eta g1 g2 g3");
  fwrite(vb, 1, 79, f);
  size_t ok = fwrite(pos, sizeof(double), (size_t)nd * dimp, f);
  ok += fwrite(w, sizeof(double), (size_t)nvar * dimp, f);
  fputc('\n', f);
  int bad = ferror(f) || ok != (size_t)(nd + nvar) * dimp;
  fclose(f);
  if (bad) return set_error(SMAUG_E_IO, "short write to %s", path);
  return SMAUG_OK;
}

}  // namespace smaug

extern "C" int smaug_read_ini(const char* path, int32_t ndim, const int32_t* n, double* w,
                              double* pos, int32_t* it, double* t) {
  smaug::clear_error();
  if (!path || !n || !w || !pos || (ndim != 2 && ndim != 3))
    return smaug::set_error(SMAUG_E_INVALID, "smaug_read_ini: bad arguments");
  return smaug::read_ini(path, ndim, n, w, pos, it, t);
}

extern "C" int smaug_write_out_host(const char* path, const smaug_params_t* p, const double* w,
                                    const double* pos, const char* name, int32_t it, double t) {
  smaug::clear_error();
  if (!path || !p || !w || !pos) return smaug::set_error(SMAUG_E_INVALID, "smaug_write_out_host: null argument");
  return smaug::write_out_host(path, p, w, pos, name, it, t);
}

extern "C" int smaug_grid_metric(int32_t ndim, const int32_t* n, double* pos, double* delx) {
  smaug::clear_error();
  if (!n || !pos || !delx || (ndim != 2 && ndim != 3))
    return smaug::set_error(SMAUG_E_INVALID, "smaug_grid_metric: bad arguments");
  return smaug::grid_metric(ndim, n, pos, delx);
}
