// fld.cpp -- field output in Neko's fld format (the Nek5000 field-file
// layout Neko writes, fld_file_write, src/io/fld_file.f90:183-620), for
// the solutions of the pressure/Helmholtz solves: mesh coordinates ('X')
// and one scalar field as the pressure ('P'), 3-D, one rank.
//
// Layout, native byte order:
//   132-byte ASCII header
//     '#std' 1x i1 1x i2 1x i2 1x i2 1x i10 1x i10 1x e20.13 1x i9 1x i6
//     1x i6 1x 10a   (real size, lx, ly, lz, nelv, nelv, time, step, 1, 1,
//     rdcode), blank-padded
//   float32 6.54321 (byte-order tag)
//   int32 element ids 1..nelv
//   'X': per element lx^3 x, then lx^3 y, then lx^3 z
//   'P': per element lx^3 values
//   metadata (float32): 'X' per element min/max of x, y, z; 'P' per element
//   min/max of the field
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "nb_internal.h"

using namespace nb;

namespace {

// Fortran Ew.d output of v (w = 20, d = 13): optional sign, "0.", d digits,
// "E", exponent sign, two exponent digits, right-justified in w columns.
std::string fortran_e(double v, int w, int d) {
  std::string body;
  if (v == 0.0) {
    body = "0." + std::string(d, '0') + "E+00";
  } else {
    // v = m 10^e with 0.1 <= |m| < 1, rounded to d digits
    char buf[64];
    snprintf(buf, sizeof(buf), "%.*e", d - 1, std::fabs(v));  // d.ddd...e+XX
    std::string s(buf);
    const size_t epos = s.find('e');
    std::string digits = s.substr(0, 1) + s.substr(2, epos - 2);
    const int ex = std::atoi(s.c_str() + epos + 1) + 1;
    char eb[8];
    snprintf(eb, sizeof(eb), "%c%02d", ex < 0 ? '-' : '+', std::abs(ex));
    body = std::string(v < 0 ? "-" : "") + "0." + digits + "E" + eb;
  }
  if ((int)body.size() < w) body = std::string(w - body.size(), ' ') + body;
  return body;
}

std::string fixed_int(long v, int w) {
  char b[32];
  snprintf(b, sizeof(b), "%*ld", w, v);
  return b;
}

nb_status err(const std::string &m) {
  set_error(m);
  return NB_ERR_ARG;
}

}  // namespace

extern "C" nb_status nb_fld_write(const char *path, int nelv, int lx, const double *x,
                                  const double *y, const double *z, const double *p, double time,
                                  int step) {
  if (!path || nelv < 1 || lx < 2 || lx > 99) return err("nb_fld_write: bad argument");
  const bool wx = x && y && z, wp = p != nullptr;
  if (!wx && !wp) return err("nb_fld_write: nothing to write");
  const long l3 = (long)lx * lx * lx;
  std::string rd = std::string(wx ? "X" : "") + (wp ? "P" : "");
  rd.resize(10, ' ');
  std::string hdr = "#std " + fixed_int(8, 1) + " " + fixed_int(lx, 2) + " " + fixed_int(lx, 2) +
                    " " + fixed_int(lx, 2) + " " + fixed_int(nelv, 10) + " " +
                    fixed_int(nelv, 10) + " " + fortran_e(time, 20, 13) + " " +
                    fixed_int(step, 9) + " " + fixed_int(1, 6) + " " + fixed_int(1, 6) + " " + rd;
  hdr.resize(132, ' ');
  FILE *f = fopen(path, "wb");
  if (!f) return err(std::string("nb_fld_write: cannot create ") + path);
  bool ok = fwrite(hdr.data(), 1, 132, f) == 132;
  const float tag = 6.54321f;
  ok = ok && fwrite(&tag, 4, 1, f) == 1;
  std::vector<int32_t> ids(nelv);
  for (int e = 0; e < nelv; e++) ids[e] = e + 1;
  ok = ok && fwrite(ids.data(), 4, nelv, f) == (size_t)nelv;
  if (wx)
    for (int e = 0; e < nelv && ok; e++)
      for (const double *a : {x, y, z}) ok = ok && fwrite(a + e * l3, 8, l3, f) == (size_t)l3;
  if (wp) ok = ok && fwrite(p, 8, (size_t)nelv * l3, f) == (size_t)nelv * l3;
  auto minmax = [&](const double *a, int e, float *o) {
    double lo = a[e * l3], hi = a[e * l3];
    for (long q = 1; q < l3; q++) {
      lo = std::min(lo, a[e * l3 + q]);
      hi = std::max(hi, a[e * l3 + q]);
    }
    o[0] = (float)lo;
    o[1] = (float)hi;
  };
  if (wx)
    for (int e = 0; e < nelv && ok; e++) {
      float m[6];
      minmax(x, e, m);
      minmax(y, e, m + 2);
      minmax(z, e, m + 4);
      ok = fwrite(m, 4, 6, f) == 6;
    }
  if (wp)
    for (int e = 0; e < nelv && ok; e++) {
      float m[2];
      minmax(p, e, m);
      ok = fwrite(m, 4, 2, f) == 2;
    }
  if (fclose(f) != 0) ok = false;
  if (!ok) return err("nb_fld_write: write failed");
  return NB_OK;
}
