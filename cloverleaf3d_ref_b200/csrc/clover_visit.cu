// VTK output of a chunk (visit.f90:103-200): legacy ASCII rectilinear grids
// with the cell fields density, energy, pressure and viscosity and the node
// velocities, one value per line in Fortran E12.4, values at or below 1e-8
// (viscosity) or 1e-8 in magnitude (velocities) written as zero, and the
// clover.visit index listing every file. The host writer runs on its own
// thread from copies of the fields (VisitFrame), so the GPU steps on while a
// frame is written.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/clover_b200.h"
#include "clover_visit.h"

namespace clover {

// Fortran E12.4: "0.dddd" mantissa in [0.1, 1) with 4 digits, "E+ee"
// exponent (three-digit exponents drop the "E"), right-aligned in 12
// characters.
void format_e12_4(double v, char out[13]) {
  char m[32];
  if (v == 0.0 || !std::isfinite(v)) {
    snprintf(out, 13, "%12s", v == 0.0 ? (std::signbit(v) ? "-0.0000E+00" : "0.0000E+00")
                                       : (std::isnan(v) ? "NaN" : (v > 0 ? "Infinity" : "-Infinity")));
    return;
  }
  // d.ddd x 10^e, rounded to four significant digits, is 0.dddd x 10^(e+1)
  snprintf(m, sizeof(m), "%.3E", v);
  const bool neg = m[0] == '-';
  const char* p = m + (neg ? 1 : 0);
  const char digits[5] = {p[0], p[2], p[3], p[4], 0};
  const int e = atoi(p + 6) + 1;
  char body[24];
  if (e >= -99 && e <= 99)
    snprintf(body, sizeof(body), "%s0.%sE%c%02d", neg ? "-" : "", digits, e < 0 ? '-' : '+',
             e < 0 ? -e : e);
  else
    snprintf(body, sizeof(body), "%s0.%s%c%03d", neg ? "-" : "", digits, e < 0 ? '-' : '+',
             e < 0 ? -e : e);
  // right-align in 12 characters (the body is at most 11: "-0.dddd+eee")
  size_t n = strlen(body);
  if (n > 12) n = 12;
  memset(out, ' ', 12);
  memcpy(out + 12 - n, body, n);
  out[12] = '\0';
}

namespace {

void put_value(FILE* f, double v) {
  char s[13];
  format_e12_4(v, s);
  fputs(s, f);
  fputc('\n', f);
}

// visit.f90: chunk and step names are i6 of 100000 + n with the first
// character turned into '.'
std::string vtk_name(int chunk, int step) {
  char c[16], s[16];
  snprintf(c, sizeof(c), "%6d", 100000 + chunk);
  snprintf(s, sizeof(s), "%6d", 100000 + step);
  c[0] = '.';
  s[0] = '.';
  return std::string("clover") + c + s + ".vtk";
}

}  // namespace

bool write_visit_frame(const VisitFrame& fr, std::string* err) {
  const std::string dir = fr.dir.empty() ? std::string(".") : fr.dir;
  // the index file: "!NBLOCKS" on the first call, then one line per file
  {
    const std::string idx = dir + "/clover.visit";
    FILE* u = fopen(idx.c_str(), fr.first ? "w" : "a");
    if (!u) {
      *err = "cannot open " + idx;
      return false;
    }
    if (fr.first) fprintf(u, "!NBLOCKS %5d\n", 0);  // parallel%task * tiles_per_chunk, task 0
    for (const VisitChunk& c : fr.chunks) fprintf(u, "%s\n", vtk_name(c.chunk, fr.step).c_str());
    fclose(u);
  }
  for (const VisitChunk& c : fr.chunks) {
    const std::string path = dir + "/" + vtk_name(c.chunk, fr.step);
    FILE* u = fopen(path.c_str(), "w");
    if (!u) {
      *err = "cannot open " + path;
      return false;
    }
    const int nxc = c.nx, nyc = c.ny, nzc = c.nz, nxv = nxc + 1, nyv = nyc + 1, nzv = nzc + 1;
    fprintf(u, "# vtk DataFile Version 3.0\nvtk output\nASCII\nDATASET RECTILINEAR_GRID\n");
    fprintf(u, "DIMENSIONS%12d%12d%12d\n", nxv, nyv, nzv);
    fprintf(u, "X_COORDINATES %5d double\n", nxv);
    for (int j = 0; j < nxv; j++) put_value(u, c.vertexx[j]);
    fprintf(u, "Y_COORDINATES %5d double\n", nyv);
    for (int k = 0; k < nyv; k++) put_value(u, c.vertexy[k]);
    fprintf(u, "Z_COORDINATES %5d double\n", nzv);
    for (int l = 0; l < nzv; l++) put_value(u, c.vertexz[l]);
    const long long ncell = (long long)nxc * nyc * nzc, nvert = (long long)nxv * nyv * nzv;
    fprintf(u, "CELL_DATA %20lld\nFIELD FieldData 4\n", ncell);
    // cell arrays in the reference layout: (nx+4) x (ny+4) x (nz+4) from min-2
    auto cell = [&](const std::vector<double>& a, int j, int k, int l) {
      return a[(size_t)(j + 2) + (size_t)(nxc + 4) * ((size_t)(k + 2) + (size_t)(nyc + 4) * (l + 2))];
    };
    auto node = [&](const std::vector<double>& a, int j, int k, int l) {
      return a[(size_t)(j + 2) + (size_t)(nxc + 5) * ((size_t)(k + 2) + (size_t)(nyc + 5) * (l + 2))];
    };
    const char* cname[4] = {"density", "energy", "pressure", "viscosity"};
    const std::vector<double>* carr[4] = {&c.density0, &c.energy0, &c.pressure, &c.viscosity};
    for (int q = 0; q < 4; q++) {
      fprintf(u, "%s 1 %20lld double\n", cname[q], ncell);
      for (int l = 0; l < nzc; l++)
        for (int k = 0; k < nyc; k++)
          for (int j = 0; j < nxc; j++) {
            double v = cell(*carr[q], j, k, l);
            if (q == 3) v = v > 0.00000001 ? v : 0.0;
            put_value(u, v);
          }
    }
    fprintf(u, "POINT_DATA %20lld\nFIELD FieldData 3\n", nvert);
    const char* vname[3] = {"x_vel", "y_vel", "z_vel"};
    const std::vector<double>* varr[3] = {&c.xvel0, &c.yvel0, &c.zvel0};
    for (int q = 0; q < 3; q++) {
      fprintf(u, "%s 1 %20lld double\n", vname[q], nvert);
      for (int l = 0; l < nzv; l++)
        for (int k = 0; k < nyv; k++)
          for (int j = 0; j < nxv; j++) {
            const double v = node(*varr[q], j, k, l);
            put_value(u, std::fabs(v) > 0.00000001 ? v : 0.0);
          }
    }
    if (fclose(u) != 0) {
      *err = "write failed: " + path;
      return false;
    }
  }
  return true;
}

}  // namespace clover

extern "C" int clover_format_e12_4(double v, char* out13) {
  clover::format_e12_4(v, out13);
  return 0;
}
