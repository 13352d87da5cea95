// GDSII stream reader and the planar-device cross-section sampler.
//
// The reference reads layouts through the vendored gdstk library
// (gdstk::read_gds(filename, 1e-6), src/core/GDSIISampler.cpp:32) and uses
// the polygons of the library's first cell.  Here the stream format is read
// directly: records are (2-byte big-endian length, record type, data type,
// payload); BOUNDARY and BOX elements of the first structure (BGNSTR ..
// ENDSTR) become polygons, their XY points scaled from database units to the
// requested unit (micrometres by default) with the UNITS record's metres per
// database unit.  The closing point that repeats the first is dropped, as
// gdstk does.  Other elements (paths, references, text) are skipped, as the
// reference's sampler only reads the cell's polygon array.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <limits>

#include "engine.h"

namespace vrc {

namespace {

enum : int {
  REC_UNITS = 0x03,
  REC_ENDLIB = 0x04,
  REC_BGNSTR = 0x05,
  REC_ENDSTR = 0x07,
  REC_BOUNDARY = 0x08,
  REC_PATH = 0x09,
  REC_SREF = 0x0A,
  REC_AREF = 0x0B,
  REC_TEXT = 0x0C,
  REC_LAYER = 0x0D,
  REC_DATATYPE = 0x0E,
  REC_XY = 0x10,
  REC_ENDEL = 0x11,
  REC_NODE = 0x15,
  REC_BOX = 0x2D,
};

uint32_t be32(const unsigned char* p) {
  return (uint32_t)p[0] << 24 | (uint32_t)p[1] << 16 | (uint32_t)p[2] << 8 | (uint32_t)p[3];
}

// 8-byte GDSII real: sign bit, 7-bit exponent (excess 64, base 16), 56-bit
// mantissa fraction: (-1)^s * (m / 2^56) * 16^(e - 64).
double gds_real(const unsigned char* p) {
  const int sign = p[0] & 0x80;
  const int expo = (p[0] & 0x7f) - 64;
  uint64_t mant = 0;
  for (int i = 1; i < 8; ++i) mant = mant << 8 | p[i];
  double v = std::ldexp((double)mant, -56) * std::pow(16.0, expo);
  return sign ? -v : v;
}

}  // namespace

std::vector<std::vector<double>> gds_read_polygons(const std::string& path, double unit, double* db_unit_m) {
  std::ifstream f(path, std::ios::binary);
  if (!f) throw StatusError(ST_EINVAL, "cannot open GDSII file");
  std::vector<unsigned char> buf((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
  std::vector<std::vector<double>> polys;
  double meters_per_db = 1e-9;  // the common default when UNITS is absent
  int structs = 0;              // structures seen (only the first is read)
  bool in_first = false, in_poly = false;
  std::vector<double> cur;
  size_t off = 0;
  while (off + 4 <= buf.size()) {
    const size_t len = (size_t)buf[off] << 8 | buf[off + 1];
    const int rec = buf[off + 2];
    if (len < 4 || off + len > buf.size()) throw StatusError(ST_EINVAL, "malformed GDSII record");
    const unsigned char* d = buf.data() + off + 4;
    const size_t dl = len - 4;
    switch (rec) {
      case REC_UNITS:
        if (dl >= 16) meters_per_db = gds_real(d + 8);
        break;
      case REC_BGNSTR:
        in_first = (structs == 0);
        ++structs;
        break;
      case REC_ENDSTR:
        in_first = false;
        break;
      case REC_BOUNDARY:
      case REC_BOX:
        in_poly = in_first;
        cur.clear();
        break;
      case REC_XY:
        if (in_poly) {
          if (dl % 8) throw StatusError(ST_EINVAL, "malformed GDSII XY record");
          for (size_t k = 0; k < dl; k += 8) {
            const int32_t x = (int32_t)be32(d + k), y = (int32_t)be32(d + k + 4);
            cur.push_back((double)x * meters_per_db / unit);
            cur.push_back((double)y * meters_per_db / unit);
          }
        }
        break;
      case REC_ENDEL:
        if (in_poly) {
          const size_t np = cur.size() / 2;
          if (np >= 2 && cur[0] == cur[2 * np - 2] && cur[1] == cur[2 * np - 1]) cur.resize(2 * (np - 1));
          if (cur.size() >= 6) polys.push_back(cur);
        }
        in_poly = false;
        break;
      case REC_ENDLIB:
        off = buf.size();
        continue;
      default:
        break;
    }
    off += len;
  }
  if (db_unit_m) *db_unit_m = meters_per_db;
  return polys;
}

// ---------------------------------------------------------------------------
// Planar device seen from above (GDSIISampler, src/core/GDSIISampler.cpp):
// the layout's y axis is the propagation coordinate z, the device layer has
// a fixed thickness along the cross-section's y, PML on all four sides.
// ---------------------------------------------------------------------------
void CellSpec::planar_region(double* xlim, double* y6) const {
  // assignSimulationRegion (GDSIISampler.cpp:48-88)
  double minX = std::numeric_limits<double>::infinity(), maxX = -minX;
  for (const auto& p : polys)
    for (size_t k = 0; k + 1 < p.size(); k += 2) {
      minX = std::min(minX, p[k]);
      maxX = std::max(maxX, p[k]);
    }
  minX += shift[0];
  maxX += shift[0];
  const double b0 = shift[1], b1 = b0 + pml_w[2];
  const double u0 = b1 + space[2] + thickness + space[3], u1 = u0 + pml_w[3];
  const double l1 = minX - space[0], l0 = l1 - pml_w[0];
  const double r0 = maxX + space[1], r1 = r0 + pml_w[1];
  xlim[0] = l0;
  xlim[1] = l1;
  xlim[2] = r0;
  xlim[3] = r1;
  // y grid of the constructor (GDSIISampler.cpp:35-42)
  y6[0] = b0;
  y6[1] = b1;
  y6[2] = b1 + space[2];
  y6[3] = y6[2] + thickness;
  y6[4] = u0;
  y6[5] = u1;
}

void CellSpec::planar_section(double z, std::vector<double>& xo, std::vector<double>& yo,
                              std::vector<cplx>* eps_out) const {
  // sampleLayout (GDSIISampler.cpp:90-140): crossings of every polygon edge
  // with the line y = z (half-open in y, unshifted layout coordinates),
  // sorted, between the PML / spacer coordinates
  constexpr double tol = 1e-12;
  std::vector<double> xs;
  for (const auto& p : polys) {
    const size_t np = p.size() / 2;
    for (size_t i = 0; i < np; ++i) {
      const double x0 = p[2 * i], y0 = p[2 * i + 1];
      const size_t j = (i + 1 == np) ? 0 : i + 1;
      const double x1 = p[2 * j], y1 = p[2 * j + 1];
      if ((y0 <= z && z < y1) || (y1 <= z && z < y0)) {
        double h = y1 - y0;
        if (std::fabs(h) < tol) h += 2.0 * tol;
        const double a = (z - y0) / h;
        xs.push_back((1.0 - a) * x0 + a * x1);
      }
    }
  }
  std::sort(xs.begin(), xs.end());
  double xl[4], y6[6];
  planar_region(xl, y6);
  const int Nx = (int)xs.size() + 4;
  xo.resize(Nx);
  xo[0] = xl[0];
  xo[1] = xl[1];
  xo[Nx - 2] = xl[2];
  xo[Nx - 1] = xl[3];
  for (int i = 2; i <= Nx - 3; ++i) xo[i] = xs[i - 2] + shift[0];
  yo.assign(y6, y6 + 6);
  if (eps_out) {
    // background everywhere; the device strip (y index 2) holds the device
    // material in every other x cell, starting at the first crossing
    eps_out->assign((size_t)5 * (Nx - 1), eps_bg);
    for (int j = 2; j <= Nx - 4; j += 2) (*eps_out)[(size_t)2 * (Nx - 1) + j] = eps_dev;
  }
}

}  // namespace vrc
