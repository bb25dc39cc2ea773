// io.cpp -- the reference's text formats (host code, no device work):
//   field dumps         MaterialGrid::PrintStrain / PrintStress /
//                       PrintLagrangeMultiplier / PrintPolarization
//                       (MaterialGrid.cpp:15-100)
//   random material     UnitTester::WriteRandomMaterial / ReadRandomMaterial
//                       (UnitTester.cpp:116-167)
//   Euler texture file  UnitTester::ReadRicardoData (UnitTester.cpp:237-265)
// Numbers go through std::ostream / std::istream with the stream defaults the
// reference uses (6 significant digits, %g style), so the files are
// byte-compatible.  Errors are returned as VPFFT_ERR_IO, never exit().
#include <cmath>
#include <fstream>
#include <string>
#include <vector>

#include "../../include/vpfft_capi.h"

namespace vpfft {
vpfft_status lib_fail(vpfft_status s, const std::string& msg);
}

namespace {

long long voxel(int x, int y, int z, int ny, int nz) { return ((long long)x * ny + y) * nz + z; }

bool dims_ok(int nx, int ny, int nz) { return nx > 0 && ny > 0 && nz > 0; }

vpfft_status io_fail(const std::string& what, const char* path) {
  return vpfft::lib_fail(VPFFT_ERR_IO, what + ": " + (path ? path : "(null)"));
}

// EigenRep's stream form: five values, each followed by a space (LinearAlgebra.cpp:902-910).
void put5(std::ostream& os, const double* v) {
  for (int c = 0; c < 5; ++c) os << v[c] << " ";
}

// SMatrix3x3::BuildActiveEulerMatrix (LinearAlgebra.cpp:160-181): angles in
// radians, single-precision cosf/sinf as the reference uses, products in double.
void active_euler(double phi, double theta, double psi, double m[9]) {
  const double cph = cosf((float)phi), cth = cosf((float)theta), cps = cosf((float)psi);
  const double sph = sinf((float)phi), sth = sinf((float)theta), sps = sinf((float)psi);
  m[0] = cph * cps - sph * cth * sps;
  m[3] = sph * cps + cph * cth * sps;
  m[6] = sth * sps;
  m[1] = -cph * sps - sph * cth * cps;
  m[4] = -sph * sps + cph * cth * cps;
  m[7] = sth * cps;
  m[2] = sph * sth;
  m[5] = -cph * sth;
  m[8] = cth;
}

}  // namespace

extern "C" {

vpfft_status vpfft_print_field(const char* path, vpfft_print_kind kind, int nx, int ny, int nz,
                               const double* re, const double* im) {
  if (!path || !re || !dims_ok(nx, ny, nz))
    return vpfft::lib_fail(VPFFT_ERR_INVALID_ARGUMENT, "bad argument");
  std::ofstream os(path);
  if (!os) return io_fail("cannot open for writing", path);
  const bool cplx = kind == VPFFT_PRINT_STRAIN || kind == VPFFT_PRINT_POLARIZATION;
  auto row = [&](int i, int j, int k) {
    const long long v = voxel(i, j, k, ny, nz);
    os << i << " " << j << " " << k << " ";
    if (cplx) {
      for (int n = 0; n < 5; ++n) os << re[v * 5 + n] << " " << (im ? im[v * 5 + n] : 0.0) << " ";
    } else {
      put5(os, re + v * 5);
    }
    os << std::endl;
  };
  switch (kind) {
    case VPFFT_PRINT_STRAIN:
    case VPFFT_PRINT_STRESS:
    case VPFFT_PRINT_POLARIZATION:  // z outermost, x innermost
      for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
          for (int i = 0; i < nx; ++i) row(i, j, k);
      break;
    case VPFFT_PRINT_LAGRANGE:  // x outermost (MaterialGrid.cpp:62-72)
      for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
          for (int k = 0; k < nz; ++k) row(i, j, k);
      break;
    default:
      return vpfft::lib_fail(VPFFT_ERR_INVALID_ARGUMENT, "unknown print kind");
  }
  os.close();
  if (!os) return io_fail("write failed", path);
  return VPFFT_OK;
}

vpfft_status vpfft_grid_print(vpfft_grid* g, vpfft_print_kind kind, const char* path) {
  int nx = 0, ny = 0, nz = 0;
  if (vpfft_status s = vpfft_grid_dims(g, &nx, &ny, &nz)) return s;
  vpfft_field f;
  switch (kind) {
    case VPFFT_PRINT_STRAIN: f = VPFFT_FIELD_STRAIN_RATE_VARIATION; break;
    case VPFFT_PRINT_STRESS: f = VPFFT_FIELD_STRESS; break;
    case VPFFT_PRINT_LAGRANGE: f = VPFFT_FIELD_LAGRANGE; break;
    case VPFFT_PRINT_POLARIZATION: f = VPFFT_FIELD_POLARIZATION; break;
    default: return vpfft::lib_fail(VPFFT_ERR_INVALID_ARGUMENT, "unknown print kind");
  }
  std::vector<double> re((size_t)nx * ny * nz * 5);
  if (vpfft_status s = vpfft_grid_get_field(g, f, re.data())) return s;
  return vpfft_print_field(path, kind, nx, ny, nz, re.data(), nullptr);
}

vpfft_status vpfft_write_random_material(const char* path, int nx, int ny, int nz,
                                         const double* R9, const double* stress5) {
  if (!path || !R9 || !stress5 || !dims_ok(nx, ny, nz))
    return vpfft::lib_fail(VPFFT_ERR_INVALID_ARGUMENT, "bad argument");
  std::ofstream os(path);
  if (!os) return io_fail("cannot open for writing", path);
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nz; ++k) {
        const long long v = voxel(i, j, k, ny, nz);
        for (int e = 0; e < 9; ++e) os << R9[v * 9 + e] << " ";
        put5(os, stress5 + v * 5);
        os << std::endl;
      }
  os.close();
  if (!os) return io_fail("write failed", path);
  return VPFFT_OK;
}

vpfft_status vpfft_read_random_material(const char* path, int nx, int ny, int nz, double* R9,
                                        double* stress5) {
  if (!path || !R9 || !stress5 || !dims_ok(nx, ny, nz))
    return vpfft::lib_fail(VPFFT_ERR_INVALID_ARGUMENT, "bad argument");
  std::ifstream is(path);
  if (!is) return io_fail("cannot open", path);
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nz; ++k) {
        const long long v = voxel(i, j, k, ny, nz);
        for (int e = 0; e < 9; ++e) is >> std::skipws >> R9[v * 9 + e];
        for (int c = 0; c < 5; ++c) is >> std::skipws >> stress5[v * 5 + c];
        if (!is) return io_fail("too few or malformed values", path);
      }
  return VPFFT_OK;
}

vpfft_status vpfft_read_euler_texture(const char* path, int nx, int ny, int nz, double* R9) {
  if (!path || !R9 || !dims_ok(nx, ny, nz))
    return vpfft::lib_fail(VPFFT_ERR_INVALID_ARGUMENT, "bad argument");
  std::ifstream is(path);
  if (!is) return io_fail("cannot open", path);
  const long long count = (long long)nx * ny * nz;
  // DEGREE_TO_RADIAN (LinearAlgebra.h:28) with PI in double
  const double to_rad = 3.14159265358979323846 / (double)180.0f;
  for (long long r = 0; r < count; ++r) {
    double e0, e1, e2;
    int x, y, z, t0, t1;
    is >> std::skipws >> e0 >> std::skipws >> e1 >> std::skipws >> e2 >> std::skipws >> x >>
        std::skipws >> y >> std::skipws >> z >> std::skipws >> t0 >> std::skipws >> t1;
    if (!is) return io_fail("too few or malformed lines", path);
    if (x < 1 || x > nx || y < 1 || y > ny || z < 1 || z > nz)
      return io_fail("voxel index out of range", path);
    active_euler(e0 * to_rad, e1 * to_rad, e2 * to_rad, R9 + voxel(x - 1, y - 1, z - 1, ny, nz) * 9);
  }
  return VPFFT_OK;
}

vpfft_status vpfft_euler_matrix(double phi, double theta, double psi, double R9[9]) {
  if (!R9) return vpfft::lib_fail(VPFFT_ERR_INVALID_ARGUMENT, "bad argument");
  active_euler(phi, theta, psi, R9);
  return VPFFT_OK;
}

// UnitTester::SetMaterialGrid (UnitTester.cpp:46-74): quadrants of the x-y
// plane alternate between two grains, Euler (-40, 0, 0) and (0, 40, 0) degrees.
vpfft_status vpfft_fixture_two_grain(int nx, int ny, int nz, double* R9) {
  if (!R9 || !dims_ok(nx, ny, nz)) return vpfft::lib_fail(VPFFT_ERR_INVALID_ARGUMENT, "bad argument");
  const double to_rad = 3.14159265358979323846 / (double)180.0f;
  double left[9], right[9];
  active_euler(-40 * to_rad, 0, 0, left);
  active_euler(0 * to_rad, 40 * to_rad, 0, right);
  const int xh = nx / 2, yh = ny / 2;
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nz; ++k) {
        const bool l = (i >= xh && j >= yh) || (i < xh && j < yh);
        const double* src = l ? left : right;
        double* dst = R9 + voxel(i, j, k, ny, nz) * 9;
        for (int e = 0; e < 9; ++e) dst[e] = src[e];
      }
  return VPFFT_OK;
}

}  // extern "C"
