// fixtures.cpp -- host-only synthetic microstructures and 3x3 <-> 5-vector maps.
//
// The reference's own generator (SetRandomMaterialGrid, UnitTester.cpp:174-231)
// draws Euler angles with rand() % 360 (not uniform on SO(3)) and seeds on
// integer lattice points with a non-periodic distance.  The synthetic
// workloads here are re-specified so that they are reproducible anywhere:
//   * pseudo-random numbers: SplitMix64 (Steele, Lea & Flood, OOPSLA 2014);
//     u in [0,1) = top 53 bits * 2^-53;
//   * per grain, in this order: seed point (u*Nx, u*Ny, u*Nz), then Shoemake's
//     uniform unit quaternion from (u1, u2, u3) (Graphics Gems III, 1992);
//   * each voxel (x, y, z) belongs to the seed with the smallest periodic
//     (minimum-image) squared distance, ties to the lower seed index.
// The Voronoi search uses a cell list and gives exactly the brute-force answer.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "../../include/vpfft_capi.h"

namespace {

struct SplitMix64 {
  uint64_t s;
  uint64_t next() {
    s += 0x9E3779B97F4A7C15ull;
    uint64_t z = s;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  double u01() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
};

// active rotation matrix of the unit quaternion (w, x, y, z), row-major
void quat_to_R(double w, double x, double y, double z, double* R) {
  R[0] = 1 - 2 * (y * y + z * z);
  R[1] = 2 * (x * y - w * z);
  R[2] = 2 * (x * z + w * y);
  R[3] = 2 * (x * y + w * z);
  R[4] = 1 - 2 * (x * x + z * z);
  R[5] = 2 * (y * z - w * x);
  R[6] = 2 * (x * z - w * y);
  R[7] = 2 * (y * z + w * x);
  R[8] = 1 - 2 * (x * x + y * y);
}

// deviatoric basis of LinearAlgebra.h:207-247 (first five elements)
void basis(double B[5][3][3]) {
  std::memset(B, 0, sizeof(double) * 45);
  const double a = 1.0 / std::sqrt(2.0), b = 1.0 / std::sqrt(6.0);
  B[0][0][0] = -1 * a;
  B[0][1][1] = 1 * a;
  B[1][0][0] = -1 * b;
  B[1][1][1] = -1 * b;
  B[1][2][2] = 2 * b;
  B[2][1][2] = B[2][2][1] = 1 * a;
  B[3][0][2] = B[3][2][0] = 1 * a;
  B[4][0][1] = B[4][1][0] = 1 * a;
}

inline double pdist2(double x, double y, double z, const double* p, int nx, int ny, int nz) {
  double dx = std::fabs(x - p[0]);
  dx = std::min(dx, nx - dx);
  double dy = std::fabs(y - p[1]);
  dy = std::min(dy, ny - dy);
  double dz = std::fabs(z - p[2]);
  dz = std::min(dz, nz - dz);
  return dx * dx + dy * dy + dz * dz;
}

}  // namespace

extern "C" {

vpfft_status vpfft_fixture_polycrystal(int nx, int ny, int nz, int ng, uint64_t seed,
                                       double* R_out, int32_t* grain_out) {
  if (nx < 1 || ny < 1 || nz < 1 || ng < 1 || !R_out) return VPFFT_ERR_INVALID_ARGUMENT;
  SplitMix64 rng{seed};
  std::vector<double> pts(3 * (size_t)ng), rot(9 * (size_t)ng);
  const double two_pi = 6.283185307179586476925286766559;
  for (int g = 0; g < ng; ++g) {
    pts[3 * g + 0] = rng.u01() * nx;
    pts[3 * g + 1] = rng.u01() * ny;
    pts[3 * g + 2] = rng.u01() * nz;
    const double u1 = rng.u01(), u2 = rng.u01(), u3 = rng.u01();
    const double a = std::sqrt(1.0 - u1), b = std::sqrt(u1);
    const double qx = a * std::sin(two_pi * u2), qy = a * std::cos(two_pi * u2);
    const double qz = b * std::sin(two_pi * u3), qw = b * std::cos(two_pi * u3);
    quat_to_R(qw, qx, qy, qz, &rot[9 * (size_t)g]);
  }
  // cell list
  const int dims[3] = {nx, ny, nz};
  int C[3];
  const int c0 = std::max(1, (int)std::floor(std::cbrt((double)ng)));
  double w[3];
  for (int a = 0; a < 3; ++a) {
    C[a] = std::max(1, std::min(dims[a], c0));
    w[a] = (double)dims[a] / C[a];
  }
  std::vector<std::vector<int>> cells((size_t)C[0] * C[1] * C[2]);
  for (int g = 0; g < ng; ++g) {
    int c[3];
    for (int a = 0; a < 3; ++a) c[a] = std::min(C[a] - 1, (int)std::floor(pts[3 * g + a] / w[a]));
    cells[((size_t)c[0] * C[1] + c[1]) * C[2] + c[2]].push_back(g);
  }
  const int rmax = std::max(C[0], std::max(C[1], C[2]));
  auto work = [&](int x0, int x1) {
    for (int x = x0; x < x1; ++x)
      for (int y = 0; y < ny; ++y)
        for (int z = 0; z < nz; ++z) {
          const double pos[3] = {(double)x, (double)y, (double)z};
          int c[3];
          for (int a = 0; a < 3; ++a) c[a] = std::min(C[a] - 1, (int)std::floor(pos[a] / w[a]));
          double best = INFINITY;
          int bi = 0x7fffffff;
          for (int r = 0; r <= rmax; ++r) {
            for (int dx = -r; dx <= r; ++dx)
              for (int dy = -r; dy <= r; ++dy)
                for (int dz = -r; dz <= r; ++dz) {
                  if (std::max(std::abs(dx), std::max(std::abs(dy), std::abs(dz))) != r) continue;
                  const int cx = ((c[0] + dx) % C[0] + C[0]) % C[0];
                  const int cy = ((c[1] + dy) % C[1] + C[1]) % C[1];
                  const int cz = ((c[2] + dz) % C[2] + C[2]) % C[2];
                  for (int g : cells[((size_t)cx * C[1] + cy) * C[2] + cz]) {
                    const double d2 = pdist2(pos[0], pos[1], pos[2], &pts[3 * (size_t)g], nx, ny, nz);
                    if (d2 < best || (d2 == best && g < bi)) {
                      best = d2;
                      bi = g;
                    }
                  }
                }
            // lower bound on the distance of any seed outside the searched block
            double lb = INFINITY;
            bool all = true;
            for (int a = 0; a < 3; ++a) {
              if (2 * r + 1 >= C[a]) continue;
              all = false;
              const double lo = (c[a] - r) * w[a], hi = (c[a] + r + 1) * w[a];
              lb = std::min(lb, std::min(pos[a] - lo, hi - pos[a]));
            }
            if (all) break;
            if (best < lb * lb) break;
          }
          const size_t v = ((size_t)x * ny + y) * nz + z;
          std::memcpy(R_out + 9 * v, &rot[9 * (size_t)bi], sizeof(double) * 9);
          if (grain_out) grain_out[v] = bi;
        }
  };
  unsigned nt = std::max(1u, std::min(std::thread::hardware_concurrency(), (unsigned)nx));
  if ((long long)nx * ny * nz < 65536) nt = 1;
  std::vector<std::thread> th;
  for (unsigned t = 0; t < nt; ++t) {
    const int x0 = (int)((long long)nx * t / nt), x1 = (int)((long long)nx * (t + 1) / nt);
    th.emplace_back(work, x0, x1);
  }
  for (auto& t : th) t.join();
  return VPFFT_OK;
}

void vpfft_edot_from_matrix(const double L[9], double out[5]) {
  double B[5][3][3];
  basis(B);
  for (int a = 0; a < 5; ++a) {
    double r = 0;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) r += L[3 * i + j] * B[a][i][j];
    out[a] = r;
  }
}

void vpfft_matrix_from_edot(const double e[5], double L[9]) {
  double B[5][3][3];
  basis(B);
  for (int k = 0; k < 9; ++k) L[k] = 0;
  for (int a = 0; a < 5; ++a)
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) L[3 * i + j] += B[a][i][j] * e[a];
}

}  // extern "C"
