// ref_io_harness.cpp -- runs the reference's own text I/O routines to produce
// golden files for the I/O parity tests (test infrastructure, not product).
//
//   vpfft_ref_io <outdir>
//
// On a 6 x 5 x 4 grid with deterministic values (written next to the outputs
// as raw doubles so a test can feed the same numbers to another writer):
//   random_material.txt      UnitTester::WriteRandomMaterial (UnitTester.cpp:116-137)
//   read_R.bin, read_S.bin   UnitTester::ReadRandomMaterial of that file (139-167)
//   stress.txt, lagrange.txt, strain.txt, polarization.txt
//                            MaterialGrid::PrintStress / PrintLagrangeMultiplier /
//                            PrintStrain / PrintPolarization (MaterialGrid.cpp:15-100)
//   texture.txt, texture_R.bin
//                            UnitTester::ReadRicardoData (UnitTester.cpp:237-265) of a
//                            generated Euler-angle file, and the orientations it set
//   two_grain_R.bin          UnitTester::SetMaterialGrid (UnitTester.cpp:46-74) on 7 x 5 x 2
// Inputs: in_R.bin (N x 9), in_S.bin (N x 5), in_L.bin (N x 5),
// in_D.bin / in_P.bin (N x 5 x 2, re/im).
#include <cmath>
#include <cstdio>
#include <fstream>
#include <string>
#include <vector>

#define private public
#define protected public
#include "MaterialGrid.h"
#include "UnitTester.h"
#undef private
#undef protected

// defined in UnitTester.cpp:46-74 (the header declares other overloads)
namespace VPFFT {
namespace UnitTester {
void SetMaterialGrid(VPFFT::LinearAlgebra::SMatrix3x3* OrientList,
                     VPFFT::LinearAlgebra::EigenRep* Stress, int NumX, int NumY, int NumZ,
                     const VPFFT::DataStructures::MaterialGrid& Grid);
}
}  // namespace VPFFT

using VPFFT::DataStructures::MaterialGrid;
using VPFFT::LinearAlgebra::EigenRep;
using VPFFT::LinearAlgebra::SMatrix3x3;

static void dump(const std::string& path, const std::vector<double>& v) {
  FILE* f = std::fopen(path.c_str(), "wb");
  std::fwrite(v.data(), sizeof(double), v.size(), f);
  std::fclose(f);
}

// values spanning many decades, both signs and exact zeros (exercise %g)
static double val(int idx, int c, int salt) {
  const double base = std::sin(1.0 + 0.37 * idx + 1.3 * c + 0.11 * salt);
  const int e = ((idx * 7 + c * 3 + salt) % 15) - 8;  // 1e-8 .. 1e6
  if ((idx + c + salt) % 23 == 0) return 0.0;
  return base * std::pow(10.0, e);
}

int main(int argc, char** argv) {
  if (argc < 2) {
    std::fprintf(stderr, "usage: vpfft_ref_io <outdir>\n");
    return 2;
  }
  const std::string out = std::string(argv[1]) + "/";
  MPI_Init(&argc, &argv);
  const int nx = 6, ny = 5, nz = 4, n = nx * ny * nz;
  MaterialGrid grid(nx, ny, nz);

  std::vector<SMatrix3x3> R(n);
  std::vector<EigenRep> S(n);
  std::vector<double> inR(n * 9), inS(n * 5), inL(n * 5), inD(n * 10), inP(n * 10);
  for (int v = 0; v < n; ++v) {
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) {
        R[v].m[a][b] = val(v, a * 3 + b, 1);
        inR[v * 9 + a * 3 + b] = R[v].m[a][b];
      }
    for (int c = 0; c < 5; ++c) {
      S[v].m[c] = val(v, c, 2);
      inS[v * 5 + c] = S[v].m[c];
      inL[v * 5 + c] = val(v, c, 3);
      inD[v * 10 + 2 * c] = val(v, c, 4);
      inD[v * 10 + 2 * c + 1] = val(v, c, 5);
      inP[v * 10 + 2 * c] = val(v, c, 6);
      inP[v * 10 + 2 * c + 1] = val(v, c, 7);
    }
  }
  dump(out + "in_R.bin", inR);
  dump(out + "in_S.bin", inS);
  dump(out + "in_L.bin", inL);
  dump(out + "in_D.bin", inD);
  dump(out + "in_P.bin", inP);

  // random material round trip
  VPFFT::UnitTester::WriteRandomMaterial(R.data(), S.data(), nx, ny, nz, grid,
                                         out + "random_material.txt");
  std::vector<SMatrix3x3> R2(n);
  std::vector<EigenRep> S2(n);
  VPFFT::UnitTester::ReadRandomMaterial(R2.data(), S2.data(), nx, ny, nz, grid,
                                        out + "random_material.txt");
  std::vector<double> rR(n * 9), rS(n * 5);
  for (int v = 0; v < n; ++v) {
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) rR[v * 9 + a * 3 + b] = R2[v].m[a][b];
    for (int c = 0; c < 5; ++c) rS[v * 5 + c] = S2[v].m[c];
  }
  dump(out + "read_R.bin", rR);
  dump(out + "read_S.bin", rS);

  // field dumps
  for (int x = 0; x < nx; ++x)
    for (int y = 0; y < ny; ++y)
      for (int z = 0; z < nz; ++z) {
        const int v = grid.ToIndex(x, y, z);
        for (int c = 0; c < 5; ++c) {
          grid.Stress(x, y, z).m[c] = inS[v * 5 + c];
          grid.LagrangeMultiplier(x, y, z).m[c] = inL[v * 5 + c];
          grid.DisplacementVariation(x, y, z, c)[0] = inD[v * 10 + 2 * c];
          grid.DisplacementVariation(x, y, z, c)[1] = inD[v * 10 + 2 * c + 1];
          grid.PolarizationField(x, y, z, c)[0] = inP[v * 10 + 2 * c];
          grid.PolarizationField(x, y, z, c)[1] = inP[v * 10 + 2 * c + 1];
        }
      }
  grid.PrintStress(out + "stress.txt");
  grid.PrintLagrangeMultiplier(out + "lagrange.txt");
  grid.PrintStrain(out + "strain.txt");
  grid.PrintPolarization(out + "polarization.txt");

  // Euler-angle texture file (the reference's ReadRicardoData format): one
  // line per voxel, angles in degrees, 1-based x y z, two trailing integers,
  // in a scrambled voxel order
  {
    std::ofstream t((out + "texture.txt").c_str());
    for (int k = 0; k < n; ++k) {
      const int v = (k * 37) % n;  // 37 is coprime with 120
      const int x = v / (ny * nz), y = (v / nz) % ny, z = v % nz;
      char line[256];
      std::snprintf(line, sizeof line, "%10.3f %9.3f %10.3f %4d %4d %4d %3d %3d\n",
                    std::fmod(17.123 * v + 3.5, 360.0), std::fmod(7.77 * v + 1.25, 180.0),
                    std::fmod(29.3 * v + 11.0, 360.0), x + 1, y + 1, z + 1, v % 5, 1);
      t << line;
    }
  }
  VPFFT::UnitTester::ReadRicardoData(out + "texture.txt", nx, ny, nz, grid);
  std::vector<double> tR(n * 9);
  for (int x = 0; x < nx; ++x)
    for (int y = 0; y < ny; ++y)
      for (int z = 0; z < nz; ++z) {
        const int v = grid.ToIndex(x, y, z);
        for (int a = 0; a < 3; ++a)
          for (int b = 0; b < 3; ++b) tR[v * 9 + a * 3 + b] = grid.Orientation(x, y, z).m[a][b];
      }
  dump(out + "texture_R.bin", tR);

  // the two-grain microstructure of the config's TwoGrainInit
  // (UnitTester::SetMaterialGrid, UnitTester.cpp:46-74), on a 7 x 5 x 2 grid
  {
    const int ax = 7, ay = 5, az = 2, an = ax * ay * az;
    MaterialGrid g2(ax, ay, az);
    std::vector<SMatrix3x3> R2g(an);
    std::vector<EigenRep> S2g(an);
    VPFFT::UnitTester::SetMaterialGrid(R2g.data(), S2g.data(), ax, ay, az, g2);
    std::vector<double> o(an * 9);
    for (int v = 0; v < an; ++v)
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) o[v * 9 + a * 3 + b] = R2g[v].m[a][b];
    dump(out + "two_grain_R.bin", o);
  }
  MPI_Finalize();
  return 0;
}
