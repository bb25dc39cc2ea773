// ref_harness.cpp -- drives the UNMODIFIED reference sources (MaterialGrid,
// Solvers, LinearAlgebra) through their own API and records what they compute.
// Test-oracle infrastructure: it is compiled together with the reference's
// Src/*.cpp and the project-written MPI/FFTW/Eigen stand-ins in ./shims by
// oracle/Makefile into oracle/_ref/vpfft_ref, and it is run only by the
// golden-fixture generator, the parity tests and the CPU baseline arm of
// bench.py.
//
// Flow, mirroring UnitTester::MPI_VPFFT_Test (UnitTester.cpp:384-457):
//   MaterialGrid(nx,ny,nz)                       MaterialGrid.h:72-78
//   material vectors set after construction      (hard-coded in
//                                                 InitializeMemory 322-336,390)
//   SendDataAndInitialize(R, sigma)              MaterialGrid.cpp:425-534
//   SetVoxelLength(h)                            MaterialGrid.h:97-102
//   RunSingleStrainStep(Edot, maxIter, dt, eps)  MaterialGrid.cpp:897-1084
//     repeated nsteps times like RunVPFFT        MaterialGrid.cpp:1202-1228
//
// Observations come from the stand-ins' hooks only:
//   * every MPI_Allreduce value (25 L0 entries per increment, then 12 per
//     fixed-point iteration: <sigma>_i and <edot>_i interleaved, then the two
//     error-norm sums; MaterialGrid.cpp:257-271, 1009-1045);
//   * the polarization / strain-rate-variation buffers just before each
//     forward FFT of polarization component 0 (MaterialGrid.cpp:639, 780):
//     at that moment they hold P and d~ produced by the previous iteration.
//
// Usage: vpfft_ref <input.bin> <outdir> [--dump-iter K]... [--dump-increments] [--quiet]
//                  [--run-vpfft] [--timing-only] [--ranks P] [--generate GRAINS SEED]
//   --run-vpfft    drive the increments through RunVPFFT (writes Stress_Strain.txt)
//   --timing-only  no copies of P and d~ at each iteration (benchmark runs)
//   --ranks P      run the reference as P MPI ranks (processes sharing memory
//                  through the stand-ins); only timing and reductions are written
//   --generate G S the input file carries no orientations: make the synthetic
//                  polycrystal with G grains and seed S (oracle/common/polycrystal.c)
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <limits>
#include <queue>
#include <sstream>
#include <string>
#include <vector>

#include <unistd.h>

#include "Eigen/Dense"
#include "fftw3-mpi.h"
#include "mpi.h"
#include "shim_hooks.h"
#include "../common/polycrystal.h"

// The harness needs read/write access to MaterialGrid's private fields
// (material parameters are hard-coded in InitializeMemory and there is no
// setter).  Access specifiers do not change the object layout under the
// Itanium C++ ABI, so this TU may see them as public while the reference's
// own TUs are compiled unchanged.
#define private public
#include "MaterialGrid.h"
#undef private

using VPFFT::DataStructures::MaterialGrid;
using VPFFT::LinearAlgebra::EigenRep;
using VPFFT::LinearAlgebra::SMatrix3x3;

static_assert(sizeof(SMatrix3x3) == 9 * sizeof(double), "SMatrix3x3 layout");
static_assert(sizeof(EigenRep) == 5 * sizeof(double), "EigenRep layout");

namespace {

struct Input {
  int nx, ny, nz, nsteps, max_iter, crss_per_voxel, edot_per_increment;
  int generated;  // no per-voxel arrays in the file: orientations from --generate
  double dt, eps, edot[5], h[3];
  std::vector<double> edot_steps;  // nsteps x 5 when edot_per_increment
  double gdot[12];
  int nexp[12];
  double tau0[12], tau1[12], theta0[12], theta1[12], H[144];
  std::vector<double> R, sigma, crss;
};

template <typename T> void rd(std::ifstream &f, T *p, size_t n) {
  f.read(reinterpret_cast<char *>(p), sizeof(T) * n);
  if (!f) {
    std::fprintf(stderr, "vpfft_ref: truncated input\n");
    std::exit(2);
  }
}

Input read_input(const char *path) {
  std::ifstream f(path, std::ios::binary);
  if (!f) {
    std::fprintf(stderr, "vpfft_ref: cannot open %s\n", path);
    std::exit(2);
  }
  char magic[8];
  rd(f, magic, 8);
  if (std::memcmp(magic, "VPFFTIN1", 8) != 0) {
    std::fprintf(stderr, "vpfft_ref: bad magic\n");
    std::exit(2);
  }
  Input in;
  int32_t hdr[8];
  rd(f, hdr, 8);
  in.nx = hdr[0];
  in.ny = hdr[1];
  in.nz = hdr[2];
  in.nsteps = hdr[3];
  in.max_iter = hdr[4];
  in.crss_per_voxel = hdr[5];
  in.edot_per_increment = hdr[6];
  in.generated = hdr[7];
  rd(f, &in.dt, 1);
  rd(f, &in.eps, 1);
  rd(f, in.edot, 5);
  rd(f, in.h, 3);
  rd(f, in.gdot, 12);
  int32_t ne[12];
  rd(f, ne, 12);
  for (int i = 0; i < 12; ++i) in.nexp[i] = ne[i];
  rd(f, in.tau0, 12);
  rd(f, in.tau1, 12);
  rd(f, in.theta0, 12);
  rd(f, in.theta1, 12);
  rd(f, in.H, 144);
  size_t N = (size_t)in.nx * in.ny * in.nz;
  if (!in.generated) {
    in.R.resize(N * 9);
    in.sigma.resize(N * 5);
    rd(f, in.R.data(), N * 9);
    rd(f, in.sigma.data(), N * 5);
  } else if (in.crss_per_voxel) {
    std::fprintf(stderr, "vpfft_ref: generated inputs take a uniform CRSS\n");
    std::exit(2);
  }
  in.crss.resize(in.crss_per_voxel ? N * 12 : 12);
  rd(f, in.crss.data(), in.crss.size());
  if (in.edot_per_increment) {
    in.edot_steps.resize((size_t)in.nsteps * 5);
    rd(f, in.edot_steps.data(), in.edot_steps.size());
  }
  return in;
}

void write_bin(const std::string &path, const double *p, size_t n) {
  FILE *f = std::fopen(path.c_str(), "wb");
  if (!f) {
    std::fprintf(stderr, "vpfft_ref: cannot write %s\n", path.c_str());
    std::exit(2);
  }
  std::fwrite(p, sizeof(double), n, f);
  std::fclose(f);
}

struct Observer {
  MaterialGrid *grid = nullptr;
  size_t N = 0;
  std::string outdir;
  int increment = 0;
  int fwd_p0_in_increment = 0;  // forward FFTs of P component 0 seen this increment
  bool snapshots = true;        // copy P and d~ at each forward FFT of P0
  std::vector<int> dump_iters;  // iteration indices of increment 0 to dump
  std::vector<double> allreduce;
  // allreduce values recorded when each increment began (RunVPFFT mode: the
  // reference's MPI_Barrier after each increment marks the boundary)
  std::vector<size_t> increment_ar_starts{0};
  std::vector<double> fwd_times;  // steady-clock seconds at each forward P0 FFT
  std::vector<double> fwd_fft_seconds;  // seconds inside fftw_execute by then
  std::vector<int> fwd_increment;
  // last snapshot of P and d~ (real parts), [N][5]
  std::vector<double> lastP, lastD;

  void snapshot(std::vector<double> &dst, MaterialGrid::FFTW_ComplexPtr *arr) {
    dst.resize(N * 5);
    for (size_t v = 0; v < N; ++v)
      for (int c = 0; c < 5; ++c) dst[v * 5 + c] = arr[c][v][0];
  }
};

Observer g_obs;

void on_exec(int sign, double (*data)[2], long, void *) {
  Observer &o = g_obs;
  if (!o.grid || sign != FFTW_FORWARD) return;
  if (data != o.grid->_PolarizationField[0]) return;
  o.fwd_times.push_back(
      std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count());
  o.fwd_fft_seconds.push_back(vpfft_shim_fft_seconds());
  o.fwd_increment.push_back(o.increment);
  // Before this forward FFT the buffers hold the previous iteration's P and d~.
  int iter = o.fwd_p0_in_increment;  // 0 = after initialisation, k = after iteration k
  ++o.fwd_p0_in_increment;
  if (!o.snapshots) return;
  o.snapshot(o.lastP, o.grid->_PolarizationField);
  o.snapshot(o.lastD, o.grid->_DisplacementVariation);
  if (o.increment == 0 &&
      std::find(o.dump_iters.begin(), o.dump_iters.end(), iter) != o.dump_iters.end()) {
    std::string pre = o.outdir + "/it" + std::to_string(iter) + "_";
    write_bin(pre + "P.bin", o.lastP.data(), o.lastP.size());
    write_bin(pre + "dtilde.bin", o.lastD.data(), o.lastD.size());
    write_bin(pre + "sigma.bin", reinterpret_cast<const double *>(o.grid->StressField), o.N * 5);
    write_bin(pre + "lambda.bin",
              reinterpret_cast<const double *>(o.grid->LagrangeMultiplierField.data()), o.N * 5);
  }
}

void on_barrier(void *) {
  g_obs.increment_ar_starts.push_back(g_obs.allreduce.size());
  ++g_obs.increment;
  g_obs.fwd_p0_in_increment = 0;
}

void on_allreduce(const double *v, int count, void *) {
  for (int i = 0; i < count; ++i) g_obs.allreduce.push_back(v[i]);
}

}  // namespace

int main(int argc, char **argv) {
  if (argc < 3) {
    std::fprintf(stderr, "usage: vpfft_ref <input.bin> <outdir> [--dump-iter K]... [--quiet]\n");
    return 2;
  }
  bool quiet = false, dump_increments = false, run_vpfft = false;
  int ranks = 1, gen_grains = 0;
  unsigned long long gen_seed = 0;
  for (int a = 3; a < argc; ++a) {
    if (!std::strcmp(argv[a], "--dump-iter") && a + 1 < argc)
      g_obs.dump_iters.push_back(std::atoi(argv[++a]));
    else if (!std::strcmp(argv[a], "--quiet"))
      quiet = true;
    else if (!std::strcmp(argv[a], "--dump-increments"))
      dump_increments = true;
    else if (!std::strcmp(argv[a], "--run-vpfft"))
      run_vpfft = true;
    else if (!std::strcmp(argv[a], "--timing-only"))
      g_obs.snapshots = false;
    else if (!std::strcmp(argv[a], "--ranks") && a + 1 < argc)
      ranks = std::atoi(argv[++a]);
    else if (!std::strcmp(argv[a], "--generate") && a + 2 < argc) {
      gen_grains = std::atoi(argv[++a]);
      gen_seed = std::strtoull(argv[++a], nullptr, 10);
    }
  }
  Input in = read_input(argv[1]);
  const size_t N = (size_t)in.nx * in.ny * in.nz;
  g_obs.N = N;
  g_obs.outdir = argv[2];
  if (in.generated && gen_grains < 1) {
    std::fprintf(stderr, "vpfft_ref: the input has no orientations; give --generate G SEED\n");
    return 2;
  }
  // With several ranks each process holds a slab of the grid; only timing,
  // the reduced values and <sigma> are written (no per-voxel fields).
  if (ranks > 1) {
    g_obs.snapshots = false;
    if (!g_obs.dump_iters.empty() || dump_increments || run_vpfft || in.crss_per_voxel) {
      std::fprintf(stderr, "vpfft_ref: --ranks > 1 writes no per-voxel output\n");
      return 2;
    }
    const size_t slab = (size_t)((in.nx + ranks - 1) / ranks) * in.ny * in.nz;
    if (vpfft_shim_configure(ranks, slab * 10 * sizeof(fftw_complex) + (1u << 20),
                             N * (sizeof(SMatrix3x3) + sizeof(EigenRep)) + (1u << 20)) != 0) {
      std::fprintf(stderr, "vpfft_ref: bad rank count %d\n", ranks);
      return 2;
    }
  }

  // The reference prints progress to std::cout; keep stdout for our summary.
  std::ofstream devnull("/dev/null");
  std::streambuf *saved = std::cout.rdbuf();
  if (quiet) std::cout.rdbuf(devnull.rdbuf());

  int argc0 = 0;
  MPI_Init(&argc0, nullptr);
  int rank = 0;
  MPI_Comm_rank(MPI_COMM_WORLD, &rank);
  MaterialGrid grid(in.nx, in.ny, in.nz);
  for (int s = 0; s < 12; ++s) {
    grid.GammaDotBase[s] = in.gdot[s];
    grid.RateSensitivity[s] = in.nexp[s];
    grid.Tau0[s] = in.tau0[s];
    grid.Tau1[s] = in.tau1[s];
    grid.Theta0[s] = in.theta0[s];
    grid.Theta1[s] = in.theta1[s];
    for (int t = 0; t < 12; ++t) grid.HardeningMatrix[s][t] = in.H[s * 12 + t];
  }
  if (rank == 0) {
    if (in.generated) {
      in.R.resize(N * 9);
      in.sigma.assign(N * 5, 0.0);
      if (oracle_polycrystal(in.nx, in.ny, in.nz, gen_grains, gen_seed, ranks, in.R.data(),
                             nullptr) != 0) {
        std::fprintf(stderr, "vpfft_ref: polycrystal generation failed\n");
        return 2;
      }
    }
    grid.SendDataAndInitialize(reinterpret_cast<SMatrix3x3 *>(in.R.data()),
                               reinterpret_cast<EigenRep *>(in.sigma.data()));
    if (ranks > 1) {  // the caller's arrays are no longer needed
      std::vector<double>().swap(in.R);
      std::vector<double>().swap(in.sigma);
    }
  } else {
    grid.RecvDataAndInitialize();
  }
  const size_t n_local = (size_t)grid.DimXLocal * grid.DimYZ;
  for (size_t v = 0; v < n_local; ++v)
    for (int s = 0; s < 12; ++s)
      grid.LocalCRSS[v][s] = in.crss_per_voxel ? in.crss[v * 12 + s] : in.crss[s];
  grid.SetVoxelLength(in.h[0], in.h[1], in.h[2]);

  g_obs.grid = &grid;
  vpfft_shim_set_exec_hook(on_exec, nullptr);
  vpfft_shim_set_allreduce_hook(on_allreduce, nullptr);
  if (run_vpfft) vpfft_shim_set_barrier_hook(on_barrier, nullptr);

  EigenRep edot(in.edot[0], in.edot[1], in.edot[2], in.edot[3], in.edot[4]);
  std::vector<double> steps;        // per increment: iters, <sigma>(5)
  std::vector<double> ar_counts;    // per increment: allreduce values recorded
  std::vector<double> step_seconds; // per increment wall time
  if (run_vpfft) {
    // the reference's own multi-increment driver (MaterialGrid.cpp:1202-1228),
    // which writes Stress_Strain.txt into the working directory
    if (chdir(g_obs.outdir.c_str()) != 0) {
      std::fprintf(stderr, "vpfft_ref: cannot enter %s\n", g_obs.outdir.c_str());
      return 2;
    }
    g_obs.increment = 0;
    auto t0 = std::chrono::steady_clock::now();
    grid.RunVPFFT(edot, in.max_iter, in.nsteps, in.dt, in.eps);
    auto t1 = std::chrono::steady_clock::now();
    // one increment opens with 25 L0 values and adds 12 per iteration; split
    // the recorded values at each L0 block (the fwd hook counts increments)
    size_t off = 0;
    for (int step = 0; step < in.nsteps; ++step) {
      size_t nvals = (step + 1 < (int)g_obs.increment_ar_starts.size())
                         ? g_obs.increment_ar_starts[step + 1] - off
                         : g_obs.allreduce.size() - off;
      steps.push_back((double)((nvals - 25) / 12));
      for (int c = 0; c < 5; ++c) steps.push_back(0.0);
      ar_counts.push_back((double)nvals);
      step_seconds.push_back(std::chrono::duration<double>(t1 - t0).count() / in.nsteps);
      off += nvals;
    }
  }
  for (int step = 0; step < (run_vpfft ? 0 : in.nsteps); ++step) {
    g_obs.increment = step;
    g_obs.fwd_p0_in_increment = 0;
    if (in.edot_per_increment) {
      const double *e = &in.edot_steps[(size_t)step * 5];
      edot = EigenRep(e[0], e[1], e[2], e[3], e[4]);
    }
    size_t ar0 = g_obs.allreduce.size();
    auto t0 = std::chrono::steady_clock::now();
    EigenRep avg = grid.RunSingleStrainStep(edot, in.max_iter, in.dt, in.eps);
    auto t1 = std::chrono::steady_clock::now();
    size_t nvals = g_obs.allreduce.size() - ar0;
    int iters = (int)((nvals - 25) / 12);
    steps.push_back(iters);
    for (int c = 0; c < 5; ++c) steps.push_back(avg(c));
    ar_counts.push_back((double)nvals);
    step_seconds.push_back(std::chrono::duration<double>(t1 - t0).count());
    // P and d~ of the last fixed-point iteration are the last snapshot taken,
    // at the forward FFT that starts OrientationEvolutionWithFFT.
    if (dump_increments) {
      const std::string pre = g_obs.outdir + "/inc" + std::to_string(step) + "_";
      write_bin(pre + "sigma.bin", reinterpret_cast<const double *>(grid.StressField), N * 5);
      write_bin(pre + "lambda.bin",
                reinterpret_cast<const double *>(grid.LagrangeMultiplierField.data()), N * 5);
      write_bin(pre + "R.bin", reinterpret_cast<const double *>(grid.OrientationField), N * 9);
      std::vector<double> cr(N * 12);
      for (size_t v = 0; v < N; ++v)
        for (int s = 0; s < 12; ++s) cr[v * 12 + s] = grid.LocalCRSS[v][s];
      write_bin(pre + "crss.bin", cr.data(), cr.size());
    }
  }
  std::cout.rdbuf(saved);
  if (rank != 0) {
    MPI_Finalize();
    return 0;
  }

  const std::string od = g_obs.outdir;
  write_bin(od + "/steps.bin", steps.data(), steps.size());
  write_bin(od + "/allreduce.bin", g_obs.allreduce.data(), g_obs.allreduce.size());
  write_bin(od + "/allreduce_counts.bin", ar_counts.data(), ar_counts.size());
  write_bin(od + "/step_seconds.bin", step_seconds.data(), step_seconds.size());
  write_bin(od + "/fwd_times.bin", g_obs.fwd_times.data(), g_obs.fwd_times.size());
  std::vector<double> fwd_inc(g_obs.fwd_increment.begin(), g_obs.fwd_increment.end());
  write_bin(od + "/fwd_increment.bin", fwd_inc.data(), fwd_inc.size());
  write_bin(od + "/fwd_fft_seconds.bin", g_obs.fwd_fft_seconds.data(),
            g_obs.fwd_fft_seconds.size());
  if (ranks > 1) {
    std::printf("{\"increments\": %d, \"ranks\": %d, \"iters\": [", in.nsteps, ranks);
    for (int s = 0; s < in.nsteps; ++s) std::printf("%s%d", s ? ", " : "", (int)steps[s * 6]);
    std::printf("]}\n");
    std::fflush(stdout);
    MPI_Finalize();
    return 0;
  }
  write_bin(od + "/sigma.bin", reinterpret_cast<const double *>(grid.StressField), N * 5);
  write_bin(od + "/lambda.bin",
            reinterpret_cast<const double *>(grid.LagrangeMultiplierField.data()), N * 5);
  write_bin(od + "/R.bin", reinterpret_cast<const double *>(grid.OrientationField), N * 9);
  std::vector<double> crss(N * 12);
  for (size_t v = 0; v < N; ++v)
    for (int s = 0; s < 12; ++s) crss[v * 12 + s] = grid.LocalCRSS[v][s];
  write_bin(od + "/crss.bin", crss.data(), crss.size());
  write_bin(od + "/accshear.bin", grid.AccumulatedShear.data(), N);
  double h[3] = {grid.XVoxelLength, grid.YVoxelLength, grid.ZVoxelLength};
  write_bin(od + "/voxlen.bin", h, 3);
  write_bin(od + "/P_last.bin", g_obs.lastP.data(), g_obs.lastP.size());
  write_bin(od + "/dtilde_last.bin", g_obs.lastD.data(), g_obs.lastD.size());
  std::vector<double> sch(N * 60);
  for (size_t v = 0; v < N; ++v)
    for (int s = 0; s < 12; ++s)
      for (int c = 0; c < 5; ++c) sch[v * 60 + s * 5 + c] = grid.LocalSchmidtTensor[v][s](c);
  write_bin(od + "/schmid.bin", sch.data(), sch.size());

  std::printf("{\"increments\": %d, \"iters\": [", in.nsteps);
  for (int s = 0; s < in.nsteps; ++s) std::printf("%s%d", s ? ", " : "", (int)steps[s * 6]);
  std::printf("], \"seconds\": [");
  for (int s = 0; s < in.nsteps; ++s) std::printf("%s%.6f", s ? ", " : "", step_seconds[s]);
  std::printf("]}\n");
  MPI_Finalize();
  return 0;
}
