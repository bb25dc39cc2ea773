// vpfft/MaterialGrid.hpp -- header-only C++ facade over vpfft_capi.h that keeps
// the reference's class and method names (MaterialGrid.h:59-577), so host
// code written against VPFFT::DataStructures::MaterialGrid keeps compiling:
//
//   VPFFT::DataStructures::MaterialGrid g(16, 16, 16);
//   g.SendDataAndInitialize(OrientList, StressList);
//   g.SetVoxelLength(1, 1, 1);
//   EigenRep avg = g.RunSingleStrainStep(Edot, 100, 0.03, 1e-5);
//
// Differences from the reference, by design: the constructor takes optional
// material/solver constants (the reference hard-codes them), failures throw
// VPFFT::Error instead of calling exit(0), the destructor frees the device
// state (the reference leaks), and the per-voxel accessors copy fields back
// from the device in bulk (Stress(), Orientation(), ...) instead of returning
// references into host arrays.
#ifndef VPFFT_MATERIALGRID_HPP
#define VPFFT_MATERIALGRID_HPP

#include <stdexcept>
#include <string>
#include <vector>

#include "../vpfft_capi.h"

namespace VPFFT {

struct Error : std::runtime_error {
  vpfft_status status;
  Error(vpfft_status s, const std::string& m) : std::runtime_error(m), status(s) {}
};

namespace LinearAlgebra {
// Layout-compatible with the reference's value types (LinearAlgebra.h:44-115, 298-521):
// arrays of them can be passed to the C ABI unchanged.
struct SMatrix3x3 {
  double m[3][3];
};
struct EigenRep {
  double m[5];
  EigenRep() : m{0, 0, 0, 0, 0} {}
  EigenRep(double a, double b, double c, double d, double e) : m{a, b, c, d, e} {}
  explicit EigenRep(const SMatrix3x3& M) { vpfft_edot_from_matrix(&M.m[0][0], m); }
  double operator()(int n) const { return m[n]; }
  double& operator()(int n) { return m[n]; }
  SMatrix3x3 ToMatrixRep() const {
    SMatrix3x3 r;
    vpfft_matrix_from_edot(m, &r.m[0][0]);
    return r;
  }
};
static_assert(sizeof(SMatrix3x3) == 9 * sizeof(double), "SMatrix3x3 layout");
static_assert(sizeof(EigenRep) == 5 * sizeof(double), "EigenRep layout");
}  // namespace LinearAlgebra

namespace detail {
inline void check(vpfft_status s, const vpfft_grid* g) {
  if (s != VPFFT_OK)
    throw Error(s, std::string(vpfft_status_string(s)) + ": " + vpfft_last_error(g));
}
}  // namespace detail

namespace DataStructures {

using LinearAlgebra::EigenRep;
using LinearAlgebra::SMatrix3x3;

class MaterialGrid {
 public:
  MaterialGrid(int DimX, int DimY, int DimZ, const vpfft_material* material = nullptr,
               vpfft_precision precision = VPFFT_PREC_FP64,
               const vpfft_solver_options* options = nullptr)
      : DimX_(DimX), DimY_(DimY), DimZ_(DimZ) {
    detail::check(vpfft_grid_create(DimX, DimY, DimZ, material, options, precision, &g_), nullptr);
  }
  ~MaterialGrid() { vpfft_grid_destroy(g_); }
  MaterialGrid(const MaterialGrid&) = delete;
  MaterialGrid& operator=(const MaterialGrid&) = delete;

  // SendDataAndInitialize (MaterialGrid.cpp:425-534)
  void SendDataAndInitialize(const SMatrix3x3* Orientations, const EigenRep* Stress) {
    detail::check(vpfft_grid_set_fields(g_, &Orientations[0].m[0][0],
                                        Stress ? &Stress[0].m[0] : nullptr),
                  g_);
  }
  // SetVoxelLength (MaterialGrid.h:97-102)
  void SetVoxelLength(double x, double y, double z) {
    detail::check(vpfft_grid_set_voxel_length(g_, x, y, z), g_);
  }
  // RunSingleStrainStep (MaterialGrid.cpp:897-1084)
  EigenRep RunSingleStrainStep(const EigenRep& MacroscopicStrainRate, int NumMaxIterations,
                               double TimeStep, double ConvergenceEpsilon,
                               vpfft_stats* stats = nullptr) {
    EigenRep avg;
    detail::check(vpfft_run_single_strain_step(g_, MacroscopicStrainRate.m, NumMaxIterations,
                                               TimeStep, ConvergenceEpsilon, avg.m, stats),
                  g_);
    return avg;
  }
  // RunVPFFT (MaterialGrid.cpp:1202-1228): writes Stress_Strain.txt like the reference
  void RunVPFFT(const EigenRep& MacroscopicStrainRate, int NumMaxIterations, int NumTimeSteps,
                double TimeStep, double ConvergenceEpsilon,
                const char* path = "Stress_Strain.txt") {
    detail::check(vpfft_run(g_, MacroscopicStrainRate.m, NumMaxIterations, NumTimeSteps, TimeStep,
                            ConvergenceEpsilon, path, nullptr, nullptr),
                  g_);
  }
  int NumX() const { return DimX_; }
  int NumY() const { return DimY_; }
  int NumZ() const { return DimZ_; }
  int ToIndex(int x, int y, int z) const { return (x * DimY_ + y) * DimZ_ + z; }

  // bulk field read-back (the reference returns references into host arrays)
  std::vector<EigenRep> Stress() { return fetch<EigenRep>(VPFFT_FIELD_STRESS); }
  std::vector<EigenRep> LagrangeMultiplier() { return fetch<EigenRep>(VPFFT_FIELD_LAGRANGE); }
  std::vector<SMatrix3x3> Orientation() { return fetch<SMatrix3x3>(VPFFT_FIELD_ORIENTATION); }

  // Print* text dumps (MaterialGrid.cpp:15-100), byte-compatible
  void PrintStrain(const std::string& f) { print(VPFFT_PRINT_STRAIN, f); }
  void PrintStress(const std::string& f) { print(VPFFT_PRINT_STRESS, f); }
  void PrintLagrangeMultiplier(const std::string& f) { print(VPFFT_PRINT_LAGRANGE, f); }
  void PrintPolarization(const std::string& f) { print(VPFFT_PRINT_POLARIZATION, f); }

  // Checkpoint of the whole grid (vpfft_grid_snapshot / vpfft_grid_restore; the
  // reference has none): a grid of the same dimensions and precision restored
  // from it continues bit for bit.
  std::vector<unsigned char> Snapshot() {
    size_t n = 0;
    detail::check(vpfft_grid_snapshot_size(g_, &n), g_);
    std::vector<unsigned char> b(n);
    detail::check(vpfft_grid_snapshot(g_, b.data(), b.size()), g_);
    return b;
  }
  void Restore(const std::vector<unsigned char>& b) {
    detail::check(vpfft_grid_restore(g_, b.data(), b.size()), g_);
  }

  vpfft_grid* handle() { return g_; }

 private:
  template <typename T>
  std::vector<T> fetch(vpfft_field f) {
    std::vector<T> v((size_t)DimX_ * DimY_ * DimZ_);
    detail::check(vpfft_grid_get_field(g_, f, reinterpret_cast<double*>(v.data())), g_);
    return v;
  }
  void print(vpfft_print_kind k, const std::string& f) {
    detail::check(vpfft_grid_print(g_, k, f.c_str()), g_);
  }
  int DimX_, DimY_, DimZ_;
  vpfft_grid* g_ = nullptr;
};

}  // namespace DataStructures
}  // namespace VPFFT

#endif
