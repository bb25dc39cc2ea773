// grid.h -- the state of one RVE on the device (struct vpfft_grid) and the
// host helpers shared by the single-grid entry points (capi.cu) and the batch
// engine (batch.cu).  Internal: not part of the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/vpfft_capi.h"
#include "kernels.h"

using vpfft::GreenParams;
using vpfft::IterCtrl;
using vpfft::LinePlan;

struct vpfft_grid {
  int device = 0;
  cudaStream_t stream = nullptr;
  int nx = 0, ny = 0, nz = 0, nh = 0;
  long long n = 0;
  vpfft_precision prec = VPFFT_PREC_FP64;
  vpfft_material mat{};
  vpfft_solver_options opt{};
  double h[3] = {1, 1, 1};
  bool fields_set = false;
  bool crss_per_voxel = false;
  bool keep_d = false;
  bool have_L0 = false;
  vpfft::LinePlan px{}, py{}, pz{};
  // device storage (element type = double for FP64, float for MIXED)
  void* R = nullptr;
  void* sigma = nullptr;
  void* lambda = nullptr;
  void* work = nullptr;
  void* dkeep = nullptr;
  void* crss = nullptr;
  double* acc = nullptr;
  void* X = nullptr;   // A: spectrum after the z pass (allocated on first use)
  void* X2 = nullptr;  // B: spectrum after the y pass
  void* twx = nullptr;
  void* twy = nullptr;
  void* twz = nullptr;
  double* partials = nullptr;
  double* sum25 = nullptr;
  double* staging = nullptr;  // voxel-major FP64 copy of one host field (N x 12 max)
  vpfft::IterCtrl* ctrl = nullptr;
  vpfft::IterCtrl* h_ctrl = nullptr;  // pinned
  double* hist = nullptr;
  int hist_cap = 0;
  double L0[25] = {0};
  double Linv[25] = {0};      // inverse(-L0): the Nyquist-plane operator
  double L0inv_sym[15] = {0}; // symmetric part of L0^-1, packed (Newton step)
  double last_edot[5] = {0};
  long long launches = 0;
  // per-kernel device timing of the fixed-point loop (vpfft_grid_set_profiling)
  bool profile = false;
  std::vector<cudaEvent_t> ev;
  double phase_ms[VPFFT_NUM_PHASES] = {0};
  int64_t phase_n[VPFFT_NUM_PHASES] = {0};
  bool in_batch = false;      // a batch request owns the grid until it completes
  // the fixed-point loop's chunk of iterations as a CUDA graph (re-captured for
  // each loop, replayed for its chunks after the first)
  cudaGraphExec_t loop_graph = nullptr;
  // the x pass's Green operator: 0 not chosen yet, 1 computed per wave
  // vector, 2 read from the stored table gtab (25 x nh ny nx values)
  int green_mode = 0;
  void* gtab = nullptr;
  double green_ms[2] = {0, 0};  // x pass computed / stored, when timed
  std::string err;
};


namespace vpfft {
namespace grid_ops {

inline MaterialParams mat_params(const vpfft_material& m) {
  MaterialParams p;
  for (int k = 0; k < kNS; ++k) {
    p.gdot[k] = m.gamma_dot_base[k];
    p.nexp[k] = m.rate_sensitivity[k];
  }
  return p;
}

template <typename S>
FieldPtrs<S> fields(const vpfft_grid* g) {
  FieldPtrs<S> f;
  f.R = (S*)g->R;
  f.sigma = (S*)g->sigma;
  f.lambda = (S*)g->lambda;
  f.work = (S*)g->work;
  f.dkeep = g->keep_d ? (S*)g->dkeep : nullptr;
  f.crss = g->crss_per_voxel ? (S*)g->crss : nullptr;
  f.acc = g->acc;
  return f;
}

template <typename S>
GreenParams<S> green_params(int nx, int ny, int nz, const double h[3], const double* L0,
                            const double* Linv) {
  GreenParams<S> gp{};
  gp.nx = nx;
  gp.ny = ny;
  gp.nz = nz;
  gp.inv_len[0] = (S)(1.0 / (nx * h[0]));
  gp.inv_len[1] = (S)(1.0 / (ny * h[1]));
  gp.inv_len[2] = (S)(1.0 / (nz * h[2]));
  for (int k = 0; k < 25; ++k) {
    gp.L0[k] = (S)L0[k];
    gp.Linv[k] = (S)Linv[k];
  }
  return gp;
}

// Spectral descriptor of the grid with the given spectrum buffers.
template <typename S>
Spectral<S> spectral(const vpfft_grid* g, void* X, void* X2) {
  Spectral<S> sp;
  sp.nx = g->nx;
  sp.ny = g->ny;
  sp.nz = g->nz;
  sp.nh = g->nh;
  sp.px = g->px;
  sp.py = g->py;
  sp.pz = g->pz;
  sp.twx = g->twx;
  sp.twy = g->twy;
  sp.twz = g->twz;
  sp.X = X;
  sp.X2 = X2;
  return sp;
}

// Bytes of one spectrum buffer (5 components, half spectrum, complex).
inline size_t spectrum_bytes(const vpfft_grid* g) {
  const size_t es = g->prec == VPFFT_PREC_FP64 ? sizeof(double) : sizeof(float);
  return 2 * es * 5 * (size_t)g->nx * g->ny * g->nh;
}

// Defined in capi.cu.
vpfft_status grid_fail(vpfft_grid* g, vpfft_status s, const std::string& msg);
VoxelParams voxel_params(const vpfft_grid* g, const double edot[5]);
NRParams nr_params(const vpfft_grid* g, const double edot[5], bool init);
PostParams post_params(const vpfft_grid* g, double dt);
// L0 from the column sums of the per-voxel inverses, then inverse(-L0) and the
// symmetric L0^-1 of the Newton step; fails on a non-finite medium.
vpfft_status finish_ref_medium(vpfft_grid* g, const double sums[25]);
// Host bookkeeping after the post-increment kernel: CRSS per voxel from now
// on, voxel lengths scaled by the strain increment.
void finish_post(vpfft_grid* g, const double edot[5], double dt);
// Control block of a fixed-point loop.
IterCtrl loop_ctrl(const vpfft_grid* g, const double edot[5], int max_iter, double eps);
vpfft_status ensure_crss_array(vpfft_grid* g);
vpfft_status ensure_hist(vpfft_grid* g, int max_iter);

}  // namespace grid_ops
}  // namespace vpfft
