// kernels.h -- host-side launch interface of the sm_100a kernels (kernels.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "device_math.cuh"
#include "nr_kernel.cuh"

namespace vpfft {

// Per-launch constants of the per-voxel phases (kernel parameter, constant bank).
struct VoxelParams {
  long long n;           // voxels
  double edot[5];        // imposed macroscopic strain rate
  double L0[25];         // reference medium, column-major
  MaterialParams mat;
  double crss[kNS];      // CRSS used when the per-voxel array is absent
  double nr_eps;         // 5e-4   (MaterialGrid.cpp:909)
  double nr_max_rss;     // 1e9    (MaterialGrid.cpp:910)
  int32_t nr_max_iter;   // 100    (MaterialGrid.cpp:911)
  int32_t init_max_iter; // 1000   (MaterialGrid.cpp:160)
  double init_eps;       // 5e-4   (MaterialGrid.cpp:159)
  double imposed_max_rss;  // max(2, 2 (edot.edot/gdot0)^(1/n_min))  (MaterialGrid.cpp:162-166)
};

// Hardening / texture constants (UpdateHardeningCRSS, MaterialGrid.cpp:1127-1157).
struct PostParams {
  long long n;
  double dt;
  MaterialParams mat;
  double crss[kNS];
  double tau0[kNS], tau1[kNS], theta0[kNS], theta1[kNS];
  double H[kNS * kNS];
};

// Device-resident control block of the fixed-point loop.  Every kernel of an
// iteration returns immediately once `done` is set, so the host may enqueue
// iterations ahead of the convergence decision.
struct IterCtrl {
  int32_t iter;       // iterations executed (StepsTaken, MaterialGrid.cpp:919)
  int32_t done;
  int32_t max_iter;
  int32_t status;     // OR of kStatus* bits
  double eps;
  double edot_norm;   // sqrt(edot.edot)
  double inv_n;       // 1/N  (unused; kept for alignment)
  double n_voxels;    // N as double
  unsigned long long nr_capped;
  double last[12];    // <sigma>(5), <edot>(5), delta_sigma, delta_eps of the last iteration
  unsigned long long nr_fp64;  // mixed precision: voxel-iterations that took the FP64 step
};
// device-side bits of IterCtrl::status; the same values as VPFFT_STATUS_MAX_RSS_TINY,
// VPFFT_STATUS_NONFINITE and VPFFT_STATUS_DEVICE_TIMEOUT of the C ABI
// (static_assert in capi.cu)
enum : int32_t { kStatusMaxRssTiny = 1, kStatusNonFinite = 2, kStatusDeviceTimeout = 4 };

// Division of 32-bit unsigned t < 2^31 by a fixed d >= 1 without a divide:
// q = (umulhi(t, mul) + t) >> shift, with shift = ceil(log2 d) and
// mul = floor(2^32 (2^shift - d) / d) + 1 (the round-up multiply method).
struct FastDiv {
  uint32_t mul;
  uint32_t shift;
};
inline FastDiv make_fast_div(uint32_t d) {
  uint32_t l = 0;
  while ((1ull << l) < d) ++l;
  const uint64_t m = (((1ull << l) - d) << 32) / d + 1;
  return FastDiv{(uint32_t)m, l};
}
#ifdef __CUDACC__
__host__ __device__ __forceinline__ uint32_t fast_div(uint32_t t, const FastDiv& f) {
#ifdef __CUDA_ARCH__
  return (__umulhi(t, f.mul) + t) >> f.shift;
#else
  return (uint32_t)((((uint64_t)t * f.mul) >> 32) + t) >> f.shift;
#endif
}
#endif

struct LinePlan {
  int n;
  int nrad;
  int rad[16];
  FastDiv by_n;          // division by n
  FastDiv by_nb[16];     // by n / rad[st]  (butterflies per line in stage st)
  FastDiv by_ns[16];     // by the stage's span Ns = rad[0] * ... * rad[st-1]
};
bool make_line_plan(int n, LinePlan* p);

template <typename S>
struct FieldPtrs {
  S* R;        // 9 x N
  S* sigma;    // 5 x N
  S* lambda;   // 5 x N
  S* work;     // 5 x N: P before the forward FFT, d~ after the inverse FFT
  S* dkeep;    // 5 x N copy of d~ (optional, may be null)
  S* crss;     // 12 x N or null
  double* acc; // N
};

// --- voxel phases (kernels.cu); each returns the number of kernels launched
template <typename S>
int launch_init(const NRParams& p, const FieldPtrs<S>& f, IterCtrl* ctrl, cudaStream_t st);
template <typename S>
int launch_ref_medium(const VoxelParams& p, const FieldPtrs<S>& f, double* partials,
                      double* out25, cudaStream_t st);
// ev (optional): 2 events recorded after the NR kernel and after the finish kernel
template <typename S>
int launch_nr_update(const NRParams& p, const FieldPtrs<S>& f, double* partials,
                     IterCtrl* ctrl, double* hist, cudaStream_t st, cudaEvent_t* ev = nullptr);
// host LU inverse of a column-major 5x5 (capi.cu)
void inverse5_colmajor(const double* a, double* out);
template <typename S>
int launch_post(const PostParams& p, const FieldPtrs<S>& f, S* crss_out, cudaStream_t st);
template <typename S>
int launch_strain_rate(const VoxelParams& p, const FieldPtrs<S>& f, S* out5, cudaStream_t st);
template <typename S>
int launch_schmid_field(long long n, const S* R, double* out60_voxel_major, cudaStream_t st);
int nr_blocks(long long n);
int ref_medium_blocks(long long n);

// --- layout conversion: host arrays are voxel-major double, device fields are
// component-major S
template <typename S>
int launch_to_soa(const double* src_vmajor, S* dst, long long n, int width, cudaStream_t st);
template <typename S>
int launch_from_soa(const S* src, double* dst_vmajor, long long n, int width, cudaStream_t st);
template <typename S>
int launch_fill(S* dst, long long count, double value, cudaStream_t st);
template <typename S>
int launch_crss_broadcast(S* dst, long long n, const double crss[kNS], cudaStream_t st);

// --- spectral phase (kernels.cu) ------------------------------------------
template <typename R>
struct Spectral {
  int nx, ny, nz, nh;
  LinePlan px, py, pz;
  const void* twx;  // twiddle tables exp(-2 pi i e / n), complex R
  const void* twy;
  const void* twz;
  void* X;          // A[c][x][kz][y]: spectrum after the z pass (complex R)
  void* X2;         // B[c][kz][ky][x]: spectrum after the y pass
};
// forward: work (P) -> X ; inverse: X -> work (d~, scaled by 1/N)
// ev (optional): 6 events recorded before the first and after each of the 5 kernels
// gtab (optional): the stored Green operator (launch_green_table); the x pass
// then reads it instead of computing the operator per wave vector.
template <typename S>
int launch_spectral_iteration(const Spectral<S>& sp, const GreenParams<S>& gp, S* work,
                              const IterCtrl* ctrl, cudaStream_t st, int ncomp,
                              cudaEvent_t* ev = nullptr, const S* gtab = nullptr);
// The stored Green operator of every wave vector of the half spectrum: 25 x
// nh ny nx values, entry (a, b) of wave vector (f = kz ny + ky, x) at
// tab[(a 5 + b) nh ny nx + f nx + x].
template <typename S>
int launch_green_table(const GreenParams<S>& gp, S* tab, int nh, cudaStream_t st);
// The x pass alone (computed or stored Green operator) on a spectrum buffer
// of B's layout, for timing the two against each other.
template <typename S>
int launch_x_pass(const Spectral<S>& sp, const GreenParams<S>& gp, const S* gtab, void* buf,
                  int ncomp, cudaStream_t st);
// The y and z passes with TMA-moved tiles (fft_tma.cu) for FP32 spectra whose
// lines on the pass's axis have 64, 128 or 256 points; false (nothing
// launched) when they do not apply.  set_tma_passes(1/0) enables / disables it process-wide (-1
// queries) and returns the previous setting.
bool launch_y_fwd_tma(const Spectral<float>& sp, const IterCtrl* ctrl, cudaStream_t st,
                      int ncomp);
bool launch_y_inv_tma(const Spectral<float>& sp, const IterCtrl* ctrl, cudaStream_t st,
                      int ncomp);
bool launch_z_r2c_tma(const Spectral<float>& sp, const float* work, const IterCtrl* ctrl,
                      cudaStream_t st, int ncomp);
bool launch_z_c2r_tma(const Spectral<float>& sp, float* work, const IterCtrl* ctrl,
                      cudaStream_t st, int ncomp);
int set_tma_passes(int enable);
// forward-only / inverse-only transforms for testing (mode 0 = forward, 1 = inverse)
template <typename S>
int launch_fft3d(const Spectral<S>& sp, S* real, int ncomp, int mode, cudaStream_t st);

// --- batches of RVEs ---------------------------------------------------------
// The fields of an RVE that the batched FFT passes read (each block copies them
// to shared memory).
template <typename S>
struct FftSlot {
  int nx, ny, nz, nh;
  FastDiv dnx, dny;  // division by nx and ny
  const void* twx;
  const void* twy;
  const void* twz;
  void* X;
  void* X2;
  S* work;
};

// One RVE ("slot") of a batch: everything a batched kernel needs, resident in
// device memory so that one launch per phase serves RVEs of different sizes.
template <typename S>
struct SlotDesc {
  NRParams nr_init;      // InitializeComputation solve
  NRParams nr;           // fixed-point loop solve
  VoxelParams vox;       // reference medium
  PostParams post;       // texture and hardening update
  GreenParams<S> gp;
  Spectral<S> sp;
  FftSlot<S> fs;         // copy of the fields of sp (and f.work) the batched passes use
  FieldPtrs<S> f;
  S* crss_out;           // per-voxel CRSS written by the post kernel
  double* partials;      // block partial sums (reference medium, loop reductions)
  double* sum25;         // reference-medium column sums
  IterCtrl* ctrl;
  double* hist;
  int init_blocks;       // block counts of the persistent kernels: the same as the
  int nr_blocks;         // single-RVE launches', so sums are formed in the same order
};
// The blocks of one batched launch: m slot indices and their cumulative block
// counts (device arrays); block b belongs to slot[i] with prefix[i] <= b < prefix[i+1].
struct BatchLaunch {
  const int* slot;
  const int* prefix;
  int m;
  int blocks;
  int per;  // blocks of every slot when all slots have the same count, else 0
};
// Dispatch value of the compile-time rate exponent (10, 20, or 0 = generic).
int uniform_exponent(const NRParams& p);
// Blocks of the persistent NR launches for n voxels (init or loop kernel).
template <typename S>
int nr_launch_blocks(const NRParams& p, bool tau, bool init);
template <typename S>
int launch_init_batch(const SlotDesc<S>* d, const BatchLaunch& bl, int nexp, bool tau,
                      cudaStream_t st);
// NR sweep + per-slot finish (bl_slots: one block per slot).  material: the
// batch's material and solver constants (every slot's NRParams agrees on them;
// the slot's strain rate and reference medium come from its descriptor).
template <typename S>
int launch_nr_update_batch(const SlotDesc<S>* d, const BatchLaunch& bl,
                           const BatchLaunch& bl_slots, const NRParams& material, int nexp,
                           bool tau, cudaStream_t st);
// reference medium: per-voxel inverse + per-slot column sums into sum25
template <typename S>
int launch_ref_medium_batch(const SlotDesc<S>* d, const BatchLaunch& bl,
                            const BatchLaunch& bl_slots, cudaStream_t st);
template <typename S>
int launch_post_batch(const SlotDesc<S>* d, const BatchLaunch& bl, cudaStream_t st);
// Blocks, dynamic shared memory, line engine ("pass set", chosen by the axis
// length) and tile family of the five batched FFT passes of one RVE.  fam:
// the tile family (0, 1, 2: about 512, 1024, 2048 complex values per buffer),
// clamped per axis to the families its engine has; -1 = the longest tiles.
struct SpectralShape {
  int blocks_z, blocks_y, blocks_x;
  size_t smem_z_r2c, smem_z_c2r, smem_y, smem_x;
  const void* set_z;
  const void* set_y;
  const void* set_x;
  int fam_z, fam_y, fam_x;
  int families;  // distinct families over the three axes (the candidates worth timing)
};
template <typename S>
SpectralShape spectral_shape(const Spectral<S>& sp, int ncomp, int fam = -1);
// The RVEs of a batch whose three axes have the same line engines and tile
// families: one launch per pass over all of them (the largest shared memory
// among them).  Chains of different classes are independent and may run on
// different streams.
struct PassChain {
  const void* set_z;
  const void* set_y;
  const void* set_x;
  BatchLaunch z, y, x;
  size_t smem_z_r2c, smem_z_c2r, smem_y, smem_x;
  int fam_z, fam_y, fam_x;
};
template <typename S>
int launch_spectral_chain(const SlotDesc<S>* d, const PassChain& c, cudaStream_t st);

// --- batched solver entry points for testing (double, voxel-major) ---------
// Loads the code of the batched Solvers kernels on the current device now
// (under lazy module loading it would load, and allocate, at first launch).
cudaError_t load_solvers_kernels();
int launch_solvers_constrained(int n, const double* s0, const double* schmid, const double* crss,
                               const MaterialParams& mp, const double edot[5],
                               const double* lambda, const double* dtilde, const double L0[25],
                               double eps, double max_rss, int max_iter, double* out,
                               double* nr_err, cudaStream_t st);
int launch_solvers_unconstrained(int n, const double* s0, const double* schmid,
                                 const double* crss, const MaterialParams& mp,
                                 const double edot[5], double eps, double max_rss, int max_iter,
                                 double* out, cudaStream_t st);
int launch_solvers_apply(int n, const double* s, const double* schmid, const double* crss,
                         const MaterialParams& mp, double* out, cudaStream_t st);
int launch_solvers_sachs(int n, const double* schmid, const double* crss, const double edot[5],
                         double* out, cudaStream_t st);
int launch_solvers_schmid(int n, const double* R, double* out, cudaStream_t st);
template <typename R>
int launch_green_batch(int n, const int32_t* kidx, const GreenParams<R>& gp, const double* phat,
                       double* dhat, cudaStream_t st);

}  // namespace vpfft
