// kernels.cu -- sm_100a kernels of the VPFFT fixed-point solve.
//
// Device layout (HBM): every per-voxel field is stored component-major
// (structure of arrays), field[c * N + v] with the reference's voxel index
// v = x*Ny*Nz + y*Nz + z, so a warp reading one component of 32 consecutive
// voxels issues one coalesced 128/256-byte request.  The half spectrum is
// X[c][x][y][kz], kz in [0, Nz/2], complex.
//
// One fixed-point iteration (MaterialGrid.cpp:930-1068) is
//   k_fft_z_r2c  : P (real)            -> z-transformed half spectrum
//   k_fft_y<-1>  : forward along y
//   k_fft_x<2>   : forward along x, Green operator, inverse along x
//   k_fft_y<+1>  : inverse along y
//   k_fft_z_c2r  : -> d~ (real, scaled by 1/N)
//   k_nr_update  : per-voxel NR + constitutive law + P and lambda update + partial sums
//   k_iter_finish: deterministic compensated reduction, error norms, stop flag
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "kernel_common.cuh"
#include "kernels.h"

namespace vpfft {

// ============================================================== line plans
// Radix-4 stages first, then 2, 3 and 5; returns false for other prime
// factors.  When at least four radix-4 stages occur, the last two become one
// radix-16 stage (two radix-4 layers in registers per pass through shared
// memory): its span is then >= 16, so its Stockham stores are contiguous
// across threads (a radix-16 first stage would store with a 16-element stride
// and 16-way bank conflicts).
bool make_line_plan(int n, LinePlan* p) {
  if (n < 1) return false;
  p->n = n;
  p->nrad = 0;
  int m = n;
  const int rs[4] = {4, 2, 3, 5};
  for (int r : rs)
    while (m % r == 0) {
      if (p->nrad >= 16) return false;
      p->rad[p->nrad++] = r;
      m /= r;
    }
  if (m != 1) return false;
  int last4 = -1, count4 = 0;
  for (int st = 0; st < p->nrad; ++st)
    if (p->rad[st] == 4) {
      ++count4;
      last4 = st;
    }
  if (count4 >= 4 && p->rad[last4 - 1] == 4) {
    p->rad[last4 - 1] = 16;
    for (int st = last4; st + 1 < p->nrad; ++st) p->rad[st] = p->rad[st + 1];
    --p->nrad;
  }
  p->by_n = make_fast_div((uint32_t)n);
  int ns = 1;
  for (int st = 0; st < p->nrad; ++st) {
    p->by_nb[st] = make_fast_div((uint32_t)(n / p->rad[st]));
    p->by_ns[st] = make_fast_div((uint32_t)ns);
    ns *= p->rad[st];
  }
  return true;
}

// Neumaier (improved Kahan) accumulator; combined pairwise in a fixed tree.
struct Neu {
  double s, c;
};
__device__ __forceinline__ void neu_add(Neu& a, double x) {
  const double t = a.s + x;
  if (fabs(a.s) >= fabs(x))
    a.c += (a.s - t) + x;
  else
    a.c += (x - t) + a.s;
  a.s = t;
}
__device__ __forceinline__ Neu neu_merge(Neu a, Neu b) {
  Neu r = a;
  neu_add(r, b.s);
  r.c += b.c;
  return r;
}


// Sum of column col of partials[nparts][width] with compensated, fixed-order
// summation (thread-strided Neumaier sums, then a fixed pairwise tree); one
// block of kFinishThreads threads.
__device__ void column_sum(const double* partials, int nparts, int width, int col, double* out) {
  __shared__ double ss[kFinishThreads], sc[kFinishThreads];
  Neu a{0.0, 0.0};
  for (int i = threadIdx.x; i < nparts; i += kFinishThreads) neu_add(a, partials[(long long)i * width + col]);
  ss[threadIdx.x] = a.s;
  sc[threadIdx.x] = a.c;
  __syncthreads();
  for (int off = kFinishThreads / 2; off > 0; off >>= 1) {
    if (threadIdx.x < off) {
      Neu x{ss[threadIdx.x], sc[threadIdx.x]}, y{ss[threadIdx.x + off], sc[threadIdx.x + off]};
      Neu z = neu_merge(x, y);
      ss[threadIdx.x] = z.s;
      sc[threadIdx.x] = z.c;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) out[col] = ss[0] + sc[0];
  __syncthreads();
}

// All columns, one after the other, in one block.
__device__ void column_sums(const double* partials, int nparts, int width, double* out) {
  for (int col = 0; col < width; ++col) column_sum(partials, nparts, width, col, out);
}

// One block per column (the same per-column order as column_sums).
__global__ void __launch_bounds__(kFinishThreads)
    k_column_sums_cols(const double* partials, int nparts, int width, double* out) {
  column_sum(partials, nparts, width, blockIdx.x, out);
}

__global__ void k_column_sums(const double* partials, int nparts, int width, double* out) {
  column_sums(partials, nparts, width, out);
}

// ============================================================== voxel phases

int nr_blocks(long long n) { return (int)((n + kVoxelBlock - 1) / kVoxelBlock); }
int ref_medium_blocks(long long n) { return nr_blocks(n); }

// BuildLinearRefMediumStiffness (MaterialGrid.cpp:219-282), per voxel:
//   (sum_s m_s (x) m_s gdot0 |r_s|^(n-1) / tau_s)^-1, block partial sums of the
// 25 entries (column-major).  The mean, the NormalizeValues clamp and the
// inverse(-L0) of the Nyquist planes are formed on the host in FP64.
template <typename S>
__device__ __forceinline__ void ref_medium_body(const VoxelParams& p, const FieldPtrs<S>& f,
                                                double* partials, int blk) {
  const long long v = (long long)blk * blockDim.x + threadIdx.x;
  double acc[25];
#pragma unroll
  for (int k = 0; k < 25; ++k) acc[k] = 0.0;
  if (v < p.n) {
    const long long n = p.n;
    double R[9], m[kNS][5], tau[kNS], s[5];
    load_R(f.R, n, v, R);
    schmid_from_R(R, m);
    load_tau(f.crss, p.crss, n, v, tau);
    load5(f.sigma, n, v, s);
    double M[5][5];
#pragma unroll
    for (int i = 0; i < 5; ++i)
#pragma unroll
      for (int j = 0; j < 5; ++j) M[i][j] = 0.0;
#pragma unroll
    for (int k = 0; k < kNS; ++k) {
      const double r = dot5(m[k], s) / tau[k];
      const double g = (p.mat.nexp[k] - 1 > 0) ? p.mat.gdot[k] * ipow(fabs(r), p.mat.nexp[k] - 1)
                                                : p.mat.gdot[k];
      const double w = g / tau[k];
#pragma unroll
      for (int i = 0; i < 5; ++i) {
        const double mw = m[k][i] * w;
#pragma unroll
        for (int j = i; j < 5; ++j) M[i][j] += mw * m[k][j];
      }
    }
#pragma unroll
    for (int i = 0; i < 5; ++i)
#pragma unroll
      for (int j = 0; j < i; ++j) M[i][j] = M[j][i];
    double Mi[5][5];
    inverse5_pp(M, Mi);
#pragma unroll
    for (int i = 0; i < 5; ++i)
#pragma unroll
      for (int j = 0; j < 5; ++j) acc[j * 5 + i] = Mi[i][j];
  }
  block_reduce_store<25, kVoxelBlock>(acc, partials + (long long)blk * 25);
}

template <typename S>
__global__ void __launch_bounds__(kVoxelBlock) k_ref_medium(VoxelParams p, FieldPtrs<S> f,
                                                            double* partials) {
  ref_medium_body<S>(p, f, partials, blockIdx.x);
}

template <typename S>
__global__ void __launch_bounds__(kVoxelBlock)
    k_ref_medium_batch(const SlotDesc<S>* __restrict__ desc, const BatchLaunch bl) {
  __shared__ VoxelParams sp;
  __shared__ FieldPtrs<S> sf;
  int lb;
  const SlotDesc<S>& d = desc[batch_slot(bl, blockIdx.x, &lb)];
  copy_struct(&sp, &d.vox);
  copy_struct(&sf, &d.f);
  __syncthreads();
  ref_medium_body<S>(sp, sf, d.partials, lb);
}

// Per-slot column sums of the reference-medium partials (block (slot, column)).
template <typename S>
__global__ void __launch_bounds__(kFinishThreads)
    k_column_sums_batch(const SlotDesc<S>* __restrict__ desc, const BatchLaunch bl) {
  const SlotDesc<S>& d = desc[bl.slot[blockIdx.x]];
  column_sum(d.partials, (int)((d.vox.n + kVoxelBlock - 1) / kVoxelBlock), 25, blockIdx.y,
             d.sum25);
}

// Reductions and convergence test of one iteration (MaterialGrid.cpp:1009-1068).
__device__ __forceinline__ void iter_finish_body(const double* partials, int nparts,
                                                 IterCtrl* ctrl, double* hist) {
  if (ctrl->done) return;
  __shared__ double sums[12];
  column_sums(partials, nparts, 12, sums);
  if (threadIdx.x == 0) {
    const double N = ctrl->n_voxels;
    double avgS[5], avgE[5];
    double errS = sums[10] / N;
    double errE = sums[11] / N;
    for (int c = 0; c < 5; ++c) {
      avgS[c] = sums[c] / N;
      avgE[c] = sums[5 + c] / N;
    }
    errS /= sqrt(dot5(avgS, avgS));
    errE /= ctrl->edot_norm;
    const int it = ctrl->iter;
    double* h = ctrl->last;
    for (int c = 0; c < 5; ++c) {
      h[c] = avgS[c];
      h[5 + c] = avgE[c];
    }
    h[10] = errS;
    h[11] = errE;
    if (hist)
      for (int k = 0; k < 12; ++k) hist[(long long)it * 12 + k] = h[k];
    bool finite = true;
    for (int k = 0; k < 12; ++k) finite = finite && isfinite(sums[k]);
    ctrl->iter = it + 1;
    if (!finite) {
      ctrl->status |= kStatusNonFinite;
      ctrl->done = 1;
    } else {
      ctrl->done = !(it + 1 < ctrl->max_iter && (errS > ctrl->eps || errE > ctrl->eps));
    }
  }
}

__global__ void __launch_bounds__(kFinishThreads) k_iter_finish(const double* partials,
                                                                int nparts, IterCtrl* ctrl,
                                                                double* hist) {
  iter_finish_body(partials, nparts, ctrl, hist);
}

// One block per slot of the batch.
template <typename S>
__global__ void __launch_bounds__(kFinishThreads)
    k_iter_finish_batch(const SlotDesc<S>* desc, BatchLaunch bl) {
  const SlotDesc<S>& d = desc[bl.slot[blockIdx.x]];
  iter_finish_body(d.partials, d.nr_blocks, d.ctrl, d.hist);
}
template __global__ void k_iter_finish_batch<double>(const SlotDesc<double>*, BatchLaunch);
template __global__ void k_iter_finish_batch<float>(const SlotDesc<float>*, BatchLaunch);

// OrientationEvolutionWithFFT (MaterialGrid.cpp:769-876) + UpdateSchmidtTensors
// + UpdateHardeningCRSS (1127-1157), fused per voxel.  The FFT part of the
// orientation update is AntiSymmetrize() of the symmetric matrix
// ToMatrixRep(d~) and therefore exactly zero (870), so
//   R += dt * W_p,   W_p from the old R, old Schmid tensors and the final stress;
// the hardening then uses the rotated Schmid tensors with the same stress
// (Solvers.cpp:314-373).
template <typename S>
__device__ __forceinline__ void post_body(const PostParams& p, const FieldPtrs<S>& f, S* crss_out,
                                          int blk) {
  const long long v = (long long)blk * blockDim.x + threadIdx.x;
  if (v >= p.n) return;
  const long long n = p.n;
  double R[9], m[kNS][5], tau[kNS], s[5];
  load_R(f.R, n, v, R);
  schmid_from_R(R, m);
  load_tau(f.crss, p.crss, n, v, tau);
  load5(f.sigma, n, v, s);
  double gs[kNS];
#pragma unroll
  for (int k = 0; k < kNS; ++k) {
    const double r = dot5(m[k], s) / tau[k];
    const double g = p.mat.nexp[k] > 0 ? p.mat.gdot[k] * ipow(fabs(r), p.mat.nexp[k]) : p.mat.gdot[k];
    gs[k] = g * (double)sgn(r);
  }
  double w[3];
  plastic_spin(R, gs, w);
  const double W[9] = {0.0, w[0], w[1], -w[0], 0.0, w[2], -w[1], -w[2], 0.0};
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    R[k] += (0.0 + W[k]) * p.dt;
    f.R[k * n + v] = (S)R[k];
  }
  schmid_from_R(R, m);
  double gd[kNS], dg = 0.0;
#pragma unroll
  for (int k = 0; k < kNS; ++k) {
    const double r = dot5(m[k], s) / tau[k];
    gd[k] = p.mat.nexp[k] > 0 ? p.mat.gdot[k] * ipow(fabs(r), p.mat.nexp[k]) : p.mat.gdot[k];
    dg += fabs(gd[k]) * p.dt;
  }
  const double a0 = f.acc[v];
#pragma unroll
  for (int i = 0; i < kNS; ++i) {
    double dtau = 0.0;
#pragma unroll
    for (int j = 0; j < kNS; ++j) dtau += p.H[i * kNS + j] * fabs(gd[j]) * p.dt;
    const double tiny = 1e-4 * p.tau0[i];
    double voce = 0.0;
    if (fabs(p.theta0[i]) > tiny) {
      voce = p.theta1[i] * dg;
      if (fabs(p.tau1[i]) > tiny) {
        const double fr = fabs(p.theta0[i] / p.tau1[i]);
        const double e_ini = exp(-a0 * fr);
        const double e_del = exp(-dg * fr);
        voce = voce - (fr * p.tau1[i] * p.theta1[i]) / fr * e_ini * (e_del - 1.0) -
               p.theta1[i] / fr * e_ini * (e_del * ((a0 + dg) * fr + 1.0) - (a0 * fr + 1.0));
      }
    }
    crss_out[i * n + v] = (S)(tau[i] + dtau * voce / dg);
  }
  f.acc[v] = a0 + dg;
}

template <typename S>
__global__ void __launch_bounds__(kVoxelBlock) k_post(PostParams p, FieldPtrs<S> f, S* crss_out) {
  post_body<S>(p, f, crss_out, blockIdx.x);
}

template <typename S>
__global__ void __launch_bounds__(kVoxelBlock)
    k_post_batch(const SlotDesc<S>* __restrict__ desc, const BatchLaunch bl) {
  __shared__ PostParams sp;
  __shared__ FieldPtrs<S> sf;
  int lb;
  const SlotDesc<S>& d = desc[batch_slot(bl, blockIdx.x, &lb)];
  copy_struct(&sp, &d.post);
  copy_struct(&sf, &d.f);
  __syncthreads();
  post_body<S>(sp, sf, d.crss_out, lb);
}

// ApplyConstitutiveEquations on the stress field (for field read-back).
template <typename S>
__global__ void k_strain_rate(VoxelParams p, FieldPtrs<S> f, S* out) {
  const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= p.n) return;
  double R[9], m[kNS][5], tau[kNS], s[5], e[5];
  load_R(f.R, p.n, v, R);
  schmid_from_R(R, m);
  load_tau(f.crss, p.crss, p.n, v, tau);
  load5(f.sigma, p.n, v, s);
  apply_constitutive(m, tau, p.mat, s, e);
  store5(out, p.n, v, e);
}

template <typename S>
__global__ void k_schmid_field(long long n, const S* R, double* out) {
  const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  double r[9], m[kNS][5];
  load_R(R, n, v, r);
  schmid_from_R(r, m);
#pragma unroll
  for (int k = 0; k < kNS; ++k)
#pragma unroll
    for (int c = 0; c < 5; ++c) out[v * 60 + k * 5 + c] = m[k][c];
}

// ---------------------------------------------------------------- conversions
template <typename S>
__global__ void k_to_soa(const double* src, S* dst, long long n, int width) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n * width) return;
  const long long v = i / width;
  const int c = (int)(i - v * width);
  dst[c * n + v] = (S)src[i];
}
template <typename S>
__global__ void k_from_soa(const S* src, double* dst, long long n, int width) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n * width) return;
  const long long v = i / width;
  const int c = (int)(i - v * width);
  dst[i] = (double)src[c * n + v];
}
template <typename S>
__global__ void k_fill(S* dst, long long count, double value) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < count) dst[i] = (S)value;
}
struct Crss12 {
  double v[kNS];
};
template <typename S>
__global__ void k_crss_broadcast(S* dst, long long n, Crss12 c) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n * kNS) return;
  dst[i] = (S)c.v[i / n];
}

static inline int grid1d(long long count, int block) { return (int)((count + block - 1) / block); }

template <typename S>
int launch_ref_medium(const VoxelParams& p, const FieldPtrs<S>& f, double* partials,
                      double* out25, cudaStream_t st) {
  const int nb = ref_medium_blocks(p.n);
  k_ref_medium<S><<<nb, kVoxelBlock, 0, st>>>(p, f, partials);
  k_column_sums_cols<<<25, kFinishThreads, 0, st>>>(partials, nb, 25, out25);
  return 2;
}
template <typename S>
int launch_ref_medium_batch(const SlotDesc<S>* d, const BatchLaunch& bl, const BatchLaunch& bls,
                            cudaStream_t st) {
  if (bl.blocks <= 0) return 0;
  k_ref_medium_batch<S><<<bl.blocks, kVoxelBlock, 0, st>>>(d, bl);
  k_column_sums_batch<S><<<dim3(bls.m, 25), kFinishThreads, 0, st>>>(d, bls);
  return 2;
}
template <typename S>
int launch_post_batch(const SlotDesc<S>* d, const BatchLaunch& bl, cudaStream_t st) {
  if (bl.blocks <= 0) return 0;
  k_post_batch<S><<<bl.blocks, kVoxelBlock, 0, st>>>(d, bl);
  return 1;
}
template <typename S>
int launch_post(const PostParams& p, const FieldPtrs<S>& f, S* crss_out, cudaStream_t st) {
  k_post<S><<<nr_blocks(p.n), kVoxelBlock, 0, st>>>(p, f, crss_out);
  return 1;
}
template <typename S>
int launch_strain_rate(const VoxelParams& p, const FieldPtrs<S>& f, S* out, cudaStream_t st) {
  k_strain_rate<S><<<nr_blocks(p.n), kVoxelBlock, 0, st>>>(p, f, out);
  return 1;
}
template <typename S>
int launch_schmid_field(long long n, const S* R, double* out, cudaStream_t st) {
  k_schmid_field<S><<<nr_blocks(n), kVoxelBlock, 0, st>>>(n, R, out);
  return 1;
}
template <typename S>
int launch_to_soa(const double* src, S* dst, long long n, int width, cudaStream_t st) {
  k_to_soa<S><<<grid1d(n * width, 256), 256, 0, st>>>(src, dst, n, width);
  return 1;
}
template <typename S>
int launch_from_soa(const S* src, double* dst, long long n, int width, cudaStream_t st) {
  k_from_soa<S><<<grid1d(n * width, 256), 256, 0, st>>>(src, dst, n, width);
  return 1;
}
template <typename S>
int launch_fill(S* dst, long long count, double value, cudaStream_t st) {
  k_fill<S><<<grid1d(count, 256), 256, 0, st>>>(dst, count, value);
  return 1;
}
template <typename S>
int launch_crss_broadcast(S* dst, long long n, const double crss[kNS], cudaStream_t st) {
  Crss12 c;
  for (int k = 0; k < kNS; ++k) c.v[k] = crss[k];
  k_crss_broadcast<S><<<grid1d(n * kNS, 256), 256, 0, st>>>(dst, n, c);
  return 1;
}

// ============================================================== Solvers batch (testing)
__device__ __forceinline__ void load_schmid(const double* schmid, long long v, double m[kNS][5]) {
#pragma unroll
  for (int k = 0; k < kNS; ++k)
#pragma unroll
    for (int c = 0; c < 5; ++c) m[k][c] = schmid[(long long)v * 60 + k * 5 + c];
}
__device__ __forceinline__ void load_crss_v(const double* crss, long long v, double tau[kNS]) {
#pragma unroll
  for (int k = 0; k < kNS; ++k) tau[k] = crss[(long long)v * kNS + k];
}
struct Vec5 {
  double v[5];
};
struct Mat25 {
  double v[25];
};

__global__ void k_solvers_apply(int n, const double* s_in, const double* schmid,
                                const double* crss, MaterialParams mp, double* out) {
  const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  double m[kNS][5], tau[kNS], s[5], e[5];
  load_schmid(schmid, v, m);
  load_crss_v(crss, v, tau);
  for (int c = 0; c < 5; ++c) s[c] = s_in[v * 5 + c];
  apply_constitutive(m, tau, mp, s, e);
  for (int c = 0; c < 5; ++c) out[v * 5 + c] = e[c];
}
__global__ void k_solvers_sachs(int n, const double* schmid, const double* crss, Vec5 edot,
                                double* out) {
  const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  double m[kNS][5], tau[kNS], g[5];
  load_schmid(schmid, v, m);
  load_crss_v(crss, v, tau);
  sachs(m, tau, edot.v, g);
  for (int c = 0; c < 5; ++c) out[v * 5 + c] = g[c];
}
__global__ void k_solvers_schmid(int n, const double* R, double* out) {
  const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  double r[9], m[kNS][5];
  for (int k = 0; k < 9; ++k) r[k] = R[(long long)v * 9 + k];
  schmid_from_R(r, m);
  for (int k = 0; k < kNS; ++k)
    for (int c = 0; c < 5; ++c) out[(long long)v * 60 + k * 5 + c] = m[k][c];
}
template <typename R>
__global__ void k_green_batch(int n, const int32_t* kidx, GreenParams<R> gp, const double* phat,
                              double* dhat) {
  const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  R pre[5], pim[5];
  for (int c = 0; c < 5; ++c) {
    pre[c] = (R)phat[(v * 5 + c) * 2];
    pim[c] = (R)phat[(v * 5 + c) * 2 + 1];
  }
  green_apply<R>(gp, kidx[v * 3], kidx[v * 3 + 1], kidx[v * 3 + 2], pre, pim);
  for (int c = 0; c < 5; ++c) {
    dhat[(v * 5 + c) * 2] = (double)pre[c];
    dhat[(v * 5 + c) * 2 + 1] = (double)pim[c];
  }
}

int launch_solvers_apply(int n, const double* s, const double* schmid, const double* crss,
                         const MaterialParams& mp, double* out, cudaStream_t st) {
  k_solvers_apply<<<grid1d(n, 128), 128, 0, st>>>(n, s, schmid, crss, mp, out);
  return 1;
}
int launch_solvers_sachs(int n, const double* schmid, const double* crss, const double edot[5],
                         double* out, cudaStream_t st) {
  Vec5 e;
  for (int c = 0; c < 5; ++c) e.v[c] = edot[c];
  k_solvers_sachs<<<grid1d(n, 128), 128, 0, st>>>(n, schmid, crss, e, out);
  return 1;
}
int launch_solvers_schmid(int n, const double* R, double* out, cudaStream_t st) {
  k_solvers_schmid<<<grid1d(n, 128), 128, 0, st>>>(n, R, out);
  return 1;
}
template <typename R>
int launch_green_batch(int n, const int32_t* kidx, const GreenParams<R>& gp, const double* phat,
                       double* dhat, cudaStream_t st) {
  k_green_batch<R><<<grid1d(n, 128), 128, 0, st>>>(n, kidx, gp, phat, dhat);
  return 1;
}

// ============================================================== instantiations
#define VPFFT_INST(S)                                                                            \
  template int launch_ref_medium<S>(const VoxelParams&, const FieldPtrs<S>&, double*, double*,   \
                                    cudaStream_t);                                               \
  template int launch_post<S>(const PostParams&, const FieldPtrs<S>&, S*, cudaStream_t);         \
  template int launch_ref_medium_batch<S>(const SlotDesc<S>*, const BatchLaunch&,                 \
                                          const BatchLaunch&, cudaStream_t);                      \
  template int launch_post_batch<S>(const SlotDesc<S>*, const BatchLaunch&, cudaStream_t);        \
  template int launch_strain_rate<S>(const VoxelParams&, const FieldPtrs<S>&, S*, cudaStream_t); \
  template int launch_schmid_field<S>(long long, const S*, double*, cudaStream_t);               \
  template int launch_to_soa<S>(const double*, S*, long long, int, cudaStream_t);                \
  template int launch_from_soa<S>(const S*, double*, long long, int, cudaStream_t);              \
  template int launch_fill<S>(S*, long long, double, cudaStream_t);                              \
  template int launch_crss_broadcast<S>(S*, long long, const double*, cudaStream_t);             \
  template int launch_green_batch<S>(int, const int32_t*, const GreenParams<S>&, const double*,  \
                                     double*, cudaStream_t);
VPFFT_INST(double)
VPFFT_INST(float)
#undef VPFFT_INST

}  // namespace vpfft
