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

// ============================================================== helpers
template <typename R>
struct CT;
template <>
struct CT<float> {
  using T = float2;
};
template <>
struct CT<double> {
  using T = double2;
};

template <typename T>
__device__ __forceinline__ T cadd(T a, T b) {
  return T{a.x + b.x, a.y + b.y};
}
template <typename T>
__device__ __forceinline__ T csub(T a, T b) {
  return T{a.x - b.x, a.y - b.y};
}
template <typename T, typename R>
__device__ __forceinline__ T cscale(T a, R s) {
  return T{a.x * s, a.y * s};
}
// v * w (SIGN < 0) or v * conj(w) (SIGN > 0); w = exp(-2 pi i e / n)
template <int SIGN, typename T>
__device__ __forceinline__ T twmul(T v, T w) {
  if (SIGN < 0) return T{v.x * w.x - v.y * w.y, v.x * w.y + v.y * w.x};
  return T{v.x * w.x + v.y * w.y, v.y * w.x - v.x * w.y};
}
// (SIGN * i) * z
template <int SIGN, typename T>
__device__ __forceinline__ T mul_si(T z) {
  if (SIGN < 0) return T{z.y, -z.x};
  return T{-z.y, z.x};
}

// Stockham autosort FFT of `nlines` lines of length pl.n held in shared
// memory (line stride `stride`), ping-ponging between a and b; returns the
// buffer holding the result in natural order.  Stage with radix R after
// radices of product Ns: butterfly j takes in[j + r n/R] * W^(r (j mod Ns) n/(Ns R))
// and writes out[(j - j mod Ns) R + j mod Ns + r Ns].
template <int SIGN, typename T>
__device__ T* stockham(T* a, T* b, const T* tw, const LinePlan& pl, int nlines, int stride) {
  using R = decltype(T{}.x);
  const int n = pl.n;
  int Ns = 1;
  for (int st = 0; st < pl.nrad; ++st) {
    const int Rr = pl.rad[st];
    const int nb = n / Rr;
    const int total = nb * nlines;
    const int tws = n / (Ns * Rr);
    for (int t = threadIdx.x; t < total; t += blockDim.x) {
      const int line = t / nb;
      const int j = t - line * nb;
      const T* in = a + line * stride;
      T* out = b + line * stride;
      const int jm = j % Ns;
      const int e = jm * tws;
      const int od = (j - jm) * Rr + jm;
      if (Rr == 4) {
        T v0 = in[j], v1 = in[j + nb], v2 = in[j + 2 * nb], v3 = in[j + 3 * nb];
        if (e) {
          v1 = twmul<SIGN>(v1, tw[e]);
          v2 = twmul<SIGN>(v2, tw[2 * e]);
          v3 = twmul<SIGN>(v3, tw[3 * e]);
        }
        const T u0 = cadd(v0, v2), u1 = csub(v0, v2), u2 = cadd(v1, v3);
        const T u3 = mul_si<SIGN>(csub(v1, v3));
        out[od] = cadd(u0, u2);
        out[od + Ns] = cadd(u1, u3);
        out[od + 2 * Ns] = csub(u0, u2);
        out[od + 3 * Ns] = csub(u1, u3);
      } else if (Rr == 2) {
        T v0 = in[j], v1 = in[j + nb];
        if (e) v1 = twmul<SIGN>(v1, tw[e]);
        out[od] = cadd(v0, v1);
        out[od + Ns] = csub(v0, v1);
      } else if (Rr == 3) {
        T v0 = in[j], v1 = in[j + nb], v2 = in[j + 2 * nb];
        if (e) {
          v1 = twmul<SIGN>(v1, tw[e]);
          v2 = twmul<SIGN>(v2, tw[2 * e]);
        }
        const T t1 = cadd(v1, v2);
        const T t2 = csub(v0, cscale(t1, R(0.5)));
        const T t3 = mul_si<SIGN>(cscale(csub(v1, v2), R(0.86602540378443864676)));
        out[od] = cadd(v0, t1);
        out[od + Ns] = cadd(t2, t3);
        out[od + 2 * Ns] = csub(t2, t3);
      } else {  // radix 5
        T v0 = in[j], v1 = in[j + nb], v2 = in[j + 2 * nb], v3 = in[j + 3 * nb],
          v4 = in[j + 4 * nb];
        if (e) {
          v1 = twmul<SIGN>(v1, tw[e]);
          v2 = twmul<SIGN>(v2, tw[2 * e]);
          v3 = twmul<SIGN>(v3, tw[3 * e]);
          v4 = twmul<SIGN>(v4, tw[4 * e]);
        }
        const R c1 = R(0.30901699437494742410), c2 = R(-0.80901699437494742410);
        const R s1 = R(0.95105651629515357212), s2 = R(0.58778525229247312917);
        const T a1 = cadd(v1, v4), a2 = cadd(v2, v3), b1 = csub(v1, v4), b2 = csub(v2, v3);
        const T p1 = cadd(v0, cadd(cscale(a1, c1), cscale(a2, c2)));
        const T p2 = cadd(v0, cadd(cscale(a1, c2), cscale(a2, c1)));
        const T q1 = mul_si<SIGN>(cadd(cscale(b1, s1), cscale(b2, s2)));
        const T q2 = mul_si<SIGN>(csub(cscale(b1, s2), cscale(b2, s1)));
        out[od] = cadd(v0, cadd(a1, a2));
        out[od + Ns] = cadd(p1, q1);
        out[od + 4 * Ns] = csub(p1, q1);
        out[od + 2 * Ns] = cadd(p2, q2);
        out[od + 3 * Ns] = csub(p2, q2);
      }
    }
    __syncthreads();
    T* tmp = a;
    a = b;
    b = tmp;
    Ns *= Rr;
  }
  return a;
}

bool make_line_plan(int n, LinePlan* p) {
  if (n < 1) return false;
  p->n = n;
  p->nrad = 0;
  int m = n;
  while (m % 4 == 0 && m > 4) {
    if (p->nrad >= 16) return false;
    p->rad[p->nrad++] = 4;
    m /= 4;
  }
  const int rs[4] = {4, 2, 3, 5};
  for (int r : rs)
    while (m % r == 0) {
      if (p->nrad >= 16) return false;
      p->rad[p->nrad++] = r;
      m /= r;
    }
  return m == 1;
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


// Column sums of partials[nparts][width] with compensated, fixed-order
// summation; one block.
__device__ void column_sums(const double* partials, int nparts, int width, double* out) {
  __shared__ double ss[kFinishThreads], sc[kFinishThreads];
  for (int col = 0; col < width; ++col) {
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
__global__ void __launch_bounds__(kVoxelBlock) k_ref_medium(VoxelParams p, FieldPtrs<S> f,
                                                            double* partials) {
  const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
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
  block_reduce_store<25, kVoxelBlock>(acc, partials + (long long)blockIdx.x * 25);
}

// Reductions and convergence test of one iteration (MaterialGrid.cpp:1009-1068).
__global__ void __launch_bounds__(kFinishThreads) k_iter_finish(const double* partials,
                                                                int nparts, IterCtrl* ctrl,
                                                                double* hist) {
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

// OrientationEvolutionWithFFT (MaterialGrid.cpp:769-876) + UpdateSchmidtTensors
// + UpdateHardeningCRSS (1127-1157), fused per voxel.  The FFT part of the
// orientation update is AntiSymmetrize() of the symmetric matrix
// ToMatrixRep(d~) and therefore exactly zero (870), so
//   R += dt * W_p,   W_p from the old R, old Schmid tensors and the final stress;
// the hardening then uses the rotated Schmid tensors with the same stress
// (Solvers.cpp:314-373).
template <typename S>
__global__ void __launch_bounds__(kVoxelBlock) k_post(PostParams p, FieldPtrs<S> f, S* crss_out) {
  const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
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
  k_column_sums<<<1, kFinishThreads, 0, st>>>(partials, nb, 25, out25);
  return 2;
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

// ============================================================== spectral phase
// Shared-memory budget per block for the line FFTs (dynamic, opted in).
constexpr size_t kSmemBudget = 96 * 1024;

// z: real lines of length nz, two packed per complex line.
template <typename S>
__global__ void __launch_bounds__(256) k_fft_z_r2c(const S* __restrict__ work,
                                                   typename CT<S>::T* __restrict__ X, LinePlan pl,
                                                   const typename CT<S>::T* __restrict__ twg,
                                                   long long nlines, int nh, int ppb,
                                                   const IterCtrl* ctrl) {
  using T = typename CT<S>::T;
  if (ctrl && ctrl->done) return;
  extern __shared__ __align__(16) unsigned char smraw[];
  const int n = pl.n;
  T* tw = reinterpret_cast<T*>(smraw);
  T* a = tw + n;
  T* b = a + ppb * n;
  for (int i = threadIdx.x; i < n; i += blockDim.x) tw[i] = twg[i];
  const long long l0 = (long long)blockIdx.x * 2 * ppb;
  for (int i = threadIdx.x; i < 2 * ppb * n; i += blockDim.x) {
    const int l = i / n, z = i - l * n;
    const long long g = l0 + l;
    const S v = g < nlines ? work[g * n + z] : S(0);
    S* dst = reinterpret_cast<S*>(&a[(l >> 1) * n + z]);
    dst[l & 1] = v;
  }
  __syncthreads();
  T* r = stockham<-1>(a, b, tw, pl, ppb, n);
  for (int i = threadIdx.x; i < 2 * ppb * nh; i += blockDim.x) {
    const int l = i / nh, k = i - l * nh;
    const long long g = l0 + l;
    if (g >= nlines) continue;
    const int pr = l >> 1;
    const T Z = r[pr * n + k];
    const T Zm = r[pr * n + (k == 0 ? 0 : n - k)];
    T o;
    if ((l & 1) == 0) {  // (Z + conj(Zm)) / 2
      o.x = (Z.x + Zm.x) * S(0.5);
      o.y = (Z.y - Zm.y) * S(0.5);
    } else {             // (Z - conj(Zm)) / (2i)
      o.x = (Z.y + Zm.y) * S(0.5);
      o.y = (Zm.x - Z.x) * S(0.5);
    }
    X[g * nh + k] = o;
  }
}

template <typename S>
__global__ void __launch_bounds__(256) k_fft_z_c2r(const typename CT<S>::T* __restrict__ X,
                                                   S* __restrict__ work, LinePlan pl,
                                                   const typename CT<S>::T* __restrict__ twg,
                                                   long long nlines, int nh, int ppb, S scale,
                                                   const IterCtrl* ctrl) {
  using T = typename CT<S>::T;
  if (ctrl && ctrl->done) return;
  extern __shared__ __align__(16) unsigned char smraw[];
  const int n = pl.n;
  T* tw = reinterpret_cast<T*>(smraw);
  T* a = tw + n;
  T* b = a + ppb * n;
  for (int i = threadIdx.x; i < n; i += blockDim.x) tw[i] = twg[i];
  const long long l0 = (long long)blockIdx.x * 2 * ppb;
  for (int i = threadIdx.x; i < ppb * n; i += blockDim.x) {
    const int pr = i / n, k = i - pr * n;
    const long long ga = l0 + 2 * pr, gb = ga + 1;
    const bool cj = k >= nh;
    const int kk = cj ? n - k : k;
    T A = ga < nlines ? X[ga * nh + kk] : T{S(0), S(0)};
    T B = gb < nlines ? X[gb * nh + kk] : T{S(0), S(0)};
    if (cj) {
      A.y = -A.y;
      B.y = -B.y;
    }
    if (k == 0 || ((n & 1) == 0 && k == n / 2)) {
      A.y = S(0);
      B.y = S(0);
    }
    a[pr * n + k] = T{A.x - B.y, A.y + B.x};
  }
  __syncthreads();
  T* r = stockham<1>(a, b, tw, pl, ppb, n);
  for (int i = threadIdx.x; i < 2 * ppb * n; i += blockDim.x) {
    const int l = i / n, z = i - l * n;
    const long long g = l0 + l;
    if (g >= nlines) continue;
    const T Z = r[(l >> 1) * n + z];
    work[g * n + z] = ((l & 1) ? Z.y : Z.x) * scale;
  }
}

// y: complex lines at fixed (c, x) and a tile of tk consecutive kz.
template <int SIGN, typename R>
__global__ void __launch_bounds__(256) k_fft_y(typename CT<R>::T* __restrict__ X, LinePlan pl,
                                               const typename CT<R>::T* __restrict__ twg, int nh,
                                               int tk, const IterCtrl* ctrl) {
  using T = typename CT<R>::T;
  if (ctrl && ctrl->done) return;
  extern __shared__ __align__(16) unsigned char smraw[];
  const int ny = pl.n;
  T* tw = reinterpret_cast<T*>(smraw);
  T* a = tw + ny;
  T* b = a + tk * ny;
  for (int i = threadIdx.x; i < ny; i += blockDim.x) tw[i] = twg[i];
  const int k0 = blockIdx.x * tk;
  const int kc = min(tk, nh - k0);
  T* base = X + (long long)blockIdx.y * ny * nh + k0;
  for (int y = threadIdx.x; y < ny; y += blockDim.x) {
    const T* src = base + (long long)y * nh;
    for (int kk = 0; kk < tk; ++kk) a[kk * ny + y] = kk < kc ? src[kk] : T{R(0), R(0)};
  }
  __syncthreads();
  T* r = stockham<SIGN>(a, b, tw, pl, tk, ny);
  for (int y = threadIdx.x; y < ny; y += blockDim.x) {
    T* dst = base + (long long)y * nh;
    for (int kk = 0; kk < kc; ++kk) dst[kk] = r[kk * ny + y];
  }
}

// x: all 5 components of the lines at fixed (y, kz tile); MODE 0 forward,
// 1 inverse, 2 forward + Green operator + inverse.
template <int MODE, typename R>
__global__ void __launch_bounds__(256) k_fft_x(typename CT<R>::T* __restrict__ X, LinePlan pl,
                                               const typename CT<R>::T* __restrict__ twg,
                                               GreenParams<R> gp, int ny, int nh, int tk,
                                               int ncomp, const IterCtrl* ctrl) {
  using T = typename CT<R>::T;
  if (ctrl && ctrl->done) return;
  extern __shared__ __align__(16) unsigned char smraw[];
  const int nx = pl.n;
  T* tw = reinterpret_cast<T*>(smraw);
  T* a = tw + nx;
  T* b = a + ncomp * tk * nx;
  for (int i = threadIdx.x; i < nx; i += blockDim.x) tw[i] = twg[i];
  const int y = blockIdx.y;
  const int k0 = blockIdx.x * tk;
  const int kc = min(tk, nh - k0);
  const long long cstride = (long long)nx * ny * nh;  // component stride
  const long long xstride = (long long)ny * nh;
  T* base = X + (long long)y * nh + k0;
  for (int i = threadIdx.x; i < ncomp * nx; i += blockDim.x) {
    const int c = i / nx, x = i - c * nx;
    const T* src = base + c * cstride + x * xstride;
    for (int kk = 0; kk < tk; ++kk) a[(c * tk + kk) * nx + x] = kk < kc ? src[kk] : T{R(0), R(0)};
  }
  __syncthreads();
  T* r = a;
  T* o = b;
  if (MODE != 1) {
    r = stockham<-1>(a, b, tw, pl, ncomp * tk, nx);
    o = (r == a) ? b : a;
  }
  if (MODE == 2) {
    for (int i = threadIdx.x; i < nx * tk; i += blockDim.x) {
      const int x = i / tk, kk = i - x * tk;
      if (kk >= kc) continue;
      R pre[5], pim[5];
#pragma unroll
      for (int c = 0; c < 5; ++c) {
        const T z = r[(c * tk + kk) * nx + x];
        pre[c] = z.x;
        pim[c] = z.y;
      }
      green_apply<R>(gp, x, y, k0 + kk, pre, pim);
#pragma unroll
      for (int c = 0; c < 5; ++c) r[(c * tk + kk) * nx + x] = T{pre[c], pim[c]};
    }
    __syncthreads();
  }
  if (MODE != 0) r = stockham<1>(r, o, tw, pl, ncomp * tk, nx);
  for (int i = threadIdx.x; i < ncomp * nx; i += blockDim.x) {
    const int c = i / nx, x = i - c * nx;
    T* dst = base + c * cstride + x * xstride;
    for (int kk = 0; kk < kc; ++kk) dst[kk] = r[(c * tk + kk) * nx + x];
  }
}

template <typename R>
size_t spectral_smem_optin(int) {
  return kSmemBudget;
}

namespace {
template <typename R>
struct Tiles {
  int ppb_z, tk_y, tk_x;
  size_t sm_z, sm_y, sm_x;
};
template <typename R>
Tiles<R> pick_tiles(const Spectral<R>& sp, int ncomp) {
  using T = typename CT<R>::T;
  Tiles<R> t;
  const size_t e = sizeof(T);
  // z: tw + 2 * ppb * nz
  t.ppb_z = (int)((kSmemBudget / e - sp.nz) / (2 * (size_t)sp.nz));
  t.ppb_z = t.ppb_z < 1 ? 1 : (t.ppb_z > 16 ? 16 : t.ppb_z);
  t.sm_z = e * (sp.nz + 2 * (size_t)t.ppb_z * sp.nz);
  t.tk_y = (int)((kSmemBudget / e - sp.ny) / (2 * (size_t)sp.ny));
  t.tk_y = t.tk_y < 1 ? 1 : (t.tk_y > 16 ? 16 : t.tk_y);
  if (t.tk_y > sp.nh) t.tk_y = sp.nh;
  t.sm_y = e * (sp.ny + 2 * (size_t)t.tk_y * sp.ny);
  t.tk_x = (int)((kSmemBudget / e - sp.nx) / (2 * (size_t)ncomp * sp.nx));
  t.tk_x = t.tk_x < 1 ? 1 : (t.tk_x > 8 ? 8 : t.tk_x);
  if (t.tk_x > sp.nh) t.tk_x = sp.nh;
  t.sm_x = e * (sp.nx + 2 * (size_t)ncomp * t.tk_x * sp.nx);
  return t;
}
template <typename R>
void optin_all() {
  static bool done = false;
  if (done) return;
  // the tiles target kSmemBudget; the longest legal lines may need more, up to
  // the 227 KB a block can have on sm_100
  const int s = 227 * 1024;
  cudaFuncSetAttribute(k_fft_z_r2c<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, s);
  cudaFuncSetAttribute(k_fft_z_c2r<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, s);
  cudaFuncSetAttribute(k_fft_y<-1, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, s);
  cudaFuncSetAttribute(k_fft_y<1, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, s);
  cudaFuncSetAttribute(k_fft_x<0, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, s);
  cudaFuncSetAttribute(k_fft_x<1, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, s);
  cudaFuncSetAttribute(k_fft_x<2, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, s);
  done = true;
}
}  // namespace

template <typename S>
int launch_spectral_iteration(const Spectral<S>& sp, const GreenParams<S>& gp, S* work,
                              const IterCtrl* ctrl, cudaStream_t st, int ncomp,
                              cudaEvent_t* ev) {
  using T = typename CT<S>::T;
  optin_all<S>();
  const Tiles<S> t = pick_tiles(sp, ncomp);
  const long long nlines = (long long)ncomp * sp.nx * sp.ny;
  T* X = reinterpret_cast<T*>(sp.X);
  const T* twx = reinterpret_cast<const T*>(sp.twx);
  const T* twy = reinterpret_cast<const T*>(sp.twy);
  const T* twz = reinterpret_cast<const T*>(sp.twz);
  const int gz = (int)((nlines + 2 * t.ppb_z - 1) / (2 * t.ppb_z));
  if (ev) cudaEventRecord(ev[0], st);
  k_fft_z_r2c<S><<<gz, 256, t.sm_z, st>>>(work, X, sp.pz, twz, nlines, sp.nh, t.ppb_z, ctrl);
  if (ev) cudaEventRecord(ev[1], st);
  dim3 gy((sp.nh + t.tk_y - 1) / t.tk_y, ncomp * sp.nx);
  k_fft_y<-1, S><<<gy, 256, t.sm_y, st>>>(X, sp.py, twy, sp.nh, t.tk_y, ctrl);
  if (ev) cudaEventRecord(ev[2], st);
  dim3 gx((sp.nh + t.tk_x - 1) / t.tk_x, sp.ny);
  k_fft_x<2, S><<<gx, 256, t.sm_x, st>>>(X, sp.px, twx, gp, sp.ny, sp.nh, t.tk_x, ncomp, ctrl);
  if (ev) cudaEventRecord(ev[3], st);
  k_fft_y<1, S><<<gy, 256, t.sm_y, st>>>(X, sp.py, twy, sp.nh, t.tk_y, ctrl);
  if (ev) cudaEventRecord(ev[4], st);
  const S scale = S(1.0 / ((double)sp.nx * sp.ny * sp.nz));
  k_fft_z_c2r<S><<<gz, 256, t.sm_z, st>>>(X, work, sp.pz, twz, nlines, sp.nh, t.ppb_z, scale, ctrl);
  if (ev) cudaEventRecord(ev[5], st);
  return 5;
}

template <typename S>
int launch_fft3d(const Spectral<S>& sp, S* real, int ncomp, int mode, cudaStream_t st) {
  using T = typename CT<S>::T;
  optin_all<S>();
  const Tiles<S> t = pick_tiles(sp, ncomp);
  const long long nlines = (long long)ncomp * sp.nx * sp.ny;
  T* X = reinterpret_cast<T*>(sp.X);
  const T* twx = reinterpret_cast<const T*>(sp.twx);
  const T* twy = reinterpret_cast<const T*>(sp.twy);
  const T* twz = reinterpret_cast<const T*>(sp.twz);
  const int gz = (int)((nlines + 2 * t.ppb_z - 1) / (2 * t.ppb_z));
  dim3 gy((sp.nh + t.tk_y - 1) / t.tk_y, ncomp * sp.nx);
  dim3 gx((sp.nh + t.tk_x - 1) / t.tk_x, sp.ny);
  GreenParams<S> gp{};
  if (mode == 0) {
    k_fft_z_r2c<S><<<gz, 256, t.sm_z, st>>>(real, X, sp.pz, twz, nlines, sp.nh, t.ppb_z, nullptr);
    k_fft_y<-1, S><<<gy, 256, t.sm_y, st>>>(X, sp.py, twy, sp.nh, t.tk_y, nullptr);
    k_fft_x<0, S><<<gx, 256, t.sm_x, st>>>(X, sp.px, twx, gp, sp.ny, sp.nh, t.tk_x, ncomp, nullptr);
  } else {
    k_fft_x<1, S><<<gx, 256, t.sm_x, st>>>(X, sp.px, twx, gp, sp.ny, sp.nh, t.tk_x, ncomp, nullptr);
    k_fft_y<1, S><<<gy, 256, t.sm_y, st>>>(X, sp.py, twy, sp.nh, t.tk_y, nullptr);
    const S scale = S(1.0 / ((double)sp.nx * sp.ny * sp.nz));
    k_fft_z_c2r<S><<<gz, 256, t.sm_z, st>>>(X, real, sp.pz, twz, nlines, sp.nh, t.ppb_z, scale,
                                            nullptr);
  }
  return 3;
}

// ============================================================== Solvers batch (testing)
__device__ __forceinline__ void load_schmid(const double* schmid, int v, double m[kNS][5]) {
#pragma unroll
  for (int k = 0; k < kNS; ++k)
#pragma unroll
    for (int c = 0; c < 5; ++c) m[k][c] = schmid[(long long)v * 60 + k * 5 + c];
}
__device__ __forceinline__ void load_crss_v(const double* crss, int v, double tau[kNS]) {
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
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
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
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n) return;
  double m[kNS][5], tau[kNS], g[5];
  load_schmid(schmid, v, m);
  load_crss_v(crss, v, tau);
  sachs(m, tau, edot.v, g);
  for (int c = 0; c < 5; ++c) out[v * 5 + c] = g[c];
}
__global__ void k_solvers_schmid(int n, const double* R, double* out) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
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
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
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
  template int launch_strain_rate<S>(const VoxelParams&, const FieldPtrs<S>&, S*, cudaStream_t); \
  template int launch_schmid_field<S>(long long, const S*, double*, cudaStream_t);               \
  template int launch_to_soa<S>(const double*, S*, long long, int, cudaStream_t);                \
  template int launch_from_soa<S>(const S*, double*, long long, int, cudaStream_t);              \
  template int launch_fill<S>(S*, long long, double, cudaStream_t);                              \
  template int launch_crss_broadcast<S>(S*, long long, const double*, cudaStream_t);             \
  template int launch_spectral_iteration<S>(const Spectral<S>&, const GreenParams<S>&, S*,       \
                                            const IterCtrl*, cudaStream_t, int, cudaEvent_t*);   \
  template int launch_fft3d<S>(const Spectral<S>&, S*, int, int, cudaStream_t);                  \
  template size_t spectral_smem_optin<S>(int);                                                   \
  template int launch_green_batch<S>(int, const int32_t*, const GreenParams<S>&, const double*,  \
                                     double*, cudaStream_t);
VPFFT_INST(double)
VPFFT_INST(float)
#undef VPFFT_INST

}  // namespace vpfft
