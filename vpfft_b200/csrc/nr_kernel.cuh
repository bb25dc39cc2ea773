// nr_kernel.cuh -- the per-voxel Newton-Raphson solves of the fixed-point loop
// and of the initialisation, arranged for sm_100a.
//
// Layout per thread: the 12 rotated Schmid 5-vectors of the voxel being solved
// live in shared memory (msm[(s*5 + c) * blockDim + tid], so a warp's loads are
// conflict-free) instead of 120 registers; the Newton state, the accumulated
// Jacobian and the 5x5 solve stay in registers.  One pass over the 12 systems
// per Newton step computes the resolved shear r_s, the admissibility test, the
// strain-rate sum S and the Jacobian sum K together.
//
// The constrained Newton step of the reference (Solvers.cpp:184-211)
//     J d = R,  J = -I - L0 K,  R = (s - lambda) + L0 (S - Edot - d~)
// is solved in its equivalent symmetric positive-definite form
//     (L0^-1 + K) d = -y,  y = L0^-1 (s - lambda) + (S - Edot - d~)
// (multiply by -L0^-1; L0 is an average of SPD matrices and K is PSD) with an
// LDL^T factorisation, which needs no pivoting; the reference's full-pivot LU
// and this give the same step up to rounding.  The unconstrained Newton of the
// initialisation (Solvers.cpp:19-101) solves K d = -R the same way and falls
// back to complete pivoting when K is singular (systems with r_s snapped to 0).
#pragma once

#include <cfloat>
#include "device_math.cuh"

namespace vpfft {

// x^E for a compile-time E >= 0 by repeated squaring
template <int E, typename T>
__device__ __forceinline__ T cpow(T x) {
  if constexpr (E == 0) {
    return T(1);
  } else if constexpr (E == 1) {
    return x;
  } else {
    const T h = cpow<E / 2>(x);
    if constexpr (E & 1)
      return h * h * x;
    else
      return h * h;
  }
}
template <typename T>
__device__ __forceinline__ T ipow_t(T x, int e) {
  T r = T(1), b = x;
  while (e > 0) {
    if (e & 1) r *= b;
    b *= b;
    e >>= 1;
  }
  return r;
}
// |r|^(n-1) with n known at compile time (NEXP > 0) or at run time (NEXP == 0)
template <int NEXP, typename T>
__device__ __forceinline__ T pow_nm1(T a, int n) {
  if constexpr (NEXP > 0) {
    return cpow<NEXP - 1>(a);
  } else {
    return n - 1 >= 0 ? ipow_t(a, n - 1) : T(1) / ipow_t(a, 1 - n);
  }
}
template <int NEXP, typename T>
__device__ __forceinline__ T pow_n(T a, int n) {
  if constexpr (NEXP > 0) {
    return cpow<NEXP>(a);
  } else {
    return ipow_t(a, n);
  }
}

// Per-launch constants of the NR kernels.
struct NRParams {
  long long n;
  double edot[5];
  double L0[25];      // column-major
  double L0inv[15];   // symmetric part of L0^-1, packed upper triangle row by row
  double gdot[kNS];
  int32_t nexp[kNS];
  double crss[kNS];   // uniform CRSS (used when the per-voxel array is absent)
  double icrss[kNS];  // 1 / crss
  double eps;         // NR relative-step tolerance
  double max_rss;     // admissibility cap of |r_s|
  int32_t max_iter;
  int32_t pad_;
  // FP32 copies for the Newton predictor of the mixed path (set_fp32_copies)
  float gdot_f[kNS];
  float icrss_f[kNS];
  float n_f[kNS];
  float eps_f;
  float max_rss_f;
  float L0inv_f[15];
  // mixed precision: the FP64 Newton step is skipped where the step estimated
  // from the FP64 residual at the predicted stress, squared, is at most
  // cert2_f |sigma|^2 (0: the step is always taken)
  float cert2_f;
};

// Fills the FP32 copies of the per-system constants from the FP64 values.
__host__ __device__ inline void set_fp32_copies(NRParams& p) {
  for (int q = 0; q < kNS; ++q) {
    p.gdot_f[q] = (float)p.gdot[q];
    p.icrss_f[q] = (float)p.icrss[q];
    p.n_f[q] = (float)p.nexp[q];
  }
  p.eps_f = (float)p.eps;
  p.max_rss_f = (float)p.max_rss;
  for (int k = 0; k < 15; ++k) p.L0inv_f[k] = (float)p.L0inv[k];
}

// The constants of a voxel solve that differ between the RVEs of a batch
// (imposed strain rate, L0, L0^-1).  A single-grid kernel reads them from its
// parameter struct (constant bank operands); a batched kernel reads its slot's
// copy in shared memory through a volatile pointer, so every use is a fresh
// load instead of a value the compiler keeps in registers across the solve.
struct ParamConsts {
  const NRParams& p;
  __device__ __forceinline__ double edot(int k) const { return p.edot[k]; }
  __device__ __forceinline__ double L0(int k) const { return p.L0[k]; }
  __device__ __forceinline__ double L0inv(int k) const { return p.L0inv[k]; }
  __device__ __forceinline__ float L0inv_f(int k) const { return p.L0inv_f[k]; }
};
struct SharedConsts {
  const volatile NRParams* p;
  __device__ __forceinline__ double edot(int k) const { return p->edot[k]; }
  __device__ __forceinline__ double L0(int k) const { return p->L0[k]; }
  __device__ __forceinline__ double L0inv(int k) const { return p->L0inv[k]; }
  __device__ __forceinline__ float L0inv_f(int k) const { return p->L0inv_f[k]; }
};

// The per-system constants in the arithmetic type of a Newton pass.
template <typename T>
struct NRConst;
template <>
struct NRConst<double> {
  __device__ static double gdot(const NRParams& p, int q) { return p.gdot[q]; }
  __device__ static double icrss(const NRParams& p, int q) { return p.icrss[q]; }
  __device__ static double n(const NRParams& p, int q) { return (double)p.nexp[q]; }
  __device__ static double max_rss(const NRParams& p) { return p.max_rss; }
};
template <>
struct NRConst<float> {
  __device__ static float gdot(const NRParams& p, int q) { return p.gdot_f[q]; }
  __device__ static float icrss(const NRParams& p, int q) { return p.icrss_f[q]; }
  __device__ static float n(const NRParams& p, int q) { return p.n_f[q]; }
  __device__ static float max_rss(const NRParams& p) { return p.max_rss_f; }
};

// packed index of (i, j), i <= j, in a symmetric 5x5
__host__ __device__ constexpr int sym5(int i, int j) {
  return i <= j ? (i * (9 - i)) / 2 + j : (j * (9 - j)) / 2 + i;
}

// Shared-memory layout of a thread's Schmid 5-vectors m(q, c) and reciprocal
// CRSS t(q), relative to the thread's base pointer (base + kThreadStride * tid):
// FP64 staging, one value per thread per row ([(q*5+c)*bs], [q*bs]); FP32
// staging, systems q and q+1 interleaved so that one 8-byte load returns
// (m(q, c), m(q+1, c)) for the paired FP32 arithmetic of the Newton predictor.
template <typename MS>
struct SL;
template <>
struct SL<double> {
  static constexpr int kThreadStride = 1;
  __device__ static int m(int q, int c, int bs) { return (q * 5 + c) * bs; }
  __device__ static int t(int q, int bs) { return q * bs; }
};
template <>
struct SL<float> {
  static constexpr int kThreadStride = 2;
  __device__ static int m(int q, int c, int bs) { return ((q >> 1) * 5 + c) * 2 * bs + (q & 1); }
  __device__ static int t(int q, int bs) { return (q >> 1) * 2 * bs + (q & 1); }
};

// Rotated Schmid 5-vectors of one voxel into shared memory (see schmid_from_R),
// computed in the staging precision MS (FP64 path: double; mixed: float).
template <typename MS>
__device__ __forceinline__ void schmid_to_smem(const MS R[9], MS* msm, int bs) {
  static_for_s<0, kNS>([&](auto sc) {
    constexpr int s = decltype(sc)::value;
    MS b[3], n[3];
    rotated_slip<s>(R, b, n);
    const MS q00 = b[0] * n[0], q11 = b[1] * n[1], q22 = b[2] * n[2];
    const MS c23 = (MS)VPFFT_INV_2SQRT3, c6 = (MS)(1.0 / 6.0);
    msm[SL<MS>::m(s, 0, bs)] = (q11 - q00) * c23;
    msm[SL<MS>::m(s, 1, bs)] = (MS(2) * q22 - q00 - q11) * c6;
    msm[SL<MS>::m(s, 2, bs)] = (b[1] * n[2] + b[2] * n[1]) * c23;
    msm[SL<MS>::m(s, 3, bs)] = (b[0] * n[2] + b[2] * n[0]) * c23;
    msm[SL<MS>::m(s, 4, bs)] = (b[0] * n[1] + b[1] * n[0]) * c23;
  });
}

// The FP32 staging of schmid_to_smem with paired arithmetic: systems q and q+1
// in the two lanes of a float2 (FMUL2/FFMA2), stored as one 8-byte value per
// component at the pair-interleaved offsets of SL<float>.  q11 - q00 is
// formed as fma(q00, -1, q11), which rounds like the subtraction.
// (A template, so that only the sm_100a device code that calls it instantiates
// the paired intrinsics.)
template <typename T = float>
__device__ __forceinline__ void schmid_to_smem_pairs(const T R[9], T* msm, int bs) {
  static_assert(sizeof(T) == 4, "FP32 staging");
  float2* m2 = reinterpret_cast<float2*>(msm);
  const float2 c23 = make_float2((float)VPFFT_INV_2SQRT3, (float)VPFFT_INV_2SQRT3);
  const float2 c6 = make_float2((float)(1.0 / 6.0), (float)(1.0 / 6.0));
  const float2 m1 = make_float2(-1.f, -1.f), two = make_float2(2.f, 2.f);
  static_for_s<0, kNS / 2>([&](auto pc) {
    constexpr int pq = decltype(pc)::value;
    float ba[3], na[3], bb[3], nb[3];
    rotated_slip<2 * pq>(R, ba, na);
    rotated_slip<2 * pq + 1>(R, bb, nb);
    float2 b[3], n[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      b[i] = make_float2(ba[i], bb[i]);
      n[i] = make_float2(na[i], nb[i]);
    }
    const float2 q00 = __fmul2_rn(b[0], n[0]), q11 = __fmul2_rn(b[1], n[1]);
    const float2 q22 = __fmul2_rn(b[2], n[2]);
    float2 t = __ffma2_rn(q00, m1, __fmul2_rn(q22, two));
    t = __ffma2_rn(q11, m1, t);
    m2[(pq * 5 + 0) * bs] = __fmul2_rn(__ffma2_rn(q00, m1, q11), c23);
    m2[(pq * 5 + 1) * bs] = __fmul2_rn(t, c6);
    m2[(pq * 5 + 2) * bs] = __fmul2_rn(__ffma2_rn(b[1], n[2], __fmul2_rn(b[2], n[1])), c23);
    m2[(pq * 5 + 3) * bs] = __fmul2_rn(__ffma2_rn(b[0], n[2], __fmul2_rn(b[2], n[0])), c23);
    m2[(pq * 5 + 4) * bs] = __fmul2_rn(__ffma2_rn(b[0], n[1], __fmul2_rn(b[1], n[0])), c23);
  });
}

template <typename MS>
__device__ __forceinline__ void load_m(const MS* msm, int bs, int s, double m[5]) {
#pragma unroll
  for (int c = 0; c < 5; ++c) m[c] = (double)msm[SL<MS>::m(s, c, bs)];
}

// 1/x: IEEE division in FP64; in FP32 (the Newton predictor, which the FP64
// step polishes) the fast reciprocal intrinsic.
__device__ __forceinline__ double recip(double x) { return 1.0 / x; }
__device__ __forceinline__ float recip(float x) { return __fdividef(1.f, x); }

// |delta| / |avg| < eps for the squared norms dn = |delta|^2, an = |avg|^2,
// compared as dn < eps^2 an; *bad when a norm is not finite or |avg| = 0
// (where the quotient would not be finite).
__device__ __forceinline__ bool small_step_f32(float dn, float an, float eps, bool* bad) {
  *bad = !(dn <= FLT_MAX) || !(an > 0.f) || !(an <= FLT_MAX);
  return dn < eps * eps * an;
}

// LDL^T factorisation of a symmetric positive-definite 5x5 A (packed upper):
// the strict lower part of L and the reciprocal pivots.  Returns false when a
// pivot is not positive (A not numerically SPD).
template <typename T>
struct Ldl5 {
  T L[5][5];  // L[i][j], i > j
  T id[5];    // 1 / d[j]
};
template <typename T>
__device__ __forceinline__ bool ldlt5_factor(const T A[15], Ldl5<T>& f) {
  T d[5];
  bool ok = true;
#pragma unroll
  for (int j = 0; j < 5; ++j) {
    T dj = A[sym5(j, j)];
#pragma unroll
    for (int k = 0; k < j; ++k) dj -= f.L[j][k] * f.L[j][k] * d[k];
    ok = ok && (dj > T(0));
    d[j] = dj;
    f.id[j] = recip(dj);
#pragma unroll
    for (int i = j + 1; i < 5; ++i) {
      T a = A[sym5(j, i)];
#pragma unroll
      for (int k = 0; k < j; ++k) a -= f.L[i][k] * f.L[j][k] * d[k];
      f.L[i][j] = a * f.id[j];
    }
  }
  return ok;
}
// x = A^-1 b from the factors of A.
template <typename T>
__device__ __forceinline__ void ldlt5_subst(const Ldl5<T>& f, const T b[5], T x[5]) {
  T z[5];
#pragma unroll
  for (int i = 0; i < 5; ++i) {
    T a = b[i];
#pragma unroll
    for (int k = 0; k < i; ++k) a -= f.L[i][k] * z[k];
    z[i] = a;
  }
#pragma unroll
  for (int i = 4; i >= 0; --i) {
    T a = z[i] * f.id[i];
#pragma unroll
    for (int k = i + 1; k < 5; ++k) a -= f.L[k][i] * x[k];
    x[i] = a;
  }
}
// LDL^T solve of A x = b; false when A is not numerically SPD.
template <typename T>
__device__ __forceinline__ bool ldlt5_solve(const T A[15], const T b[5], T x[5]) {
  Ldl5<T> f;
  const bool ok = ldlt5_factor(A, f);
  ldlt5_subst(f, b, x);
  return ok;
}

// 1/CRSS of system q: per voxel from shared memory (stride bs) or uniform
// from the launch parameters.
template <bool kTauSmem, typename MS>
__device__ __forceinline__ double itau_of(const MS* tsm, int bs, const NRParams& p, int q) {
  if constexpr (kTauSmem)
    return (double)tsm[SL<MS>::t(q, bs)];
  else
    return p.icrss[q];
}

// One pass over the systems: r_s, admissibility, S = sum m gdot r, K = sum n gdot/tau m m^T,
// in arithmetic type T (double, or float for the predictor of the mixed path).
// snap: set |r| < 1e-10 to 0 (the unconstrained solver does, Solvers.cpp:50-51).
// rmax (kRmax): max_s |r_s| at s.
template <int NEXP, bool kSnap, bool kTauSmem, typename T, typename MS, bool kRmax = false>
__device__ __forceinline__ bool accumulate(const MS* msm, const MS* tsm, int bs,
                                           const NRParams& p, const T s[5], T S[5], T K[15],
                                           T* rmax = nullptr) {
  using C = NRConst<T>;
  bool adm = true;
  T rm = T(0);
#pragma unroll
  for (int c = 0; c < 5; ++c) S[c] = T(0);
#pragma unroll
  for (int k = 0; k < 15; ++k) K[k] = T(0);
#pragma unroll 2
  for (int q = 0; q < kNS; ++q) {
    T m[5];
#pragma unroll
    for (int c = 0; c < 5; ++c) m[c] = (T)msm[SL<MS>::m(q, c, bs)];
    T it;
    if constexpr (kTauSmem)
      it = (T)tsm[SL<MS>::t(q, bs)];
    else
      it = C::icrss(p, q);
    T r = (m[0] * s[0] + m[1] * s[1] + m[2] * s[2] + m[3] * s[3] + m[4] * s[4]) * it;
    if (kSnap) r = fabs(r) < T(1e-10) ? T(0) : r;
    adm = adm && !(fabs(r) > C::max_rss(p));
    if constexpr (kRmax) rm = fmax(rm, fabs(r));
    const int n = p.nexp[q];
    // the constrained solver tests n != 1, the unconstrained n - 1 > 0 (Solvers.cpp:66,177)
    const bool power = kSnap ? (n - 1 > 0) : (n != 1);
    const T g = power ? C::gdot(p, q) * pow_nm1<NEXP>(fabs(r), n) : C::gdot(p, q);
    const T gr = g * r;
    const T w = C::n(p, q) * g * it;
#pragma unroll
    for (int i = 0; i < 5; ++i) {
      S[i] += m[i] * gr;
      const T mw = m[i] * w;
#pragma unroll
      for (int j = i; j < 5; ++j) K[sym5(i, j)] += mw * m[j];
    }
  }
  if constexpr (kRmax) *rmax = rm;
  return adm;
}

// x^E for both lanes of a float2 (E >= 0 at compile time), paired multiplies.
template <int E>
__device__ __forceinline__ float2 cpow2(float2 x) {
  if constexpr (E == 0) {
    return make_float2(1.f, 1.f);
  } else if constexpr (E == 1) {
    return x;
  } else {
    const float2 h = cpow2<E / 2>(x);
    if constexpr (E & 1)
      return __fmul2_rn(__fmul2_rn(h, h), x);
    else
      return __fmul2_rn(h, h);
  }
}

// The predictor's pass over the systems with paired FP32 arithmetic: lane 0
// of every float2 carries system q, lane 1 system q+1 (FFMA2/FMUL2 issue two
// FMAs per instruction); the two partial sums of S and K are added at the end.
// Compile-time rate exponent NEXP > 1 (the power branch of Solvers.cpp:177).
// kFull: the pass over the 6 pairs fully unrolled (the single-grid kernel,
// which has the registers for it: measured 3 % faster) or by 2 (the batched
// kernel at 4 blocks per SM, where the full unroll spills).
template <int NEXP, bool kTauSmem, bool kFull = true>
__device__ __forceinline__ bool accumulate_pairs(const float* msm, const float* tsm, int bs,
                                                 const NRParams& p, const float s[5], float S[5],
                                                 float K[15], float* rmax) {
  static_assert(NEXP > 1, "paired predictor needs a compile-time exponent > 1");
  const float2* m2p = reinterpret_cast<const float2*>(msm);
  const float2* t2p = reinterpret_cast<const float2*>(tsm);
  float2 S2[5], K2[15], s2[5];
#pragma unroll
  for (int c = 0; c < 5; ++c) {
    S2[c] = make_float2(0.f, 0.f);
    s2[c] = make_float2(s[c], s[c]);
  }
#pragma unroll
  for (int k = 0; k < 15; ++k) K2[k] = make_float2(0.f, 0.f);
  const float2 nn = make_float2((float)NEXP, (float)NEXP);
  const float mr = p.max_rss_f;
  bool adm = true;
  float rm = 0.f;
  auto pair = [&](int pq) {
    float2 m[5];
#pragma unroll
    for (int c = 0; c < 5; ++c) m[c] = m2p[(pq * 5 + c) * bs];
    float2 it;
    if constexpr (kTauSmem)
      it = t2p[pq * bs];
    else
      it = make_float2(p.icrss_f[2 * pq], p.icrss_f[2 * pq + 1]);
    float2 r = __fmul2_rn(m[0], s2[0]);
#pragma unroll
    for (int c = 1; c < 5; ++c) r = __ffma2_rn(m[c], s2[c], r);
    r = __fmul2_rn(r, it);
    const float ax = fabsf(r.x), ay = fabsf(r.y);
    adm = adm && !(ax > mr) && !(ay > mr);
    rm = fmaxf(rm, fmaxf(ax, ay));
    const float2 pw = cpow2<NEXP - 1>(make_float2(ax, ay));
    const float2 g = __fmul2_rn(make_float2(p.gdot_f[2 * pq], p.gdot_f[2 * pq + 1]), pw);
    const float2 gr = __fmul2_rn(g, r);
    const float2 w = __fmul2_rn(__fmul2_rn(nn, g), it);
#pragma unroll
    for (int i = 0; i < 5; ++i) {
      S2[i] = __ffma2_rn(m[i], gr, S2[i]);
      const float2 mw = __fmul2_rn(m[i], w);
#pragma unroll
      for (int j = i; j < 5; ++j) K2[sym5(i, j)] = __ffma2_rn(mw, m[j], K2[sym5(i, j)]);
    }
  };
  if constexpr (kFull) {
#pragma unroll
    for (int pq = 0; pq < kNS / 2; ++pq) pair(pq);
  } else {
#pragma unroll 2
    for (int pq = 0; pq < kNS / 2; ++pq) pair(pq);
  }
#pragma unroll
  for (int c = 0; c < 5; ++c) S[c] = S2[c].x + S2[c].y;
#pragma unroll
  for (int k = 0; k < 15; ++k) K[k] = K2[k].x + K2[k].y;
  *rmax = rm;
  return adm;
}

// Newton predictor of the constrained solve in FP32 (mixed precision only):
// the reference's iteration and stopping rule in single precision.  Returns
// true and the iterate in s_io when it converged with finite values; the
// caller then takes the accepted step with FP64 residual and Jacobian.
// *rmax0 gets max_s |r_s| at the starting point.
// fac (optional): the LDL^T factors of the converged step's Newton matrix.
// l32, e32: lambda and Edot + d~ rounded to FP32; cur: the starting stress in,
// the converged iterate out (undefined when the predictor fails).
template <int NEXP, bool kTauSmem, bool kFull = true, typename MS, class C>
__device__ __forceinline__ bool nr_predict_fp32(const MS* msm, const MS* tsm, int bs,
                                                const NRParams& p, const C& cs,
                                                const float l32[5], const float e32[5],
                                                float cur[5], int max_steps, float* rmax0,
                                                Ldl5<float>* fac = nullptr) {
  *rmax0 = 0.f;
  for (int it = 0; it < max_steps; ++it) {
    float S[5], K[15], rm;
    bool adm;
    if constexpr (NEXP > 1 && sizeof(MS) == 4)
      adm = accumulate_pairs<NEXP, kTauSmem, kFull>(msm, tsm, bs, p, cur, S, K, &rm);
    else
      adm = accumulate<NEXP, false, kTauSmem, float, MS, true>(msm, tsm, bs, p, cur, S, K, &rm);
    if (it == 0) *rmax0 = rm;
    if (!adm) return false;
    float y[5];
#pragma unroll
    for (int i = 0; i < 5; ++i) {
      float a = S[i] - e32[i];
#pragma unroll
      for (int j = 0; j < 5; ++j) a += cs.L0inv_f(sym5(i, j)) * (cur[j] - l32[j]);
      y[i] = -a;
    }
#pragma unroll
    for (int k = 0; k < 15; ++k) K[k] += cs.L0inv_f(k);
    float delta[5];
    Ldl5<float> f;
    if (!ldlt5_factor(K, f)) return false;
    ldlt5_subst(f, y, delta);
    float dn = 0.f, an = 0.f;
#pragma unroll
    for (int c = 0; c < 5; ++c) {
      const float nw = cur[c] + delta[c];
      const float av = (nw + cur[c]) * 0.5f;
      dn += delta[c] * delta[c];
      an += av * av;
      cur[c] = nw;
    }
    bool bad;
    const bool small = small_step_f32(dn, an, p.eps_f, &bad);
    if (bad) return false;
    if (small) {
      if (fac) *fac = f;
      return true;
    }
  }
  return false;
}

// The strain rate S(s) = sum_s m_s gdot_s |r_s|^(n-1) r_s in FP64 and the
// admissibility of s (every |r_s| within the cap): the FP64 residual pass of
// the mixed path, the S half of `accumulate` for the constrained solver.
// kFull: the pass over the 12 systems fully unrolled (the single-grid sweep:
// measured 4.7 % faster at 256^3 than by 2), else by 4 (the batched sweep,
// which has 128 registers: 388 solves/s against 377-384 by 2 and 382 fully
// unrolled on the 256-RVE workload).
template <int NEXP, bool kTauSmem, bool kFull = true, typename MS>
__device__ __forceinline__ bool strain_rate_fp64(const MS* msm, const MS* tsm, int bs,
                                                 const NRParams& p, const double s[5],
                                                 double S[5]) {
  bool adm = true;
#pragma unroll
  for (int c = 0; c < 5; ++c) S[c] = 0.0;
#pragma unroll(kFull ? kNS : 4)
  for (int q = 0; q < kNS; ++q) {
    double m[5];
    load_m(msm, bs, q, m);
    const double it = itau_of<kTauSmem>(tsm, bs, p, q);
    const double r = (m[0] * s[0] + m[1] * s[1] + m[2] * s[2] + m[3] * s[3] + m[4] * s[4]) * it;
    adm = adm && !(fabs(r) > p.max_rss);
    const int n = p.nexp[q];
    const double g = n != 1 ? p.gdot[q] * pow_nm1<NEXP>(fabs(r), n) : p.gdot[q];
    const double gr = g * r;
#pragma unroll
    for (int i = 0; i < 5; ++i) S[i] += m[i] * gr;
  }
  return adm;
}

// SolveConstrainedConstitutiveEquations (Solvers.cpp:111-222).  ed = Edot + d~.
// Returns the Newton steps taken; *capped when the iteration budget ran out.
// The stopping test |delta| / |avg| < eps is taken on the squared norms
// (|delta|^2 < eps^2 |avg|^2); *rel_out (optional) gets the last step's ratio,
// *tight (optional) whether it was below 1e-5.
// kSolveF32: the Newton system, formed in FP64 (residual and Jacobian), is
// solved by an FP32 LDL^T (the mixed path's final step, which is small: the
// step's relative error ~1e-6 is a relative change of sigma far below FP32
// storage, and the next step, if any, sees the FP64 residual); otherwise by
// an FP64 LDL^T (the FP64 path, the reference's arithmetic).
template <int NEXP, bool kTauSmem, typename MS, class C = ParamConsts, bool kSolveF32 = false>
__device__ __forceinline__ int nr_constrained_smem(const MS* msm, const MS* tsm, int bs,
                                                   const NRParams& p, const C& cs,
                                                   const double lam[5],
                                                   const double ed[5], double s_io[5],
                                                   double* rel_out, bool* capped,
                                                   double* e_lin = nullptr,
                                                   bool* tight = nullptr) {
  double cur[5], saved[5], nw[5] = {-1.0, -3.0, -7.0, -9.0, -11.0};
#pragma unroll
  for (int c = 0; c < 5; ++c) cur[c] = saved[c] = s_io[c];
  const double eps2 = p.eps * p.eps;
  double dn = 1e10, an = 1.0;  // a ratio of 1e5 before the first step
  bool conv = false;
  int remaining = p.max_iter, steps = 0;
  *capped = false;
  while (remaining > 0) {
    double S[5], K[15];
    // admissibility loop (Solvers.cpp:147-172): back off towards the saved
    // state while some |r_s| exceeds the cap; every pass costs one iteration
    for (;;) {
      const bool adm = accumulate<NEXP, false, kTauSmem, double>(msm, tsm, bs, p, cur, S, K);
      if (!adm) {
#pragma unroll
        for (int c = 0; c < 5; ++c) cur[c] = saved[c] + (cur[c] - saved[c]) * 0.2;
      }
      remaining--;
      if (remaining < 0) {
        *capped = true;
        if (rel_out) *rel_out = sqrt(dn) / sqrt(an);
        if (tight) *tight = false;
#pragma unroll
        for (int c = 0; c < 5; ++c) s_io[c] = cur[c];
        return steps;
      }
      if (adm) break;
    }
    // y = L0^-1 (cur - lambda) + (S - Edot - d~);  (L0^-1 + K) delta = -y
    double dl[5], y[5];
#pragma unroll
    for (int c = 0; c < 5; ++c) dl[c] = cur[c] - lam[c];
#pragma unroll
    for (int i = 0; i < 5; ++i) {
      double a = S[i] - ed[i];
#pragma unroll
      for (int j = 0; j < 5; ++j) a += cs.L0inv(sym5(i, j)) * dl[j];
      y[i] = -a;
    }
#pragma unroll
    for (int k = 0; k < 15; ++k) K[k] += cs.L0inv(k);
    double delta[5];
    if constexpr (kSolveF32) {
      float Kf[15], yf[5], df[5];
#pragma unroll
      for (int k = 0; k < 15; ++k) Kf[k] = (float)K[k];
#pragma unroll
      for (int c = 0; c < 5; ++c) yf[c] = (float)y[c];
      ldlt5_solve<float>(Kf, yf, df);
#pragma unroll
      for (int c = 0; c < 5; ++c) delta[c] = (double)df[c];
    } else {
      ldlt5_solve<double>(K, y, delta);
    }
    dn = 0.0;
    an = 0.0;
#pragma unroll
    for (int c = 0; c < 5; ++c) {
      saved[c] = cur[c];
      nw[c] = cur[c] + delta[c];
      const double df = nw[c] - saved[c];
      const double av = (nw[c] + saved[c]) * 0.5;
      dn += df * df;
      an += av * av;
      cur[c] = nw[c];
    }
    steps++;
    conv = dn < eps2 * an;
    if (conv) break;
  }
  if (rel_out) *rel_out = sqrt(dn) / sqrt(an);
  if (tight) *tight = dn < 1e-10 * an;
  *capped = !conv;
#pragma unroll
  for (int c = 0; c < 5; ++c) s_io[c] = nw[c];
  if (e_lin) {
    // strain rate at the new point from the last Newton linearisation:
    // S + K delta = ed - L0^-1 (sigma_new - lambda)  (error O(|delta|^2))
#pragma unroll
    for (int i = 0; i < 5; ++i) {
      double a = ed[i];
#pragma unroll
      for (int j = 0; j < 5; ++j) a -= cs.L0inv(sym5(i, j)) * (nw[j] - lam[j]);
      e_lin[i] = a;
    }
  }
  return steps;
}

// Complete-pivoting fallback of the unconstrained step (singular K).
static __device__ __noinline__ void solve_neg_K_fullpiv(const double K[15], const double res[5],
                                                 double delta[5]) {
  double A[5][5], b[5];
#pragma unroll
  for (int i = 0; i < 5; ++i) {
    b[i] = res[i];
#pragma unroll
    for (int j = 0; j < 5; ++j) A[i][j] = -K[sym5(i, j)];
  }
  solve5_fullpiv(A, b, delta);
}

// SolveConstitutiveEquations (Solvers.cpp:19-101): -K delta = R, R = S - Edot.
template <int NEXP, bool kTauSmem, typename MS>
__device__ __forceinline__ int nr_unconstrained_smem(const MS* msm, const MS* tsm, int bs,
                                                     const NRParams& p, const double edot[5],
                                                     double s_io[5], bool* capped) {
  double cur[5], nw[5], saved[5];
#pragma unroll
  for (int c = 0; c < 5; ++c) {
    cur[c] = nw[c] = s_io[c];
    saved[c] = 0.0;
  }
  int remaining = p.max_iter, steps = 0;
  bool conv = false;
  while (remaining > 0) {
    double S[5], K[15];
    for (;;) {
      const bool adm = accumulate<NEXP, true, kTauSmem, double>(msm, tsm, bs, p, cur, S, K);
      if (!adm) {
#pragma unroll
        for (int c = 0; c < 5; ++c) cur[c] = saved[c] + (cur[c] - saved[c]) * 0.2;
      }
      remaining--;
      if (remaining < 0) {  // the reference returns NewStressState here (Solvers.cpp:59-60)
        *capped = true;
#pragma unroll
        for (int c = 0; c < 5; ++c) s_io[c] = nw[c];
        return steps;
      }
      if (adm) break;
    }
    // J = -K, R = S - Edot:  K delta = -R
    double res[5], mres[5], delta[5];
#pragma unroll
    for (int c = 0; c < 5; ++c) {
      res[c] = S[c] - edot[c];
      mres[c] = -res[c];
    }
    if (!ldlt5_solve<double>(K, mres, delta)) solve_neg_K_fullpiv(K, res, delta);
    double dn = 0.0, sn = 0.0;
#pragma unroll
    for (int c = 0; c < 5; ++c) {
      saved[c] = cur[c];
      nw[c] = cur[c] + delta[c];
      const double sm = nw[c] + cur[c];
      dn += delta[c] * delta[c];
      sn += sm * sm;
      cur[c] = nw[c];
    }
    steps++;
    // 2 |delta| / |new + old| < eps, on the squared norms
    if (4.0 * dn < p.eps * p.eps * sn) {
      conv = true;
      break;
    }
  }
  *capped = !conv;
#pragma unroll
  for (int c = 0; c < 5; ++c) s_io[c] = nw[c];
  return steps;
}

// Newton predictor of the unconstrained solve in FP32 (mixed precision only):
// the reference's iteration (Solvers.cpp:19-101: admissibility back-off towards
// the previous iterate, K delta = -(S - Edot), stop at 2|delta|/|new + old| <
// eps) in single precision.  Returns true with the iterate in s_io when it
// converged; the caller then runs the FP64 iteration from there.
template <int NEXP, bool kTauSmem, typename MS>
__device__ __forceinline__ bool nr_predict_unconstrained_fp32(const MS* msm, const MS* tsm,
                                                              int bs, const NRParams& p,
                                                              const double edot[5],
                                                              double s_io[5], int max_steps) {
  float cur[5], saved[5], e32[5];
#pragma unroll
  for (int c = 0; c < 5; ++c) {
    cur[c] = (float)s_io[c];
    saved[c] = 0.f;
    e32[c] = (float)edot[c];
  }
  for (int it = 0; it < max_steps; ++it) {
    float S[5], K[15], rm;
    for (int back = 0;; ++back) {
      bool adm;
      if constexpr (NEXP > 1 && sizeof(MS) == 4)
        adm = accumulate_pairs<NEXP, kTauSmem>(msm, tsm, bs, p, cur, S, K, &rm);
      else
        adm = accumulate<NEXP, false, kTauSmem, float, MS, true>(msm, tsm, bs, p, cur, S, K, &rm);
      if (adm) break;
      if (back >= 40) return false;
#pragma unroll
      for (int c = 0; c < 5; ++c) cur[c] = saved[c] + (cur[c] - saved[c]) * 0.2f;
    }
    float mres[5], delta[5];
#pragma unroll
    for (int c = 0; c < 5; ++c) mres[c] = e32[c] - S[c];
    if (!ldlt5_solve(K, mres, delta)) return false;
    float dn = 0.f, sn = 0.f;
#pragma unroll
    for (int c = 0; c < 5; ++c) {
      saved[c] = cur[c];
      const float nw = cur[c] + delta[c];
      const float sm = nw + cur[c];
      dn += delta[c] * delta[c];
      sn += sm * sm;
      cur[c] = nw;
    }
    // 2 |delta| / |sum| < eps
    bool bad;
    const bool small = small_step_f32(4.f * dn, sn, p.eps_f, &bad);
    if (bad) return false;
    if (small) {
#pragma unroll
      for (int c = 0; c < 5; ++c) s_io[c] = (double)cur[c];
      return true;
    }
  }
  return false;
}

// GetMaxRSS (MaterialGrid.h:550-566) and the Sachs bound (Solvers.cpp:234-240):
// max_s |m_s . x| / tau_s
template <bool kTauSmem, typename MS>
__device__ __forceinline__ double max_resolved(const MS* msm, const MS* tsm, int bs,
                                               const NRParams& p, const double x[5]) {
  double mx = 0.0;
#pragma unroll 4
  for (int q = 0; q < kNS; ++q) {
    double m[5];
    load_m(msm, bs, q, m);
    const double a =
        fabs((m[0] * x[0] + m[1] * x[1] + m[2] * x[2] + m[3] * x[3] + m[4] * x[4]) *
             itau_of<kTauSmem>(tsm, bs, p, q));
    mx = (a < mx) ? mx : a;
  }
  return mx;
}

// ApplyConstitutiveEquations (Solvers.cpp:255-274)
template <int NEXP, bool kTauSmem, typename MS>
__device__ __forceinline__ void apply_smem(const MS* msm, const MS* tsm, int bs, const NRParams& p,
                                           const double s[5], double e[5]) {
#pragma unroll
  for (int c = 0; c < 5; ++c) e[c] = 0.0;
#pragma unroll 2
  for (int q = 0; q < kNS; ++q) {
    double m[5];
    load_m(msm, bs, q, m);
    const double r = (m[0] * s[0] + m[1] * s[1] + m[2] * s[2] + m[3] * s[3] + m[4] * s[4]) *
                     itau_of<kTauSmem>(tsm, bs, p, q);
    const int n = p.nexp[q];
    const double g = n > 0 ? p.gdot[q] * pow_n<NEXP>(fabs(r), n) : p.gdot[q];
    const double f = g * (double)sgn(r);
#pragma unroll
    for (int c = 0; c < 5; ++c) e[c] += m[c] * f;
  }
}

}  // namespace vpfft
