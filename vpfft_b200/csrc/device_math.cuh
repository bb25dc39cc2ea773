// device_math.cuh -- per-voxel crystal-plasticity arithmetic for sm_100a.
//
// Everything here runs in registers of one thread per voxel.  The
// Newton-Raphson solves, the reference-medium inverse and the reductions are
// FP64 in every precision mode; only storage, FFT and Green operator switch to
// FP32 in mixed mode.
//
// Reference routines restated (file:line in exmatex/VPFFT Src/):
//   deviatoric basis            LinearAlgebra.h:207-247
//   FCC slip systems            BurgerVectorBasis.h:16-75, 126-151
//   local Schmid tensors        MaterialGrid.cpp:107-124
//   GetMaxRSS                   MaterialGrid.h:550-566
//   SolveSachEquation           Solvers.cpp:230-243
//   SolveConstitutiveEquations  Solvers.cpp:19-101
//   SolveConstrained...         Solvers.cpp:111-222
//   ApplyConstitutiveEquations  Solvers.cpp:255-274
//   LU_Solver (full pivoting)   LinearAlgebra.cpp:1171-1187
//   ConstructGreensOperator     MaterialGrid.cpp:583-615 (+ Symmetrize/projection 717)
#pragma once

#include <type_traits>

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

namespace vpfft {

// a * b + c with one rounding, spelled out: the line transforms and the Green
// operator use it for every product-sum so that their arithmetic does not
// depend on the compiler's choice of contractions (their translation units are
// built with contraction off), which makes every compiled copy of a pass --
// the single-grid tiles and each batched tile family -- give the same bits.
__host__ __device__ __forceinline__ float fmad(float a, float b, float c) {
#ifdef __CUDA_ARCH__
  return __fmaf_rn(a, b, c);
#else
  return fmaf(a, b, c);
#endif
}
__host__ __device__ __forceinline__ double fmad(double a, double b, double c) {
#ifdef __CUDA_ARCH__
  return __fma_rn(a, b, c);
#else
  return fma(a, b, c);
#endif
}

constexpr int kNS = 12;

// FCC {111}<110> slip systems in the reference's order: Burgers direction b_s
// and plane normal n_s (unnormalised integer vectors, BurgerVectorBasis.h:16-75).
// The Schmid tensor is sym(b (x) n)/(2 sqrt 6) and the anti-Schmid tensor
// skew(b (x) n)/(2 sqrt 6) (BurgerVectorBasis.h:126-151); with |b||n| = sqrt 6
// both have unit-normalised directions.
__host__ __device__ constexpr int slip_b(int s, int i) {
  // clang-format off
  return (s == 0) ? (i == 0 ? 0 : 1)
       : (s == 1) ? (i == 1 ? 0 : 1)
       : (s == 2) ? (i == 0 ? 1 : i == 1 ? -1 : 0)
       : (s == 3) ? (i == 0 ? 0 : i == 1 ? 1 : -1)
       : (s == 4) ? (i == 1 ? 0 : 1)
       : (s == 5) ? (i == 2 ? 0 : 1)
       : (s == 6) ? (i == 0 ? 0 : 1)
       : (s == 7) ? (i == 0 ? 1 : i == 1 ? 0 : -1)
       : (s == 8) ? (i == 2 ? 0 : 1)
       : (s == 9) ? (i == 0 ? 0 : i == 1 ? 1 : -1)
       : (s == 10) ? (i == 0 ? 1 : i == 1 ? 0 : -1)
       : (i == 0 ? 1 : i == 1 ? -1 : 0);
  // clang-format on
}
__host__ __device__ constexpr int slip_n(int s, int i) {
  // planes: (1,1,-1) s=0..2, (1,-1,-1) s=3..5, (1,-1,1) s=6..8, (1,1,1) s=9..11
  return (i == 0) ? 1
       : (i == 1) ? ((s < 3 || s >= 9) ? 1 : -1)
                  : ((s < 6) ? -1 : 1);
}

// c0 x0 + c1 x1 + c2 x2 for compile-time coefficients in {-1, 0, 1}, summed in
// index order: the same roundings as the multiply-add chain over the integer
// slip vectors, without the multiplications by 0 and 1.
template <int C0, int C1, int C2, typename T>
__host__ __device__ __forceinline__ T signed_sum3(T x0, T x1, T x2) {
  static_assert(C0 != 0 || C1 != 0 || C2 != 0, "zero vector");
  static_assert(C0 >= -1 && C0 <= 1 && C1 >= -1 && C1 <= 1 && C2 >= -1 && C2 <= 1, "signs");
  auto term = [](auto c, T x) { return c < 0 ? -x : x; };
  if constexpr (C0 != 0) {
    T r = term(C0, x0);
    if constexpr (C1 > 0) r = r + x1;
    if constexpr (C1 < 0) r = r - x1;
    if constexpr (C2 > 0) r = r + x2;
    if constexpr (C2 < 0) r = r - x2;
    return r;
  } else if constexpr (C1 != 0) {
    T r = term(C1, x1);
    if constexpr (C2 > 0) r = r + x2;
    if constexpr (C2 < 0) r = r - x2;
    return r;
  } else {
    return term(C2, x2);
  }
}

template <int I, int N, typename F>
__host__ __device__ __forceinline__ void static_for_s(F&& f) {
  if constexpr (I < N) {
    f(std::integral_constant<int, I>{});
    static_for_s<I + 1, N>(f);
  }
}

// Rotated slip direction b' = R b and plane normal n' = R n of system S (R
// row-major), from the integer vectors of slip_b / slip_n.
template <int S, typename T>
__host__ __device__ __forceinline__ void rotated_slip(const T R[9], T b[3], T n[3]) {
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    b[i] = signed_sum3<slip_b(S, 0), slip_b(S, 1), slip_b(S, 2)>(R[3 * i], R[3 * i + 1],
                                                                 R[3 * i + 2]);
    n[i] = signed_sum3<slip_n(S, 0), slip_n(S, 1), slip_n(S, 2)>(R[3 * i], R[3 * i + 1],
                                                                 R[3 * i + 2]);
  }
}

// 1/(2 sqrt 3) and 1/6: the coefficients that map q_ij = b'_i n'_j (rotated
// vectors) to the 5 deviatoric-basis components of sym(b' (x) n')/(2 sqrt 6).
#define VPFFT_INV_2SQRT3 0.28867513459481288225
#define VPFFT_INV_2SQRT6 0.20412414523193150818

// m_s = EigenRep(R M_s R^T) for the 12 systems (MaterialGrid.cpp:107-124).
// R M_s R^T = sym((R b) (x) (R n))/(2 sqrt 6), also for non-orthogonal R (the
// texture update is additive and does not re-orthonormalise, MaterialGrid.cpp:870).
// Projection on the basis of LinearAlgebra.h:207-247:
//   m0 = (S11 - S00)/sqrt2, m1 = (2 S22 - S00 - S11)/sqrt6,
//   m2 = sqrt2 S12, m3 = sqrt2 S02, m4 = sqrt2 S01.
__device__ __forceinline__ void schmid_from_R(const double R[9], double m[kNS][5]) {
  static_for_s<0, kNS>([&](auto sc) {
    constexpr int s = decltype(sc)::value;
    double b[3], n[3];
    rotated_slip<s>(R, b, n);
    const double q00 = b[0] * n[0], q11 = b[1] * n[1], q22 = b[2] * n[2];
    m[s][0] = (q11 - q00) * VPFFT_INV_2SQRT3;
    m[s][1] = (2.0 * q22 - q00 - q11) * (1.0 / 6.0);
    m[s][2] = (b[1] * n[2] + b[2] * n[1]) * VPFFT_INV_2SQRT3;
    m[s][3] = (b[0] * n[2] + b[2] * n[0]) * VPFFT_INV_2SQRT3;
    m[s][4] = (b[0] * n[1] + b[1] * n[0]) * VPFFT_INV_2SQRT3;
  });
}

// Plastic spin of MaterialGrid::ShearRate (MaterialGrid.cpp:1098-1119) and
// Solvers::CalculateShearRate (Solvers.cpp:282-302):
//   W = sum_s (R A_s R^T) gdot0 |r_s|^n sgn(r_s),  R A_s R^T = skew((Rb)(x)(Rn))/(2 sqrt6)
// Only the 3 independent entries of the skew matrix are returned:
//   w01 = W[0][1], w02 = W[0][2], w12 = W[1][2]  (W[j][i] = -W[i][j]).
__device__ __forceinline__ void plastic_spin(const double R[9], const double gs[kNS],
                                             double w[3]) {
  w[0] = w[1] = w[2] = 0.0;
#pragma unroll
  for (int s = 0; s < kNS; ++s) {
    double b[3], n[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      b[i] = R[3 * i + 0] * slip_b(s, 0) + R[3 * i + 1] * slip_b(s, 1) + R[3 * i + 2] * slip_b(s, 2);
      n[i] = R[3 * i + 0] * slip_n(s, 0) + R[3 * i + 1] * slip_n(s, 1) + R[3 * i + 2] * slip_n(s, 2);
    }
    const double f = gs[s] * VPFFT_INV_2SQRT6;
    w[0] += (b[0] * n[1] - n[0] * b[1]) * f;
    w[1] += (b[0] * n[2] - n[0] * b[2]) * f;
    w[2] += (b[1] * n[2] - n[1] * b[2]) * f;
  }
}

__device__ __forceinline__ double dot5(const double* a, const double* b) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2] + a[3] * b[3] + a[4] * b[4];
}
__device__ __forceinline__ double norm5(const double* a) { return sqrt(dot5(a, a)); }

// |x|^e for a non-negative integer e by binary exponentiation (the reference
// calls std::pow(double, int), Solvers.cpp:67,178,268; agreement is a few ulp).
__device__ __forceinline__ double ipow(double x, int e) {
  double r = 1.0;
  double b = x;
  while (e > 0) {
    if (e & 1) r *= b;
    b *= b;
    e >>= 1;
  }
  return r;
}
// the reference's power for possibly negative exponents (n - 1 < 0 is legal input)
__device__ __forceinline__ double rpow(double x, int e) {
  return e >= 0 ? ipow(x, e) : 1.0 / ipow(x, -e);
}

__device__ __forceinline__ int sgn(double v) { return (0.0 < v) - (v < 0.0); }

// Material constants of one grid, passed by value into kernels (constant bank).
struct MaterialParams {
  double gdot[kNS];
  int32_t nexp[kNS];
};

// ---------------------------------------------------------------- 5x5 solves
// A x = b with complete pivoting (the algorithm of the reference's
// fullPivLu().solve, LinearAlgebra.cpp:1182): pivot = largest |a_ij| in the
// trailing block, first in row-major order on ties; zero pivots leave the
// corresponding unknown at zero.  A is row-major A[i][j] and is destroyed.
// Written with compile-time indices and selects so it stays in registers.
__device__ __forceinline__ void solve5_fullpiv(double A[5][5], double b[5], double x[5]) {
  int colp[5] = {0, 1, 2, 3, 4};
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    double best = -1.0;
    int pi = k, pj = k;
#pragma unroll
    for (int i = k; i < 5; ++i)
#pragma unroll
      for (int j = k; j < 5; ++j) {
        const double a = fabs(A[i][j]);
        const bool better = a > best;
        best = better ? a : best;
        pi = better ? i : pi;
        pj = better ? j : pj;
      }
#pragma unroll
    for (int i = k + 1; i < 5; ++i) {
      const bool sw = (pi == i);
#pragma unroll
      for (int j = 0; j < 5; ++j) {
        const double t = A[k][j];
        A[k][j] = sw ? A[i][j] : t;
        A[i][j] = sw ? t : A[i][j];
      }
      const double t = b[k];
      b[k] = sw ? b[i] : t;
      b[i] = sw ? t : b[i];
    }
#pragma unroll
    for (int j = k + 1; j < 5; ++j) {
      const bool sw = (pj == j);
#pragma unroll
      for (int i = 0; i < 5; ++i) {
        const double t = A[i][k];
        A[i][k] = sw ? A[i][j] : t;
        A[i][j] = sw ? t : A[i][j];
      }
      const int tc = colp[k];
      colp[k] = sw ? colp[j] : tc;
      colp[j] = sw ? tc : colp[j];
    }
    const double piv = A[k][k];
    const bool ok = piv != 0.0;
#pragma unroll
    for (int i = k + 1; i < 5; ++i) {
      const double l = ok ? A[i][k] / piv : A[i][k];
      A[i][k] = l;
#pragma unroll
      for (int j = k + 1; j < 5; ++j) A[i][j] = ok ? A[i][j] - l * A[k][j] : A[i][j];
      b[i] = ok ? b[i] - l * b[k] : b[i];
    }
  }
  double z[5];
#pragma unroll
  for (int i = 4; i >= 0; --i) {
    double s = b[i];
#pragma unroll
    for (int j = i + 1; j < 5; ++j) s -= A[i][j] * z[j];
    z[i] = (A[i][i] == 0.0) ? 0.0 : s / A[i][i];
  }
#pragma unroll
  for (int t = 0; t < 5; ++t) {
    double v = 0.0;
#pragma unroll
    for (int i = 0; i < 5; ++i) v = (colp[i] == t) ? z[i] : v;
    x[t] = v;
  }
}

// Inverse by LU with row pivoting (the algorithm the reference's Eigen
// inverse() uses for 5x5 matrices, MaterialGrid.cpp:245-248).  Row-major.
__device__ __forceinline__ void inverse5_pp(double A[5][5], double Ainv[5][5]) {
  int perm[5] = {0, 1, 2, 3, 4};
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    double best = fabs(A[k][k]);
    int piv = k;
#pragma unroll
    for (int i = k + 1; i < 5; ++i) {
      const double a = fabs(A[i][k]);
      const bool better = a > best;
      best = better ? a : best;
      piv = better ? i : piv;
    }
#pragma unroll
    for (int i = k + 1; i < 5; ++i) {
      const bool sw = (piv == i);
#pragma unroll
      for (int j = 0; j < 5; ++j) {
        const double t = A[k][j];
        A[k][j] = sw ? A[i][j] : t;
        A[i][j] = sw ? t : A[i][j];
      }
      const int tp = perm[k];
      perm[k] = sw ? perm[i] : tp;
      perm[i] = sw ? tp : perm[i];
    }
#pragma unroll
    for (int i = k + 1; i < 5; ++i) {
      A[i][k] = A[i][k] / A[k][k];
#pragma unroll
      for (int j = k + 1; j < 5; ++j) A[i][j] -= A[i][k] * A[k][j];
    }
  }
#pragma unroll
  for (int col = 0; col < 5; ++col) {
    double y[5];
#pragma unroll
    for (int i = 0; i < 5; ++i) {
      double s = (perm[i] == col) ? 1.0 : 0.0;
#pragma unroll
      for (int j = 0; j < i; ++j) s -= A[i][j] * y[j];
      y[i] = s;
    }
#pragma unroll
    for (int i = 4; i >= 0; --i) {
      double s = y[i];
#pragma unroll
      for (int j = i + 1; j < 5; ++j) s -= A[i][j] * y[j];
      y[i] = s / A[i][i];
    }
#pragma unroll
    for (int i = 0; i < 5; ++i) Ainv[i][col] = y[i];
  }
}

// ---------------------------------------------------------------- constitutive law
// Resolved shear stress over CRSS for all systems.
__device__ __forceinline__ void resolved(const double m[kNS][5], const double tau[kNS],
                                         const double s[5], double r[kNS]) {
#pragma unroll
  for (int k = 0; k < kNS; ++k) r[k] = dot5(m[k], s) / tau[k];
}

// GetMaxRSS (MaterialGrid.h:550-566), without the exit on < 1e-10.
__device__ __forceinline__ double max_rss(const double m[kNS][5], const double tau[kNS],
                                          const double s[5]) {
  double mx = 0.0;
#pragma unroll
  for (int k = 0; k < kNS; ++k) {
    const double a = fabs(dot5(m[k], s) / tau[k]);
    mx = (a < mx) ? mx : a;
  }
  return mx;
}

// SolveSachEquation (Solvers.cpp:230-243)
__device__ __forceinline__ void sachs(const double m[kNS][5], const double tau[kNS],
                                      const double edot[5], double out[5]) {
  double mx = 0.0;
#pragma unroll
  for (int k = 0; k < kNS; ++k) {
    const double a = fabs(dot5(edot, m[k]) / tau[k]);
    mx = (a < mx) ? mx : a;
  }
#pragma unroll
  for (int c = 0; c < 5; ++c) out[c] = edot[c] / mx;
}

// ApplyConstitutiveEquations (Solvers.cpp:255-274):
//   edot = sum_s m_s gdot0 |r|^n sgn(r)
__device__ __forceinline__ void apply_constitutive(const double m[kNS][5], const double tau[kNS],
                                                   const MaterialParams& mp, const double s[5],
                                                   double e[5]) {
#pragma unroll
  for (int c = 0; c < 5; ++c) e[c] = 0.0;
#pragma unroll
  for (int k = 0; k < kNS; ++k) {
    const double r = dot5(m[k], s) / tau[k];
    const double g = mp.nexp[k] > 0 ? mp.gdot[k] * ipow(fabs(r), mp.nexp[k]) : mp.gdot[k];
    const double f = g * (double)sgn(r);
#pragma unroll
    for (int c = 0; c < 5; ++c) e[c] += m[k][c] * f;
  }
}

// Result flags of the per-voxel solves.
enum : int { NR_OK = 0, NR_CAPPED = 1 };

// SolveConstitutiveEquations (Solvers.cpp:19-101): Newton-Raphson on
//   sum_s m_s gdot0 |r_s|^(n-1) r_s = edot,  r_s = m_s.s / tau_s,
// with |r_s| < 1e-10 snapped to 0 and the admissibility back-off
// s <- s_saved + 0.2 (s - s_saved) whenever some |r_s| > max_rss.
// Returns the number of Newton steps; *flag = NR_CAPPED if the iteration
// budget ran out.
__device__ __forceinline__ int nr_unconstrained(const double m[kNS][5], const double tau[kNS],
                                                const MaterialParams& mp, const double edot[5],
                                                double eps, double max_rss_cap, int max_iter,
                                                double s_io[5], int* flag) {
  double cur[5], nw[5], saved[5];
#pragma unroll
  for (int c = 0; c < 5; ++c) {
    cur[c] = s_io[c];
    nw[c] = s_io[c];
    saved[c] = 0.0;
  }
  int remaining = max_iter, steps = 0;
  bool conv = false;
  *flag = NR_OK;
  while (remaining > 0) {
    double r[kNS];
    bool admissible;
    do {
      admissible = true;
#pragma unroll
      for (int k = 0; k < kNS; ++k) {
        double v = dot5(m[k], cur) / tau[k];
        v = fabs(v) < 1e-10 ? 0.0 : v;
        admissible = admissible && !(fabs(v) > max_rss_cap);
        r[k] = v;
      }
      if (!admissible) {
#pragma unroll
        for (int c = 0; c < 5; ++c) cur[c] = saved[c] + (cur[c] - saved[c]) * 0.2;
      }
      remaining--;
      if (remaining < 0) {
        *flag = NR_CAPPED;
#pragma unroll
        for (int c = 0; c < 5; ++c) s_io[c] = nw[c];
        return steps;
      }
    } while (!admissible);
    double res[5] = {0, 0, 0, 0, 0};
    double J[5][5];
#pragma unroll
    for (int i = 0; i < 5; ++i)
#pragma unroll
      for (int j = 0; j < 5; ++j) J[i][j] = 0.0;
#pragma unroll
    for (int k = 0; k < kNS; ++k) {
      const double g = (mp.nexp[k] - 1 > 0) ? mp.gdot[k] * ipow(fabs(r[k]), mp.nexp[k] - 1)
                                             : mp.gdot[k];
      const double gr = g * r[k];
      const double w = (double)mp.nexp[k] * g / tau[k];
#pragma unroll
      for (int i = 0; i < 5; ++i) {
        res[i] += m[k][i] * gr;
#pragma unroll
        for (int j = 0; j < 5; ++j) J[i][j] -= m[k][i] * m[k][j] * w;
      }
    }
#pragma unroll
    for (int c = 0; c < 5; ++c) {
      res[c] -= edot[c];
      saved[c] = cur[c];
    }
    double delta[5];
    solve5_fullpiv(J, res, delta);
    double sum[5];
#pragma unroll
    for (int c = 0; c < 5; ++c) {
      nw[c] = cur[c] + delta[c];
      sum[c] = nw[c] + cur[c];
    }
    const double rel = 2.0 * norm5(delta) / norm5(sum);
#pragma unroll
    for (int c = 0; c < 5; ++c) cur[c] = nw[c];
    steps++;
    if (rel < eps) {
      conv = true;
      break;
    }
  }
  *flag = conv ? NR_OK : NR_CAPPED;
#pragma unroll
  for (int c = 0; c < 5; ++c) s_io[c] = nw[c];
  return steps;
}

// SolveConstrainedConstitutiveEquations (Solvers.cpp:111-222): Newton-Raphson on
//   R(s) = s - lambda + L0 (sum_s m_s gdot0 |r_s|^(n-1) r_s - edot - d~) = 0
//   J    = -I - L0 sum_s n gdot0 |r_s|^(n-1) / tau_s  m_s (x) m_s
// with the admissibility back-off (coefficient 0.2, cap max_rss_cap) and the
// relative-step test |s_new - s_old| / |(s_new + s_old)/2| < eps.
// L0 is column-major (L0[j*5+i] = L0(i,j)).
__device__ __forceinline__ int nr_constrained(const double m[kNS][5], const double tau[kNS],
                                              const MaterialParams& mp, const double edot[5],
                                              const double lam[5], const double d[5],
                                              const double* L0, double eps, double max_rss_cap,
                                              int max_iter, double s_io[5], double* rel_out,
                                              int* flag) {
  double cur[5], nw[5] = {-1.0, -3.0, -7.0, -9.0, -11.0}, saved[5];
#pragma unroll
  for (int c = 0; c < 5; ++c) {
    cur[c] = s_io[c];
    saved[c] = s_io[c];
  }
  // constant part of the residual: -(edot + d~)
  double ed[5];
#pragma unroll
  for (int c = 0; c < 5; ++c) ed[c] = edot[c] + d[c];
  double rel = 1e5;
  int remaining = max_iter, steps = 0;
  *flag = NR_OK;
  while (remaining > 0) {
    double r[kNS];
    bool admissible;
    do {
      admissible = true;
#pragma unroll
      for (int k = 0; k < kNS; ++k) {
        r[k] = dot5(m[k], cur) / tau[k];
        admissible = admissible && !(fabs(r[k]) > max_rss_cap);
      }
      if (!admissible) {
#pragma unroll
        for (int c = 0; c < 5; ++c) cur[c] = saved[c] + (cur[c] - saved[c]) * 0.2;
      }
      remaining--;
      if (remaining < 0) {
        *flag = NR_CAPPED;
        *rel_out = rel;
#pragma unroll
        for (int c = 0; c < 5; ++c) s_io[c] = cur[c];
        return steps;
      }
    } while (!admissible);
    double S[5] = {0, 0, 0, 0, 0};
    double K[5][5];
#pragma unroll
    for (int i = 0; i < 5; ++i)
#pragma unroll
      for (int j = 0; j < 5; ++j) K[i][j] = 0.0;
#pragma unroll
    for (int k = 0; k < kNS; ++k) {
      const double g = (mp.nexp[k] != 1) ? mp.gdot[k] * rpow(fabs(r[k]), mp.nexp[k] - 1)
                                          : mp.gdot[k];
      const double gr = g * r[k];
      const double w = (double)mp.nexp[k] * g / tau[k];
#pragma unroll
      for (int i = 0; i < 5; ++i) {
        S[i] += m[k][i] * gr;
        const double mw = m[k][i] * w;
#pragma unroll
        for (int j = i; j < 5; ++j) K[i][j] += mw * m[k][j];
      }
    }
#pragma unroll
    for (int i = 0; i < 5; ++i)
#pragma unroll
      for (int j = 0; j < i; ++j) K[i][j] = K[j][i];
    // J = -I - L0 K ; res = (cur - lambda) + L0 (S - edot - d~)
    double J[5][5], res[5], t[5];
#pragma unroll
    for (int c = 0; c < 5; ++c) t[c] = S[c] - ed[c];
#pragma unroll
    for (int i = 0; i < 5; ++i) {
      double acc = 0.0;
#pragma unroll
      for (int k = 0; k < 5; ++k) acc += L0[k * 5 + i] * t[k];
      res[i] = (cur[i] - lam[i]) + acc;
#pragma unroll
      for (int j = 0; j < 5; ++j) {
        double lk = 0.0;
#pragma unroll
        for (int k = 0; k < 5; ++k) lk += L0[k * 5 + i] * K[k][j];
        J[i][j] = ((i == j) ? -1.0 : -0.0) - lk;
      }
    }
#pragma unroll
    for (int c = 0; c < 5; ++c) saved[c] = cur[c];
    double delta[5];
    solve5_fullpiv(J, res, delta);
    double diff[5], avg[5];
#pragma unroll
    for (int c = 0; c < 5; ++c) {
      nw[c] = cur[c] + delta[c];
      diff[c] = nw[c] - saved[c];
      avg[c] = (nw[c] + saved[c]) * 0.5;
    }
    rel = norm5(diff) / norm5(avg);
#pragma unroll
    for (int c = 0; c < 5; ++c) cur[c] = nw[c];
    steps++;
    if (rel < eps) break;
  }
  if (!(rel < eps)) *flag = NR_CAPPED;
  *rel_out = rel;
#pragma unroll
  for (int c = 0; c < 5; ++c) s_io[c] = nw[c];
  return steps;
}

// ---------------------------------------------------------------- Green operator
// For a non-zero wave vector k the reference builds (MaterialGrid.cpp:583-615)
//   A_ik = sum_jl k_j k_l L_ijkl,  L = sum_ab L0_ab B_a (x) B_b
//   Gamma_ijkl = -k_j k_l [A k; k^T 0]^{-1}_ik
// then symmetrises and projects it on the basis (717).  With v_a = B_a k this
// is Ghat_ab = -v_a^T Bk v_b where A = V L0 V^T and Bk = A^-1 - u w^T/(k^T A^-1 k)
// (u = A^-1 k, w^T = k^T A^-1) is the upper-left block of the bordered inverse;
// so  dhat = -Ghat phat = V^T Bk (V phat).
// On the Nyquist planes (index N/2 or N/2+1 of an even axis, 710-713) the
// reference uses inverse(-L0) instead, and taking the real part of its c2c
// inverse transform equals applying Gbar(k) = (Op(k) + Op(-k))/2 on the
// Hermitian half spectrum; the DC term is zero (733-740).
template <typename R>
struct GreenParams {
  int nx, ny, nz;
  R inv_len[3];  // 1 / (N_i h_i)
  R L0[25];      // column-major
  R Linv[25];    // inverse(-L0), column-major
};

__host__ __device__ __forceinline__ bool nyq_override(int i, int n) {
  return ((n & 1) == 0) && (i == n / 2 || i == n / 2 + 1);
}

template <typename R>
struct cpx2 {
  R x, y;
};

// The operator of one wave vector comes in three parts, so that the x pass
// can compute it or read its expensive middle from a stored table and still
// perform the same operations on the same values (the same bits either way):
//   green_geometry  weights of Gamma and of inverse(-L0) (Nyquist planes) and
//                   the unit wave vector;
//   green_core      A = V L0 V^T and its inverse C (9 values, scaled by
//                   1/det) and 1/(k.C k) -- the kGreenStored values a table
//                   keeps per wave vector;
//   green_finish    u = C k, w = C^T k, and the application to phat.
constexpr int kGreenStored = 10;

template <typename R>
struct GreenPoint {
  R wg, wl;   // weights of Gamma and of inverse(-L0)
  R kv[3];    // unit wave vector (valid when wg != 0)
  R V[3][5];  // columns v_a = B_a k (valid when wg != 0)
};

// The four structural zeros of V: adding 0 * x to a sum leaves it unchanged
// for finite x, so skipping them gives the results of the full products.
__host__ __device__ __forceinline__ constexpr bool green_vz(int i, int a) {
  return (i == 0 && a == 2) || (i == 1 && a == 3) || (i == 2 && (a == 0 || a == 4));
}

// false for the DC term (whose operator is zero).
template <typename R>
__device__ __forceinline__ bool green_geometry(const GreenParams<R>& gp, int ix, int iy, int iz,
                                               GreenPoint<R>& q) {
  if (ix == 0 && iy == 0 && iz == 0) return false;
  // index of -k (indices are in [0, n))
  const int mx = ix ? gp.nx - ix : 0, my = iy ? gp.ny - iy : 0, mz = iz ? gp.nz - iz : 0;
  const bool ovk = nyq_override(ix, gp.nx) || nyq_override(iy, gp.ny) || nyq_override(iz, gp.nz);
  const bool ovm = nyq_override(mx, gp.nx) || nyq_override(my, gp.ny) || nyq_override(mz, gp.nz);
  q.wg = R(0.5) * R((ovk ? 0 : 1) + (ovm ? 0 : 1));
  q.wl = R(0.5) * R((ovk ? 1 : 0) + (ovm ? 1 : 0));
  if (q.wg == R(0)) return true;
  R k0 = R(ix > gp.nx / 2 ? ix - gp.nx : ix) * gp.inv_len[0];
  R k1 = R(iy > gp.ny / 2 ? iy - gp.ny : iy) * gp.inv_len[1];
  R k2 = R(iz > gp.nz / 2 ? iz - gp.nz : iz) * gp.inv_len[2];
  R il;
  const R kk = fmad(k2, k2, fmad(k1, k1, k0 * k0));
  if constexpr (sizeof(R) == 4)
    il = rsqrtf(kk);
  else
    il = R(1) / sqrt(kk);
  k0 *= il;
  k1 *= il;
  k2 *= il;
  q.kv[0] = k0;
  q.kv[1] = k1;
  q.kv[2] = k2;
  const R is2 = R(0.70710678118654752440), is6 = R(0.40824829046386301637);
  q.V[0][0] = -k0 * is2; q.V[1][0] = k1 * is2;  q.V[2][0] = R(0);
  q.V[0][1] = -k0 * is6; q.V[1][1] = -k1 * is6; q.V[2][1] = R(2) * k2 * is6;
  q.V[0][2] = R(0);      q.V[1][2] = k2 * is2;  q.V[2][2] = k1 * is2;
  q.V[0][3] = k2 * is2;  q.V[1][3] = R(0);      q.V[2][3] = k0 * is2;
  q.V[0][4] = k1 * is2;  q.V[1][4] = k0 * is2;  q.V[2][4] = R(0);
  return true;
}

// C = (V L0 V^T)^-1 and ikak = 1/(k.C k) of a point with wg != 0.
template <typename R>
__device__ __forceinline__ void green_core(const GreenParams<R>& gp, const GreenPoint<R>& q,
                                           R C[3][3], R& ikak) {
  R VL[3][5];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int b = 0; b < 5; ++b) {
      R acc = R(0);
#pragma unroll
      for (int a = 0; a < 5; ++a)
        if (!green_vz(i, a)) acc = fmad(q.V[i][a], gp.L0[b * 5 + a], acc);
      VL[i][b] = acc;
    }
  R A[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      R acc = R(0);
#pragma unroll
      for (int b = 0; b < 5; ++b)
        if (!green_vz(k, b)) acc = fmad(VL[i][b], q.V[k][b], acc);
      A[i][k] = acc;
    }
  // A^-1 by the adjugate; x*y - z*w as fmad(x, y, -(z*w))
  auto det2 = [](R x, R y, R z, R w) { return fmad(x, y, -(z * w)); };
  C[0][0] = det2(A[1][1], A[2][2], A[1][2], A[2][1]);
  C[0][1] = det2(A[0][2], A[2][1], A[0][1], A[2][2]);
  C[0][2] = det2(A[0][1], A[1][2], A[0][2], A[1][1]);
  C[1][0] = det2(A[1][2], A[2][0], A[1][0], A[2][2]);
  C[1][1] = det2(A[0][0], A[2][2], A[0][2], A[2][0]);
  C[1][2] = det2(A[0][2], A[1][0], A[0][0], A[1][2]);
  C[2][0] = det2(A[1][0], A[2][1], A[1][1], A[2][0]);
  C[2][1] = det2(A[0][1], A[2][0], A[0][0], A[2][1]);
  C[2][2] = det2(A[0][0], A[1][1], A[0][1], A[1][0]);
  const R idet = R(1) / fmad(A[0][2], C[2][0], fmad(A[0][1], C[1][0], A[0][0] * C[0][0]));
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int k = 0; k < 3; ++k) C[i][k] *= idet;
  const R* kv = q.kv;
  R u[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) u[i] = fmad(C[i][2], kv[2], fmad(C[i][1], kv[1], C[i][0] * kv[0]));
  ikak = R(1) / fmad(kv[2], u[2], fmad(kv[1], u[1], kv[0] * u[0]));
}

// dhat = wg V^T Bk (V phat) - wl inverse(-L0) phat in place on (pre, pim);
// C and ikak are used only when wg != 0.
template <typename R>
__device__ __forceinline__ void green_finish(const GreenParams<R>& gp, const GreenPoint<R>& q,
                                             const R C[3][3], R ikak, R pre[5], R pim[5]) {
  R dre[5] = {0, 0, 0, 0, 0}, dim[5] = {0, 0, 0, 0, 0};
  if (q.wg != R(0)) {
    const R* kv = q.kv;
    R u[3], w[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      u[i] = fmad(C[i][2], kv[2], fmad(C[i][1], kv[1], C[i][0] * kv[0]));
      w[i] = fmad(kv[2], C[2][i], fmad(kv[1], C[1][i], kv[0] * C[0][i]));
    }
    // q = V phat (3 complex), t = Bk q = A^-1 q - u (w.q)/(k.A^-1 k)
    R qr[3], qi[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      R ar = R(0), ai = R(0);
#pragma unroll
      for (int b = 0; b < 5; ++b) {
        if (green_vz(i, b)) continue;
        ar = fmad(q.V[i][b], pre[b], ar);
        ai = fmad(q.V[i][b], pim[b], ai);
      }
      qr[i] = ar;
      qi[i] = ai;
    }
    const R wqr = fmad(w[2], qr[2], fmad(w[1], qr[1], w[0] * qr[0])) * ikak;
    const R wqi = fmad(w[2], qi[2], fmad(w[1], qi[1], w[0] * qi[0])) * ikak;
    R tr[3], ti[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      tr[i] = fmad(-u[i], wqr, fmad(C[i][2], qr[2], fmad(C[i][1], qr[1], C[i][0] * qr[0])));
      ti[i] = fmad(-u[i], wqi, fmad(C[i][2], qi[2], fmad(C[i][1], qi[1], C[i][0] * qi[0])));
    }
#pragma unroll
    for (int a = 0; a < 5; ++a) {
      dre[a] = q.wg * fmad(q.V[2][a], tr[2], fmad(q.V[1][a], tr[1], q.V[0][a] * tr[0]));
      dim[a] = q.wg * fmad(q.V[2][a], ti[2], fmad(q.V[1][a], ti[1], q.V[0][a] * ti[0]));
    }
  }
  if (q.wl != R(0)) {
#pragma unroll
    for (int a = 0; a < 5; ++a) {
      R ar = R(0), ai = R(0);
#pragma unroll
      for (int b = 0; b < 5; ++b) {
        ar = fmad(gp.Linv[b * 5 + a], pre[b], ar);
        ai = fmad(gp.Linv[b * 5 + a], pim[b], ai);
      }
      dre[a] = fmad(-q.wl, ar, dre[a]);
      dim[a] = fmad(-q.wl, ai, dim[a]);
    }
  }
#pragma unroll
  for (int c = 0; c < 5; ++c) {
    pre[c] = dre[c];
    pim[c] = dim[c];
  }
}

// The Green constants as green_apply reads them: from a GreenParams (a kernel
// parameter: constant-bank operands), or through GreenShared, a view of a
// GreenParams in shared memory read at each use, so that a batched pass keeps
// no registers for the 50 matrix entries.
template <typename R>
__device__ __forceinline__ R green_l0(const GreenParams<R>& g, int i) {
  return g.L0[i];
}
template <typename R>
__device__ __forceinline__ R green_linv(const GreenParams<R>& g, int i) {
  return g.Linv[i];
}
template <typename R>
struct GreenShared {
  const GreenParams<R>* p;
  int nx, ny, nz;
  R inv_len[3];
  __device__ explicit GreenShared(const GreenParams<R>* q)
      : p(q), nx(q->nx), ny(q->ny), nz(q->nz), inv_len{q->inv_len[0], q->inv_len[1], q->inv_len[2]} {}
};
template <typename R>
__device__ __forceinline__ R green_l0(const GreenShared<R>& g, int i) {
  return *reinterpret_cast<const volatile R*>(&g.p->L0[i]);
}
template <typename R>
__device__ __forceinline__ R green_linv(const GreenShared<R>& g, int i) {
  return *reinterpret_cast<const volatile R*>(&g.p->Linv[i]);
}

// dh[c] (in: phat, out: dhat) for wave-vector indices (ix, iy, iz) of the full grid.
// The geometry, green_core and green_finish written out in one body (the
// compiler schedules this form better: 72 instead of 80 registers in the
// 256-point x pass, and a faster pass); every value is formed by the same
// operations as in those parts, so the stored-table path gives the same bits.
template <typename R, class G>
__device__ __forceinline__ void green_apply(const G& gp, int ix, int iy, int iz, R pre[5],
                                            R pim[5]) {
  if (ix == 0 && iy == 0 && iz == 0) {
#pragma unroll
    for (int c = 0; c < 5; ++c) pre[c] = pim[c] = R(0);
    return;
  }
  // index of -k (indices are in [0, n))
  const int mx = ix ? gp.nx - ix : 0, my = iy ? gp.ny - iy : 0, mz = iz ? gp.nz - iz : 0;
  const bool ovk = nyq_override(ix, gp.nx) || nyq_override(iy, gp.ny) || nyq_override(iz, gp.nz);
  const bool ovm = nyq_override(mx, gp.nx) || nyq_override(my, gp.ny) || nyq_override(mz, gp.nz);
  const R wg = R(0.5) * R((ovk ? 0 : 1) + (ovm ? 0 : 1));  // weight of Gamma
  const R wl = R(0.5) * R((ovk ? 1 : 0) + (ovm ? 1 : 0));  // weight of inverse(-L0)
  R dre[5] = {0, 0, 0, 0, 0}, dim[5] = {0, 0, 0, 0, 0};
  if (wg != R(0)) {
    R k0 = R(ix > gp.nx / 2 ? ix - gp.nx : ix) * gp.inv_len[0];
    R k1 = R(iy > gp.ny / 2 ? iy - gp.ny : iy) * gp.inv_len[1];
    R k2 = R(iz > gp.nz / 2 ? iz - gp.nz : iz) * gp.inv_len[2];
    R il;
    const R kk = fmad(k2, k2, fmad(k1, k1, k0 * k0));
    if constexpr (sizeof(R) == 4)
      il = rsqrtf(kk);
    else
      il = R(1) / sqrt(kk);
    k0 *= il;
    k1 *= il;
    k2 *= il;
    const R is2 = R(0.70710678118654752440), is6 = R(0.40824829046386301637);
    // columns v_a = B_a k
    R V[3][5];
    V[0][0] = -k0 * is2; V[1][0] = k1 * is2;  V[2][0] = R(0);
    V[0][1] = -k0 * is6; V[1][1] = -k1 * is6; V[2][1] = R(2) * k2 * is6;
    V[0][2] = R(0);      V[1][2] = k2 * is2;  V[2][2] = k1 * is2;
    V[0][3] = k2 * is2;  V[1][3] = R(0);      V[2][3] = k0 * is2;
    V[0][4] = k1 * is2;  V[1][4] = k0 * is2;  V[2][4] = R(0);
    // A = V L0 V^T.  The four structural zeros of V (vz) are skipped: adding
    // 0 * x to a sum leaves it unchanged for finite x, so the results are the
    // same as with the full products.
    auto vz = [](int i, int a) {
      return (i == 0 && a == 2) || (i == 1 && a == 3) || (i == 2 && (a == 0 || a == 4));
    };
    R VL[3][5];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int b = 0; b < 5; ++b) {
        R acc = R(0);
#pragma unroll
        for (int a = 0; a < 5; ++a)
          if (!vz(i, a)) acc = fmad(V[i][a], green_l0(gp, b * 5 + a), acc);
        VL[i][b] = acc;
      }
    R A[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        R acc = R(0);
#pragma unroll
        for (int b = 0; b < 5; ++b)
          if (!vz(k, b)) acc = fmad(VL[i][b], V[k][b], acc);
        A[i][k] = acc;
      }
    // A^-1 by the adjugate; x*y - z*w as fmad(x, y, -(z*w))
    auto det2 = [](R x, R y, R z, R w) { return fmad(x, y, -(z * w)); };
    R C[3][3];
    C[0][0] = det2(A[1][1], A[2][2], A[1][2], A[2][1]);
    C[0][1] = det2(A[0][2], A[2][1], A[0][1], A[2][2]);
    C[0][2] = det2(A[0][1], A[1][2], A[0][2], A[1][1]);
    C[1][0] = det2(A[1][2], A[2][0], A[1][0], A[2][2]);
    C[1][1] = det2(A[0][0], A[2][2], A[0][2], A[2][0]);
    C[1][2] = det2(A[0][2], A[1][0], A[0][0], A[1][2]);
    C[2][0] = det2(A[1][0], A[2][1], A[1][1], A[2][0]);
    C[2][1] = det2(A[0][1], A[2][0], A[0][0], A[2][1]);
    C[2][2] = det2(A[0][0], A[1][1], A[0][1], A[1][0]);
    const R idet =
        R(1) / fmad(A[0][2], C[2][0], fmad(A[0][1], C[1][0], A[0][0] * C[0][0]));
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int k = 0; k < 3; ++k) C[i][k] *= idet;
    const R kv[3] = {k0, k1, k2};
    R u[3], w[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      u[i] = fmad(C[i][2], kv[2], fmad(C[i][1], kv[1], C[i][0] * kv[0]));
      w[i] = fmad(kv[2], C[2][i], fmad(kv[1], C[1][i], kv[0] * C[0][i]));
    }
    const R ikak = R(1) / fmad(kv[2], u[2], fmad(kv[1], u[1], kv[0] * u[0]));
    // q = V phat (3 complex), t = Bk q = A^-1 q - u (w.q)/(k.A^-1 k)
    R qr[3], qi[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      R ar = R(0), ai = R(0);
#pragma unroll
      for (int b = 0; b < 5; ++b) {
        if (vz(i, b)) continue;
        ar = fmad(V[i][b], pre[b], ar);
        ai = fmad(V[i][b], pim[b], ai);
      }
      qr[i] = ar;
      qi[i] = ai;
    }
    const R wqr = fmad(w[2], qr[2], fmad(w[1], qr[1], w[0] * qr[0])) * ikak;
    const R wqi = fmad(w[2], qi[2], fmad(w[1], qi[1], w[0] * qi[0])) * ikak;
    R tr[3], ti[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      tr[i] = fmad(-u[i], wqr, fmad(C[i][2], qr[2], fmad(C[i][1], qr[1], C[i][0] * qr[0])));
      ti[i] = fmad(-u[i], wqi, fmad(C[i][2], qi[2], fmad(C[i][1], qi[1], C[i][0] * qi[0])));
    }
#pragma unroll
    for (int a = 0; a < 5; ++a) {
      dre[a] = wg * fmad(V[2][a], tr[2], fmad(V[1][a], tr[1], V[0][a] * tr[0]));
      dim[a] = wg * fmad(V[2][a], ti[2], fmad(V[1][a], ti[1], V[0][a] * ti[0]));
    }
  }
  if (wl != R(0)) {
#pragma unroll
    for (int a = 0; a < 5; ++a) {
      R ar = R(0), ai = R(0);
#pragma unroll
      for (int b = 0; b < 5; ++b) {
        ar = fmad(green_linv(gp, b * 5 + a), pre[b], ar);
        ai = fmad(green_linv(gp, b * 5 + a), pim[b], ai);
      }
      dre[a] = fmad(-wl, ar, dre[a]);
      dim[a] = fmad(-wl, ai, dim[a]);
    }
  }
#pragma unroll
  for (int c = 0; c < 5; ++c) {
    pre[c] = dre[c];
    pim[c] = dim[c];
  }
}

// The same with C and ikak read from a stored table: value j of the wave
// vector at position `at` of the half spectrum (M positions) at tab[j M + at],
// C row-major in j = 0..8, ikak in j = 9.
template <typename R>
__device__ __forceinline__ void green_apply_stored(const GreenParams<R>& gp, int ix, int iy,
                                                   int iz, const R* __restrict__ tab, long long M,
                                                   long long at, R pre[5], R pim[5]) {
  GreenPoint<R> q;
  if (!green_geometry(gp, ix, iy, iz, q)) {
#pragma unroll
    for (int c = 0; c < 5; ++c) pre[c] = pim[c] = R(0);
    return;
  }
  R C[3][3], ikak = R(0);
  if (q.wg != R(0)) {
#pragma unroll
    for (int j = 0; j < 9; ++j) C[j / 3][j % 3] = tab[j * M + at];
    ikak = tab[9 * M + at];
  }
  green_finish(gp, q, C, ikak, pre, pim);
}

}  // namespace vpfft
