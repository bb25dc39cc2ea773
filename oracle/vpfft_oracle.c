/*
 * vpfft_oracle.c -- plain-C restatement of the reference solve.  TEST ORACLE
 * ONLY (see vpfft_oracle.h).  Every routine cites the reference routine it
 * restates; expression evaluation order follows the reference's C++ operator
 * overloads so results match the reference build bit for bit.
 */
#include "vpfft_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "common/dft.h"

#define NS ORACLE_NSYS

/* ------------------------------------------------------------ basis tables */

/* EigenBasis::BuildBasisList (LinearAlgebra.h:207-247): scalar * SMatrix3x3
 * multiplies every entry by the scalar. */
void oracle_basis(double B[6][3][3]) {
  static const double raw[6][3][3] = {
      {{-1, 0, 0}, {0, 1, 0}, {0, 0, 0}}, {{-1, 0, 0}, {0, -1, 0}, {0, 0, 2}},
      {{0, 0, 0}, {0, 0, 1}, {0, 1, 0}},  {{0, 0, 1}, {0, 0, 0}, {1, 0, 0}},
      {{0, 1, 0}, {1, 0, 0}, {0, 0, 0}},  {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}}};
  const double f[6] = {1.0 / sqrt(2.0), 1.0 / sqrt(6.0), 1.0 / sqrt(2.0),
                       1.0 / sqrt(2.0), 1.0 / sqrt(2.0), 1.0 / sqrt(3.0)};
  for (int a = 0; a < 6; ++a)
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) B[a][i][j] = raw[a][i][j] * f[a];
}

/* FCC 12 {111}<110> systems in the reference's order (BurgerVectorBasis.h:16-75) */
static const double kBurgers[NS][3] = {{0, 1, 1},  {1, 0, 1},  {1, -1, 0}, {0, 1, -1},
                                       {1, 0, 1},  {1, 1, 0},  {0, 1, 1},  {1, 0, -1},
                                       {1, 1, 0},  {0, 1, -1}, {1, 0, -1}, {1, -1, 0}};
static const double kNormals[NS][3] = {{1, 1, -1}, {1, 1, -1}, {1, 1, -1}, {1, -1, -1},
                                       {1, -1, -1}, {1, -1, -1}, {1, -1, 1}, {1, -1, 1},
                                       {1, -1, 1},  {1, 1, 1},   {1, 1, 1},  {1, 1, 1}};

/* FCC_SchmidtBasis::BuildBasisList / BuildAntiBasisList (BurgerVectorBasis.h:126-151):
 * (b (x) n +/- n (x) b) / (2 sqrt 6), elementwise sum then elementwise divide. */
void oracle_schmid_crystal(double M[NS][3][3], double A[NS][3][3]) {
  const double d = 2.0 * sqrt(6.0);
  for (int s = 0; s < NS; ++s)
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        double m1 = kBurgers[s][i] * kNormals[s][j];
        double m2 = kNormals[s][i] * kBurgers[s][j];
        M[s][i][j] = (m1 + m2) / d;
        A[s][i][j] = (m1 - m2) / d;
      }
}

typedef struct {
  double B[6][3][3];
  double M[NS][3][3];
  double A[NS][3][3];
  int ready;
} tables_t;
static tables_t g_tab;

static const tables_t *tables(void) {
  if (!g_tab.ready) {
    oracle_basis(g_tab.B);
    oracle_schmid_crystal(g_tab.M, g_tab.A);
    g_tab.ready = 1;
  }
  return &g_tab;
}

/* ------------------------------------------------------------ 3x3 helpers */
/* SMatrix3x3::operator*(SMatrix3x3) (LinearAlgebra.cpp:419-439) */
static void mat3_mul(const double a[3][3], const double b[3][3], double r[3][3]) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r[i][j] = a[i][0] * b[0][j] + a[i][1] * b[1][j] + a[i][2] * b[2][j];
}
/* EigenRep(const SMatrix3x3&) (LinearAlgebra.h:307-312) with InnerProduct
 * over 3x3 (LinearAlgebra.cpp:812-820) */
static void eigenrep(const double m[3][3], double out[5]) {
  const tables_t *t = tables();
  for (int a = 0; a < 5; ++a) {
    double r = 0;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) r += m[i][j] * t->B[a][i][j];
    out[a] = r;
  }
}
/* EigenRep::ToMatrixRep (LinearAlgebra.h:352-360) */
static void to_matrix(const double v[5], double m[3][3]) {
  const tables_t *t = tables();
  memset(m, 0, sizeof(double) * 9);
  for (int a = 0; a < 5; ++a)
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) m[i][j] += t->B[a][i][j] * v[a];
}

/* MaterialGrid::UpdateSchmidtTensors (MaterialGrid.cpp:107-124) */
void oracle_schmid_sample(const double R9[9], double m[NS * 5]) {
  const tables_t *t = tables();
  double R[3][3], Rt[3][3], T1[3][3], T2[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      R[i][j] = R9[i * 3 + j];
      Rt[j][i] = R9[i * 3 + j];
    }
  for (int s = 0; s < NS; ++s) {
    mat3_mul(R, t->M[s], T1);
    mat3_mul(T1, Rt, T2);
    eigenrep(T2, m + 5 * s);
  }
}

/* ------------------------------------------------------------ 5-vectors */
static double inner5(const double *a, const double *b) {
  double r = 0;
  for (int i = 0; i < 5; ++i) r += a[i] * b[i];
  return r;
}
static double norm5(const double *a) {
  return sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2] + a[3] * a[3] + a[4] * a[4]);
}
/* operator*(SMatrix5x5, EigenRep) (LinearAlgebra.cpp:1120-1127); column-major */
static void matvec5(const double *L, const double *x, double *y) {
  double r[5] = {0, 0, 0, 0, 0};
  for (int i = 0; i < 5; ++i)
    for (int j = 0; j < 5; ++j) r[i] += L[j * 5 + i] * x[j];
  memcpy(y, r, sizeof(r));
}
static int sgn(double v) { return (0.0 < v) - (v < 0.0); } /* Solvers.h:23-25 */

/* ------------------------------------------------------------ dense solvers
 * The same textbook algorithms as the Eigen stand-in (oracle/shims/Eigen/Dense):
 * LU with row pivoting for inverses of n > 4, adjugate for 4x4, complete
 * pivoting for A x = b. */
static void inverse_lu(const double *a, double *out, int N) {
  double lu[5][5];
  int perm[5];
  for (int i = 0; i < N; ++i) {
    perm[i] = i;
    for (int j = 0; j < N; ++j) lu[i][j] = a[j * N + i];
  }
  for (int k = 0; k < N; ++k) {
    int piv = k;
    double best = fabs(lu[k][k]);
    for (int i = k + 1; i < N; ++i)
      if (fabs(lu[i][k]) > best) {
        best = fabs(lu[i][k]);
        piv = i;
      }
    if (piv != k) {
      for (int j = 0; j < N; ++j) {
        double tmp = lu[k][j];
        lu[k][j] = lu[piv][j];
        lu[piv][j] = tmp;
      }
      int tp = perm[k];
      perm[k] = perm[piv];
      perm[piv] = tp;
    }
    for (int i = k + 1; i < N; ++i) {
      lu[i][k] /= lu[k][k];
      for (int j = k + 1; j < N; ++j) lu[i][j] -= lu[i][k] * lu[k][j];
    }
  }
  for (int col = 0; col < N; ++col) {
    double y[5];
    for (int i = 0; i < N; ++i) {
      double s = (perm[i] == col) ? 1.0 : 0.0;
      for (int j = 0; j < i; ++j) s -= lu[i][j] * y[j];
      y[i] = s;
    }
    for (int i = N - 1; i >= 0; --i) {
      double s = y[i];
      for (int j = i + 1; j < N; ++j) s -= lu[i][j] * y[j];
      y[i] = s / lu[i][i];
    }
    for (int i = 0; i < N; ++i) out[col * N + i] = y[i];
  }
}
void oracle_inverse5(const double *a, double *out) { inverse_lu(a, out, 5); }

static void inverse4(const double *a, double *out) {
#define A_(i, j) a[(j) * 4 + (i)]
  double s0 = A_(0, 0) * A_(1, 1) - A_(1, 0) * A_(0, 1);
  double s1 = A_(0, 0) * A_(1, 2) - A_(1, 0) * A_(0, 2);
  double s2 = A_(0, 0) * A_(1, 3) - A_(1, 0) * A_(0, 3);
  double s3 = A_(0, 1) * A_(1, 2) - A_(1, 1) * A_(0, 2);
  double s4 = A_(0, 1) * A_(1, 3) - A_(1, 1) * A_(0, 3);
  double s5 = A_(0, 2) * A_(1, 3) - A_(1, 2) * A_(0, 3);
  double c5 = A_(2, 2) * A_(3, 3) - A_(3, 2) * A_(2, 3);
  double c4 = A_(2, 1) * A_(3, 3) - A_(3, 1) * A_(2, 3);
  double c3 = A_(2, 1) * A_(3, 2) - A_(3, 1) * A_(2, 2);
  double c2 = A_(2, 0) * A_(3, 3) - A_(3, 0) * A_(2, 3);
  double c1 = A_(2, 0) * A_(3, 2) - A_(3, 0) * A_(2, 2);
  double c0 = A_(2, 0) * A_(3, 1) - A_(3, 0) * A_(2, 1);
  double det = s0 * c5 - s1 * c4 + s2 * c3 + s3 * c2 - s4 * c1 + s5 * c0;
  double inv = 1.0 / det;
  double B[4][4];
  B[0][0] = (A_(1, 1) * c5 - A_(1, 2) * c4 + A_(1, 3) * c3) * inv;
  B[0][1] = (-A_(0, 1) * c5 + A_(0, 2) * c4 - A_(0, 3) * c3) * inv;
  B[0][2] = (A_(3, 1) * s5 - A_(3, 2) * s4 + A_(3, 3) * s3) * inv;
  B[0][3] = (-A_(2, 1) * s5 + A_(2, 2) * s4 - A_(2, 3) * s3) * inv;
  B[1][0] = (-A_(1, 0) * c5 + A_(1, 2) * c2 - A_(1, 3) * c1) * inv;
  B[1][1] = (A_(0, 0) * c5 - A_(0, 2) * c2 + A_(0, 3) * c1) * inv;
  B[1][2] = (-A_(3, 0) * s5 + A_(3, 2) * s2 - A_(3, 3) * s1) * inv;
  B[1][3] = (A_(2, 0) * s5 - A_(2, 2) * s2 + A_(2, 3) * s1) * inv;
  B[2][0] = (A_(1, 0) * c4 - A_(1, 1) * c2 + A_(1, 3) * c0) * inv;
  B[2][1] = (-A_(0, 0) * c4 + A_(0, 1) * c2 - A_(0, 3) * c0) * inv;
  B[2][2] = (A_(3, 0) * s4 - A_(3, 1) * s2 + A_(3, 3) * s0) * inv;
  B[2][3] = (-A_(2, 0) * s4 + A_(2, 1) * s2 - A_(2, 3) * s0) * inv;
  B[3][0] = (-A_(1, 0) * c3 + A_(1, 1) * c1 - A_(1, 2) * c0) * inv;
  B[3][1] = (A_(0, 0) * c3 - A_(0, 1) * c1 + A_(0, 2) * c0) * inv;
  B[3][2] = (-A_(3, 0) * s3 + A_(3, 1) * s1 - A_(3, 2) * s0) * inv;
  B[3][3] = (A_(2, 0) * s3 - A_(2, 1) * s1 + A_(2, 2) * s0) * inv;
#undef A_
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) out[j * 4 + i] = B[i][j];
}

/* LU_Solver (LinearAlgebra.cpp:1171-1187): fullPivLu().solve(b) */
static void solve_fullpiv5(const double *a, const double *b, double *x) {
  double lu[5][5];
  int rowp[5], colp[5];
  for (int i = 0; i < 5; ++i) {
    rowp[i] = i;
    colp[i] = i;
    for (int j = 0; j < 5; ++j) lu[i][j] = a[j * 5 + i];
  }
  for (int k = 0; k < 5; ++k) {
    int pi = k, pj = k;
    double best = -1;
    for (int i = k; i < 5; ++i)
      for (int j = k; j < 5; ++j)
        if (fabs(lu[i][j]) > best) {
          best = fabs(lu[i][j]);
          pi = i;
          pj = j;
        }
    if (pi != k) {
      for (int j = 0; j < 5; ++j) {
        double tmp = lu[k][j];
        lu[k][j] = lu[pi][j];
        lu[pi][j] = tmp;
      }
      int tp = rowp[k];
      rowp[k] = rowp[pi];
      rowp[pi] = tp;
    }
    if (pj != k) {
      for (int i = 0; i < 5; ++i) {
        double tmp = lu[i][k];
        lu[i][k] = lu[i][pj];
        lu[i][pj] = tmp;
      }
      int tp = colp[k];
      colp[k] = colp[pj];
      colp[pj] = tp;
    }
    if (lu[k][k] == 0.0) continue;
    for (int i = k + 1; i < 5; ++i) {
      lu[i][k] /= lu[k][k];
      for (int j = k + 1; j < 5; ++j) lu[i][j] -= lu[i][k] * lu[k][j];
    }
  }
  double y[5], z[5];
  for (int i = 0; i < 5; ++i) {
    double s = b[rowp[i]];
    for (int j = 0; j < i; ++j) s -= lu[i][j] * y[j];
    y[i] = s;
  }
  for (int i = 4; i >= 0; --i) {
    double s = y[i];
    for (int j = i + 1; j < 5; ++j) s -= lu[i][j] * z[j];
    z[i] = lu[i][i] == 0.0 ? 0.0 : s / lu[i][i];
  }
  for (int i = 0; i < 5; ++i) x[colp[i]] = z[i];
}

/* ------------------------------------------------------------ Solvers.cpp */

void oracle_sachs(const double *m, const double *crss, const double edot[5], double out[5]) {
  double maxc = 0;
  for (int s = 0; s < NS; ++s) {
    double rss = inner5(edot, m + 5 * s) / crss[s];
    double a = fabs(rss);
    maxc = (a < maxc) ? maxc : a; /* std::max(fabs(RSS), MaxCRSS) */
  }
  for (int c = 0; c < 5; ++c) out[c] = edot[c] / maxc;
}

double oracle_max_rss(const double sigma[5], const double *m, const double *crss) {
  double mx = 0;
  for (int s = 0; s < NS; ++s) {
    double rss = inner5(m + 5 * s, sigma);
    double a = fabs(rss / crss[s]);
    mx = (a < mx) ? mx : a;
  }
  return mx;
}

/* SolveConstitutiveEquations (Solvers.cpp:19-101) */
int oracle_solve_unconstrained(const double s0[5], const double *m, const double *crss,
                               const oracle_material *mat, const double edot[5], double eps,
                               double max_rss, int max_iter, double out[5]) {
  const double coeff = 0.2;
  double cur[5], nw[5], saved[5] = {0, 0, 0, 0, 0};
  memcpy(cur, s0, sizeof(cur));
  memcpy(nw, s0, sizeof(nw));
  int remaining = max_iter, steps = 0;
  while (remaining > 0) {
    double rss[NS];
    int admissible;
    do {
      admissible = 1;
      for (int s = 0; s < NS; ++s) {
        rss[s] = inner5(m + 5 * s, cur) / crss[s];
        if (fabs(rss[s]) < 1e-10) rss[s] = 0;
        if (fabs(rss[s]) > max_rss) admissible = 0;
      }
      if (!admissible)
        for (int c = 0; c < 5; ++c) cur[c] = saved[c] + (cur[c] - saved[c]) * coeff;
      remaining--;
      if (remaining < 0) {
        memcpy(out, nw, sizeof(nw));
        return steps;
      }
    } while (!admissible);
    double gd[NS];
    for (int s = 0; s < NS; ++s) {
      if (mat->rate_sensitivity[s] - 1 > 0)
        gd[s] = mat->gamma_dot_base[s] * pow(fabs(rss[s]), (double)(mat->rate_sensitivity[s] - 1));
      else
        gd[s] = mat->gamma_dot_base[s];
    }
    double res[5] = {0, 0, 0, 0, 0}, J[25];
    memset(J, 0, sizeof(J));
    for (int s = 0; s < NS; ++s) {
      const double *ms = m + 5 * s;
      for (int c = 0; c < 5; ++c) res[c] += ms[c] * gd[s] * rss[s];
      for (int i = 0; i < 5; ++i)
        for (int j = 0; j < 5; ++j)
          J[j * 5 + i] -= ms[i] * ms[j] * (double)mat->rate_sensitivity[s] * gd[s] / crss[s];
    }
    for (int c = 0; c < 5; ++c) res[c] = res[c] - edot[c];
    memcpy(saved, cur, sizeof(cur));
    double delta[5];
    solve_fullpiv5(J, res, delta);
    double sum[5];
    for (int c = 0; c < 5; ++c) nw[c] = cur[c] + delta[c];
    for (int c = 0; c < 5; ++c) sum[c] = nw[c] + cur[c];
    double rel = 2.0 * norm5(delta) / norm5(sum);
    memcpy(cur, nw, sizeof(nw));
    steps++;
    if (rel < eps) break;
  }
  memcpy(out, nw, sizeof(nw));
  return steps;
}

/* SolveConstrainedConstitutiveEquations (Solvers.cpp:111-222) */
int oracle_solve_constrained(const double s0[5], const double *m, const double *crss,
                             const oracle_material *mat, const double edot[5],
                             const double lambda[5], const double dtilde[5], const double L0[25],
                             double eps, double max_rss, int max_iter, double out[5],
                             double *nr_error) {
  const double coeff = 0.2;
  double cur[5], nw[5] = {-1, -3, -7, -9, -11}, saved[5];
  memcpy(cur, s0, sizeof(cur));
  memcpy(saved, s0, sizeof(saved));
  double rel = 1e5;
  int remaining = max_iter, steps = 0;
  while (remaining > 0) {
    double rss[NS];
    int admissible;
    do {
      admissible = 1;
      for (int s = 0; s < NS; ++s) {
        rss[s] = inner5(m + 5 * s, cur) / crss[s];
        if (fabs(rss[s]) > max_rss) admissible = 0;
      }
      if (!admissible)
        for (int c = 0; c < 5; ++c) cur[c] = saved[c] + (cur[c] - saved[c]) * coeff;
      remaining--;
      if (remaining < 0) {
        memcpy(out, cur, sizeof(cur));
        if (nr_error) *nr_error = rel; /* never written by the reference on this path */
        return -steps - 1;
      }
    } while (!admissible);
    double gd[NS];
    for (int s = 0; s < NS; ++s) {
      if (mat->rate_sensitivity[s] != 1)
        gd[s] = mat->gamma_dot_base[s] * pow(fabs(rss[s]), (double)(mat->rate_sensitivity[s] - 1));
      else
        gd[s] = mat->gamma_dot_base[s];
    }
    double S[5] = {0, 0, 0, 0, 0}, K[25];
    memset(K, 0, sizeof(K));
    for (int s = 0; s < NS; ++s) {
      const double *ms = m + 5 * s;
      for (int c = 0; c < 5; ++c) S[c] += ms[c] * gd[s] * rss[s];
      for (int i = 0; i < 5; ++i)
        for (int j = 0; j < 5; ++j)
          K[j * 5 + i] += ms[i] * ms[j] * (double)mat->rate_sensitivity[s] * gd[s] / crss[s];
    }
    /* J = -I - L0 K  (SMatrix5x5 operator*, LinearAlgebra.cpp:1106-1115) */
    double LK[25], J[25];
    for (int i = 0; i < 5; ++i)
      for (int j = 0; j < 5; ++j) {
        double a = 0;
        for (int k = 0; k < 5; ++k) a += L0[k * 5 + i] * K[j * 5 + k];
        LK[j * 5 + i] = a;
      }
    for (int i = 0; i < 5; ++i)
      for (int j = 0; j < 5; ++j) {
        double mi = -((i == j) ? 1.0 : 0.0);
        J[j * 5 + i] = mi - LK[j * 5 + i];
      }
    /* R = (s - lambda) + L0 ((S - Edot) - dtilde) */
    double t[5], Lt[5], res[5];
    for (int c = 0; c < 5; ++c) t[c] = (S[c] - edot[c]) - dtilde[c];
    matvec5(L0, t, Lt);
    for (int c = 0; c < 5; ++c) res[c] = (cur[c] - lambda[c]) + Lt[c];
    memcpy(saved, cur, sizeof(cur));
    double delta[5];
    solve_fullpiv5(J, res, delta);
    double diff[5], avg[5];
    for (int c = 0; c < 5; ++c) nw[c] = cur[c] + delta[c];
    for (int c = 0; c < 5; ++c) {
      diff[c] = nw[c] - saved[c];
      avg[c] = (nw[c] + saved[c]) * 0.5;
    }
    rel = norm5(diff) / norm5(avg);
    memcpy(cur, nw, sizeof(nw));
    steps++;
    if (rel < eps) break;
  }
  if (nr_error) *nr_error = rel;
  memcpy(out, nw, sizeof(nw));
  return steps;
}

/* ApplyConstitutiveEquations (Solvers.cpp:255-274) */
void oracle_apply_constitutive(const double s[5], const double *m, const double *crss,
                               const oracle_material *mat, double out[5]) {
  double e[5] = {0, 0, 0, 0, 0};
  for (int k = 0; k < NS; ++k) {
    double rss = inner5(m + 5 * k, s) / crss[k];
    double gd;
    if (mat->rate_sensitivity[k] > 0)
      gd = mat->gamma_dot_base[k] * pow(fabs(rss), (double)mat->rate_sensitivity[k]);
    else
      gd = mat->gamma_dot_base[k];
    double sg = (double)sgn(rss);
    for (int c = 0; c < 5; ++c) e[c] += m[5 * k + c] * gd * sg;
  }
  memcpy(out, e, sizeof(e));
}

/* CalculateShearRate (Solvers.cpp:282-302) with the local anti-Schmid
 * tensors R A_s R^T of MaterialGrid::ShearRate (MaterialGrid.cpp:1098-1119) */
static void shear_rate(const double R9[9], const double s[5], const double *m,
                       const double *crss, const oracle_material *mat, double W[3][3]) {
  const tables_t *t = tables();
  double R[3][3], Rt[3][3], T1[3][3], Aloc[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      R[i][j] = R9[i * 3 + j];
      Rt[j][i] = R9[i * 3 + j];
    }
  memset(W, 0, sizeof(double) * 9);
  for (int k = 0; k < NS; ++k) {
    mat3_mul(R, t->A[k], T1);
    mat3_mul(T1, Rt, Aloc);
    double rss = inner5(m + 5 * k, s) / crss[k];
    double gd;
    if (mat->rate_sensitivity[k] > 0)
      gd = mat->gamma_dot_base[k] * pow(fabs(rss), (double)mat->rate_sensitivity[k]);
    else
      gd = mat->gamma_dot_base[k];
    double sg = (double)sgn(rss);
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) W[i][j] += Aloc[i][j] * gd * sg;
  }
}

/* CalculateHardening (Solvers.cpp:314-373) */
static void hardening(double *acc, double dt, const double s[5], const double *m,
                      const double *crss, const oracle_material *mat, double *crss_out) {
  double gd[NS], dg = 0;
  for (int k = 0; k < NS; ++k) {
    double rss = inner5(m + 5 * k, s) / crss[k];
    if (mat->rate_sensitivity[k] > 0)
      gd[k] = mat->gamma_dot_base[k] * pow(fabs(rss), (double)mat->rate_sensitivity[k]);
    else
      gd[k] = mat->gamma_dot_base[k];
    dg += fabs(gd[k]) * dt;
  }
  for (int i = 0; i < NS; ++i) {
    double dtau = 0;
    for (int j = 0; j < NS; ++j) dtau += mat->hardening[i * NS + j] * fabs(gd[j]) * dt;
    double tiny = 1e-4 * mat->tau0[i];
    double voce = 0;
    if (fabs(mat->theta0[i]) > tiny) {
      voce = mat->theta1[i] * dg;
      if (fabs(mat->tau1[i]) > tiny) {
        double fr = fabs(mat->theta0[i] / mat->tau1[i]);
        double e_ini = exp(-*acc * fr);
        double e_del = exp(-dg * fr);
        voce = voce - (fr * mat->tau1[i] * mat->theta1[i]) / fr * e_ini * (e_del - 1.0) -
               mat->theta1[i] / fr * e_ini * (e_del * ((*acc + dg) * fr + 1.0) - (*acc * fr + 1.0));
      }
    }
    crss_out[i] = crss[i] + dtau * voce / dg;
  }
  *acc += dg;
}

/* ------------------------------------------------------------ Green operator */

/* SMatrix5x5::ToTensor4RankRep (LinearAlgebra.h:583-599), T[i*27+j*9+k*3+l] */
static void to_tensor4(const double *L, double *T) {
  const tables_t *t = tables();
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      for (int k = 0; k < 3; ++k)
        for (int l = 0; l < 3; ++l) {
          double acc = 0;
          for (int a = 0; a < 5; ++a)
            for (int b = 0; b < 5; ++b) acc += L[b * 5 + a] * t->B[a][i][j] * t->B[b][k][l];
          T[i * 27 + j * 9 + k * 3 + l] = acc;
        }
}
/* Symmetrize(Tensor4Rank) (LinearAlgebra.cpp:868-879) then SMatrix5x5(T)
 * (LinearAlgebra.h:541-554) */
static void sym_project(const double *T, double *G) {
  const tables_t *t = tables();
  double S[81];
#define T4(i, j, k, l) T[(i) * 27 + (j) * 9 + (k) * 3 + (l)]
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      for (int k = 0; k < 3; ++k)
        for (int l = 0; l < 3; ++l)
          S[i * 27 + j * 9 + k * 3 + l] =
              (T4(i, j, k, l) + T4(j, i, k, l) + T4(i, j, l, k) + T4(j, i, l, k)) / 4.0;
#undef T4
  for (int a = 0; a < 5; ++a)
    for (int b = 0; b < 5; ++b) {
      double acc = 0;
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
          for (int k = 0; k < 3; ++k)
            for (int l = 0; l < 3; ++l)
              acc += S[i * 27 + j * 9 + k * 3 + l] * t->B[a][i][j] * t->B[b][k][l];
      G[b * 5 + a] = acc;
    }
}
/* ConstructGreensOperator (MaterialGrid.cpp:583-615) given L as a tensor */
static void green_from_tensor(const double *Lt, const double W[3], double *G4) {
  double A[16];
  memset(A, 0, sizeof(A));
  for (int k = 0; k < 3; ++k)
    for (int l = 0; l < 3; ++l)
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) A[k * 4 + i] += W[l] * W[j] * Lt[i * 27 + j * 9 + k * 3 + l];
  for (int i = 0; i < 3; ++i) {
    A[i * 4 + 3] = W[i]; /* A(3,i) */
    A[3 * 4 + i] = W[i]; /* A(i,3) */
  }
  A[15] = 0;
  double Ai[16];
  inverse4(A, Ai);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      for (int k = 0; k < 3; ++k)
        for (int l = 0; l < 3; ++l)
          G4[i * 27 + j * 9 + k * 3 + l] = -W[j] * W[l] * Ai[k * 4 + i];
}
void oracle_green(const double L0[25], const double k[3], double G[25]) {
  double Lt[81], G4[81];
  to_tensor4(L0, Lt);
  green_from_tensor(Lt, k, G4);
  sym_project(G4, G);
}

/* ------------------------------------------------------------ the grid */
struct oracle_grid {
  int nx, ny, nz;
  size_t n;
  oracle_material mat;
  double *R, *sigma, *lambda, *crss, *acc, *schmid;
  oracle_cplx *P[5], *D[5];
  double h[3];
  double L0[25];
  double L0_sums[25]; /* the 25 values the reference allreduces: M(i,j)*DimXLocal, i-major */
  oracle_iter_hook hook;
  void *hook_user;
};

oracle_grid *oracle_grid_create(int nx, int ny, int nz, const oracle_material *mat) {
  oracle_grid *g = (oracle_grid *)calloc(1, sizeof(*g));
  g->nx = nx;
  g->ny = ny;
  g->nz = nz;
  g->n = (size_t)nx * ny * nz;
  g->mat = *mat;
  g->R = (double *)calloc(g->n * 9, sizeof(double));
  g->sigma = (double *)calloc(g->n * 5, sizeof(double));
  g->lambda = (double *)calloc(g->n * 5, sizeof(double));
  g->crss = (double *)calloc(g->n * NS, sizeof(double));
  g->acc = (double *)calloc(g->n, sizeof(double));
  g->schmid = (double *)calloc(g->n * NS * 5, sizeof(double));
  for (int c = 0; c < 5; ++c) {
    g->P[c] = (oracle_cplx *)calloc(g->n, sizeof(oracle_cplx));
    g->D[c] = (oracle_cplx *)calloc(g->n, sizeof(oracle_cplx));
  }
  g->h[0] = g->h[1] = g->h[2] = 1.0;
  return g;
}

void oracle_grid_free(oracle_grid *g) {
  if (!g) return;
  free(g->R);
  free(g->sigma);
  free(g->lambda);
  free(g->crss);
  free(g->acc);
  free(g->schmid);
  for (int c = 0; c < 5; ++c) {
    free(g->P[c]);
    free(g->D[c]);
  }
  free(g);
}

static void update_schmid(oracle_grid *g) {
  for (size_t v = 0; v < g->n; ++v) oracle_schmid_sample(g->R + 9 * v, g->schmid + 60 * v);
}

void oracle_grid_set(oracle_grid *g, const double *R, const double *sigma, const double *crss,
                     int per_voxel, const double h[3]) {
  memcpy(g->R, R, sizeof(double) * 9 * g->n);
  memcpy(g->sigma, sigma, sizeof(double) * 5 * g->n);
  for (size_t v = 0; v < g->n; ++v)
    for (int s = 0; s < NS; ++s) g->crss[v * NS + s] = per_voxel ? crss[v * NS + s] : crss[s];
  if (h) memcpy(g->h, h, sizeof(double) * 3);
  update_schmid(g); /* SendDataAndInitialize, MaterialGrid.cpp:455 */
}

void oracle_grid_set_iter_hook(oracle_grid *g, oracle_iter_hook h, void *user) {
  g->hook = h;
  g->hook_user = user;
}

static void set_polarization(oracle_grid *g, size_t v, const double *s) {
  for (int c = 0; c < 5; ++c) {
    g->P[c][v].re = s[c];
    g->P[c][v].im = 0;
  }
}

/* InitializeComputation (MaterialGrid.cpp:153-210); returns -1 when a voxel's
 * MaxRSS < 1e-10 (the reference exits there). */
static int initialize_computation(oracle_grid *g, const double edot[5]) {
  int min_n = g->mat.rate_sensitivity[0];
  for (int s = 1; s < NS; ++s)
    if (g->mat.rate_sensitivity[s] < min_n) min_n = g->mat.rate_sensitivity[s];
  double imposed = 2.0 * pow(inner5(edot, edot) / g->mat.gamma_dot_base[0],
                             (double)(1. / (float)min_n));
  imposed = (2.0 < imposed) ? imposed : 2.0; /* std::max(2.0, x) */
  for (size_t v = 0; v < g->n; ++v) {
    const double *m = g->schmid + 60 * v;
    const double *cr = g->crss + NS * v;
    double guess[5];
    oracle_sachs(m, cr, edot, guess);
    double mx = oracle_max_rss(guess, m, cr);
    if (mx > 1.1)
      for (int c = 0; c < 5; ++c) guess[c] /= mx;
    if (mx < 1e-10) return -1;
    oracle_solve_unconstrained(guess, m, cr, &g->mat, edot, 5e-4, imposed, 1000,
                               g->sigma + 5 * v);
    memcpy(g->lambda + 5 * v, g->sigma + 5 * v, sizeof(double) * 5);
    set_polarization(g, v, g->sigma + 5 * v);
  }
  return 0;
}

/* BuildLinearRefMediumStiffness (MaterialGrid.cpp:219-282) */
static void build_ref_medium(oracle_grid *g, double *M, double *sums) {
  memset(M, 0, sizeof(double) * 25);
  for (size_t v = 0; v < g->n; ++v) {
    const double *m = g->schmid + 60 * v;
    const double *cr = g->crss + NS * v;
    const double *s = g->sigma + 5 * v;
    double ML[25];
    memset(ML, 0, sizeof(ML));
    for (int k = 0; k < NS; ++k) {
      double rss = inner5(m + 5 * k, s) / cr[k];
      double gd;
      if (g->mat.rate_sensitivity[k] - 1 > 0)
        gd = g->mat.gamma_dot_base[k] * pow(fabs(rss), (double)(g->mat.rate_sensitivity[k] - 1));
      else
        gd = g->mat.gamma_dot_base[k];
      for (int i = 0; i < 5; ++i)
        for (int j = 0; j < 5; ++j) ML[j * 5 + i] += m[5 * k + i] * m[5 * k + j] * gd / cr[k];
    }
    double Mi[25];
    oracle_inverse5(ML, Mi);
    /* MovingAverage (LinearAlgebra.cpp:981-988) */
    for (int i = 0; i < 5; ++i)
      for (int j = 0; j < 5; ++j)
        M[j * 5 + i] += (Mi[j * 5 + i] - M[j * 5 + i]) / (double)(v + 1);
  }
  for (int i = 0; i < 5; ++i)
    for (int j = 0; j < 5; ++j) {
      double tmp = M[j * 5 + i] * (double)g->nx; /* * DimXLocal, one rank */
      sums[i * 5 + j] = tmp;
      M[j * 5 + i] = tmp / (double)g->nx;
    }
  for (int i = 0; i < 25; ++i)
    if (fabs(M[i]) < 1e-10) M[i] = 0; /* NormalizeValues */
}

static int is_override(int idx, int n) { return (n % 2 == 0) && (idx == n / 2 || idx == n / 2 + 1); }

/* StrainRateEvolutionWithFFT (MaterialGrid.cpp:624-761) */
static void strain_rate_evolution(oracle_grid *g, const double *L0) {
  double Linv_in[25], Linv[25];
  for (int i = 0; i < 25; ++i) Linv_in[i] = -L0[i];
  oracle_inverse5(Linv_in, Linv);
  for (int c = 0; c < 5; ++c)
    oracle_dft3d_inplace(g->P[c], (size_t)g->nx, (size_t)g->ny, (size_t)g->nz, -1);
  const int cx = g->nx / 2, cy = g->ny / 2, cz = g->nz / 2;
  double Lt[81], Linv_t[81], Gover[25];
  to_tensor4(L0, Lt);
  to_tensor4(Linv, Linv_t);
  sym_project(Linv_t, Gover);
  for (int x = 0; x < g->nx; ++x)
    for (int y = 0; y < g->ny; ++y)
      for (int z = 0; z < g->nz; ++z) {
        size_t v = ((size_t)x * g->ny + y) * g->nz + z;
        if (x != 0 || y != 0 || z != 0) {
          double W[3] = {(double)x, (double)y, (double)z};
          if (x > cx) W[0] -= g->nx;
          if (y > cy) W[1] -= g->ny;
          if (z > cz) W[2] -= g->nz;
          W[0] /= (g->nx * g->h[0]);
          W[1] /= (g->ny * g->h[1]);
          W[2] /= (g->nz * g->h[2]);
          /* SVector3::Normalize with the float sqrtf of GetLength
           * (LinearAlgebra.cpp:545-560) */
          double len = (double)sqrtf((float)(W[0] * W[0] + W[1] * W[1] + W[2] * W[2]));
          W[0] /= len;
          W[1] /= len;
          W[2] /= len;
          double G5[25];
          if (is_override(x, g->nx) || is_override(y, g->ny) || is_override(z, g->nz)) {
            memcpy(G5, Gover, sizeof(G5));
          } else {
            double G4[81];
            green_from_tensor(Lt, W, G4);
            sym_project(G4, G5);
          }
          for (int i = 0; i < 5; ++i) {
            double re = 0, im = 0;
            for (int j = 0; j < 5; ++j) {
              re -= G5[j * 5 + i] * g->P[j][v].re;
              im -= G5[j * 5 + i] * g->P[j][v].im;
            }
            g->D[i][v].re = re;
            g->D[i][v].im = im;
          }
        } else {
          for (int i = 0; i < 5; ++i) {
            g->D[i][v].re = 0;
            g->D[i][v].im = 0;
          }
        }
      }
  for (int c = 0; c < 5; ++c)
    oracle_dft3d_inplace(g->D[c], (size_t)g->nx, (size_t)g->ny, (size_t)g->nz, +1);
  const double norm = 1.0 / (double)(g->nx * g->ny * g->nz);
  for (int c = 0; c < 5; ++c)
    for (size_t v = 0; v < g->n; ++v) g->D[c][v].re *= norm;
}

int oracle_grid_run_increment(oracle_grid *g, const double edot[5], int max_iter, double dt,
                              double eps, double avg_stress[5]) {
  update_schmid(g);
  if (initialize_computation(g, edot) != 0) return -1;
  double L0[25];
  build_ref_medium(g, L0, g->L0_sums);
  memcpy(g->L0, L0, sizeof(L0));
  if (g->hook) g->hook(-1, NULL, g->hook_user);
  int steps = 0;
  double errS, errE, totavg[5] = {0, 0, 0, 0, 0};
  const double nvox = (double)(g->nx * g->ny * g->nz);
  do {
    double avgS[5] = {0, 0, 0, 0, 0}, avgE[5] = {0, 0, 0, 0, 0};
    errS = 0;
    errE = 0;
    strain_rate_evolution(g, L0);
    for (size_t v = 0; v < g->n; ++v) {
      const double *m = g->schmid + 60 * v;
      const double *cr = g->crss + NS * v;
      double *s = g->sigma + 5 * v;
      double *lam = g->lambda + 5 * v;
      double d[5];
      for (int c = 0; c < 5; ++c) d[c] = g->D[c][v].re;
      double mx = oracle_max_rss(s, m, cr);
      for (int c = 0; c < 5; ++c) s[c] /= mx;
      double nr_err = 0;
      double snew[5];
      oracle_solve_constrained(s, m, cr, &g->mat, edot, lam, d, L0, 5e-4, 1e9, 100, snew, &nr_err);
      memcpy(s, snew, sizeof(snew));
      double e[5];
      oracle_apply_constitutive(s, m, cr, &g->mat, e);
      double Ld[5], p[5];
      matvec5(L0, d, Ld);
      for (int c = 0; c < 5; ++c) p[c] = s[c] - Ld[c];
      set_polarization(g, v, p);
      /* UpdateLagrangeMultiplier (MaterialGrid.cpp:1169-1184) */
      double T[5], LT[5];
      for (int c = 0; c < 5; ++c) T[c] = edot[c] + d[c] - e[c];
      matvec5(L0, T, LT);
      for (int c = 0; c < 5; ++c) lam[c] += LT[c];
      double se[5], ee[5];
      for (int c = 0; c < 5; ++c) {
        avgS[c] += s[c];
        avgE[c] += e[c];
        ee[c] = e[c] - edot[c] - d[c];
        se[c] = s[c] - lam[c];
      }
      errS += sqrt(inner5(se, se));
      errE += sqrt(inner5(ee, ee));
    }
    if (g->hook) {
      double sums[12];
      for (int c = 0; c < 5; ++c) {
        sums[2 * c] = avgS[c];
        sums[2 * c + 1] = avgE[c];
      }
      sums[10] = errS;
      sums[11] = errE;
      g->hook(steps, sums, g->hook_user);
    }
    errS = errS / nvox;
    errE = errE / nvox;
    for (int c = 0; c < 5; ++c) {
      avgS[c] /= nvox;
      avgE[c] /= nvox;
    }
    memcpy(totavg, avgS, sizeof(totavg));
    errS /= sqrt(inner5(avgS, avgS));
    errE /= sqrt(inner5(edot, edot));
    steps++;
  } while (steps < max_iter && (errS > eps || errE > eps));

  /* OrientationEvolutionWithFFT (MaterialGrid.cpp:769-876): the FFT term is
   * AntiSymmetrize() of a symmetric matrix and hence exactly zero, so only the
   * plastic spin contributes; it uses the old R and old Schmid tensors. */
  for (size_t v = 0; v < g->n; ++v) {
    double W[3][3];
    shear_rate(g->R + 9 * v, g->sigma + 5 * v, g->schmid + 60 * v, g->crss + NS * v, &g->mat, W);
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) g->R[9 * v + 3 * i + j] += (0.0 + W[i][j]) * dt;
  }
  update_schmid(g);
  /* UpdateVoxelLength (MaterialGrid.cpp:1190-1196) */
  double E[3][3];
  to_matrix(edot, E);
  g->h[0] *= (1.0 + E[0][0] * dt);
  g->h[1] *= (1.0 + E[1][1] * dt);
  g->h[2] *= (1.0 + E[2][2] * dt);
  /* UpdateHardeningCRSS (MaterialGrid.cpp:1127-1157) */
  for (size_t v = 0; v < g->n; ++v) {
    double out[NS];
    hardening(g->acc + v, dt, g->sigma + 5 * v, g->schmid + 60 * v, g->crss + NS * v, &g->mat,
              out);
    memcpy(g->crss + NS * v, out, sizeof(out));
  }
  memcpy(avg_stress, totavg, sizeof(totavg));
  return steps;
}

int oracle_grid_get(const oracle_grid *g, const char *which, double *dst) {
  size_t n = g->n;
  if (!strcmp(which, "sigma")) memcpy(dst, g->sigma, sizeof(double) * 5 * n);
  else if (!strcmp(which, "lambda")) memcpy(dst, g->lambda, sizeof(double) * 5 * n);
  else if (!strcmp(which, "R")) memcpy(dst, g->R, sizeof(double) * 9 * n);
  else if (!strcmp(which, "crss")) memcpy(dst, g->crss, sizeof(double) * NS * n);
  else if (!strcmp(which, "accshear")) memcpy(dst, g->acc, sizeof(double) * n);
  else if (!strcmp(which, "schmid")) memcpy(dst, g->schmid, sizeof(double) * 60 * n);
  else if (!strcmp(which, "L0")) memcpy(dst, g->L0, sizeof(double) * 25);
  else if (!strcmp(which, "L0_sums")) memcpy(dst, g->L0_sums, sizeof(double) * 25);
  else if (!strcmp(which, "voxlen")) memcpy(dst, g->h, sizeof(double) * 3);
  else if (!strcmp(which, "P") || !strcmp(which, "dtilde")) {
    oracle_cplx *const *src = which[0] == 'P' ? g->P : g->D;
    for (size_t v = 0; v < n; ++v)
      for (int c = 0; c < 5; ++c) dst[v * 5 + c] = src[c][v].re;
  } else
    return -1;
  return 0;
}
