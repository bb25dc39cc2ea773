/*
 * vpfft_oracle.h -- plain-C restatement of the reference's fixed-point solve
 * (exmatex/VPFFT Src/MaterialGrid.cpp, Solvers.cpp, LinearAlgebra.*,
 * BurgerVectorBasis.h).
 *
 * TEST ORACLE ONLY.  It is the checker used by tests/, __graft_entry__.smoke()
 * and the CPU-baseline leg of bench.py; the product (vpfft_b200) never links,
 * loads or calls it.  Each function restates one reference routine and keeps
 * its floating-point operation order (no FMA contraction: build without
 * -march so the x86-64 baseline ISA applies), so that on the same inputs it
 * reproduces the reference compiled against the stand-ins in oracle/shims
 * bit for bit; the parity tests check exactly that.
 *
 * Layouts follow the reference: voxel index x*Ny*Nz + y*Nz + z
 * (MaterialGrid.h:121-124); 3x3 row-major m[3][3] (LinearAlgebra.h:114);
 * 5-vector in the deviatoric basis (LinearAlgebra.h:207-247); 5x5 matrices
 * column-major m[j*5+i] (LinearAlgebra.h:574).
 */
#ifndef VPFFT_ORACLE_H
#define VPFFT_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

#define ORACLE_NSYS 12

typedef struct {
  double gamma_dot_base[ORACLE_NSYS];
  int rate_sensitivity[ORACLE_NSYS];
  double tau0[ORACLE_NSYS], tau1[ORACLE_NSYS], theta0[ORACLE_NSYS], theta1[ORACLE_NSYS];
  double hardening[ORACLE_NSYS * ORACLE_NSYS]; /* h[s*12+t] */
} oracle_material;

/* --- building blocks (per voxel) --------------------------------------- */
/* deviatoric basis B_a, a = 0..5 (LinearAlgebra.h:207-247) */
void oracle_basis(double B[6][3][3]);
/* crystal-frame Schmid (sym) and anti-Schmid tensors (BurgerVectorBasis.h:126-151) */
void oracle_schmid_crystal(double M[ORACLE_NSYS][3][3], double A[ORACLE_NSYS][3][3]);
/* m_s = EigenRep(R M_s R^T) (MaterialGrid.cpp:107-124) */
void oracle_schmid_sample(const double R[9], double m[ORACLE_NSYS * 5]);
/* Sachs guess (Solvers.cpp:230-243) */
void oracle_sachs(const double *m, const double *crss, const double edot[5], double out[5]);
/* GetMaxRSS without the exit (MaterialGrid.h:550-566) */
double oracle_max_rss(const double sigma[5], const double *m, const double *crss);
/* SolveConstitutiveEquations (Solvers.cpp:19-101); returns NR steps taken */
int oracle_solve_unconstrained(const double s0[5], const double *m, const double *crss,
                               const oracle_material *mat, const double edot[5], double eps,
                               double max_rss, int max_iter, double out[5]);
/* SolveConstrainedConstitutiveEquations (Solvers.cpp:111-222); L0 column-major */
int oracle_solve_constrained(const double s0[5], const double *m, const double *crss,
                             const oracle_material *mat, const double edot[5],
                             const double lambda[5], const double dtilde[5], const double L0[25],
                             double eps, double max_rss, int max_iter, double out[5],
                             double *nr_error);
/* ApplyConstitutiveEquations (Solvers.cpp:255-274) */
void oracle_apply_constitutive(const double s[5], const double *m, const double *crss,
                               const oracle_material *mat, double out[5]);
/* symmetrised, projected Green operator at wave vector k (MaterialGrid.cpp:583-615,
 * 717), before the Nyquist override; G column-major */
void oracle_green(const double L0[25], const double k[3], double G[25]);
/* 5x5 inverse (the LU algorithm of the Eigen stand-in), column-major */
void oracle_inverse5(const double *a, double *out);

/* --- whole grid --------------------------------------------------------- */
typedef struct oracle_grid oracle_grid;
oracle_grid *oracle_grid_create(int nx, int ny, int nz, const oracle_material *mat);
void oracle_grid_free(oracle_grid *g);
/* R: N*9, sigma: N*5, crss: N*12 (per_voxel) or 12 */
void oracle_grid_set(oracle_grid *g, const double *R, const double *sigma, const double *crss,
                     int crss_per_voxel, const double h[3]);
/* one RunSingleStrainStep (MaterialGrid.cpp:897-1084). Returns iterations. */
int oracle_grid_run_increment(oracle_grid *g, const double edot[5], int max_iter, double dt,
                              double eps, double avg_stress[5]);
/* observation: called once after initialisation and L0 with iter = -1 and
 * sums = NULL, then after the reductions of every fixed-point iteration with
 * the 12 reduced sums in the reference's allreduce order */
typedef void (*oracle_iter_hook)(int iter, const double sums[12], void *user);
void oracle_grid_set_iter_hook(oracle_grid *g, oracle_iter_hook h, void *user);
/* field access: which = "sigma","lambda","R","crss","accshear","P","dtilde","schmid","L0","voxlen" */
int oracle_grid_get(const oracle_grid *g, const char *which, double *dst);

#ifdef __cplusplus
}
#endif

#endif
