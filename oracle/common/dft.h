/*
 * dft.h -- double-precision mixed-radix complex DFT used ONLY by the test
 * oracle (the FFTW stand-in that the reference is compiled against, and the
 * plain-C restatement of the solve).  It is test infrastructure: the product
 * library never links it.
 *
 * Conventions follow FFTW 3.3 (the library the reference links,
 * Makefile.make:70): unnormalised transforms,
 *   sign = -1 (FFTW_FORWARD):  X[k] = sum_j x[j] exp(-2 pi i j k / n)
 *   sign = +1 (FFTW_BACKWARD): X[k] = sum_j x[j] exp(+2 pi i j k / n)
 * Multi-dimensional transforms use C (row-major) order with the last index
 * fastest, as fftw_mpi_plan_dft_3d does (MaterialGrid.cpp:356-375).
 *
 * Algorithm: recursive decimation-in-time Cooley-Tukey over the prime-power
 * factorisation n = p1*p2*...; each combine step is a direct p-point DFT
 * (radix 2,3,4,5 and a generic O(p^2) fallback for other primes), with
 * twiddles taken from a table computed in long double.
 */
#ifndef VPFFT_ORACLE_DFT_H
#define VPFFT_ORACLE_DFT_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { double re, im; } oracle_cplx;

typedef struct oracle_dft1d oracle_dft1d;

/* Plan a length-n 1D transform with the given sign (-1 or +1). */
oracle_dft1d *oracle_dft1d_plan(size_t n, int sign);
void oracle_dft1d_free(oracle_dft1d *p);
/* out[k] = DFT(in)[k]; in has element stride `is`, out stride `os`. in != out. */
void oracle_dft1d_exec(const oracle_dft1d *p, const oracle_cplx *in, size_t is,
                       oracle_cplx *out, size_t os);

/* In-place 3D transform of an n0 x n1 x n2 array (last index fastest). */
void oracle_dft3d_inplace(oracle_cplx *data, size_t n0, size_t n1, size_t n2, int sign);

#ifdef __cplusplus
}
#endif

#endif
