/*
 * fftw3-mpi.h -- single-process stand-in for the FFTW 3.3 / fftw3_mpi subset
 * the reference uses (MaterialGrid.h:11, 63-65, 320-330; MaterialGrid.cpp:
 * 293-297, 315, 344-376, 436, 549, 639, 746, 780, 856).  Project-written test
 * infrastructure.  Plans record (dims, buffer, sign); fftw_execute runs the
 * oracle's double-precision mixed-radix DFT in place, unnormalised, with
 * FFTW's sign convention.  Each execute is reported to an optional hook so
 * the harness can observe the reference's FFT buffers.
 */
#ifndef VPFFT_SHIM_FFTW3_MPI_H
#define VPFFT_SHIM_FFTW3_MPI_H

#include <stddef.h>
#include "mpi.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct vpfft_shim_plan_s *fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)
#define FFTW_DESTROY_INPUT (1U << 0)

void fftw_mpi_init(void);
ptrdiff_t fftw_mpi_local_size_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2, MPI_Comm comm,
                                 ptrdiff_t *local_n0, ptrdiff_t *local_0_start);
fftw_complex *fftw_alloc_complex(size_t n);
void *fftw_malloc(size_t n);
void fftw_free(void *p);
fftw_plan fftw_mpi_plan_dft_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2, fftw_complex *in,
                               fftw_complex *out, MPI_Comm comm, int sign, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
void fftw_cleanup(void);

#ifdef __cplusplus
}
#endif

#endif
