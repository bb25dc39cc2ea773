/*
 * shim_hooks.h -- observation hooks of the MPI/FFTW stand-ins, used by the
 * oracle harness (ref_harness.cpp) to read the reference's reductions and
 * FFT buffers without modifying the reference's sources.  Test-only.
 */
#ifndef VPFFT_SHIM_HOOKS_H
#define VPFFT_SHIM_HOOKS_H

#ifdef __cplusplus
extern "C" {
#endif

/* Called before every fftw_execute with the plan's sign and its buffer. */
typedef void (*vpfft_shim_exec_hook)(int sign, double (*data)[2], long n_total, void *user);
void vpfft_shim_set_exec_hook(vpfft_shim_exec_hook h, void *user);

/* Called after every MPI_Allreduce on doubles with the reduced values. */
typedef void (*vpfft_shim_allreduce_hook)(const double *values, int count, void *user);
void vpfft_shim_set_allreduce_hook(vpfft_shim_allreduce_hook h, void *user);

long vpfft_shim_exec_count(void);
long vpfft_shim_allreduce_count(void);

#ifdef __cplusplus
}
#endif

#endif
