/*
 * shim_hooks.h -- observation hooks of the MPI/FFTW stand-ins, used by the
 * oracle harness (ref_harness.cpp) to read the reference's reductions and
 * FFT buffers without modifying the reference's sources.  Test-only.
 */
#ifndef VPFFT_SHIM_HOOKS_H
#define VPFFT_SHIM_HOOKS_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Called before every fftw_execute with the plan's sign and its buffer. */
typedef void (*vpfft_shim_exec_hook)(int sign, double (*data)[2], long n_total, void *user);
void vpfft_shim_set_exec_hook(vpfft_shim_exec_hook h, void *user);

/* Called after every MPI_Allreduce on doubles with the reduced values. */
typedef void (*vpfft_shim_allreduce_hook)(const double *values, int count, void *user);
void vpfft_shim_set_allreduce_hook(vpfft_shim_allreduce_hook h, void *user);

/* Called after every MPI_Barrier. */
typedef void (*vpfft_shim_barrier_hook)(void *user);
void vpfft_shim_set_barrier_hook(vpfft_shim_barrier_hook h, void *user);

/* Seconds spent inside fftw_execute by this rank so far. */
double vpfft_shim_fft_seconds(void);

/* Run the reference as `ranks` processes (call before MPI_Init, which forks
 * them): each rank's FFTW buffers come from its share of a shared arena
 * (arena_bytes_per_rank), point-to-point messages from a shared mailbox of
 * mailbox_bytes.  Returns 0 on success. */
int vpfft_shim_configure(int ranks, size_t arena_bytes_per_rank, size_t mailbox_bytes);

long vpfft_shim_exec_count(void);
long vpfft_shim_allreduce_count(void);

#ifdef __cplusplus
}
#endif

#endif
