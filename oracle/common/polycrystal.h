/*
 * polycrystal.h -- the synthetic microstructure of the benchmark workloads,
 * generated on the oracle side so that the reference build can make its own
 * inputs (the product's generator is vpfft_fixture_polycrystal in the CUDA
 * library; the reference arm of the benchmark must not load that library).
 * TEST-ORACLE INFRASTRUCTURE: used by the reference harness and the port CLI,
 * never by the product.
 *
 * Recipe (the same one vpfft_fixture_polycrystal documents; a CPU test checks
 * the two bit for bit):
 *   pseudo-random numbers  SplitMix64 (Steele, Lea & Flood, OOPSLA 2014),
 *                          u in [0,1) = top 53 bits * 2^-53;
 *   per grain, in order    seed point (u*Nx, u*Ny, u*Nz), then Shoemake's
 *                          uniform unit quaternion from (u1, u2, u3);
 *   voxel (x, y, z)        belongs to the seed at the smallest periodic
 *                          (minimum-image) squared distance, ties to the lower
 *                          seed index; its orientation is the grain's active
 *                          rotation matrix, row-major.
 * The search here is a brute-force scan over a seed list sorted into a
 * periodic bucket grid, visited in rings until no closer seed can exist.
 */
#ifndef VPFFT_ORACLE_POLYCRYSTAL_H
#define VPFFT_ORACLE_POLYCRYSTAL_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* R_out: nx*ny*nz*9 doubles (voxel index x*ny*nz + y*nz + z); grain_out may
 * be NULL.  threads <= 1 runs on the calling thread.  Returns 0 on success. */
int oracle_polycrystal(int nx, int ny, int nz, int grains, uint64_t seed, int threads,
                       double *R_out, int32_t *grain_out);

#ifdef __cplusplus
}
#endif

#endif
