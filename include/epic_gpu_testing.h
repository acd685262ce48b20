/*
 * epic_gpu_testing.h -- known-answer hooks of the B200 EPIC library.
 *
 * Not part of the reference's interface; they let tests run single device
 * routines on given inputs.
 */
#ifndef EPIC_GPU_TESTING_H
#define EPIC_GPU_TESTING_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Scherzinger eigen decomposition (scherzinger.f90:31-147) of n symmetric
 * matrices given as rows (A11, A12, A13, A22, A23, A33).  D: (n, 3)
 * descending; V: (n, 9), eigenvector j in V[9i + 3j .. 9i + 3j + 2].
 * exact != 0 selects the non-contracted arithmetic used for decisions. */
int epic_gpu_test_eigen(int64_t n, const double* A6, double* D, double* V, int exact, int values_only);

struct epic_ctx;
/* diverge (inversion.f90:410-455) of a given field phi ((nz+3) x ny x nx,
 * z fastest) on the context's grid; grad receives 3 fields of that shape
 * with the halo rows extrapolated like apply_laplace. */
int epic_gpu_test_diverge(struct epic_ctx* ctx, const double* phi, double* grad);

/* fftxyp2s, lapinv1 and fftxys2p (sta3dfft.f90:134-257,
 * inversion_utils.f90:567-589) of a physical field f ((nz+3) x ny x nx, z
 * fastest, rows 0 .. nz) into out (op 0; test_lapinv1.f90).  Other ops are
 * the oracle's (epic_oracle_test_spectral): the device has no standalone
 * vertical differences, they are fused into the inversion's column kernels. */
int epic_gpu_test_spectral(struct epic_ctx* ctx, int op, const double* f, double* out);

/* parcel_delete (parcel_container.f90:413-458) of n distinct parcels given
 * by their 0-based container indices (test_mpi_parcel_delete.f90). */
int epic_gpu_test_delete(struct epic_ctx* ctx, int64_t n, const int32_t* idx);

/* apply_reflective_bc (parcel_bc.f90:45-57) on every parcel. */
int epic_gpu_test_reflective_bc(struct epic_ctx* ctx);

/* Selects the horizontal FFT implementation of the context: 0 (default) the
 * 2-D plane kernel for square grids of 16, 32, 64 or 128 points, else the
 * tiled line kernel; 1 the tiled line kernel (power-of-two axes 16 .. 256);
 * 2 the batched Stockham line kernels (any even size with factors 2, 3, 5);
 * 3 the half-plane kernel (a cluster of two CTAs per plane, square 64 or 128).
 * Each falls back to the next where it does not apply; all compute
 * fftxyp2s / fftxys2p (sta3dfft.f90:134-257). */
int epic_gpu_test_set_fft_path(struct epic_ctx* ctx, int path);

/* Lane mapping of the scatter kernels: lanes take groups of 2^lg consecutive
 * parcels (lg in 0..5) for vol2grid, par2grid and the fused stage.  Any
 * setting computes the same sums; it only changes the memory access order. */
int epic_gpu_test_set_scatter_groups(struct epic_ctx* ctx, int lg_vol2grid, int lg_par2grid, int lg_stage);

/* Free the second parcel store, as when the device had no room for it: the
 * box sort then permutes slot by slot through scratch memory. */
/* Support vectors by a kernel of their own before a scatter that recomputes
 * them (1, default) or inside the scatter kernel (0); same results. */
int epic_gpu_test_set_vectors_kernel(struct epic_ctx* ctx, int on);
/* Mixed form only: the spectral work (FFTs, column transforms, spectral
 * algebra) in FP64 instead of FP32, to measure that part's share of the
 * form's error against FP64. */
int epic_gpu_test_set_spectral_fp64(struct epic_ctx* ctx, int on);
/* Stage kernel (split form) gathers from the box's records staged in shared
 * memory (1) or from global memory (0, default); same results. */
int epic_gpu_test_set_stage_window(struct epic_ctx* ctx, int on);
/* Split-form stage kernel computes the support vectors of the advanced shapes
 * for the next par2grid (1) or a separate kernel does (0, default); same
 * results.  Both non-default variants measured slower on the B200 (plain and
 * mixed, early and developed flows) and are kept for the parity tests. */
int epic_gpu_test_set_stage_vectors(struct epic_ctx* ctx, int on);
int epic_gpu_test_drop_sort_store(struct epic_ctx* ctx);

#ifdef __cplusplus
}
#endif

#endif
