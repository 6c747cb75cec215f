/* fftw3-mpi.h -- the FFTW 3 (and FFTW-MPI, one process) calls of the reference
 * solver (adalbal/SpNS src/FFTW_package.cpp:47-56, src/HIT_LES.cpp:557-572,
 * src/util.cpp:128-142), so that its sources compile unchanged into a CPU
 * executable under oracle/_ref/.  TEST INFRASTRUCTURE ONLY.
 *
 * The transforms are the oracle's mixed-radix FFT (orc_rfft3d / orc_irfft3d,
 * OpenMP over lines) behind FFTW's layouts and conventions: unnormalised,
 * forward sign -1; the MPI r2c real array padded to 2 (n2/2+1) in its last
 * dimension; FFTW_MPI_TRANSPOSED_OUT / _IN swap the first two dimensions of the
 * complex array ([n1][n0][n2/2+1]).  FFTW itself is not in this image; the
 * planner flags are accepted and ignored.  Double precision only (BYTES=8). */
#ifndef SPNS_REF_SHIM_FFTW3_MPI_H
#define SPNS_REF_SHIM_FFTW3_MPI_H

#include <stddef.h>
#include <stdlib.h>

#include "mpi.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct spns_ref_fftw_plan *fftw_plan;

#define FFTW_MEASURE (0U)
#define FFTW_DESTROY_INPUT (1U << 0)
#define FFTW_PATIENT (1U << 5)
#define FFTW_ESTIMATE (1U << 6)
#define FFTW_MPI_TRANSPOSED_IN (1U << 29)
#define FFTW_MPI_TRANSPOSED_OUT (1U << 30)

void *fftw_malloc(size_t n);
void fftw_free(void *p);
double *fftw_alloc_real(size_t n);
fftw_complex *fftw_alloc_complex(size_t n);
float *fftwf_alloc_real(size_t n);   /* single-precision input files (src/HIT_LES.cpp:663-676) */
void fftwf_free(void *p);
int fftw_init_threads(void);
void fftw_plan_with_nthreads(int nthreads);
void fftw_mpi_init(void);

ptrdiff_t fftw_mpi_local_size_3d_transposed(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2, MPI_Comm comm, ptrdiff_t *local_n0,
                                            ptrdiff_t *local_0_start, ptrdiff_t *local_n1, ptrdiff_t *local_1_start);
fftw_plan fftw_mpi_plan_dft_r2c_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2, double *in, fftw_complex *out, MPI_Comm comm,
                                   unsigned flags);
fftw_plan fftw_mpi_plan_dft_c2r_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2, fftw_complex *in, double *out, MPI_Comm comm,
                                   unsigned flags);
void fftw_mpi_execute_dft_r2c(const fftw_plan p, double *in, fftw_complex *out);
void fftw_mpi_execute_dft_c2r(const fftw_plan p, fftw_complex *in, double *out);
fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double *in, fftw_complex *out, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);

#ifdef __cplusplus
}
#endif

#endif
