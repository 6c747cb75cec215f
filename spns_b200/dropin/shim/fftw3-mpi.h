/* fftw3-mpi.h -- the FFTW names the reference driver and headers need when the
 * transforms run on the GPU through libspns: the complex and plan types that
 * src/HIT_LES.h and src/FFTW_package.h declare members with, the aligned
 * allocators src/MAIN.cpp uses for host arrays, and the threading set-up calls
 * of src/util.cpp (no-ops: no FFTW plan is ever made). */
#ifndef SPNS_SHIM_FFTW3_MPI_H
#define SPNS_SHIM_FFTW3_MPI_H

#include <stddef.h>
#include <stdlib.h>

#include "mpi.h"

typedef double fftw_complex[2];
typedef float fftwf_complex[2];
typedef struct spns_no_fftw_plan *fftw_plan;
typedef struct spns_no_fftwf_plan *fftwf_plan;

#define FFTW_MEASURE (0U)
#define FFTW_DESTROY_INPUT (1U << 0)
#define FFTW_PATIENT (1U << 5)
#define FFTW_ESTIMATE (1U << 6)
#define FFTW_MPI_TRANSPOSED_IN (1U << 29)
#define FFTW_MPI_TRANSPOSED_OUT (1U << 30)

static inline void *spns_aligned_alloc(size_t bytes) {
    void *p = NULL;
    if (posix_memalign(&p, 64, bytes ? bytes : 64) != 0) return NULL;
    return p;
}
static inline double *fftw_alloc_real(size_t n) { return (double *)spns_aligned_alloc(n * sizeof(double)); }
static inline float *fftwf_alloc_real(size_t n) { return (float *)spns_aligned_alloc(n * sizeof(float)); }
static inline fftw_complex *fftw_alloc_complex(size_t n) { return (fftw_complex *)spns_aligned_alloc(n * sizeof(fftw_complex)); }
static inline fftwf_complex *fftwf_alloc_complex(size_t n) { return (fftwf_complex *)spns_aligned_alloc(n * sizeof(fftwf_complex)); }
static inline void *fftw_malloc(size_t n) { return spns_aligned_alloc(n); }
static inline void *fftwf_malloc(size_t n) { return spns_aligned_alloc(n); }
static inline void fftw_free(void *p) { free(p); }
static inline void fftwf_free(void *p) { free(p); }
static inline int fftw_init_threads(void) { return 1; }
static inline int fftwf_init_threads(void) { return 1; }
static inline void fftw_mpi_init(void) {}
static inline void fftwf_mpi_init(void) {}
static inline void fftw_plan_with_nthreads(int n) { (void)n; }
static inline void fftwf_plan_with_nthreads(int n) { (void)n; }

#endif
