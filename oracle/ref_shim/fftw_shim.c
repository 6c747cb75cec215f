/* fftw_shim.c -- FFTW 3 stand-in for the CPU build of the reference solver
 * (declarations and conventions in fftw3-mpi.h).  TEST INFRASTRUCTURE ONLY.
 *
 * Every plan remembers its sizes, arrays and kind; execution converts between
 * FFTW's layouts and the oracle's numpy-rfftn layout ([n0][n1][n2] real,
 * [n0][n1][n2/2+1] complex, unnormalised c2r) and runs orc_rfft3d /
 * orc_irfft3d. */
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "fftw3-mpi.h"
#include "../spns_oracle.h"

enum { KIND_MPI_R2C, KIND_MPI_C2R, KIND_R2C };

struct spns_ref_fftw_plan {
    int kind;
    ptrdiff_t n0, n1, n2;
    int transposed;      /* complex side is [n1][n0][n2/2+1] */
    double *real;        /* arrays given at planning (fftw_execute) */
    fftw_complex *cplx;
};

void *fftw_malloc(size_t n) {
    void *p = NULL;
    if (posix_memalign(&p, 64, n ? n : 64) != 0) return NULL;
    return p;
}
void fftw_free(void *p) { free(p); }
double *fftw_alloc_real(size_t n) { return (double *)fftw_malloc(n * sizeof(double)); }
fftw_complex *fftw_alloc_complex(size_t n) { return (fftw_complex *)fftw_malloc(n * sizeof(fftw_complex)); }
float *fftwf_alloc_real(size_t n) { return (float *)fftw_malloc(n * sizeof(float)); }
void fftwf_free(void *p) { free(p); }
int fftw_init_threads(void) { return 1; }
/* The reference's OMP_Threads parameter bounds the threads of the transforms, as
 * it bounds FFTW's. */
void fftw_plan_with_nthreads(int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
}
void fftw_mpi_init(void) {}

/* One process holds every plane: local_n0 = n0 (real x planes), local_n1 = n1
 * (transposed complex ky rows); the count is the complex elements to allocate. */
ptrdiff_t fftw_mpi_local_size_3d_transposed(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2, MPI_Comm comm, ptrdiff_t *local_n0,
                                            ptrdiff_t *local_0_start, ptrdiff_t *local_n1, ptrdiff_t *local_1_start) {
    (void)comm;
    *local_n0 = n0; *local_0_start = 0;
    *local_n1 = n1; *local_1_start = 0;
    return n0 * n1 * n2;
}

static fftw_plan make_plan(int kind, ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2, int transposed, double *real, fftw_complex *cplx) {
    fftw_plan p = (fftw_plan)calloc(1, sizeof(*p));
    p->kind = kind; p->n0 = n0; p->n1 = n1; p->n2 = n2; p->transposed = transposed;
    p->real = real; p->cplx = cplx;
    return p;
}
fftw_plan fftw_mpi_plan_dft_r2c_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2, double *in, fftw_complex *out, MPI_Comm comm,
                                   unsigned flags) {
    (void)comm;
    return make_plan(KIND_MPI_R2C, n0, n1, n2, (flags & FFTW_MPI_TRANSPOSED_OUT) != 0, in, out);
}
fftw_plan fftw_mpi_plan_dft_c2r_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2, fftw_complex *in, double *out, MPI_Comm comm,
                                   unsigned flags) {
    (void)comm;
    return make_plan(KIND_MPI_C2R, n0, n1, n2, (flags & FFTW_MPI_TRANSPOSED_IN) != 0, out, in);
}
fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double *in, fftw_complex *out, unsigned flags) {
    (void)flags;
    return make_plan(KIND_R2C, n0, n1, n2, 0, in, out);
}
void fftw_destroy_plan(fftw_plan p) { free(p); }

/* [n0][n1][h] <-> [n1][n0][h] complex */
static void swap01(const double *src, double *dst, ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t h) {
#pragma omp parallel for
    for (ptrdiff_t i = 0; i < n0; i++)
        for (ptrdiff_t j = 0; j < n1; j++) memcpy(dst + 2 * (j * n0 + i) * h, src + 2 * (i * n1 + j) * h, sizeof(double) * 2 * h);
}

static void r2c(const fftw_plan p, const double *in, fftw_complex *out, int padded) {
    const ptrdiff_t n0 = p->n0, n1 = p->n1, n2 = p->n2, h = n2 / 2 + 1, pad = padded ? 2 * h : n2;
    double *real = (double *)malloc(sizeof(double) * n0 * n1 * n2);
#pragma omp parallel for
    for (ptrdiff_t ij = 0; ij < n0 * n1; ij++) memcpy(real + ij * n2, in + ij * pad, sizeof(double) * n2);
    if (p->transposed) {
        double *tmp = (double *)malloc(sizeof(double) * 2 * n0 * n1 * h);
        orc_rfft3d((int)n0, (int)n1, (int)n2, real, tmp);
        swap01(tmp, (double *)out, n0, n1, h);
        free(tmp);
    } else {
        orc_rfft3d((int)n0, (int)n1, (int)n2, real, (double *)out);
    }
    free(real);
}

void fftw_mpi_execute_dft_r2c(const fftw_plan p, double *in, fftw_complex *out) { r2c(p, in, out, 1); }

void fftw_mpi_execute_dft_c2r(const fftw_plan p, fftw_complex *in, double *out) {
    const ptrdiff_t n0 = p->n0, n1 = p->n1, n2 = p->n2, h = n2 / 2 + 1;
    const double *src = (const double *)in;
    double *tmp = NULL;
    if (p->transposed) {
        tmp = (double *)malloc(sizeof(double) * 2 * n0 * n1 * h);
        swap01(src, tmp, n1, n0, h);
        src = tmp;
    }
    double *real = (double *)malloc(sizeof(double) * n0 * n1 * n2);
    orc_irfft3d((int)n0, (int)n1, (int)n2, src, real);
#pragma omp parallel for
    for (ptrdiff_t ij = 0; ij < n0 * n1; ij++) memcpy(out + ij * 2 * h, real + ij * n2, sizeof(double) * n2);
    free(real);
    free(tmp);
}

void fftw_execute(const fftw_plan p) {
    if (p->kind == KIND_R2C) r2c(p, p->real, p->cplx, 0);
    else if (p->kind == KIND_MPI_R2C) fftw_mpi_execute_dft_r2c(p, p->real, p->cplx);
    else fftw_mpi_execute_dft_c2r(p, p->cplx, p->real);
}
