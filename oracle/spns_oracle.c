/*
 * spns_oracle.c -- CPU oracle: plain-C restatement of the reference solver.
 *
 * TEST INFRASTRUCTURE ONLY (see spns_oracle.h).  Every routine cites the
 * reference function it restates (paths relative to the adalbal/SpNS tree).
 * Memory layout, masks, loop order and the advective form of the convective
 * term follow the reference so that this code is a faithful, slow checker.
 */
#define _GNU_SOURCE
#include "spns_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define PI_REF 3.141592653589793238462643 /* src/util.h:56 */

/* ===================================================================== */
/* 1-D FFT: Stockham autosort, mixed radix, exact-angle twiddle table     */
/* ===================================================================== */
typedef struct {
    int n, nf, fac[40];
    double *tw; /* tw[2m], tw[2m+1] = cos, -sin of 2*pi*m/n  (forward kernel) */
} fplan;

#define MAXPLANS 64
static fplan g_plans[MAXPLANS];
static int g_nplans = 0;

static void make_plan(fplan *p, int n) {
    p->n = n;
    p->nf = 0;
    int m = n;
    static const int pref[] = {4, 2, 3, 5};
    for (int i = 0; i < 4; i++)
        while (m % pref[i] == 0) { p->fac[p->nf++] = pref[i]; m /= pref[i]; }
    for (int f = 7; m > 1; f += 2)
        while (m % f == 0) { p->fac[p->nf++] = f; m /= f; }
    p->tw = (double *)malloc(sizeof(double) * 2 * (size_t)n);
    for (int k = 0; k < n; k++) {
        long double ang = 2.0L * 3.14159265358979323846264338327950288L * (long double)k / (long double)n;
        p->tw[2 * k] = (double)cosl(ang);
        p->tw[2 * k + 1] = (double)(-sinl(ang));
    }
}

static const fplan *get_plan(int n) {
    const fplan *res = NULL;
#pragma omp critical(orc_plan)
    {
        for (int i = 0; i < g_nplans; i++)
            if (g_plans[i].n == n) res = &g_plans[i];
        if (!res) {
            if (g_nplans >= MAXPLANS) { fprintf(stderr, "oracle: too many FFT sizes\n"); abort(); }
            make_plan(&g_plans[g_nplans], n);
            res = &g_plans[g_nplans];
            g_nplans++;
        }
    }
    return res;
}

/* x: n complex (interleaved), w: work of n complex.  sign=-1 forward, +1 backward. */
static void fft_exec(const fplan *p, double *x, double *w, int sign) {
    const int n = p->n;
    double *in = x, *out = w;
    int Ns = 1;
    double vr[64], vi[64], yr[64], yi[64];
    for (int s = 0; s < p->nf; s++) {
        const int R = p->fac[s];
        const int nR = n / R;
        const int twstep = n / (Ns * R);
        for (int j = 0; j < nR; j++) {
            const int k = j % Ns;
            for (int r = 0; r < R; r++) {
                double ar = in[2 * (j + r * nR)], ai = in[2 * (j + r * nR) + 1];
                int m = (int)(((long)r * k * twstep) % n);
                double c = p->tw[2 * m], sn = p->tw[2 * m + 1] * (sign < 0 ? 1.0 : -1.0);
                vr[r] = ar * c - ai * sn;
                vi[r] = ar * sn + ai * c;
            }
            if (R == 2) {
                yr[0] = vr[0] + vr[1]; yi[0] = vi[0] + vi[1];
                yr[1] = vr[0] - vr[1]; yi[1] = vi[0] - vi[1];
            } else if (R == 4) {
                double t0r = vr[0] + vr[2], t0i = vi[0] + vi[2];
                double t1r = vr[0] - vr[2], t1i = vi[0] - vi[2];
                double t2r = vr[1] + vr[3], t2i = vi[1] + vi[3];
                double t3r = vr[1] - vr[3], t3i = vi[1] - vi[3];
                /* multiply t3 by -i*sign... forward (sign=-1): W4 = -i */
                double ur = (sign < 0) ? t3i : -t3i;
                double ui = (sign < 0) ? -t3r : t3r;
                yr[0] = t0r + t2r; yi[0] = t0i + t2i;
                yr[2] = t0r - t2r; yi[2] = t0i - t2i;
                yr[1] = t1r + ur;  yi[1] = t1i + ui;
                yr[3] = t1r - ur;  yi[3] = t1i - ui;
            } else if (R == 3) {
                const double c3 = -0.5;
                const double s3 = (sign < 0 ? -1.0 : 1.0) * 0.86602540378443864676372317075294;
                double sr = vr[1] + vr[2], si = vi[1] + vi[2];
                double dr = vr[1] - vr[2], di = vi[1] - vi[2];
                yr[0] = vr[0] + sr; yi[0] = vi[0] + si;
                double mr = vr[0] + c3 * sr, mi = vi[0] + c3 * si;
                /* i*s3*d */
                double er = -s3 * di, ei = s3 * dr;
                yr[1] = mr + er; yi[1] = mi + ei;
                yr[2] = mr - er; yi[2] = mi - ei;
            } else {
                const int st = n / R;
                for (int q = 0; q < R; q++) {
                    double accr = 0.0, acci = 0.0;
                    for (int r = 0; r < R; r++) {
                        int m = (int)(((long)r * q % R) * st);
                        double c = p->tw[2 * m], sn = p->tw[2 * m + 1] * (sign < 0 ? 1.0 : -1.0);
                        accr += vr[r] * c - vi[r] * sn;
                        acci += vr[r] * sn + vi[r] * c;
                    }
                    yr[q] = accr; yi[q] = acci;
                }
            }
            const int base = (j / Ns) * Ns * R + k;
            for (int r = 0; r < R; r++) {
                out[2 * (base + r * Ns)] = yr[r];
                out[2 * (base + r * Ns) + 1] = yi[r];
            }
        }
        double *t = in; in = out; out = t;
        Ns *= R;
    }
    if (in != x) memcpy(x, in, sizeof(double) * 2 * (size_t)n);
}

void orc_fft1d(int n, double *data, int sign) {
    const fplan *p = get_plan(n);
    double *w = (double *)malloc(sizeof(double) * 2 * (size_t)n);
    fft_exec(p, data, w, sign);
    free(w);
}

/* real -> half complex (n/2+1 outputs) */
static void rfft_line(const fplan *p, const double *in, int istride, double *out, int ostride, double *buf, double *w) {
    const int n = p->n;
    for (int i = 0; i < n; i++) { buf[2 * i] = in[(size_t)i * istride]; buf[2 * i + 1] = 0.0; }
    fft_exec(p, buf, w, -1);
    for (int k = 0; k <= n / 2; k++) {
        out[2 * (size_t)k * ostride] = buf[2 * k];
        out[2 * (size_t)k * ostride + 1] = buf[2 * k + 1];
    }
}

/* half complex -> real, unnormalised; imaginary parts of DC and (even n)
 * Nyquist are ignored, as a c2r transform of a Hermitian signal does. */
static void irfft_line(const fplan *p, const double *in, int istride, double *out, int ostride, double *buf, double *w) {
    const int n = p->n;
    buf[0] = in[0]; buf[1] = 0.0;
    for (int k = 1; k <= (n - 1) / 2; k++) {
        double re = in[2 * (size_t)k * istride], im = in[2 * (size_t)k * istride + 1];
        buf[2 * k] = re; buf[2 * k + 1] = im;
        buf[2 * (n - k)] = re; buf[2 * (n - k) + 1] = -im;
    }
    if (n % 2 == 0) { buf[n] = in[2 * (size_t)(n / 2) * istride]; buf[n + 1] = 0.0; }
    fft_exec(p, buf, w, +1);
    for (int i = 0; i < n; i++) out[(size_t)i * ostride] = buf[2 * i];
}

/* complex line with stride (in complex units), in place */
static void cfft_line(const fplan *p, double *data, long stride, double *buf, double *w, int sign) {
    const int n = p->n;
    for (int i = 0; i < n; i++) { buf[2 * i] = data[2 * i * stride]; buf[2 * i + 1] = data[2 * i * stride + 1]; }
    fft_exec(p, buf, w, sign);
    for (int i = 0; i < n; i++) { data[2 * i * stride] = buf[2 * i]; data[2 * i * stride + 1] = buf[2 * i + 1]; }
}

/* numpy rfftn layout: in real [n0][n1][n2], out complex [n0][n1][n2/2+1] */
void orc_rfft3d(int n0, int n1, int n2, const double *in, double *out) {
    const int h = n2 / 2 + 1;
    const fplan *p0 = get_plan(n0), *p1 = get_plan(n1), *p2 = get_plan(n2);
    int mx = n0 > n1 ? n0 : n1; if (n2 > mx) mx = n2;
#pragma omp parallel
    {
        double *buf = (double *)malloc(sizeof(double) * 2 * mx), *w = (double *)malloc(sizeof(double) * 2 * mx);
#pragma omp for
        for (long ij = 0; ij < (long)n0 * n1; ij++)
            rfft_line(p2, in + ij * n2, 1, out + 2 * ij * h, 1, buf, w);
#pragma omp for
        for (long ik = 0; ik < (long)n0 * h; ik++) {
            long i = ik / h, k = ik % h;
            cfft_line(p1, out + 2 * (i * n1 * h + k), h, buf, w, -1);
        }
#pragma omp for
        for (long jk = 0; jk < (long)n1 * h; jk++)
            cfft_line(p0, out + 2 * jk, (long)n1 * h, buf, w, -1);
        free(buf); free(w);
    }
}

void orc_irfft3d(int n0, int n1, int n2, const double *in, double *out) {
    const int h = n2 / 2 + 1;
    const fplan *p0 = get_plan(n0), *p1 = get_plan(n1), *p2 = get_plan(n2);
    double *tmp = (double *)malloc(sizeof(double) * 2 * (size_t)n0 * n1 * h);
    memcpy(tmp, in, sizeof(double) * 2 * (size_t)n0 * n1 * h);
    int mx = n0 > n1 ? n0 : n1; if (n2 > mx) mx = n2;
#pragma omp parallel
    {
        double *buf = (double *)malloc(sizeof(double) * 2 * mx), *w = (double *)malloc(sizeof(double) * 2 * mx);
#pragma omp for
        for (long jk = 0; jk < (long)n1 * h; jk++)
            cfft_line(p0, tmp + 2 * jk, (long)n1 * h, buf, w, +1);
#pragma omp for
        for (long ik = 0; ik < (long)n0 * h; ik++) {
            long i = ik / h, k = ik % h;
            cfft_line(p1, tmp + 2 * (i * n1 * h + k), h, buf, w, +1);
        }
#pragma omp for
        for (long ij = 0; ij < (long)n0 * n1; ij++)
            irfft_line(p2, tmp + 2 * ij * h, 1, out + ij * n2, 1, buf, w);
        free(buf); free(w);
    }
    free(tmp);
}

/* ===================================================================== */
/* The HIT state (src/HIT_LES.h:203-245), single rank                    */
/* ===================================================================== */
typedef double cplx[2];

struct orc {
    orc_args A;
    long ActualNx, ActualNy, ActualNz, ActualMx, ActualMy, ActualMz;
    long Nx, Ny, Nz, Nx_2, Ny_2, Nz_2, Mx, My, Mz, Mx_2, Mz_2, last_rad, last_rad_max;
    long ActualNx_file, ActualNy_file, ActualNz_file, Nx_file, Ny_file, Nz_file;
    double nu, ReLambda, delta, C_Smag, C_At, Ax, Ay, Az;
    int Lx_factor, Ly_factor, Lz_factor;
    double omega_x, omega_y, omega_z;
    double time, MaxVel, At;
    double Ah, t1, kappa, k[2], phi[3], c[14], phi0, _kappa05;
    long alloc_local, local_n0, local_n1;
    double *u, *v, *w, *gradu[3], *gradv[3], *gradw[3], *convx, *convy, *convz;
    cplx *uk_aux, *vk_aux, *wk_aux, *uk_0, *vk_0, *wk_0, *uk_1, *vk_1, *wk_1;
    cplx *gradu_k[3], *gradv_k[3], *gradw_k[3], *convx_k, *convy_k, *convz_k;
    cplx *Rx0_k, *Ry0_k, *Rz0_k, *Rx1_k, *Ry1_k, *Rz1_k;
    unsigned char *dealiased, *conjugate;
    double *rad2, *local_acumField, *global_acumField, *Ek;
    double Ok_Tot, Ek_Tot, Ek_init, Ek_init_file, Enstrophy_init_file;
    double *nu_eddy, *SGS_11, *SGS_21, *SGS_22, *SGS_31, *SGS_32, *SGS_33;
    cplx *SGS_11_k, *SGS_21_k, *SGS_22_k, *SGS_31_k, *SGS_32_k, *SGS_33_k, *divSGSx_k, *divSGSy_k, *divSGSz_k;
    long iter; /* file-scope 'iter' of src/HIT_LES.cpp:3 */
    const fplan *px, *py, *pz;
    int nthreads;
};

static long fourier_freq(long a, long M) { return (a <= M / 2) ? a : (a - M); } /* src/util.h:67 */
#define LOOP_FOURIER(o) for (long b = 0; b < (o)->local_n1; b++) for (long a = 0; a < (o)->Mx; a++) for (long k3 = 0; k3 < (o)->Mz_2 + 1; k3++)
#define IND_F(o) ((b * (o)->Mx + a) * ((o)->Mz_2 + 1) + k3)
#define LOOP_REAL(o) for (long i = 0; i < (o)->local_n0; i++) for (long j = 0; j < (o)->My; j++) for (long kk = 0; kk < (o)->Mz; kk++)
#define IND_R(o) ((i * (o)->My + j) * 2 * ((o)->Mz_2 + 1) + kk)

static double *alloc_real(long n) { double *p = (double *)calloc((size_t)n, sizeof(double)); if (!p) { fprintf(stderr, "oracle: out of memory\n"); abort(); } return p; }
static cplx *alloc_complex(long n) { return (cplx *)alloc_real(2 * n); }

static void crash(const char *msg) { fprintf(stderr, "oracle crash: %s\n", msg); abort(); }

/* ------------------------------------------------------------------- */
/* FFT_package (src/FFTW_package.cpp): transposed-out r2c / transposed-in c2r */
/* ------------------------------------------------------------------- */
/* IFFTWc2r (src/FFTW_package.cpp:12-14): in C[b][a][k3] (destroyed), out R[x][y][z+pad].
 * Order: inverse along kx, inverse along ky, then c2r along kz (the c2r of the
 * k3=0 and k3=Mz/2 entries keeps only their real parts). */
static void fft_c2r(orc *o, cplx *cin, double *rout) {
    const long Mx = o->Mx, My = o->My, Mz = o->Mz, H = o->Mz_2 + 1;
    double *C = (double *)cin;
    long mx = Mx > My ? Mx : My; if (Mz > mx) mx = Mz;
#pragma omp parallel num_threads(o->nthreads)
    {
        double *buf = (double *)malloc(sizeof(double) * 2 * mx), *w = (double *)malloc(sizeof(double) * 2 * mx);
#pragma omp for
        for (long bk = 0; bk < My * H; bk++) {
            long b = bk / H, k3 = bk % H;
            cfft_line(o->px, C + 2 * (b * Mx * H + k3), H, buf, w, +1);
        }
#pragma omp for
        for (long ak = 0; ak < Mx * H; ak++) {
            long a = ak / H, k3 = ak % H;
            cfft_line(o->py, C + 2 * (a * H + k3), Mx * H, buf, w, +1);
        }
#pragma omp for
        for (long xy = 0; xy < Mx * My; xy++) {
            long x = xy / My, y = xy % My;
            irfft_line(o->pz, C + 2 * ((y * Mx + x) * H), 1, rout + (x * My + y) * 2 * H, 1, buf, w);
        }
        free(buf); free(w);
    }
}

/* FFTWr2c (src/FFTW_package.cpp:7-9): in R[x][y][z+pad], out C[b][a][k3], unnormalised. */
static void fft_r2c(orc *o, const double *rin, cplx *cout) {
    const long Mx = o->Mx, My = o->My, Mz = o->Mz, H = o->Mz_2 + 1;
    double *C = (double *)cout;
    long mx = Mx > My ? Mx : My; if (Mz > mx) mx = Mz;
#pragma omp parallel num_threads(o->nthreads)
    {
        double *buf = (double *)malloc(sizeof(double) * 2 * mx), *w = (double *)malloc(sizeof(double) * 2 * mx);
#pragma omp for
        for (long xy = 0; xy < Mx * My; xy++) {
            long x = xy / My, y = xy % My;
            rfft_line(o->pz, rin + (x * My + y) * 2 * H, 1, C + 2 * ((y * Mx + x) * H), 1, buf, w);
        }
#pragma omp for
        for (long ak = 0; ak < Mx * H; ak++) {
            long a = ak / H, k3 = ak % H;
            cfft_line(o->py, C + 2 * (a * H + k3), Mx * H, buf, w, -1);
        }
#pragma omp for
        for (long bk = 0; bk < My * H; bk++) {
            long b = bk / H, k3 = bk % H;
            cfft_line(o->px, C + 2 * (b * Mx * H + k3), H, buf, w, -1);
        }
        free(buf); free(w);
    }
}

/* Fourier_Normalization(COMPLEX*, relevant) (src/FFTW_package.cpp:33-42) */
static void fourier_normalization(orc *o, cplx *phi) {
    const double norm_Fourier = (double)(o->Mx * o->My * o->Mz);
    LOOP_FOURIER(o) {
        long ind = IND_F(o);
        if (o->dealiased[ind]) { phi[ind][0] /= norm_Fourier; phi[ind][1] /= norm_Fourier; }
    }
}

/* ------------------------------------------------------------------- */
/* Integrals (src/HIT_LES.cpp:1137-1214, 991-1003, 1254-1266, 490-495)  */
/* ------------------------------------------------------------------- */
static double kinetic_energy(const orc *o, long ind) {
    const cplx *u = o->uk_1, *v = o->vk_1, *w = o->wk_1;
    return 0.5 * (u[ind][0] * u[ind][0] + u[ind][1] * u[ind][1] + v[ind][0] * v[ind][0] + v[ind][1] * v[ind][1] +
                  w[ind][0] * w[ind][0] + w[ind][1] * w[ind][1]);
}
static double enstrophy_fn(const orc *o, long ind) { return 2 * o->rad2[ind] * kinetic_energy(o, ind); }

/* which: 0 kinetic energy, 1 enstrophy.  acum != NULL => spectrum into acum[Kmin..Kmax]. */
static double integrate_field(orc *o, int which, double *acum, int Kmin, int Kmax) {
    if (Kmin < 0) crash("Invalid Kmin<0");
    if (Kmax > o->last_rad_max) crash("Invalid Kmax>last_rad_max");
    double sum_glo;
    if (acum) {
        double *ptr_loc = o->local_acumField;
        for (int K = Kmin; K <= Kmax; K++) { ptr_loc[K] = 0.0; acum[K] = 0.0; }
        LOOP_FOURIER(o) {
            long ind = IND_F(o);
            if (o->dealiased[ind]) {
                int K = (int)round(sqrt(o->rad2[ind]));
                if (Kmin <= K && K <= Kmax) {
                    double aux = which ? enstrophy_fn(o, ind) : kinetic_energy(o, ind);
                    if (o->conjugate[ind]) ptr_loc[K] += (2 * aux); else ptr_loc[K] += aux;
                }
            }
        }
        for (int K = Kmin; K <= Kmax; K++) acum[K] = ptr_loc[K]; /* MPI_Allreduce on one rank */
        sum_glo = 0.0;
        for (int K = Kmin; K <= Kmax; K++) sum_glo += acum[K];
    } else {
        double sum_loc = 0.0;
        LOOP_FOURIER(o) {
            long ind = IND_F(o);
            if (o->dealiased[ind]) {
                int K = (int)round(sqrt(o->rad2[ind]));
                if (Kmin <= K && K <= Kmax) {
                    double aux = which ? enstrophy_fn(o, ind) : kinetic_energy(o, ind);
                    if (o->conjugate[ind]) sum_loc += (2 * aux); else sum_loc += aux;
                }
            }
        }
        sum_glo = sum_loc;
    }
    return sum_glo;
}

double orc_recalculate_energy(orc *o) { o->Ek_Tot = integrate_field(o, 0, NULL, 0, (int)o->last_rad_max); return o->Ek_Tot; }
double orc_recalculate_energy_cascade(orc *o, double *Ek_out) {
    o->Ek_Tot = integrate_field(o, 0, o->Ek, 0, (int)o->last_rad_max);
    if (Ek_out) memcpy(Ek_out, o->Ek, sizeof(double) * (size_t)(o->last_rad_max + 1));
    return o->Ek_Tot;
}
double orc_recalculate_enstrophy(orc *o) { o->Ok_Tot = integrate_field(o, 1, NULL, 1, (int)o->last_rad_max); return o->Ok_Tot; }

/* src/HIT_LES.cpp:478-489 */
double orc_recalculate_reynolds_lambda(orc *o) {
    orc_recalculate_energy(o);
    orc_recalculate_enstrophy(o);
    o->ReLambda = o->Ek_Tot / o->nu * sqrt(20.0 / 3.0 / o->Ok_Tot);
    return o->ReLambda;
}
void orc_forcing_reynolds_lambda(orc *o, double relambda) {
    orc_recalculate_energy(o);
    orc_recalculate_enstrophy(o);
    o->nu = o->Ek_Tot / relambda * sqrt(20.0 / 3.0 / o->Ok_Tot);
}

/* ------------------------------------------------------------------- */
/* Step pieces (src/HIT_LES.cpp:34-359)                                 */
/* ------------------------------------------------------------------- */
static void velocity_gradients(orc *o) { /* :34-58 */
    LOOP_FOURIER(o) {
        long ind = IND_F(o);
        double k1 = (double)fourier_freq(a, o->Mx), k2 = (double)fourier_freq(b, o->My), kz = (double)k3;
        if (o->dealiased[ind]) {
            cplx *src[3] = {o->uk_1, o->vk_1, o->wk_1};
            cplx **dst[3] = {o->gradu_k, o->gradv_k, o->gradw_k};
            double kk[3] = {k1, k2, kz};
            for (int c = 0; c < 3; c++)
                for (int d = 0; d < 3; d++) {
                    dst[c][d][ind][0] = -kk[d] * src[c][ind][1];
                    dst[c][d][ind][1] = kk[d] * src[c][ind][0];
                }
        } else {
            for (int d = 0; d < 3; d++) {
                o->gradu_k[d][ind][0] = o->gradu_k[d][ind][1] = 0.0;
                o->gradv_k[d][ind][0] = o->gradv_k[d][ind][1] = 0.0;
                o->gradw_k[d][ind][0] = o->gradw_k[d][ind][1] = 0.0;
            }
        }
    }
}

void orc_velocity_antitransform(orc *o) { /* :60-69 */
    size_t bytes = sizeof(cplx) * (size_t)o->alloc_local;
    memcpy(o->uk_aux, o->uk_1, bytes);
    memcpy(o->vk_aux, o->vk_1, bytes);
    memcpy(o->wk_aux, o->wk_1, bytes);
    fft_c2r(o, o->uk_aux, o->u);
    fft_c2r(o, o->vk_aux, o->v);
    fft_c2r(o, o->wk_aux, o->w);
}

static void convective(orc *o) { /* :74-125 */
    velocity_gradients(o);
    orc_velocity_antitransform(o);
    for (int coord = 0; coord < 3; coord++) {
        double **g = coord == 0 ? o->gradu : coord == 1 ? o->gradv : o->gradw;
        cplx **gk = coord == 0 ? o->gradu_k : coord == 1 ? o->gradv_k : o->gradw_k;
        double *conv = coord == 0 ? o->convx : coord == 1 ? o->convy : o->convz;
        cplx *conv_k = coord == 0 ? o->convx_k : coord == 1 ? o->convy_k : o->convz_k;
        for (int s = 0; s < 3; s++) fft_c2r(o, gk[s], g[s]);
        LOOP_REAL(o) {
            long ind = IND_R(o);
            conv[ind] = o->u[ind] * g[0][ind] + o->v[ind] * g[1][ind] + o->w[ind] * g[2][ind];
        }
        fft_r2c(o, conv, conv_k);
        fourier_normalization(o, conv_k);
    }
}

/* Velocity-gradient invariants of G_ij = d_j u_i (src/HIT_LES.cpp:1297-1319 with
 * the definitions of src/tensor_algebra.cpp:165-306, 356-358): Q_G, Q_S second
 * invariants 1/2 (tr(T)^2 - tr(T T)) of G and of S = (G + G^T)/2; R_G, R_S their
 * determinants; V^2 = 4 (tr(S^2 Omega^2) - 2 Q_S Q_Omega), Omega = G - S,
 * Q_Omega = Q_G - Q_S. */
static double second_invariant3(double T[3][3]) {
    double tr = T[0][0] + T[1][1] + T[2][2], tr2 = 0.0;
    for (int i = 0; i < 3; i++)
        for (int k = 0; k < 3; k++) tr2 += T[i][k] * T[k][i];
    return 0.5 * (tr * tr - tr2);
}
static double determinant3(double t[3][3]) {
    double det = 0.0;
    det += t[0][0] * t[1][1] * t[2][2];
    det += t[0][1] * t[1][2] * t[2][0];
    det += t[0][2] * t[1][0] * t[2][1];
    det -= t[0][2] * t[1][1] * t[2][0];
    det -= t[0][1] * t[1][0] * t[2][2];
    det -= t[0][0] * t[1][2] * t[2][1];
    return det;
}
static void grad_invariants(double G[3][3], double out[5]) {
    double S[3][3], O[3][3], S2[3][3], O2[3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) { S[i][j] = 0.5 * G[i][j] + 0.5 * G[j][i]; O[i][j] = G[i][j] - S[i][j]; }
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            S2[i][j] = 0.0; O2[i][j] = 0.0;
            for (int k = 0; k < 3; k++) { S2[i][j] += S[i][k] * S[k][j]; O2[i][j] += O[i][k] * O[k][j]; }
        }
    double trS2O2 = 0.0;
    for (int i = 0; i < 3; i++)
        for (int k = 0; k < 3; k++) trS2O2 += S2[i][k] * O2[k][i];
    const double QG = second_invariant3(G), QS = second_invariant3(S);
    out[0] = QG;
    out[1] = QS;
    out[2] = determinant3(G);
    out[3] = determinant3(S);
    out[4] = 4.0 * (trS2O2 - 2.0 * QS * (QG - QS));
}

void orc_invariant_spectra(orc *o, double *out) {
    velocity_gradients(o);
    cplx **gks[3] = {o->gradu_k, o->gradv_k, o->gradw_k};
    double **gs[3] = {o->gradu, o->gradv, o->gradw};
    for (int c = 0; c < 3; c++)
        for (int d = 0; d < 3; d++) fft_c2r(o, gks[c][d], gs[c][d]);
    double *inv[5];
    for (int c = 0; c < 5; c++) inv[c] = alloc_real(2 * o->alloc_local);
    LOOP_REAL(o) {
        long ind = IND_R(o);
        double G[3][3], q[5];
        for (int c = 0; c < 3; c++)
            for (int d = 0; d < 3; d++) G[c][d] = gs[c][d][ind];
        grad_invariants(G, q);
        for (int c = 0; c < 5; c++) inv[c][ind] = q[c];
    }
    cplx *fk = alloc_complex(o->alloc_local);
    const long nb = o->last_rad_max + 1;
    for (int c = 0; c < 5; c++) {
        fft_r2c(o, inv[c], fk);
        fourier_normalization(o, fk);
        double *acc = out + c * nb;
        for (long K = 0; K < nb; K++) acc[K] = 0.0;
        LOOP_FOURIER(o) {
            long ind = IND_F(o);
            if (!o->dealiased[ind]) continue;
            int K = (int)round(sqrt(o->rad2[ind]));
            if (K > o->last_rad_max) continue;
            double aux = fk[ind][0] * fk[ind][0] + fk[ind][1] * fk[ind][1];
            acc[K] += o->conjugate[ind] ? 2 * aux : aux;
        }
        free(inv[c]);
    }
    free(fk);
}

/* Eddy-viscosity statistics over the grid: mean, root mean square and maximum of
 * nu_t = (C_s Delta)^2 sqrt(2 S_ij S_ij) of the current state (the nu_t of
 * Recalculate_Eddy_Viscosity, src/HIT_LES.cpp:130-142, same expression order). */
void orc_eddy_viscosity_stats(orc *o, double *out) {
    velocity_gradients(o);
    cplx **gks[3] = {o->gradu_k, o->gradv_k, o->gradw_k};
    double **gs[3] = {o->gradu, o->gradv, o->gradw};
    for (int c = 0; c < 3; c++)
        for (int d = 0; d < 3; d++) fft_c2r(o, gks[c][d], gs[c][d]);
    const double ct = o->C_Smag * o->C_Smag * o->delta * o->delta;
    double **gu = o->gradu, **gv = o->gradv, **gw = o->gradw;
    double sum = 0.0, sq = 0.0, mx = 0.0;
    long n = 0;
    LOOP_REAL(o) {
        long ind = IND_R(o);
        double ne = 2.0 * gu[0][ind] * gu[0][ind];
        ne += 2.0 * gv[1][ind] * gv[1][ind];
        ne += 2.0 * gw[2][ind] * gw[2][ind];
        ne += (gu[1][ind] + gv[0][ind]) * (gu[1][ind] + gv[0][ind]);
        ne += (gu[2][ind] + gw[0][ind]) * (gu[2][ind] + gw[0][ind]);
        ne += (gv[2][ind] + gw[1][ind]) * (gv[2][ind] + gw[1][ind]);
        const double nt = ct * sqrt(ne);
        sum += nt; sq += nt * nt; mx = nt > mx ? nt : mx; n++;
    }
    out[0] = sum / (double)n;
    out[1] = sqrt(sq / (double)n);
    out[2] = mx;
}

static void sgs_divergence(orc *o) { /* :130-192 */
    const double ct = o->C_Smag * o->C_Smag * o->delta * o->delta;
    double **gu = o->gradu, **gv = o->gradv, **gw = o->gradw;
    LOOP_REAL(o) { /* Recalculate_Eddy_Viscosity :130-142 */
        long ind = IND_R(o);
        double ne = 2.0 * gu[0][ind] * gu[0][ind];
        ne += 2.0 * gv[1][ind] * gv[1][ind];
        ne += 2.0 * gw[2][ind] * gw[2][ind];
        ne += (gu[1][ind] + gv[0][ind]) * (gu[1][ind] + gv[0][ind]);
        ne += (gu[2][ind] + gw[0][ind]) * (gu[2][ind] + gw[0][ind]);
        ne += (gv[2][ind] + gw[1][ind]) * (gv[2][ind] + gw[1][ind]);
        o->nu_eddy[ind] = ct * sqrt(ne);
    }
    LOOP_REAL(o) { /* Recalculate_SGS_Tensor_Components :144-154 */
        long ind = IND_R(o);
        double ne = o->nu_eddy[ind];
        o->SGS_11[ind] = (-2.0) * ne * gu[0][ind];
        o->SGS_21[ind] = (-1.0) * ne * (gu[1][ind] + gv[0][ind]);
        o->SGS_22[ind] = (-2.0) * ne * gv[1][ind];
        o->SGS_31[ind] = (-1.0) * ne * (gu[2][ind] + gw[0][ind]);
        o->SGS_32[ind] = (-1.0) * ne * (gv[2][ind] + gw[1][ind]);
        o->SGS_33[ind] = (-2.0) * ne * gw[2][ind];
    }
    /* Recalculate_SGS_Tensor_Transform :156-171 */
    fft_r2c(o, o->SGS_11, o->SGS_11_k); fft_r2c(o, o->SGS_21, o->SGS_21_k); fft_r2c(o, o->SGS_22, o->SGS_22_k);
    fft_r2c(o, o->SGS_31, o->SGS_31_k); fft_r2c(o, o->SGS_32, o->SGS_32_k); fft_r2c(o, o->SGS_33, o->SGS_33_k);
    fourier_normalization(o, o->SGS_11_k); fourier_normalization(o, o->SGS_21_k); fourier_normalization(o, o->SGS_22_k);
    fourier_normalization(o, o->SGS_31_k); fourier_normalization(o, o->SGS_32_k); fourier_normalization(o, o->SGS_33_k);
    LOOP_FOURIER(o) { /* :179-191 */
        long ind = IND_F(o);
        double k1 = (double)fourier_freq(a, o->Mx), k2 = (double)fourier_freq(b, o->My), kz = (double)k3;
        if (o->dealiased[ind]) {
            o->divSGSx_k[ind][0] = -k1 * o->SGS_11_k[ind][1] - k2 * o->SGS_21_k[ind][1] - kz * o->SGS_31_k[ind][1];
            o->divSGSx_k[ind][1] = k1 * o->SGS_11_k[ind][0] + k2 * o->SGS_21_k[ind][0] + kz * o->SGS_31_k[ind][0];
            o->divSGSy_k[ind][0] = -k1 * o->SGS_21_k[ind][1] - k2 * o->SGS_22_k[ind][1] - kz * o->SGS_32_k[ind][1];
            o->divSGSy_k[ind][1] = k1 * o->SGS_21_k[ind][0] + k2 * o->SGS_22_k[ind][0] + kz * o->SGS_32_k[ind][0];
            o->divSGSz_k[ind][0] = -k1 * o->SGS_31_k[ind][1] - k2 * o->SGS_32_k[ind][1] - kz * o->SGS_33_k[ind][1];
            o->divSGSz_k[ind][1] = k1 * o->SGS_31_k[ind][0] + k2 * o->SGS_32_k[ind][0] + kz * o->SGS_33_k[ind][0];
        }
    }
}

static void r_vector(orc *o) { /* :196-280 */
    size_t bytes = sizeof(cplx) * (size_t)o->alloc_local;
    memcpy(o->Rx0_k, o->Rx1_k, bytes);
    memcpy(o->Ry0_k, o->Ry1_k, bytes);
    memcpy(o->Rz0_k, o->Rz1_k, bytes);
    convective(o);
    LOOP_FOURIER(o) {
        long ind = IND_F(o);
        if (o->dealiased[ind]) {
            double ct = o->nu * o->rad2[ind];
            int isMean = !(o->rad2[ind] > 0.0);
            for (int ic = 0; ic <= 1; ic++) {
                o->Rx1_k[ind][ic] = -(isMean ? 0.0 : o->convx_k[ind][ic]) - ct * o->uk_1[ind][ic];
                o->Ry1_k[ind][ic] = -(isMean ? 0.0 : o->convy_k[ind][ic]) - ct * o->vk_1[ind][ic];
                o->Rz1_k[ind][ic] = -(isMean ? 0.0 : o->convz_k[ind][ic]) - ct * o->wk_1[ind][ic];
            }
        }
    }
    if (o->A.isLES) {
        sgs_divergence(o);
        LOOP_FOURIER(o) {
            long ind = IND_F(o);
            if (o->dealiased[ind])
                for (int ic = 0; ic <= 1; ic++) {
                    o->Rx1_k[ind][ic] -= o->divSGSx_k[ind][ic];
                    o->Ry1_k[ind][ic] -= o->divSGSy_k[ind][ic];
                    o->Rz1_k[ind][ic] -= o->divSGSz_k[ind][ic];
                }
        }
    }
    if (o->A.isRotating) {
        LOOP_FOURIER(o) {
            long ind = IND_F(o);
            if (o->dealiased[ind])
                for (int ic = 0; ic <= 1; ic++) {
                    o->Rx1_k[ind][ic] += 2 * (o->omega_z * o->vk_1[ind][ic] - o->omega_y * o->wk_1[ind][ic]);
                    o->Ry1_k[ind][ic] += 2 * (o->omega_x * o->wk_1[ind][ic] - o->omega_z * o->uk_1[ind][ic]);
                    o->Rz1_k[ind][ic] += 2 * (o->omega_y * o->uk_1[ind][ic] - o->omega_x * o->vk_1[ind][ic]);
                }
        }
    }
    if (o->A.eps_forcing > 0.0) { /* restatement of the disabled block :243-278 with eps_in as a parameter */
        const int Kfmin = o->A.eps_kmin, Kfmax = o->A.eps_kmax;
        double Ef = integrate_field(o, 0, o->Ek, Kfmin, Kfmax);
        const double tiny = 1e-30;
        double alpha = 0.0;
        if (Ef > tiny) alpha = o->A.eps_forcing / (2.0 * Ef);
        LOOP_FOURIER(o) {
            long ind = IND_F(o);
            int K = (int)round(sqrt(o->rad2[ind]));
            if (o->dealiased[ind]) {
                if (Kfmin <= K && K <= Kfmax) {
                    for (int ic = 0; ic <= 1; ic++) {
                        o->Rx1_k[ind][ic] += alpha * o->uk_1[ind][ic];
                        o->Ry1_k[ind][ic] += alpha * o->vk_1[ind][ic];
                        o->Rz1_k[ind][ic] += alpha * o->wk_1[ind][ic];
                    }
                } else if (K == 0) {
                    for (int ic = 0; ic <= 1; ic++) o->Rx1_k[ind][ic] = o->Ry1_k[ind][ic] = o->Rz1_k[ind][ic] = 0.0;
                }
            }
        }
    }
}

static void predictor(orc *o) { /* :295-339 */
    size_t bytes = sizeof(cplx) * (size_t)o->alloc_local;
    if (o->A.isSelfAdaptive) {
        if (o->iter > 0) {
            memcpy(o->uk_aux, o->uk_0, bytes);
            memcpy(o->vk_aux, o->vk_0, bytes);
            memcpy(o->wk_aux, o->wk_0, bytes);
        } else {
            /* The reference reads here the c2r-destroyed copy of u^n left by
             * Recalculate_Velocity_Antitransform (FFTW-internal contents).  The
             * intended history (comment at :298) is u^{-1}=u^0, used here. */
            memcpy(o->uk_aux, o->uk_1, bytes);
            memcpy(o->vk_aux, o->vk_1, bytes);
            memcpy(o->wk_aux, o->wk_1, bytes);
        }
        memcpy(o->uk_0, o->uk_1, bytes);
        memcpy(o->vk_0, o->vk_1, bytes);
        memcpy(o->wk_0, o->wk_1, bytes);
        o->_kappa05 = (1.0 / (o->kappa + 0.5));
        const double kappa = o->kappa, At = o->At, k05 = o->_kappa05;
        LOOP_FOURIER(o) {
            long ind = IND_F(o);
            if (o->dealiased[ind])
                for (int ic = 0; ic <= 1; ic++) {
                    o->uk_1[ind][ic] = k05 * (2.0 * kappa * o->uk_0[ind][ic] + At * ((1.0 + kappa) * o->Rx1_k[ind][ic] - kappa * o->Rx0_k[ind][ic]) - (kappa - 0.5) * o->uk_aux[ind][ic]);
                    o->vk_1[ind][ic] = k05 * (2.0 * kappa * o->vk_0[ind][ic] + At * ((1.0 + kappa) * o->Ry1_k[ind][ic] - kappa * o->Ry0_k[ind][ic]) - (kappa - 0.5) * o->vk_aux[ind][ic]);
                    o->wk_1[ind][ic] = k05 * (2.0 * kappa * o->wk_0[ind][ic] + At * ((1.0 + kappa) * o->Rz1_k[ind][ic] - kappa * o->Rz0_k[ind][ic]) - (kappa - 0.5) * o->wk_aux[ind][ic]);
                }
        }
    } else {
        memcpy(o->uk_0, o->uk_1, bytes);
        memcpy(o->vk_0, o->vk_1, bytes);
        memcpy(o->wk_0, o->wk_1, bytes);
        const double At = o->At;
        LOOP_FOURIER(o) {
            long ind = IND_F(o);
            if (o->dealiased[ind])
                for (int ic = 0; ic <= 1; ic++) {
                    o->uk_1[ind][ic] = o->uk_0[ind][ic] + At * (1.5 * o->Rx1_k[ind][ic] - 0.5 * o->Rx0_k[ind][ic]);
                    o->vk_1[ind][ic] = o->vk_0[ind][ic] + At * (1.5 * o->Ry1_k[ind][ic] - 0.5 * o->Ry0_k[ind][ic]);
                    o->wk_1[ind][ic] = o->wk_0[ind][ic] + At * (1.5 * o->Rz1_k[ind][ic] - 0.5 * o->Rz0_k[ind][ic]);
                }
        }
    }
}

static void projection(orc *o) { /* :346-359 */
    LOOP_FOURIER(o) {
        long ind = IND_F(o);
        double k1 = (double)fourier_freq(a, o->Mx), k2 = (double)fourier_freq(b, o->My), kz = (double)k3;
        if (o->dealiased[ind])
            for (int ic = 0; ic <= 1; ic++) {
                double aux = ((o->rad2[ind] > 0) ? ((k1 * o->uk_1[ind][ic] + k2 * o->vk_1[ind][ic] + kz * o->wk_1[ind][ic]) / o->rad2[ind]) : 0.0);
                o->uk_1[ind][ic] -= aux * k1;
                o->vk_1[ind][ic] -= aux * k2;
                o->wk_1[ind][ic] -= aux * kz;
            }
    }
}

/* Self-adaptive helpers (src/HIT_LES.h:249-269) */
static double FuL(double x, double x0, double x1, double f0, double f1) { return f0 + (x - x0) * (f1 - f0) / (x1 - x0); }
static double FuQ(double x, double x0, double x1) { return (x - x0) * (x - x1); }
static double FuG(double x, double a, double b, double c, double x0, double x1, double f0, double f1) {
    return (a * x * x + b * x + c) * FuQ(x, x0, x1) + FuL(x, x0, x1, f0, f1);
}
static double Topt(orc *o, double phi0) {
    if (phi0 >= 0.0 && phi0 < o->phi[0]) return FuG(phi0, 0.0, o->c[0], o->c[1], 0.0, o->phi[0], 4.0 / 3.0, o->t1);
    if (phi0 >= o->phi[0] && phi0 <= PI_REF / 2.0) return FuG(phi0, o->c[2], o->c[3], o->c[4], o->phi[0], PI_REF / 2.0, o->t1, 1.0);
    crash("Topt fail!"); return 0;
}
static double Kopt(orc *o, double phi0) {
    if (phi0 >= 0.0 && phi0 <= o->phi[0]) return 1.0;
    if (phi0 > o->phi[0] && phi0 <= o->phi[1]) return FuG(phi0, o->c[5], o->c[6], o->c[7], o->phi[0], o->phi[1], 1.0, o->k[0]);
    if (phi0 > o->phi[1] && phi0 <= o->phi[2]) return FuG(phi0, o->c[8], o->c[9], o->c[10], o->phi[1], o->phi[2], o->k[0], o->k[1]);
    if (phi0 > o->phi[2] && phi0 <= PI_REF / 2.0) return FuG(phi0, o->c[11], o->c[12], o->c[13], o->phi[2], PI_REF / 2.0, o->k[1], 0.0);
    crash("Kopt fail!"); return 0;
}

void orc_recalculate_timestep(orc *o) { /* :365-403 */
    if (o->A.fixed_dt > 0.0) { o->At = o->A.fixed_dt; return; }
    double local_MaxVel = 0.0;
    if (o->A.isSelfAdaptive) {
        LOOP_REAL(o) {
            long ind = IND_R(o);
            local_MaxVel = fmax(local_MaxVel, (fabs(o->u[ind]) / o->Ax + fabs(o->v[ind]) / o->Ay + fabs(o->w[ind]) / o->Az));
        }
        o->MaxVel = local_MaxVel;
        o->phi0 = atan(o->MaxVel * o->Ah * o->Ah / (0.35 * o->nu * 12.0));
        o->At = Topt(o, o->phi0) / sqrt((o->MaxVel * o->MaxVel) / (0.35 * 0.35) + (144.0 * o->nu * o->nu / (o->Ah * o->Ah * o->Ah * o->Ah)));
        o->kappa = Kopt(o, o->phi0);
        o->At = o->C_At * o->At;
    } else {
        LOOP_REAL(o) {
            long ind = IND_R(o);
            local_MaxVel = fmax(local_MaxVel, fmax(fabs(o->u[ind]) / o->Ax, fmax(fabs(o->v[ind]) / o->Ay, fabs(o->w[ind]) / o->Az)));
        }
        o->MaxVel = local_MaxVel;
        double C_visc = 0.2 * fmin(o->Ax * o->Ax, fmin(o->Ay * o->Ay, o->Az * o->Az)) / o->nu;
        double C_conv = 0.35 / o->MaxVel;
        o->At = fmin(C_visc, C_conv);
        o->At = o->C_At * o->At;
    }
}

void orc_step(orc *o) { /* New_Fractional_Step_Method :9-25 (without the QA-only energy check) */
    r_vector(o);
    predictor(o);
    projection(o);
    orc_recalculate_timestep(o);
    o->time = o->time + o->At;
    o->iter++;
}

/* ------------------------------------------------------------------- */
/* Forcing and conjugate correction (src/HIT_LES.cpp:410-476)           */
/* ------------------------------------------------------------------- */
void orc_complex_conjugate_correction(orc *o) {
    const long Mx = o->Mx, My = o->My, H = o->Mz_2 + 1;
    cplx *pl[3] = {o->uk_1, o->vk_1, o->wk_1};
    cplx *copy = alloc_complex(3 * Mx * My);
    for (int c = 0; c < 3; c++)
        for (long b = 0; b < My; b++)
            for (long a = 0; a < Mx; a++) {
                copy[c * Mx * My + b * Mx + a][0] = pl[c][(b * Mx + a) * H][0];
                copy[c * Mx * My + b * Mx + a][1] = pl[c][(b * Mx + a) * H][1];
            }
    for (long b = 0; b < My; b++)
        for (long a = 0; a < Mx; a++) {
            long k1 = fourier_freq(a, Mx), k2 = fourier_freq(b, My);
            if (k1 < 0 || (k1 == 0 && k2 < 0)) {
                long k1c = -k1, k2c = -k2;
                long ind = (b * Mx + a) * H;
                long a_c = k1c, b_c = (k2c >= 0) ? k2c : (My + k2c);
                long ic0 = b_c * Mx + a_c;
                for (int c = 0; c < 3; c++) {
                    pl[c][ind][0] = copy[c * Mx * My + ic0][0];
                    pl[c][ind][1] = -copy[c * Mx * My + ic0][1];
                }
            }
        }
    free(copy);
}

void orc_forcing_energy_cascade(orc *o, const double *Forced_Ek, int last_input_rad, int nullify) {
    orc_recalculate_energy_cascade(o, NULL);
    int last_eff_rad = (int)((last_input_rad < o->last_rad) ? last_input_rad : o->last_rad);
    double *FT = alloc_real(last_eff_rad + 1);
    for (int K = 0; K <= last_eff_rad; K++) FT[K] = ((o->Ek[K] > 0.0) ? sqrt(Forced_Ek[K] / o->Ek[K]) : 0.0);
    LOOP_FOURIER(o) {
        long ind = IND_F(o);
        if (o->dealiased[ind]) {
            int K = (int)round(sqrt(o->rad2[ind]));
            if (K <= last_eff_rad) {
                for (int ic = 0; ic <= 1; ic++) { o->uk_1[ind][ic] *= FT[K]; o->vk_1[ind][ic] *= FT[K]; o->wk_1[ind][ic] *= FT[K]; }
            } else if (nullify) {
                for (int ic = 0; ic <= 1; ic++) { o->uk_1[ind][ic] = 0.0; o->vk_1[ind][ic] = 0.0; o->wk_1[ind][ic] = 0.0; }
            }
        }
    }
    free(FT);
    if (o->A.isComplexConjugateCorrected) orc_complex_conjugate_correction(o);
}

/* ------------------------------------------------------------------- */
/* Initial fields (src/HIT_LES.cpp:502-763, 1268-1294)                 */
/* ------------------------------------------------------------------- */
static void input_k41(orc *o) { /* :502-540, with the per-rank srand(0) of a P-rank run */
    const int P = o->A.k41_ranks > 0 ? o->A.k41_ranks : 1;
    const long blk = (o->My + P - 1) / P; /* FFTW-MPI default block for the transposed dimension */
    for (int r = 0; r < P; r++) {
        long b0 = r * blk, b1 = (r + 1) * blk;
        if (b1 > o->My) b1 = o->My;
        srand(0);
        for (long b = b0; b < b1; b++)
            for (long a = 0; a < o->Mx; a++)
                for (long k3 = 0; k3 < o->Mz_2 + 1; k3++) {
                    long ind = IND_F(o);
                    for (int ic = 0; ic <= 1; ic++) {
                        if (o->dealiased[ind]) {
                            int K = (int)round(sqrt(o->rad2[ind]));
                            if (K <= o->last_rad) {
                                o->uk_1[ind][ic] = (((double)rand() / RAND_MAX) * 2.0 - 1.0);
                                o->vk_1[ind][ic] = (((double)rand() / RAND_MAX) * 2.0 - 1.0);
                                o->wk_1[ind][ic] = (((double)rand() / RAND_MAX) * 2.0 - 1.0);
                            } else {
                                o->uk_1[ind][ic] = o->vk_1[ind][ic] = o->wk_1[ind][ic] = 0.0;
                            }
                        } else {
                            o->uk_1[ind][ic] = o->vk_1[ind][ic] = o->wk_1[ind][ic] = 0.0;
                        }
                    }
                }
    }
    orc_complex_conjugate_correction(o);
    double *K41_Ek = alloc_real(o->last_rad + 1);
    K41_Ek[0] = 0.0;
    for (int K = 1; K <= o->last_rad; K++) K41_Ek[K] = pow(K, -5.0 / 3.0);
    /* Forcing_Energy_Cascade(K41_Ek, last_rad, false) */
    orc_forcing_energy_cascade(o, K41_Ek, (int)o->last_rad, 0);
    free(K41_Ek);
}

static void calculate_ek_init_file(orc *o, const cplx *uk, const cplx *vk, const cplx *wk) { /* :1268-1294 */
    o->Ek_init_file = 0.0;
    o->Enstrophy_init_file = 0.0;
    const long Nxf = o->Nx_file, Nyf = o->Ny_file, Nzf = o->Nz_file;
    for (long a = 0; a < Nxf; a++)
        for (long b = 0; b < Nyf; b++)
            for (long k3 = 0; k3 < Nzf / 2 + 1; k3++) {
                long ind = (a * Nyf + b) * (Nzf / 2 + 1) + k3;
                long k1 = fourier_freq(a, Nxf), k2 = fourier_freq(b, Nyf);
                long rad2_file = k1 * k1 + k2 * k2 + k3 * k3;
                int relevant = ((k1 % o->Lx_factor == 0) && (k2 % o->Ly_factor == 0) && (k3 % o->Lz_factor == 0));
                if (relevant) {
                    int conj = (k3 != 0) && !((Nzf % 2 == 0) && (k3 == Nzf / 2));
                    double E = (uk[ind][0] * uk[ind][0]) + (uk[ind][1] * uk[ind][1]);
                    E += (vk[ind][0] * vk[ind][0]) + (vk[ind][1] * vk[ind][1]);
                    E += (wk[ind][0] * wk[ind][0]) + (wk[ind][1] * wk[ind][1]);
                    E *= 0.5;
                    if (conj) { o->Ek_init_file += 2 * E; o->Enstrophy_init_file += 2 * (2 * rad2_file * E); }
                    else { o->Ek_init_file += E; o->Enstrophy_init_file += (2 * rad2_file * E); }
                }
            }
}

static void input_real_field(orc *o, const double *file_uvw) { /* :542-599, 604-732, 738-763 */
    const long Nxf = o->Nx_file, Nyf = o->Ny_file, Nzf = o->Nz_file;
    const long nf = Nxf * Nyf * Nzf, hf = Nzf / 2 + 1;
    const long nact = o->ActualNx_file * o->ActualNy_file * o->ActualNz_file;
    double *uvw_file[3];
    for (int c = 0; c < 3; c++) {
        uvw_file[c] = alloc_real(nf);
        const double *rd = file_uvw + c * nact;
        if (o->A.isNotCubic) { /* :710-731 periodic repetition of the file box */
            for (long i = 0; i < Nxf; i++)
                for (long j = 0; j < Nyf; j++)
                    for (long k = 0; k < Nzf; k++) {
                        long ind = (i * Nyf + j) * Nzf + k;
                        if (i < o->ActualNx_file && j < o->ActualNy_file && k < o->ActualNz_file) {
                            uvw_file[c][ind] = rd[(i * o->ActualNy_file + j) * o->ActualNz_file + k];
                        } else {
                            long i_ = (i < o->ActualNx_file) ? i : i - o->ActualNx_file;
                            long j_ = (j < o->ActualNy_file) ? j : j - o->ActualNy_file;
                            long k_ = (k < o->ActualNz_file) ? k : k - o->ActualNz_file;
                            uvw_file[c][ind] = uvw_file[c][(i_ * Nyf + j_) * Nzf + k_];
                        }
                    }
        } else {
            memcpy(uvw_file[c], rd, sizeof(double) * (size_t)nf);
        }
    }
    cplx *uvwk[3];
    for (int c = 0; c < 3; c++) {
        uvwk[c] = alloc_complex(Nxf * Nyf * hf);
        orc_rfft3d((int)Nxf, (int)Nyf, (int)Nzf, uvw_file[c], (double *)uvwk[c]);
        free(uvw_file[c]);
        for (long ind = 0; ind < Nxf * Nyf * hf; ind++)
            for (int ic = 0; ic <= 1; ic++) uvwk[c][ind][ic] /= (double)(Nxf * Nyf * Nzf);
    }
    calculate_ek_init_file(o, uvwk[0], uvwk[1], uvwk[2]);
    cplx *dst[3] = {o->uk_1, o->vk_1, o->wk_1};
    LOOP_FOURIER(o) { /* Truncate_Input_File_Fourier_Coefficients :738-763 */
        long ind = IND_F(o);
        long k1 = fourier_freq(a, o->Mx), k2 = fourier_freq(b, o->My);
        for (int ic = 0; ic <= 1; ic++) {
            if (o->dealiased[ind]) {
                if ((labs(k1) <= (Nxf - 1) / 2) && (labs(k2) <= (Nyf - 1) / 2) && (k3 <= (Nzf - 1) / 2)) {
                    long a_file = (k1 >= 0) ? a : (Nxf + k1);
                    long b_file = (k2 >= 0) ? b : (Nyf + k2);
                    long c_file = k3;
                    long ind_file = (a_file * Nyf + b_file) * hf + c_file;
                    for (int c = 0; c < 3; c++) dst[c][ind][ic] = uvwk[c][ind_file][ic];
                } else {
                    for (int c = 0; c < 3; c++) dst[c][ind][ic] = 0.0;
                }
            } else {
                for (int c = 0; c < 3; c++) dst[c][ind][ic] = 0.0;
            }
        }
    }
    for (int c = 0; c < 3; c++) free(uvwk[c]);
}

/* ------------------------------------------------------------------- */
/* Construction (src/HIT_LES.h:23-84, src/HIT_LES.cpp:770-1092)          */
/* ------------------------------------------------------------------- */
static long actual(long n, long L) { return (n % 2 == 0) ? n / L : (n - 1) / L + 1; }

orc *orc_create(const orc_args *A, const double *file_uvw) {
    orc *o = (orc *)calloc(1, sizeof(orc));
    o->A = *A;
    o->nthreads = A->nthreads > 0 ? A->nthreads : 1;
    o->Lx_factor = A->Lx; o->Ly_factor = A->Ly; o->Lz_factor = A->Lz;
    o->ActualNx = actual(A->Nx, A->Lx); o->ActualNy = actual(A->Ny, A->Ly); o->ActualNz = actual(A->Nz, A->Lz);
    o->ActualMx = actual(A->Mx, A->Lx); o->ActualMy = actual(A->My, A->Ly); o->ActualMz = actual(A->Mz, A->Lz);
    o->Nx = A->Nx; o->Ny = A->Ny; o->Nz = A->Nz;
    o->Nx_2 = A->Nx / 2; o->Ny_2 = A->Ny / 2; o->Nz_2 = A->Nz / 2;
    o->Mx = A->Mx; o->My = A->My; o->Mz = A->Mz; o->Mx_2 = A->Mx / 2; o->Mz_2 = A->Mz / 2;
    {
        long a = (A->Nx - 1) / 2, b = (A->Ny - 1) / 2, c = (A->Nz - 1) / 2;
        long m = b < c ? b : c; o->last_rad = a < m ? a : m;
    }
    o->last_rad_max = (long)ceil(sqrt(1.0 * o->Nx_2 * o->Nx_2 + 1.0 * o->Ny_2 * o->Ny_2 + 1.0 * o->Nz_2 * o->Nz_2));
    o->nu = A->nu;
    o->delta = 2.0 * PI_REF / cbrt((double)(A->Lx * A->Ly * A->Lz * o->ActualMx * o->ActualMy * o->ActualMz));
    o->C_Smag = A->C_Smag; o->C_At = A->C_At;
    o->Ax = 2.0 * PI_REF / o->ActualMx / A->Lx;
    o->Ay = 2.0 * PI_REF / o->ActualMy / A->Ly;
    o->Az = 2.0 * PI_REF / o->ActualMz / A->Lz;
    o->omega_x = A->omega_x; o->omega_y = A->omega_y; o->omega_z = A->omega_z;
    o->ActualNx_file = actual(A->Nx_file, A->Lx); o->ActualNy_file = actual(A->Ny_file, A->Ly); o->ActualNz_file = actual(A->Nz_file, A->Lz);
    o->Nx_file = A->Nx_file; o->Ny_file = A->Ny_file; o->Nz_file = A->Nz_file;
    o->time = 0.0;
    o->kappa = 0.5;
    o->px = get_plan((int)o->Mx); o->py = get_plan((int)o->My); o->pz = get_plan((int)o->Mz);

    /* 1. memory (:775-827) */
    o->alloc_local = o->Mx * o->My * (o->Mz_2 + 1);
    o->local_n0 = o->Mx; o->local_n1 = o->My;
    long AL = o->alloc_local;
    o->u = alloc_real(2 * AL); o->v = alloc_real(2 * AL); o->w = alloc_real(2 * AL);
    for (int c = 0; c < 3; c++) { o->gradu[c] = alloc_real(2 * AL); o->gradv[c] = alloc_real(2 * AL); o->gradw[c] = alloc_real(2 * AL); }
    o->convx = alloc_real(2 * AL); o->convy = alloc_real(2 * AL); o->convz = alloc_real(2 * AL);
    o->rad2 = alloc_real(AL);
    o->local_acumField = alloc_real(o->last_rad_max + 1);
    o->global_acumField = alloc_real(o->last_rad_max + 1);
    o->Ek = alloc_real(o->last_rad_max + 1);
    o->uk_aux = alloc_complex(AL); o->vk_aux = alloc_complex(AL); o->wk_aux = alloc_complex(AL);
    o->uk_0 = alloc_complex(AL); o->vk_0 = alloc_complex(AL); o->wk_0 = alloc_complex(AL);
    o->uk_1 = alloc_complex(AL); o->vk_1 = alloc_complex(AL); o->wk_1 = alloc_complex(AL);
    for (int c = 0; c < 3; c++) { o->gradu_k[c] = alloc_complex(AL); o->gradv_k[c] = alloc_complex(AL); o->gradw_k[c] = alloc_complex(AL); }
    o->convx_k = alloc_complex(AL); o->convy_k = alloc_complex(AL); o->convz_k = alloc_complex(AL);
    o->Rx0_k = alloc_complex(AL); o->Ry0_k = alloc_complex(AL); o->Rz0_k = alloc_complex(AL);
    o->Rx1_k = alloc_complex(AL); o->Ry1_k = alloc_complex(AL); o->Rz1_k = alloc_complex(AL);
    o->dealiased = (unsigned char *)calloc((size_t)AL, 1);
    o->conjugate = (unsigned char *)calloc((size_t)AL, 1);

    /* 2. masks (:833-881) */
    LOOP_FOURIER(o) {
        long ind = IND_F(o);
        long k1 = fourier_freq(a, o->Mx), k2 = fourier_freq(b, o->My);
        o->rad2[ind] = (double)(k1 * k1 + k2 * k2 + k3 * k3);
        int d = (labs(k1) <= o->Nx_2 && labs(k2) <= o->Ny_2 && k3 <= o->Nz_2);
        if (A->isNotCubic)
            if ((k1 % A->Lx != 0) || (k2 % A->Ly != 0) || (k3 % A->Lz != 0)) d = 0;
        o->dealiased[ind] = (unsigned char)d;
        o->conjugate[ind] = (unsigned char)(d && (k3 != 0) && !((o->Mz % 2 == 0) && (k3 == o->Mz_2)));
    }
    /* 3. LES memory (:940-959) */
    if (A->isLES) {
        o->nu_eddy = alloc_real(2 * AL);
        o->SGS_11 = alloc_real(2 * AL); o->SGS_21 = alloc_real(2 * AL); o->SGS_22 = alloc_real(2 * AL);
        o->SGS_31 = alloc_real(2 * AL); o->SGS_32 = alloc_real(2 * AL); o->SGS_33 = alloc_real(2 * AL);
        o->SGS_11_k = alloc_complex(AL); o->SGS_21_k = alloc_complex(AL); o->SGS_22_k = alloc_complex(AL);
        o->SGS_31_k = alloc_complex(AL); o->SGS_32_k = alloc_complex(AL); o->SGS_33_k = alloc_complex(AL);
        o->divSGSx_k = alloc_complex(AL); o->divSGSy_k = alloc_complex(AL); o->divSGSz_k = alloc_complex(AL);
    }
    /* 6. initial field (:1030-1044) */
    if (A->isInitialFieldFromFile) {
        if (!file_uvw) crash("file initial field requested without data");
        input_real_field(o, file_uvw);
    } else {
        input_k41(o);
    }
    /* R1 = 0 (:1038-1044): calloc already zeroed it */
    /* 7. timestep constants (:1049-1078) */
    if (A->isSelfAdaptive) {
        o->Ah = (o->Ax + o->Ay + o->Az) / 3.0;
        o->t1 = 0.9302468;
        o->kappa = 0.5;
        o->k[0] = 0.73782212; o->k[1] = 0.44660387;
        o->phi[0] = atan(164.0 / 99.0); o->phi[1] = PI_REF / 3.0; o->phi[2] = PI_REF * 3.0 * 3.0 / (5.0 * 5.0);
        static const double cc[14] = {0.0647998, -0.386022, 3.72945, -9.38143, 7.06574, 2403400.0, -5018490.0,
                                      2620140.0, 2945.0, -6665.76, 3790.54, 4.80513, -16.9473, 15.0155};
        memcpy(o->c, cc, sizeof(cc));
    }
    orc_velocity_antitransform(o);
    if (!A->isReLambda) orc_recalculate_timestep(o);
    o->Ek_init = orc_recalculate_energy(o);
    return o;
}

void orc_destroy(orc *o) {
    if (!o) return;
    double *reals[] = {o->u, o->v, o->w, o->convx, o->convy, o->convz, o->rad2, o->local_acumField, o->global_acumField, o->Ek,
                       o->nu_eddy, o->SGS_11, o->SGS_21, o->SGS_22, o->SGS_31, o->SGS_32, o->SGS_33};
    for (size_t i = 0; i < sizeof(reals) / sizeof(reals[0]); i++) free(reals[i]);
    cplx *cs[] = {o->uk_aux, o->vk_aux, o->wk_aux, o->uk_0, o->vk_0, o->wk_0, o->uk_1, o->vk_1, o->wk_1, o->convx_k, o->convy_k,
                  o->convz_k, o->Rx0_k, o->Ry0_k, o->Rz0_k, o->Rx1_k, o->Ry1_k, o->Rz1_k, o->SGS_11_k, o->SGS_21_k, o->SGS_22_k,
                  o->SGS_31_k, o->SGS_32_k, o->SGS_33_k, o->divSGSx_k, o->divSGSy_k, o->divSGSz_k};
    for (size_t i = 0; i < sizeof(cs) / sizeof(cs[0]); i++) free(cs[i]);
    for (int c = 0; c < 3; c++) {
        free(o->gradu[c]); free(o->gradv[c]); free(o->gradw[c]);
        free(o->gradu_k[c]); free(o->gradv_k[c]); free(o->gradw_k[c]);
    }
    free(o->dealiased); free(o->conjugate);
    free(o);
}

/* Check_PhysFour_Energy (src/HIT_LES.cpp:1216-1252): returns 0 if within atol */
int orc_check_physfour_energy(orc *o, double atol, double *d1, double *d2) {
    double EkFour = 0.0;
    LOOP_FOURIER(o) {
        long ind = IND_F(o);
        if (o->dealiased[ind]) {
            double aux = kinetic_energy(o, ind);
            if (o->conjugate[ind]) EkFour += 2 * aux; else EkFour += aux;
        }
    }
    orc_velocity_antitransform(o);
    double EkReal = 0.0;
    LOOP_REAL(o) {
        long ind = IND_R(o);
        EkReal += o->u[ind] * o->u[ind] + o->v[ind] * o->v[ind] + o->w[ind] * o->w[ind];
    }
    EkReal = 0.5 * EkReal / (double)(o->Mx * o->My * o->Mz);
    double EkSpNS = orc_recalculate_energy(o);
    double diff1 = fabs(EkReal - EkFour), diff2 = fabs(EkSpNS - EkFour);
    if (d1) *d1 = diff1;
    if (d2) *d2 = diff2;
    return (diff1 > atol || diff2 > atol) ? 1 : 0;
}

void orc_get_scalars(const orc *o, double *s) {
    s[0] = o->time; s[1] = o->At; s[2] = o->nu; s[3] = o->Ek_Tot; s[4] = o->Ok_Tot; s[5] = o->ReLambda;
    s[6] = o->Ek_init; s[7] = o->Ek_init_file; s[8] = o->Enstrophy_init_file; s[9] = o->kappa; s[10] = o->MaxVel;
    s[11] = (double)o->last_rad; s[12] = (double)o->last_rad_max; s[13] = (double)o->iter;
}
void orc_set_nu(orc *o, double nu) { o->nu = nu; }

static long kx_count(const orc *o) { return 2 * o->Nx_2 + 1; }
static long ky_count(const orc *o) { return 2 * o->Ny_2 + 1; }
long orc_compact_size(const orc *o) { return kx_count(o) * ky_count(o) * (o->Nz_2 + 1); }

static void compact_map(const orc *o, int to_compact, double *buf) {
    const long Kx = kx_count(o), Ky = ky_count(o), Kz = o->Nz_2 + 1, S = Kx * Ky * Kz;
    cplx *f[3] = {o->uk_1, o->vk_1, o->wk_1};
    for (long iy = 0; iy < Ky; iy++) {
        long k2 = (iy <= o->Ny_2) ? iy : iy - Ky;
        long b = (k2 >= 0) ? k2 : o->My + k2;
        for (long ix = 0; ix < Kx; ix++) {
            long k1 = (ix <= o->Nx_2) ? ix : ix - Kx;
            long a = (k1 >= 0) ? k1 : o->Mx + k1;
            for (long kz = 0; kz < Kz; kz++) {
                long ind = (b * o->Mx + a) * (o->Mz_2 + 1) + kz;
                long ci = (iy * Kx + ix) * Kz + kz;
                for (int c = 0; c < 3; c++) {
                    if (to_compact) {
                        buf[2 * (c * S + ci)] = f[c][ind][0];
                        buf[2 * (c * S + ci) + 1] = f[c][ind][1];
                    } else {
                        f[c][ind][0] = buf[2 * (c * S + ci)];
                        f[c][ind][1] = buf[2 * (c * S + ci) + 1];
                    }
                }
            }
        }
    }
}
void orc_get_compact(const orc *o, double *out) { compact_map(o, 1, out); }
void orc_set_compact(orc *o, const double *in) { compact_map(o, 0, (double *)in); }

void orc_get_physical(const orc *o, double *out) {
    const long n = o->Mx * o->My * o->Mz;
    const double *f[3] = {o->u, o->v, o->w};
    for (int c = 0; c < 3; c++)
        for (long i = 0; i < o->Mx; i++)
            for (long j = 0; j < o->My; j++)
                for (long k = 0; k < o->Mz; k++)
                    out[c * n + (i * o->My + j) * o->Mz + k] = f[c][(i * o->My + j) * 2 * (o->Mz_2 + 1) + k];
}
