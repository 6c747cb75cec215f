/*
 * spns_oracle.h -- CPU oracle for the SpNS pseudospectral step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * solver's algorithm (class HIT in src/HIT_LES.{h,cpp} of adalbal/SpNS and the
 * FFT wrapper src/FFTW_package.cpp), used by tests/, by the smoke check and by
 * bench.py's CPU-baseline leg as the checker.  The product path (libspns) never
 * links, loads or calls it.
 *
 * Parity pin: the oracle reproduces the reference's own QA golden logs
 * (QA/TEST_1_DHIT_DNS/REF/stdout.0, QA/TEST_2_DHIT_SMAGORINSKY/REF/stdout.0 and
 * the K41-initialised QA tests through a P-rank emulation of the K41 field),
 * which were produced by the reference built against FFTW 3 (version not
 * pinned by the reference) on 4 MPI ranks.  The FFT here is project-written
 * (mixed radix 2/3/4/5/generic Stockham) and is checked against numpy.fft.
 *
 * Layout is the reference's single-rank FFTW-MPI transposed layout:
 *   spectral  C[b][a][k3], ind=(b*Mx+a)*(Mz/2+1)+k3   (src/util.h:75-77)
 *   physical  R[i][j][k],  ind=(i*My+j)*2*(Mz/2+1)+k  (src/util.h:78-80)
 */
#ifndef SPNS_ORACLE_H
#define SPNS_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Arguments of the HIT constructor (src/HIT_LES.h:23-29) after the driver's
 * derivations (src/MAIN.cpp:174-318), plus oracle-harness options. */
typedef struct orc_args {
    int Nx, Ny, Nz;          /* retained modes (after length-factor expansion) */
    int Mx, My, Mz;          /* FFT grid (3N/2, after length-factor expansion) */
    double nu, C_Smag, C_At;
    int Lx, Ly, Lz;          /* length factors as the HIT ctor receives them   */
    double omega_x, omega_y, omega_z;
    int Nx_file, Ny_file, Nz_file;
    int isReLambda, isInitialFieldFromFile, isNotCubic, isRotating, isLES;
    int isComplexConjugateCorrected, isSelfAdaptive;
    /* harness options (not in the reference's constructor) */
    int k41_ranks;           /* number of MPI ranks whose K41 field is emulated (>=1) */
    int nthreads;            /* OpenMP threads used inside the FFTs (as FFTW threads) */
    double fixed_dt;         /* >0: time step fixed to this value (no CFL)          */
    double eps_forcing;      /* >0: constant-power forcing of src/HIT_LES.cpp:244-278 */
    int eps_kmin, eps_kmax;  /* forced shell range for eps_forcing (reference: 1, 2) */
} orc_args;

typedef struct orc orc;

/* file_uvw: physical velocity of the initial-field file, 3 components stored one
 * after another, each ActualN_file^3 values in [x][y][z] order (exactly what
 * src/HIT_LES.cpp:604-732 reads); NULL for the K41 initial field. */
orc *orc_create(const orc_args *a, const double *file_uvw);
void orc_destroy(orc *o);

void orc_step(orc *o);                                     /* New_Fractional_Step_Method */
void orc_recalculate_timestep(orc *o);
void orc_forcing_energy_cascade(orc *o, const double *Ek, int last_input_rad, int nullify);
void orc_forcing_reynolds_lambda(orc *o, double relambda);
double orc_recalculate_reynolds_lambda(orc *o);
double orc_recalculate_energy(orc *o);
double orc_recalculate_enstrophy(orc *o);
double orc_recalculate_energy_cascade(orc *o, double *Ek_out); /* Ek_out[0..last_rad_max] */
/* Recalculate_Invariants_Distribution: spectra of Q_G, Q_S, R_G, R_S, V^2 of the
 * current state, out[c*(last_rad_max+1) + K]. */
void orc_invariant_spectra(orc *o, double *out);
void orc_eddy_viscosity_stats(orc *o, double *out);
void orc_velocity_antitransform(orc *o);
void orc_complex_conjugate_correction(orc *o);
int orc_check_physfour_energy(orc *o, double atol, double *diff1, double *diff2);

/* scalars: [time, At, nu, Ek_Tot, Ok_Tot, ReLambda, Ek_init, Ek_init_file,
 *           Enstrophy_init_file, kappa, MaxVel, last_rad, last_rad_max, iter] */
void orc_get_scalars(const orc *o, double *out14);
void orc_set_nu(orc *o, double nu);

/* Dealiased box of the spectral velocity in the compact layout
 * [iy][ix][kz] (iy<Ky=2*(Ny/2)+1, ix<Kx=2*(Nx/2)+1, kz<=Nz/2), interleaved
 * re/im, 3 components one after another. */
long orc_compact_size(const orc *o);
void orc_get_compact(const orc *o, double *out);
void orc_set_compact(orc *o, const double *in);
/* physical velocity u,v,w on the M grid, [x][y][z] without padding */
void orc_get_physical(const orc *o, double *out);

/* Plain 1-D and 3-D transforms (checked against numpy.fft in tests). */
void orc_fft1d(int n, double *data, int sign);               /* in place, unnormalised */
void orc_rfft3d(int n0, int n1, int n2, const double *in, double *out); /* numpy rfftn layout */
void orc_irfft3d(int n0, int n1, int n2, const double *in, double *out);/* unnormalised c2r  */

#ifdef __cplusplus
}
#endif
#endif
