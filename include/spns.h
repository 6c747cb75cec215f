/*
 * spns.h -- C ABI of libspns, the B200-native (sm_100a) pseudospectral time step.
 *
 * One handle = one periodic box solved the way the reference's class HIT
 * (src/HIT_LES.h:21-246 of adalbal/SpNS) solves it, on one GPU, with no MPI.
 * Each entry point replaces one HIT member (cited per function) so that a
 * HIT_LES.cpp replacement can forward every call the reference driver
 * (src/MAIN.cpp) makes.  Plain pointers and sizes only; host arrays belong to
 * the caller and are copied; the handle owns every device buffer.
 *
 * Status codes: 0 = success, negative = error (see spns_status); the message of
 * the last error of a handle is returned by spns_last_error().
 */
#ifndef SPNS_H
#define SPNS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum spns_status {
    SPNS_OK = 0,
    SPNS_ERR_INVALID_ARGUMENT = -1,
    SPNS_ERR_UNSUPPORTED_SIZE = -2, /* an FFT length outside the compiled set   */
    SPNS_ERR_CUDA = -3,             /* a CUDA runtime call failed               */
    SPNS_ERR_OUT_OF_MEMORY = -4,    /* device allocation refused                */
    SPNS_ERR_NONFINITE = -5,        /* NaN/Inf met in the CFL maximum           */
    SPNS_ERR_DOMAIN = -6,           /* time-step angle outside [0, pi/2] (crash "Topt fail!") */
    SPNS_ERR_TIMEOUT = -7           /* a bounded device-side wait gave up (staged copy never arrived) */
} spns_status;

typedef enum spns_precision {
    SPNS_FP64 = 0,      /* plain form: every array and FFT in double            */
    SPNS_FP32_HILO = 1  /* FFTs/products in float; spectral state as float hi/lo pair;
                           reductions, CFL and forcing normalisation in double */
} spns_precision;

/* Arguments of the HIT constructor (src/HIT_LES.h:23-29), as src/MAIN.cpp:325
 * passes them after its derivations (length-factor expansion of N and M,
 * flags), plus options the reference does not have (marked "extension"). */
typedef struct spns_hit_args {
    int Nx, Ny, Nz;          /* retained modes per axis (expanded by length factors) */
    int Mx, My, Mz;          /* 3/2-rule FFT grid per axis (expanded)                 */
    double nu, C_Smag, C_At;
    int Lx_factor, Ly_factor, Lz_factor;
    double omega_x, omega_y, omega_z;
    int Nx_file, Ny_file, Nz_file;
    int isReLambda, isInitialFieldFromFile, isNotCubic, isRotating, isLES;
    int isComplexConjugateCorrected, isSelfAdaptive;
    /* extensions */
    int precision;           /* spns_precision                                          */
    int device;              /* CUDA device ordinal                                     */
    int k41_ranks;           /* K41 initial field as generated by this many MPI ranks (>=1); a negative
                                value starts from a zero state instead, for callers that set the state
                                themselves (spns_set_spectral, spns_seed_field, spns_checkpoint_load) */
    double fixed_dt;         /* >0: constant time step instead of the CFL/self-adaptive one */
    double eps_forcing;      /* >0: constant-power forcing on shells [eps_kmin, eps_kmax]   */
    int eps_kmin, eps_kmax;  /*     (the disabled block src/HIT_LES.cpp:243-278, eps_in=eps) */
    int nonlinear_form;      /* DNS only.  0 (default): rotational omega x u (6 inverse
                                transforms) plus the exact aliasing correction of the +-N/2
                                planes, which equals the reference's advective u.grad(u)
                                (src/HIT_LES.cpp:74-125) after the projection;
                                1: rotational without the correction (equal only while the
                                +-N/2 modes carry no energy); 2: advective, 12 inverse
                                transforms, the reference's arithmetic */
    int stream_priority;     /* CUDA stream priority of the handle's work (0 = default;
                                lower values run first, clamped to the device's range).
                                A serving loop gives short runs precedence this way. */
} spns_hit_args;

typedef struct spns_handle spns_handle;

/* Scalars of the solver (getters of src/HIT_LES.h:187-201). */
typedef struct spns_scalars {
    double time, At, nu, Ek_Tot, Ok_Tot, ReLambda, Ek_init, Ek_init_file, Enstrophy_init_file;
    double kappa, MaxVel;
    int64_t iter, last_rad, last_rad_max;
} spns_scalars;

/* HIT::HIT + HIT_init (src/HIT_LES.h:23-84, src/HIT_LES.cpp:770-1092).
 * file_uvw: initial physical velocity from the input file, three components one
 * after another, each ActualNx_file*ActualNy_file*ActualNz_file doubles in
 * [x][y][z] order (what src/HIT_LES.cpp:604-732 reads); NULL selects the K41
 * initial field (src/HIT_LES.cpp:502-540). */
int spns_create(const spns_hit_args *args, const double *file_uvw, spns_handle **out);
/* HIT::~HIT (src/HIT_LES.h:86-88) */
int spns_destroy(spns_handle *h);

/* HIT::New_Fractional_Step_Method (src/HIT_LES.cpp:9-25), nsteps times. */
int spns_step(spns_handle *h, int nsteps);
/* HIT::Recalculate_TimeStep (src/HIT_LES.cpp:365-403) from the physical
 * velocity of the last inverse transform. */
int spns_recalculate_timestep(spns_handle *h);
/* HIT::Forcing_Energy_Cascade (src/HIT_LES.cpp:410-444); Forced_Ek[0..last_input_rad]. */
int spns_forcing_energy_cascade(spns_handle *h, const double *Forced_Ek, int last_input_rad, int nullify_missing);
/* HIT::Forcing_Reynolds_Lambda (src/HIT_LES.cpp:485-489) */
int spns_forcing_reynolds_lambda(spns_handle *h, double relambda);
/* HIT::Recalculate_Reynolds_Lambda (src/HIT_LES.cpp:478-483) */
int spns_recalculate_reynolds_lambda(spns_handle *h, double *relambda);
/* HIT::Recalculate_Energy (src/HIT_LES.cpp:1254-1259) */
int spns_recalculate_energy(spns_handle *h, double *ek_tot);
/* HIT::Recalculate_Enstrophy (src/HIT_LES.cpp:490-495) */
int spns_recalculate_enstrophy(spns_handle *h, double *ok_tot);
/* HIT::Recalculate_Energy_Cascade (src/HIT_LES.cpp:1261-1266): Ek[0..last_rad_max]. */
int spns_recalculate_energy_cascade(spns_handle *h, double *Ek, double *ek_tot);
/* HIT::Recalculate_Velocity_Antitransform (src/HIT_LES.cpp:60-69): refreshes
 * the physical velocity (and its CFL maximum) from the spectral state. */
int spns_velocity_antitransform(spns_handle *h);
/* HIT::Complex_Conjugate_Correction (src/HIT_LES.cpp:446-476) */
int spns_complex_conjugate_correction(spns_handle *h);
/* HIT::Check_PhysFour_Energy (src/HIT_LES.cpp:1216-1252): energies by the
 * Fourier sum, the physical sum and the shell integral; *ok = all within atol. */
int spns_check_physfour_energy(spns_handle *h, double atol, int *ok, double *diff1, double *diff2);

/* HIT::Recalculate_Invariants_Distribution (src/HIT_LES.cpp:1297-1319, invariant
 * definitions src/tensor_algebra.cpp:165-306, 356-358): spectra[c*(last_rad_max+1) + K]
 * for c = Q_G, Q_S, R_G, R_S, V^2 of the velocity-gradient tensor G_ij = d_j u_i,
 * each the shell integral of |F_c(k)|^2 (conjugate weight 2 for kz > 0) of the
 * normalised transform.  Computed from the current spectral state (the reference
 * uses the gradients of the last step's start).  The first call allocates work
 * buffers of the advective step's size (6 S1 + 9 S2 fields), kept until destroy. */
int spns_invariant_spectra(spns_handle *h, double *spectra);
/* Eddy-viscosity statistics of the current state: stats[0] mean, stats[1] root
 * mean square, stats[2] maximum over the grid of nu_t = (C_s Delta)^2
 * sqrt(2 S_ij S_ij), the nu_t of Recalculate_Eddy_Viscosity
 * (src/HIT_LES.cpp:130-142); zero for a DNS handle.  Runs the invariant passes
 * (same work buffers as spns_invariant_spectra).  The reference writes no such
 * statistics; they carry the FP32-against-FP64 comparison of an LES run. */
int spns_eddy_viscosity_stats(spns_handle *h, double *stats);

/* ---- Slab decomposition of one box over several GPUs (one process per GPU) ----
 * Replaces the reference's FFTW-MPI transposed slab layout
 * (src/FFTW_package.cpp:47-56: fftw_mpi_local_size_3d_transposed and the
 * TRANSPOSED_OUT/IN plans; src/FFTW_package.h:60-64: local_n0 x planes in
 * physical space, local_n1 ky rows in spectral space) and its one all-to-all
 * per 3-D transform.  Rank `rank` of `nranks` holds the compact ky rows
 * [y0, y0+ny) of the state, the x pass's rows and the spectral sweep; between
 * the inverse and the forward y pass it holds the x planes [x0, x0+nx) (y and z
 * passes).  Both splits are FFTW-MPI's default block, ceil(n/nranks) per rank
 * (spns_slab_block).  A step is the reference's two transposes around the y/z
 * passes as two all-to-alls of the staging arrays, made by the caller (NCCL, or
 * any transport) between the phases:
 *   SPNS_SLAB_A, all-to-all, [sum ds.ef over ranks], SPNS_SLAB_B,
 *   all-to-all, max of the 4 CFL words and of nonfinite over ranks, SPNS_SLAB_C.
 * The first time step: SPNS_SLAB_VEL_A, all-to-all, SPNS_SLAB_VEL_B, max of the
 * CFL words, SPNS_SLAB_DT (HIT::Recalculate_Velocity_Antitransform and
 * Recalculate_TimeStep, src/HIT_LES.cpp:60-69, 365-403).
 * The all-to-all moves block s of the sender's staging array (offsets from the
 * block sizes in rank order) to the receiver's staging array, block r from rank
 * r in rank order; spns_slab_exchange gives the counts.  Slab handles run the
 * advective arithmetic (nonlinear_form 2) or LES, with AB2 or the kappa scheme,
 * rotation and constant-power forcing; the state is set with spns_set_spectral
 * on the rank's rows ([3][ny][Kx][Kz]); conjugate correction, Re_lambda forcing,
 * K41 and file initial fields are not available (SPNS_ERR_INVALID_ARGUMENT).
 * spns_step is refused on a slab handle. */
enum spns_slab_phase_id {
    SPNS_SLAB_VEL_A = 0, SPNS_SLAB_VEL_B = 1, SPNS_SLAB_DT = 2,
    SPNS_SLAB_A = 3, SPNS_SLAB_B = 4, SPNS_SLAB_C = 5
};
/* [start, start+count) of block `rank` when n items are split over nranks
 * (FFTW-MPI's default block size ceil(n/nranks)); host only, no device needed. */
int spns_slab_block(int n, int nranks, int rank, int *start, int *count);
int spns_slab_create(const spns_hit_args *args, int nranks, int rank, spns_handle **out);
/* This rank's rows and planes. */
int spns_slab_layout(spns_handle *h, int *y0, int *ny, int *x0, int *nx);
int spns_slab_phase(spns_handle *h, int phase);
/* Element counts (complex values of the handle's precision) this rank sends to
 * and receives from every rank in the exchange after `phase` (SPNS_SLAB_VEL_A,
 * SPNS_SLAB_A or SPNS_SLAB_B): send[s], recv[s] for s < nranks. */
int spns_slab_exchange(spns_handle *h, int phase, long long *send, long long *recv);
/* The same counts for any box and rank without a handle (host only): nf fields,
 * back = 0 for the ky-rows -> x-planes exchange, 1 for the way back. */
int spns_slab_counts(int Ky, int Mx, int Kz, int nranks, int rank, int nf, int back, long long *send, long long *recv);
/* Device staging arrays (send, recv; `elems` complex values each) and the device
 * address of the solver scalars with the byte offsets of the fields the caller
 * reduces: off[0] the 4 CFL words (uint64 bit patterns of non-negative doubles:
 * their maximum is the integer maximum), off[1] nonfinite (int), off[2] ef (double). */
int spns_slab_buffers(spns_handle *h, void **send, void **recv, size_t *elems, void **scalars, size_t *off);

/* getters / HIT::setnu (src/HIT_LES.h:187-201) */
int spns_get_scalars(spns_handle *h, spns_scalars *out);
int spns_set_nu(spns_handle *h, double nu);

/* State access (HIT::FourierVelocity_to_BinaryFile / RealVelocity_to_BinaryFile
 * data, src/HIT_LES_output.cpp:8-14).  Spectral layout: 3 components one after
 * another, each [iy][ix][kz] with ix<Kx=2*(Nx'/2)+1, iy<Ky=2*(Ny'/2)+1,
 * kz<=Nz'/2 (N' = retained modes before length-factor expansion), interleaved
 * re/im doubles; ix maps to k1=ix (ix<=Nx'/2) or ix-Kx.  Physical layout: 3
 * components, each [x][y][z] on the true FFT grid (ActualMx, ActualMy, ActualMz). */
int spns_spectral_dims(spns_handle *h, int *Kx, int *Ky, int *Kz);
int spns_physical_dims(spns_handle *h, int *Mx, int *My, int *Mz);
int spns_get_spectral(spns_handle *h, double *uvw);
int spns_set_spectral(spns_handle *h, const double *uvw);
int spns_get_physical(spns_handle *h, double *uvw);

/* Device-resident state for callers that keep their own device buffers:
 * pointers to the three spectral components (layout as spns_get_spectral,
 * element type double2 for SPNS_FP64; for SPNS_FP32_HILO the float2 high parts
 * of the hi + lo pairs). */
int spns_device_state(spns_handle *h, void **u, void **v, void **w);
/* The CUDA stream all work of the handle is issued on (cudaStream_t). */
int spns_stream(spns_handle *h, void **stream);
/* Number of kernels issued by the last spns_step call (per step). */
int spns_kernels_per_step(spns_handle *h, int *count);

/* Device bytes a handle with these arguments allocates (state, history, work
 * buffers, edge planes, twiddles), for admission against a memory budget.  The
 * physical-field buffer of spns_get_physical is allocated later, on first use. */
int spns_estimate_device_bytes(const spns_hit_args *args, size_t *bytes);

/* Seeded initial field (no counterpart in the reference, which starts from its
 * K41 draw or a file): complex Gaussian modes from Philox4x32-10 (key = seed,
 * counter = compact mode index and draw number), projected onto k-perp, zero for
 * |m_i| > (N_i-1)/2 and at k=0, Hermitian on kz=0, shells scaled to
 * E(K) ~ K^4 exp(-2 (K/kp)^2) with total energy 3/2 urms^2.  Replaces the state;
 * call spns_velocity_antitransform and spns_recalculate_timestep afterwards, as
 * after spns_set_spectral. */
int spns_seed_field(spns_handle *h, uint64_t seed, double kp, double urms);

/* Asynchronous stepping for callers that keep many handles busy at once:
 * spns_step_async enqueues nsteps steps on the handle's stream and returns;
 * spns_query reports whether they have finished (*idle = 1); spns_synchronize
 * waits and returns the status of the steps (as spns_step does). */
int spns_step_async(spns_handle *h, int nsteps);
int spns_query(spns_handle *h, int *idle);
int spns_synchronize(spns_handle *h);

/* Exact checkpoint of a handle: scalars (time, dt, kappa, iteration, ...),
 * the state (hi and lo parts in FP32_HILO), R^{n-1} and, for the kappa scheme,
 * u^{n-1}; loading it into a handle created with the same arguments resumes the
 * run bit for bit. */
int spns_checkpoint_bytes(spns_handle *h, size_t *bytes);
int spns_checkpoint_save(spns_handle *h, void *buf, size_t bytes);
int spns_checkpoint_load(spns_handle *h, const void *buf, size_t bytes);

/* Ensembles (no counterpart in the reference, which runs one box per job):
 * members of any sizes and precisions on one device advance together, one CUDA
 * graph per step in which every member's step is an independent branch, so the
 * kernels of small boxes run concurrently.  Each member's result equals the
 * one it reaches stepped alone.  spns_ensemble_step synchronises and returns the
 * first failing member's status (message from spns_ensemble_last_error). */
typedef struct spns_ensemble spns_ensemble;
int spns_ensemble_create(spns_handle *const *members, int n, spns_ensemble **out);
int spns_ensemble_step(spns_ensemble *e, int nsteps);
int spns_ensemble_destroy(spns_ensemble *e);
const char *spns_ensemble_last_error(spns_ensemble *e);
/* Batched classes (off by default): members of one class -- same precision, box,
 * form (advective or LES) and launch shapes, Adams-Bashforth, no constant-power
 * forcing -- step in one launch per pass for the whole class (blockIdx.z selects
 * the member from a device table of its buffers and constants) instead of one
 * graph branch each.  Results are bit for bit those of the branches.  Measured on
 * a B200 with FP32 LES boxes: 64 boxes of 32^3 73.0k against 72.4k box-steps/s,
 * 64 of 48^3 29.4k against 30.2k, the 64-box mix of 32..96^3 7.9k against 8.4k:
 * the boxes' own kernels bound an ensemble, not launches. */
int spns_ensemble_set_batched(spns_ensemble *e, int on);

/* Per-kernel CUDA-event profile of the next max_steps calls of one step
 * (events recorded on the handle's stream between the kernels of a step). */
/* Autotuner of the launch shapes (FFT radix plan and tile per pass).  For each
 * of the passes K1..K5 whose length has an alternate compiled shape (E = 6
 * values per thread for lengths <= 192 in the step forms), times the default
 * and the alternate over `steps` real steps of this handle (per-kernel CUDA
 * events), keeps the faster per pass and restores the state it found, so the
 * run is unchanged.  Choices are cached per process by precision, form and box;
 * a later call or a handle created later for the same key uses them without
 * timing.  `choice` (5 ints, or NULL) receives 0 (default) / 1 (alternate) for
 * K1..K5.  Call it before an ensemble that holds the handle is stepped.
 * It stands where the reference measures its FFT plans (FFTW_MEASURE,
 * src/FFTW_package.h:12, at plan creation src/FFTW_package.cpp:53-55). */
int spns_autotune(spns_handle *h, int steps, int *choice);
/* Forgets the process-wide tuning cache (handles keep their shapes). */
int spns_autotune_forget(void);
/* Sets the shapes of K1..K5 directly (0 default, 1 alternate where compiled). */
int spns_set_shapes(spns_handle *h, const int *choice);

int spns_profile_begin(spns_handle *h, int max_steps);
/* ms[s*nkernels + k] = duration of kernel k in profiled step s (synchronises). */
int spns_profile_read(spns_handle *h, float *ms, int cap, int *nkernels, int *nsteps);
const char *spns_profile_kernel_name(spns_handle *h, int i);

const char *spns_last_error(spns_handle *h);
const char *spns_status_string(int status);

/* Energy spectrum without device allocation.  No counterpart in the reference.
 * For callers that cannot allocate device memory when they need E(K): host
 * frameworks that own all device memory through their own caching pool (a
 * foreign cudaMalloc fails once the pool holds the free memory, or fragments
 * it), and loops that must not stall other streams (cudaMalloc and cudaFree can
 * synchronise the device).  Computes Ek[K], K=0..nbins-1 (host array;
 * K=round(|k|), conjugate weight 2 for kz>0, as spns_recalculate_energy_cascade)
 * and *ek_tot from a compact spectral velocity already on the device (uvw_dev:
 * 3 components one after another, each Ky*Kx*Kz double2 in the layout of
 * spns_get_spectral; wavenumbers scaled by the length factors), on `stream`
 * (cudaStream_t, NULL = default stream).  It copies E(K) to the host and
 * synchronises that stream before returning.
 * The input must be FP64 state (double2).  The compensated FP32 form keeps a
 * float2 hi/lo pair, which this call cannot read: for such handles use
 * spns_recalculate_energy_cascade.
 * Working memory is a fixed array of SPNS_NOALLOC_MAX_BINS x 2 doubles compiled
 * into the library (held by every device that loads it until exit); nbins
 * above SPNS_NOALLOC_MAX_BINS is rejected with SPNS_ERR_UNSUPPORTED_SIZE.  The
 * first call on a device looks up the array's device address and the device's
 * SM count (cudaGetSymbolAddress, cudaDeviceGetAttribute) and keeps them for
 * the life of the process: make that first call before any stream capture is
 * under way on the device, and do not call it after cudaDeviceReset on that
 * device.  All calls share the array: calls whose GPU work overlaps race and
 * must be serialised by the caller.  Error text: spns_last_error(NULL). */
#define SPNS_NOALLOC_MAX_BINS 2048
int spns_energy_cascade_noalloc_f64(const void *uvw_dev, int Kx, int Ky, int Kz, int Lx_factor, int Ly_factor,
                                    int Lz_factor, double *Ek, int nbins, double *ek_tot, void *stream);

/* Building block exposed for tests: batched 1-D complex FFT of `batch` contiguous
 * length-n lines of device memory (double2), in place, unnormalised; sign=-1
 * forward, +1 backward.  Replaces nothing in the reference (FFTW's 1-D plans,
 * src/FFTW_package.cpp:47-56, are internal to its 3-D transforms). */
int spns_fft1d_batch_f64(void *data_dev, int n, int batch, int sign);

#ifdef __cplusplus
}
#endif
#endif /* SPNS_H */
