// hit_forwarding.cpp -- the members of the reference class HIT (src/HIT_LES.h of
// adalbal/SpNS, compiled unchanged) implemented by forwarding to libspns, so
// that the reference driver src/MAIN.cpp runs its time loop on one B200.
//
// This unit replaces src/HIT_LES.cpp and src/HIT_LES_output.cpp.  HIT_LES.h has
// no slot for a libspns handle, so the handle of each HIT object lives in a
// table keyed by the object's address.  The header's inline getters read the
// private scalars (time, At, nu, Ek_Tot, ...); every forwarding member copies
// them back from the device after its call.  HIT::setnu is inline in the header
// and only writes the member, so the viscosity is pushed to the device before
// any call that depends on it.
//
// Options the reference does not have, read from the environment:
//   SPNS_DEVICE        CUDA device ordinal (default 0)
//   SPNS_PRECISION     fp64 (default) or fp32 (float transforms, float hi+lo state)
//   SPNS_K41_RANKS     build the K41 initial field as a run of that many MPI ranks
//                      does (srand(0) per rank over its slab; default 1)
//   SPNS_NONLINEAR_FORM 0 rotational + exact +-N/2 correction (default), 2 advective
#include "HIT_LES.h"
#include "spns.h"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <string>
#include <vector>

namespace {

struct Binding {
    spns_handle *h = nullptr;
    double nu_on_device = 0.0;
};
std::map<const HIT *, Binding> g_bindings;
std::mutex g_bindings_mutex;

Binding &binding_of(const HIT *p) {
    std::lock_guard<std::mutex> lock(g_bindings_mutex);
    auto it = g_bindings.find(p);
    if (it == g_bindings.end()) crash("libspns: no handle bound to this HIT object");
    return it->second;
}

int env_int(const char *name, int dflt) {
    const char *v = getenv(name);
    return (v && *v) ? atoi(v) : dflt;
}

void check(spns_handle *h, int status, const char *what) {
    if (status != SPNS_OK) crash("libspns: %s failed (%s): %s", what, spns_status_string(status), spns_last_error(h));
}

// Initial physical velocity as src/HIT_LES.cpp:604-709 reads it: the
// ActualN*_file box, components one after another, [x][y][z].  Binary files hold
// float64 or float32 values (told apart by the file size); ASCII files one
// "u v w" row per point.
std::vector<double> read_initial_field(const char *ascii, const char *binary, bool from_binary, long nx, long ny, long nz) {
    const size_t n = (size_t)nx * ny * nz;
    std::vector<double> uvw(3 * n);
    if (from_binary) {
        FILE *f = fopen(binary, "rb");
        if (!f) crash("Error opening \"%s\"!!\n", binary);
        fseek(f, 0, SEEK_END);
        const long long size = ftell(f);
        fseek(f, 0, SEEK_SET);
        if (size == (long long)(3 * n * sizeof(double))) {
            if (fread(uvw.data(), sizeof(double), 3 * n, f) != 3 * n) crash("Short read of \"%s\"", binary);
        } else if (size == (long long)(3 * n * sizeof(float))) {
            std::vector<float> tmp(3 * n);
            if (fread(tmp.data(), sizeof(float), 3 * n, f) != 3 * n) crash("Short read of \"%s\"", binary);
            for (size_t i = 0; i < 3 * n; i++) uvw[i] = tmp[i];
        } else {
            crash("Incorrect size of \"%s\"!! %lld bytes instead of %zu bytes (for single-precision) or %zu bytes (for double-precision).\n",
                  binary, size, 3 * n * sizeof(float), 3 * n * sizeof(double));
        }
        fclose(f);
    } else {
        std::ifstream in(ascii);
        if (in.fail()) crash("Error opening \"%s\"!!\n", ascii);
        for (size_t row = 0; row < n && !in.eof(); row++) in >> uvw[row] >> uvw[n + row] >> uvw[2 * n + row];
    }
    return uvw;
}

}  // namespace

// HIT::HIT_init (src/HIT_LES.cpp:770-1092): the solver state lives on the GPU.
void HIT::HIT_init() {
    if (numprocs != 1) crash("libspns drop-in runs one box per process (found %d MPI ranks)", numprocs);
    spns_hit_args a;
    memset(&a, 0, sizeof(a));
    a.Nx = (int)Nx; a.Ny = (int)Ny; a.Nz = (int)Nz;
    a.Mx = (int)Mx; a.My = (int)My; a.Mz = (int)Mz;
    a.nu = nu; a.C_Smag = C_Smag; a.C_At = C_At;
    a.Lx_factor = Lx_factor; a.Ly_factor = Ly_factor; a.Lz_factor = Lz_factor;
    a.omega_x = omega_x; a.omega_y = omega_y; a.omega_z = omega_z;
    a.Nx_file = (int)Nx_file; a.Ny_file = (int)Ny_file; a.Nz_file = (int)Nz_file;
    a.isReLambda = isReLambda;
    a.isInitialFieldFromFile = isInitialFieldFromBinaryFile || isInitialFieldFromASCIIFile;
    a.isNotCubic = isNotCubic; a.isRotating = isRotating; a.isLES = isLES;
    a.isComplexConjugateCorrected = isComplexConjugateCorrected; a.isSelfAdaptive = isSelfAdaptive;
    const char *prec = getenv("SPNS_PRECISION");
    a.precision = (prec && (strcmp(prec, "fp32") == 0 || strcmp(prec, "1") == 0)) ? SPNS_FP32_HILO : SPNS_FP64;
    a.device = env_int("SPNS_DEVICE", 0);
    a.k41_ranks = env_int("SPNS_K41_RANKS", 1);
    a.nonlinear_form = env_int("SPNS_NONLINEAR_FORM", 0);

    std::vector<double> file_uvw;
    if (a.isInitialFieldFromFile)
        file_uvw = read_initial_field(ASCII_Input_Filename, Binary_Input_Filename, isInitialFieldFromBinaryFile, ActualNx_file,
                                      ActualNy_file, ActualNz_file);
    spns_handle *h = nullptr;
    check(nullptr, spns_create(&a, a.isInitialFieldFromFile ? file_uvw.data() : nullptr, &h), "spns_create");
    {
        std::lock_guard<std::mutex> lock(g_bindings_mutex);
        Binding &b = g_bindings[this];
        b.h = h;
        b.nu_on_device = nu;
    }
    Ek = alloc_real(last_rad_max + 1);
    for (ptrdiff_t K = 0; K <= last_rad_max; K++) Ek[K] = 0.0;
    spns_scalars s;
    check(h, spns_get_scalars(h, &s), "spns_get_scalars");
    time = s.time; At = s.At; Ek_init = s.Ek_init; Ek_init_file = s.Ek_init_file;
    Enstrophy_init_file = s.Enstrophy_init_file; Ek_Tot = s.Ek_Tot; Ok_Tot = 0.0; ReLambda = 0.0;
    kappa = s.kappa; MaxVel = s.MaxVel;
}

void HIT::HIT_destroy() {
    spns_handle *h = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_bindings_mutex);
        auto it = g_bindings.find(this);
        if (it != g_bindings.end()) { h = it->second.h; g_bindings.erase(it); }
    }
    if (h) spns_destroy(h);
    FREE(Ek);
    Ek = nullptr;
}

// Pushes a viscosity set through the inline HIT::setnu, then runs the call.
#define SPNS_FORWARD(call, what)                                                   \
    do {                                                                           \
        Binding &b_ = binding_of(this);                                            \
        if (nu != b_.nu_on_device) {                                               \
            check(b_.h, spns_set_nu(b_.h, nu), "spns_set_nu");                    \
            b_.nu_on_device = nu;                                                  \
        }                                                                          \
        spns_handle *h = b_.h;                                                     \
        check(h, (call), what);                                                    \
    } while (0)

// Copies the device scalars into the members the inline getters return.
static void pull_scalars(const HIT *self, spns_scalars &s) {
    Binding &b = binding_of(self);
    check(b.h, spns_get_scalars(b.h, &s), "spns_get_scalars");
    b.nu_on_device = s.nu;
}
#define SPNS_PULL()                                                                \
    do {                                                                           \
        spns_scalars s_;                                                           \
        pull_scalars(this, s_);                                                    \
        time = s_.time; At = s_.At; nu = s_.nu; kappa = s_.kappa; MaxVel = s_.MaxVel; \
    } while (0)

void HIT::New_Fractional_Step_Method() {
#if (QA)
    // The reference's QA build checks, before every step, that the energy of the
    // spectral state equals that of its physical field to 1e-13 and crashes if not
    // (src/HIT_LES.cpp:10-12, 1216-1252).
    Check_PhysFour_Energy(1e-13);
#endif
    SPNS_FORWARD(spns_step(h, 1), "New_Fractional_Step_Method");
    SPNS_PULL();
}

void HIT::Recalculate_TimeStep() {
    SPNS_FORWARD(spns_recalculate_timestep(h), "Recalculate_TimeStep");
    SPNS_PULL();
}

void HIT::Recalculate_Velocity_Antitransform() {
    SPNS_FORWARD(spns_velocity_antitransform(h), "Recalculate_Velocity_Antitransform");
}

void HIT::Forcing_Energy_Cascade(REAL const *const Forced_Ek, const ptrdiff_t &last_input_rad, const bool &isNullifyMissingEk) {
    SPNS_FORWARD(spns_forcing_energy_cascade(h, Forced_Ek, (int)last_input_rad, isNullifyMissingEk ? 1 : 0), "Forcing_Energy_Cascade");
    spns_scalars s;
    pull_scalars(this, s);
    Ek_Tot = s.Ek_Tot;
}

void HIT::Complex_Conjugate_Correction() {
    SPNS_FORWARD(spns_complex_conjugate_correction(h), "Complex_Conjugate_Correction");
}

REAL HIT::Recalculate_Reynolds_Lambda() {
    double re = 0.0;
    SPNS_FORWARD(spns_recalculate_reynolds_lambda(h, &re), "Recalculate_Reynolds_Lambda");
    spns_scalars s;
    pull_scalars(this, s);
    ReLambda = re; Ek_Tot = s.Ek_Tot; Ok_Tot = s.Ok_Tot;
    return ReLambda;
}

void HIT::Forcing_Reynolds_Lambda(const REAL ReLambda_) {
    SPNS_FORWARD(spns_forcing_reynolds_lambda(h, ReLambda_), "Forcing_Reynolds_Lambda");
    spns_scalars s;
    pull_scalars(this, s);
    nu = s.nu; Ek_Tot = s.Ek_Tot; Ok_Tot = s.Ok_Tot;
}

REAL HIT::Recalculate_Enstrophy() {
    double ok = 0.0;
    SPNS_FORWARD(spns_recalculate_enstrophy(h, &ok), "Recalculate_Enstrophy");
    Ok_Tot = ok;
    return Ok_Tot;
}

REAL HIT::Recalculate_Energy() {
    double ek = 0.0;
    SPNS_FORWARD(spns_recalculate_energy(h, &ek), "Recalculate_Energy");
    Ek_Tot = ek;
    return Ek_Tot;
}

// src/HIT_LES.cpp:1137-1214 / :1261-1266: Ek[K] for K=0..last_rad_max, written as
// "K<TAB>Ek[K]" lines when a file name is given.
REAL HIT::Recalculate_Energy_Cascade(const char *filename) {
    double tot = 0.0;
    SPNS_FORWARD(spns_recalculate_energy_cascade(h, Ek, &tot), "Recalculate_Energy_Cascade");
    Ek_Tot = tot;
    if (filename) {
        std::ofstream out(filename);
        if (!out.is_open()) printf("WARNING: HIT::Integrate_Field(): Error opening \"%s\".\n", filename);
        for (ptrdiff_t K = 0; K <= last_rad_max; K++) out << K << "\t" << Ek[K] << "\n";
    }
    return Ek_Tot;
}

void HIT::Check_PhysFour_Energy(const REAL atol) {
    int ok = 0;
    double d1 = 0.0, d2 = 0.0;
    SPNS_FORWARD(spns_check_physfour_energy(h, atol, &ok, &d1, &d2), "Check_PhysFour_Energy");
    spns_scalars s;
    pull_scalars(this, s);
    Ek_Tot = s.Ek_Tot;   // the reference's check runs Recalculate_Energy (src/HIT_LES.cpp:1242)
    if (!ok) crash("Ek differences exceed tolerance [EkReal vs EkFour %e, EkSpNS vs EkFour: %e]\n", d1, d2);
}

// src/HIT_LES.cpp:1297-1319: spectra of Q_G, Q_S, R_G, R_S and V^2 of the
// velocity-gradient tensor, each written as "K<TAB>value" lines (the format of
// src/HIT_LES.cpp:1180-1187) when its file name is given.  They are computed
// from the current spectral state.
void HIT::Recalculate_Invariants_Distribution(const char *filename[5]) {
    std::vector<double> sp(5 * (size_t)(last_rad_max + 1));
    SPNS_FORWARD(spns_invariant_spectra(h, sp.data()), "Recalculate_Invariants_Distribution");
    if (!filename) return;
    for (int c = 0; c < 5; c++) {
        if (!filename[c]) continue;
        std::ofstream out(filename[c]);
        if (!out.is_open()) printf("WARNING: HIT::Integrate_Field(): Error opening \"%s\".\n", filename[c]);
        for (ptrdiff_t K = 0; K <= last_rad_max; K++) out << K << "\t" << sp[c * (size_t)(last_rad_max + 1) + K] << "\n";
    }
}

// src/HIT_LES_output.cpp:8-10, 20-64: the retained Fourier coefficients of
// u, v, w in the reference's dealiased order ([ky][kx][kz], FFT order, which is
// the compact layout of libspns), components one after another.  Each
// component takes exactly its number of retained modes; the reference reserves
// ActualNx*ActualNy*(ActualNz/2+1) modes per component, which for even N is
// fewer than it writes (the components overlap), so files from even-N runs differ.
void HIT::FourierVelocity_to_BinaryFile(char const *const filename) const {
    Binding &b = binding_of(this);
    int Kx = 0, Ky = 0, Kz = 0;
    check(b.h, spns_spectral_dims(b.h, &Kx, &Ky, &Kz), "spns_spectral_dims");
    std::vector<double> uvw(3 * 2 * (size_t)Kx * Ky * Kz);
    check(b.h, spns_get_spectral(b.h, uvw.data()), "spns_get_spectral");
    FILE *f = fopen(filename, "wb");
    if (!f) crash("FourierVelocity_to_BinaryFile(): cannot open \"%s\"", filename);
    if (fwrite(uvw.data(), sizeof(double), uvw.size(), f) != uvw.size()) crash("short write to \"%s\"", filename);
    fclose(f);
}

// src/HIT_LES_output.cpp:12-14, 67-115: u, v, w on the true FFT grid
// (ActualMx x ActualMy x ActualMz, [x][y][z]), components one after another.
// The grid values are computed from the current spectral state.
void HIT::RealVelocity_to_BinaryFile(char const *const filename) const {
    Binding &b = binding_of(this);
    int mx = 0, my = 0, mz = 0;
    check(b.h, spns_physical_dims(b.h, &mx, &my, &mz), "spns_physical_dims");
    std::vector<double> uvw(3 * (size_t)mx * my * mz);
    check(b.h, spns_get_physical(b.h, uvw.data()), "spns_get_physical");
    FILE *f = fopen(filename, "wb");
    if (!f) crash("RealVelocity_to_BinaryFile(): cannot open \"%s\"", filename);
    if (fwrite(uvw.data(), sizeof(double), uvw.size(), f) != uvw.size()) crash("short write to \"%s\"", filename);
    fclose(f);
}
