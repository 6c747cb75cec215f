// fft_package_forwarding.cpp -- the members of the reference class FFT_package
// (src/FFTW_package.h of adalbal/SpNS, compiled unchanged) for the GPU drop-in:
// the transforms run inside libspns, so the package plans nothing and allocates
// nothing.  This unit replaces src/FFTW_package.cpp.  HIT_LES.h embeds an
// FFT_package member; constructing it must stay cheap, and any direct
// transform request is an error.
#include "FFTW_package.h"

void FFT_package::FFT_init() {
    alloc_local = 0;
    local_n0 = Mx;        // one rank holds every x plane and every ky row
    local_0_start = 0;
    local_n1 = My;
    local_1_start = 0;
    r2c_plan = nullptr;
    c2r_plan = nullptr;
    complex_3D = nullptr;
    real_3D = nullptr;
}

void FFT_package::FFT_destroy() {}

void FFT_package::FFTWr2c(REAL *rin, COMPLEX *cout) {
    (void)rin; (void)cout;
    crash("FFT_package::FFTWr2c: host transforms are not available in the libspns drop-in");
}

void FFT_package::IFFTWc2r(COMPLEX *cin, REAL *rout) {
    (void)cin; (void)rout;
    crash("FFT_package::IFFTWc2r: host transforms are not available in the libspns drop-in");
}

void FFT_package::Fourier_Normalization(REAL *phi, bool const *const relevant) {
    (void)phi; (void)relevant;
    crash("FFT_package::Fourier_Normalization: not available in the libspns drop-in");
}

void FFT_package::Fourier_Normalization(COMPLEX *phi, bool const *const relevant) {
    (void)phi; (void)relevant;
    crash("FFT_package::Fourier_Normalization: not available in the libspns drop-in");
}

void FFT_package::Fourier_Normalization(REAL *phi) {
    (void)phi;
    crash("FFT_package::Fourier_Normalization: not available in the libspns drop-in");
}
