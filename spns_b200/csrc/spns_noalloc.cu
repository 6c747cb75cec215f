// spns_noalloc.cu -- energy spectrum of a spectral velocity without any device
// allocation.
//
// Some callers cannot call cudaMalloc when they need the spectrum:
//   * a host framework that owns all device memory through its own pool (a
//     caching allocator that has reserved the free memory): a foreign
//     cudaMalloc then fails for want of memory, or fragments the pool;
//   * a latency-critical loop that must not stall the other streams of the
//     device: cudaMalloc and cudaFree can synchronise the whole device.
// For them spns_energy_cascade_noalloc_f64 computes E(K) straight from device
// pointers they already own, with its working bins in a fixed array compiled
// into the library.  The call copies E(K) to the host and synchronises the
// given stream before it returns.
//
// The working array is a file-scope __device__ array of SPNS_NOALLOC_MAX_BINS
// energy bins plus as many enstrophy bins (32 KiB): every GPU that loads the
// library holds it until the process exits.  All calls on a device share it and
// it keeps the contents of the last call, so each call clears it first; calls
// whose work overlaps on the GPU (different streams, or different host threads
// on one device) race on it and must be serialised by the caller.  The array's
// device address and the device's SM count are looked up by the first call on
// each device and kept for the life of the process: that first call should come
// before any stream capture is under way on the device, and the entry point must
// not be used after the host program calls cudaDeviceReset on that device.
#include "spns.h"
#include "solver_kernels.cuh"

#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

using namespace spns;

static __device__ __align__(256) double g_noalloc_bins[2 * SPNS_NOALLOC_MAX_BINS];

// Error text of calls without a handle, returned by spns_last_error(NULL) (spns.cu).
void spns_set_handleless_error(const char *msg);

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
double *g_bins_addr[kMaxDevices] = {nullptr};
int g_sm_count[kMaxDevices] = {0};

int noalloc_fail(int code, const char *msg) {
    spns_set_handleless_error(msg);
    return code;
}

// Device address of the working array on the current device, and the device's
// SM count (grid size of the shell sums).  The host-side symbol is only a
// stand-in for the array, so the address is looked up once per device, with
// that device current, and cached.
int bins_address(int dev, double **out, int *sms) {
    if (dev < 0 || dev >= kMaxDevices) return noalloc_fail(SPNS_ERR_INVALID_ARGUMENT, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_bins_addr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_bins);
        if (e != cudaSuccess) {
            char buf[256];
            snprintf(buf, sizeof(buf), "cudaGetSymbolAddress of the working bins failed: %s", cudaGetErrorString(e));
            return noalloc_fail(SPNS_ERR_CUDA, buf);
        }
        int n = 0;
        e = cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess || n < 1) return noalloc_fail(SPNS_ERR_CUDA, "cudaDeviceGetAttribute(SM count) failed");
        g_sm_count[dev] = n;
        g_bins_addr[dev] = static_cast<double *>(p);
    }
    *out = g_bins_addr[dev];
    *sms = g_sm_count[dev];
    return SPNS_OK;
}
} // namespace

extern "C" int spns_energy_cascade_noalloc_f64(const void *uvw_dev, int Kx, int Ky, int Kz, int Lx_factor, int Ly_factor,
                                              int Lz_factor, double *Ek, int nbins, double *ek_tot, void *stream) {
    if (!uvw_dev || !Ek || nbins < 1 || Kx < 1 || Ky < 1 || Kz < 1 || (Kx % 2) == 0 || (Ky % 2) == 0 || Lx_factor < 1 ||
        Ly_factor < 1 || Lz_factor < 1)
        return noalloc_fail(SPNS_ERR_INVALID_ARGUMENT, "invalid argument (null pointer, non-positive or even size)");
    if (nbins > SPNS_NOALLOC_MAX_BINS) {
        char buf[200];
        snprintf(buf, sizeof(buf), "nbins=%d exceeds the %d bins of the fixed working array", nbins, SPNS_NOALLOC_MAX_BINS);
        return noalloc_fail(SPNS_ERR_UNSUPPORTED_SIZE, buf);
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return noalloc_fail(SPNS_ERR_CUDA, cudaGetErrorString(e));
    double *bins = nullptr;
    int sms = 0;
    int rc = bins_address(dev, &bins, &sms);
    if (rc) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    Geo g{};
    g.Kx = Kx; g.Ky = Ky; g.Kz = Kz;
    g.hx = (Kx - 1) / 2; g.hy = (Ky - 1) / 2; g.hz = Kz - 1;
    g.sx = Lx_factor; g.sy = Ly_factor; g.sz = Lz_factor;
    g.S0 = (long long)Kx * Ky * Kz;
    g.y0 = 0;
    g.Kyg = Ky;
    const double2 *u = static_cast<const double2 *>(uvw_dev);

    // The array keeps the previous call's sums: clear the bins used here.
    e = cudaMemsetAsync(bins, 0, sizeof(double) * 2 * (size_t)nbins, st);
    if (e != cudaSuccess) return noalloc_fail(SPNS_ERR_CUDA, cudaGetErrorString(e));
    const long long n = g.S0;
    const long long cap = (long long)SHELL_BLOCKS_PER_SM * sms;   // one wave of resident blocks
    const int blocks = (int)((n + 255) / 256 < cap ? (n + 255) / 256 : cap);
    k_shell_sums<double><<<blocks, 256, sizeof(double) * 2 * nbins, st>>>(
        g, (const cx<double> *)u, (const cx<double> *)(u + g.S0), (const cx<double> *)(u + 2 * g.S0), nullptr, nullptr, nullptr, nbins - 1, bins,
        bins + nbins);
    e = cudaGetLastError();
    if (e != cudaSuccess) return noalloc_fail(SPNS_ERR_CUDA, cudaGetErrorString(e));
    e = cudaMemcpyAsync(Ek, bins, sizeof(double) * nbins, cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return noalloc_fail(SPNS_ERR_CUDA, cudaGetErrorString(e));
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return noalloc_fail(SPNS_ERR_CUDA, cudaGetErrorString(e));
    if (ek_tot) {
        double s = 0.0;
        for (int K = 0; K < nbins; K++) s += Ek[K];
        *ek_tot = s;
    }
    return SPNS_OK;
}
