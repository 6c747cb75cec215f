// handle.h -- the solver handle of libspns and the launch machinery shared by
// the translation units (spns.cu: C ABI; spns_f64.cu / spns_f32.cu: the passes
// of one step instantiated for one precision).
#pragma once
#include "spns.h"
#include "solver_kernels.cuh"

#include <type_traits>
#include "edge_kernels.cuh"
#include "zpass_staged.cuh"
#include "axis_tma.cuh"

#include <cuda_runtime.h>

#include <cmath>
#include <map>
#include <string>
#include <utility>
#include <vector>

// ---------------------------------------------------------------------------
// Compiled FFT lengths and launch shapes
// ---------------------------------------------------------------------------
#define SPNS_FOR_EACH_LENGTH(X) X(48) X(72) X(96) X(144) X(192) X(288) X(384) X(768) X(1536)

inline bool spns_length_supported(int L) {
#define SPNS_CASE(n) if (L == n) return true;
    SPNS_FOR_EACH_LENGTH(SPNS_CASE)
#undef SPNS_CASE
    return false;
}

// Tile shapes per pass (complex values per thread E, threads per block),
// chosen by timing the N=512 step on B200.
template <typename T, int L, int E_, int THR> struct ShapeT {
    static constexpr int E = E_;             // complex values per thread
    static constexpr int Q = L / E;          // threads per pencil
    static constexpr int P0 = THR / Q;
    static constexpr int P = P0 >= 32 ? 32 : P0 >= 16 ? 16 : P0 >= 8 ? 8 : 4; // pencils per block
    static constexpr int THREADS = P * Q;
    static constexpr size_t SMEM_ROW = (size_t)L * P * sizeof(spns::cx<T>);
    static constexpr size_t SMEM_PEN = (size_t)spns::SmPencil<T, L, E_>::PITCH * P * sizeof(spns::cx<T>);
};
// Double precision shapes (E, threads per block); single precision has its own
// (half the register and shared-memory footprint per value).
#ifndef SPNS_F32_K1_E
#define SPNS_F32_K1_E 12
#endif
#ifndef SPNS_F32_K1_T
#define SPNS_F32_K1_T 256
#endif
#ifndef SPNS_K1_E
#define SPNS_K1_E 12          // double inverse x pass: complex values per thread
#endif
#ifndef SPNS_K5_E
#define SPNS_K5_E 24          // double forward x pass: complex values per thread
#endif
#ifndef SPNS_K5_T
#define SPNS_K5_T 128         // double forward x pass: threads per block
#endif
#ifndef SPNS_K1_T
#define SPNS_K1_T 256         // double inverse x pass: threads per block
#endif
#ifndef SPNS_K2_E
#define SPNS_K2_E 24          // double y passes: complex values per thread
#endif
#ifndef SPNS_K2_T
#define SPNS_K2_T 256         // double y passes: threads per block
#endif
#ifndef SPNS_F32_K2_E
#define SPNS_F32_K2_E 24
#endif
#ifndef SPNS_F32_K2_T
#define SPNS_F32_K2_T 512
#endif
#ifndef SPNS_F32_K5_E
#define SPNS_F32_K5_E 24
#endif
#ifndef SPNS_F32_K5_T
#define SPNS_F32_K5_T 256
#endif
#ifndef SPNS_F32_Z_E
#define SPNS_F32_Z_E 12
#endif
#ifndef SPNS_F32_Z_T
#define SPNS_F32_Z_T 128
#endif
#ifndef SPNS_Z_THREADS
#define SPNS_Z_THREADS 128    // threads per block in the double z pass (2 blocks per SM)
#endif
#ifndef SPNS_Z_E
#define SPNS_Z_E 12           // complex values per thread in the double z pass (3 pairs in registers)
#endif
#ifndef SPNS_Z_STAGE
#define SPNS_Z_STAGE 1        // double z pass: stage the six input fields in shared memory
#endif
#ifndef SPNS_F32_Z_STAGE
#define SPNS_F32_Z_STAGE 1
#endif
#ifndef SPNS_Z_E_ROT
#define SPNS_Z_E_ROT SPNS_Z_E
#endif
#ifndef SPNS_F32_Z_E_ROT
#define SPNS_F32_Z_E_ROT 12
#endif
template <typename T> struct ShapeSel {
    static constexpr bool D = sizeof(T) == 8;
    static constexpr int K1_E = D ? SPNS_K1_E : SPNS_F32_K1_E, K1_T = D ? SPNS_K1_T : SPNS_F32_K1_T;
    static constexpr int K2_E = D ? SPNS_K2_E : SPNS_F32_K2_E, K2_T = D ? SPNS_K2_T : SPNS_F32_K2_T;
    static constexpr int K5_E = D ? SPNS_K5_E : SPNS_F32_K5_E, K5_T = D ? SPNS_K5_T : SPNS_F32_K5_T;
    static constexpr int Z_E = D ? SPNS_Z_E : SPNS_F32_Z_E, Z_T = D ? SPNS_Z_THREADS : SPNS_F32_Z_T;
    static constexpr bool Z_STAGE = D ? SPNS_Z_STAGE : SPNS_F32_Z_STAGE;
    static constexpr int Z_E_ROT = D ? SPNS_Z_E_ROT : SPNS_F32_Z_E_ROT;   // rotational/velocity z pass
};
template <typename T, int L> using ShapeK1 = ShapeT<T, L, ShapeSel<T>::K1_E, ShapeSel<T>::K1_T>;   // inverse x
template <typename T, int L> using ShapeK2 = ShapeT<T, L, ShapeSel<T>::K2_E, ShapeSel<T>::K2_T>;   // inverse y (and forward y)
template <typename T, int L> using ShapeK5 = ShapeT<T, L, ShapeSel<T>::K5_E, ShapeSel<T>::K5_T>;   // forward x
template <typename T, int L> using Shape = ShapeT<T, L, 24, 128>;                                   // edge planes, test lines
// Alternate shapes the autotuner (spns_autotune) can pick per pass for short
// lengths: E = 6 values per thread (radix plan 6 x 2 x ... or 6 x 6 x ...),
// four times the threads per pencil of the default E = 24, which small boxes
// need to fill the GPU.  Compiled for the step forms at L <= SPNS_ALT_MAX_L.
#ifndef SPNS_ALT_MAX_L
#define SPNS_ALT_MAX_L 192
#endif
constexpr int SPNS_ALT_E = 6;
template <int L, int MODE> constexpr bool shape_alt_ok() {
    return L <= SPNS_ALT_MAX_L && (MODE == spns::MODE_ROT || MODE == spns::MODE_ADV || MODE == spns::MODE_LES);
}
template <typename T, int L, int ALT> using ShapeK1A = typename std::conditional<ALT != 0, ShapeT<T, L, SPNS_ALT_E, ShapeSel<T>::K1_T>, ShapeK1<T, L>>::type;
template <typename T, int L, int ALT> using ShapeK2A = typename std::conditional<ALT != 0, ShapeT<T, L, SPNS_ALT_E, ShapeSel<T>::K2_T>, ShapeK2<T, L>>::type;
template <typename T, int L, int ALT> using ShapeK5A = typename std::conditional<ALT != 0, ShapeT<T, L, SPNS_ALT_E, ShapeSel<T>::K5_T>, ShapeK5<T, L>>::type;

// Rotational z pass with pair-by-pair bulk-copy staging, persistent
// (k3_rot_staged, zpass_staged.cuh): used at lengths from SPNS_ZS_MIN_L up to 768.
// Per precision: E values per thread, PB pencils per block, SLOTS physical slots
// in shared memory (of four), MINB resident blocks per SM for the register budget.
#ifndef SPNS_ZS_MIN_L
#define SPNS_ZS_MIN_L 768         // double: measured 14.65 against 14.93 ms at 768, slower at 384
#endif
#ifndef SPNS_F32_ZS_MIN_L
#define SPNS_F32_ZS_MIN_L 100000  // single: off (12.29 against 11.61 ms at 768)
#endif
#ifndef SPNS_ZS_E
#define SPNS_ZS_E 12
#endif
// Double at 768, N=512: one pencil per block, two of the four slots in shared memory and
// 6 blocks per SM (12 warps) 12.97 ms; two pencils per block with one slot and 3 blocks
// 13.74, with no slot and 2 blocks 13.94; one pencil with one slot 13.19 (6 blocks), 14.42 (7).
#ifndef SPNS_ZS_PB
#define SPNS_ZS_PB 1
#endif
#ifndef SPNS_ZS_SLOTS
#define SPNS_ZS_SLOTS 2
#endif
#ifndef SPNS_ZS_MINB
#define SPNS_ZS_MINB 6
#endif
#ifndef SPNS_F32_ZS_E
#define SPNS_F32_ZS_E 12
#endif
#ifndef SPNS_F32_ZS_PB
#define SPNS_F32_ZS_PB 2
#endif
#ifndef SPNS_F32_ZS_SLOTS
#define SPNS_F32_ZS_SLOTS 0
#endif
#ifndef SPNS_F32_ZS_MINB
#define SPNS_F32_ZS_MINB 4
#endif
template <typename T, int L> struct ZStagedShape {
    static constexpr bool D = sizeof(T) == 8;
    static constexpr int E = D ? SPNS_ZS_E : SPNS_F32_ZS_E;
    static constexpr int PB = D ? SPNS_ZS_PB : SPNS_F32_ZS_PB;
    static constexpr int SLOTS = D ? SPNS_ZS_SLOTS : SPNS_F32_ZS_SLOTS;
    static constexpr int MINB = D ? SPNS_ZS_MINB : SPNS_F32_ZS_MINB;
    static constexpr bool ON = L >= (D ? SPNS_ZS_MIN_L : SPNS_F32_ZS_MIN_L) && L <= 768 && L % E == 0 && spns::n_stages(L, E) > 0;
};

// x/y passes with TMA-moved tiles (k_axis_tma, axis_tma.cuh): double precision,
// lengths from SPNS_AX_TMA_MIN_L, E values per thread and P pencils per block.
// Off by default: two whole-field tiles per block leave one block (8 warps) per
// SM, and at N=512 the y pass took 11.65 ms against 7.03 ms for k2_inv_y (E=12,
// 512 threads: 11.13 ms; P=4: 19.0 ms).  Build with -DSPNS_AX_TMA_MIN_L=384 to use it.
#ifndef SPNS_AX_TMA_MIN_L
#define SPNS_AX_TMA_MIN_L 100000
#endif
#ifndef SPNS_AX_TMA_E
#define SPNS_AX_TMA_E 24
#endif
#ifndef SPNS_AX_TMA_P
#define SPNS_AX_TMA_P 8
#endif
#ifndef SPNS_AX_TMA_R
#define SPNS_AX_TMA_R 128        // rows per TMA box
#endif
template <typename T, int L> struct AxisTmaShape {
    static constexpr int E = SPNS_AX_TMA_E, P = SPNS_AX_TMA_P;
    static constexpr bool ON = sizeof(T) == 8 && L >= SPNS_AX_TMA_MIN_L && L % E == 0 && L % SPNS_AX_TMA_R == 0 &&
                               spns::n_stages(L, E) > 0 && 2 * (size_t)L * P * sizeof(spns::cx<T>) + 160 <= 227 * 1024;
    static constexpr size_t SMEM = 2 * (size_t)L * P * sizeof(spns::cx<T>) + 128 + 2 * sizeof(unsigned long long);
};

// z pass: pencils per block limited by the shared memory of the exchange
// buffer plus the physical fields kept per pencil.
template <typename T, int L, int MODE, int ALT = 0> struct Shape3 {
    static constexpr int E = ALT ? SPNS_ALT_E : (MODE == spns::MODE_ROT || MODE == spns::MODE_VEL) ? ShapeSel<T>::Z_E_ROT : ShapeSel<T>::Z_E;
    static constexpr int Q = L / E;
    static constexpr int ZT = ShapeSel<T>::Z_T / Q;
    static constexpr int P0 = ZT >= 32 ? 32 : ZT >= 16 ? 16 : ZT >= 8 ? 8 : ZT >= 4 ? 4 : ZT >= 2 ? 2 : 1;
    static constexpr size_t PER_PEN = (size_t)spns::pencil_pitch<T, L, E>() * sizeof(spns::cx<T>) + (size_t)spns::K3Reg<T, MODE, E>::NSM * L * sizeof(T);
    static constexpr int PMAX = (int)((200 * 1024) / PER_PEN);
    static constexpr int P = P0 <= PMAX ? P0 : PMAX >= 16 ? 16 : PMAX >= 8 ? 8 : PMAX >= 4 ? 4 : PMAX >= 2 ? 2 : 1;
    static constexpr int THREADS = P * Q;
    static constexpr size_t SMEM = PER_PEN * P;
};

// ---------------------------------------------------------------------------
// Handle
// ---------------------------------------------------------------------------
// Device buffers are typed by the precision of the handle: element cx<double>
// (SPNS_FP64) or cx<float> (SPNS_FP32_HILO; the spectral state and the
// kappa-scheme history then carry a low part Ulo/Uplo with u = hi + lo).
struct spns_handle {
    spns_hit_args a;
    int prec = SPNS_FP64;
    size_t csz = 16;                                 // bytes per complex element
    spns::Geo g;
    spns::StepConsts c;
    int last_rad = 0, last_rad_max = 0;
    double delta = 0, Ek_init = 0, Ek_init_file = 0, Enstrophy_init_file = 0;
    cudaStream_t st = nullptr;
    spns::DevScalars *ds = nullptr;
    void *U = nullptr, *Ulo = nullptr;               // state u^n (3 fields of S0)
    void *Up = nullptr, *Uplo = nullptr;             // u^{n-1} (kappa scheme)
    void *R = nullptr;                               // R^{n-1}
    void *B1 = nullptr, *B2 = nullptr;               // S1 and S2 work buffers
    int nB1 = 0, nB2 = 0;
    double *bins = nullptr;                          // Ek[0..Kmax], Om[0..Kmax]
    double *FT = nullptr, *forced = nullptr;
    int forced_cap = 0;
    double *phys = nullptr;
    void *edge = nullptr;                            // edge-correction planes (rotational form)
    void *inv_B1 = nullptr, *inv_B2 = nullptr;       // invariant spectra: advective-size work buffers (on first use)
    double *inv_bins = nullptr;                      // 5 spectra, then the nu_t accumulators
    double nut_stats[3] = {0.0, 0.0, 0.0};           // mean, rms, max of nu_t at the last invariant pass
    bool edge_axis[3] = {false, false, false};       // axes whose +-N/2 planes alias (M = 3h)
    std::map<int, void *> tw;                        // twiddle tables per length (precision of the handle)
    std::map<std::pair<int, const void *>, CUtensorMap> tmaps;   // TMA tensor maps per (pass, input buffer)
    int sms = 0;                                     // SM count of the handle's device
    // slab decomposition (spns_slab_create): this rank holds the compact ky rows
    // [g.y0, g.y0 + g.Ky) of the state and, in the y and z passes, the x planes
    // [x0, x0 + gx.Mx); B1 holds the x pass's rows, B1x/B2x the x planes' S1/S2
    // fields (B2 = B2x, also the nonlinear term), XS/XR the all-to-all staging
    int slab_ranks = 0, slab_rank = 0, x0 = 0;
    spns::Geo gx;
    void *B1x = nullptr, *XS = nullptr, *XR = nullptr;
    size_t xelems = 0;                               // complex elements of XS and of XR
    spns::SlabRanges yr, xr;                         // every rank's ky rows and x planes
    std::string err;
    int kernels_per_step = 0;
    int edge_launches = 0;                           // launches of the edge correction in the last step
    // CUDA graphs of one step, per parity of the state-buffer swap (kappa scheme)
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    // launch shape per pass (index 1..5 = K1..K5): 0 default, 1 the alternate of
    // shape_alt_ok lengths; set by spns_autotune or from its per-process cache
    unsigned char shape_alt[6] = {0, 0, 0, 0, 0, 0};
    void *U0 = nullptr;                              // state buffer of parity 0
    bool use_graphs = true;
    // optional per-kernel event profile of the next steps (spns_profile_*)
    std::vector<cudaEvent_t> prof_ev;
    std::vector<std::string> prof_names;
    int prof_cap_steps = 0, prof_steps = 0, prof_nk = 0;
};

// Records the error text (handle, or the handle-less slot) and returns code.
int spns_fail(spns_handle *h, int code, const char *fmt, ...);

#define CK(call)                                                                                   \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            return spns_fail(h, e_ == cudaErrorMemoryAllocation ? SPNS_ERR_OUT_OF_MEMORY : SPNS_ERR_CUDA, \
                             "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
    } while (0)

#define CKL()                                                                                      \
    do {                                                                                           \
        cudaError_t e_ = cudaGetLastError();                                                       \
        if (e_ != cudaSuccess)                                                                     \
            return spns_fail(h, SPNS_ERR_CUDA, "kernel launch failed: %s (%s:%d)", cudaGetErrorString(e_), \
                             __FILE__, __LINE__);                                                  \
    } while (0)

#define LAUNCH(expr)                                                                              \
    do {                                                                                          \
        cudaError_t e_ = (expr);                                                                  \
        if (e_ != cudaSuccess)                                                                    \
            return spns_fail(h, SPNS_ERR_CUDA, "launch failed: %s (%s:%d)", cudaGetErrorString(e_), __FILE__, __LINE__); \
    } while (0)

#define DISPATCH(Lval, call)                                                                 \
    switch (Lval) {                                                                          \
    case 48: { constexpr int LL = 48; call; } break;                                         \
    case 72: { constexpr int LL = 72; call; } break;                                         \
    case 96: { constexpr int LL = 96; call; } break;                                         \
    case 144: { constexpr int LL = 144; call; } break;                                       \
    case 192: { constexpr int LL = 192; call; } break;                                       \
    case 288: { constexpr int LL = 288; call; } break;                                       \
    case 384: { constexpr int LL = 384; call; } break;                                       \
    case 768: { constexpr int LL = 768; call; } break;                                       \
    case 1536: { constexpr int LL = 1536; call; } break;                                     \
    default: return spns_fail(h, SPNS_ERR_UNSUPPORTED_SIZE, "FFT length %d is not compiled", Lval); \
    }

// Twiddle table w_L^m = exp(-2 pi i m / L), computed in extended precision, followed
// by the per-stage sub-tables w_n^m = w_L^{m L/n} (copies of base entries) for every
// divisor n < L of L, in increasing n (spns::tw_sub_offset), and the power tables
// w_n^{r k} for r = 2, 4, 8 (spns::tw_pow_offset); allocated in stream
// order on `st` (no device-wide synchronisation).
template <typename T> inline void *spns_make_twiddles(int L, cudaStream_t st) {
    const int total = spns::tw_full_size(L);
    std::vector<spns::cx<T>> t(total);
    for (int m = 0; m < L; m++) {
        long double ang = 2.0L * 3.14159265358979323846264338327950288L * (long double)m / (long double)L;
        t[m].x = (T)cosl(ang);
        t[m].y = (T)(-sinl(ang));
    }
    for (int n = 2; n < L; n++) {
        if (L % n) continue;
        const int off = spns::tw_sub_offset(L, n);
        for (int m = 0; m < n; m++) t[off + m] = t[(long long)m * (L / n)];
    }
    for (int r = 2; r <= 8; r *= 2)
        for (int n = 2; n <= L; n++) {
            if (L % n) continue;
            const int off = spns::tw_pow_offset(L, n, r);
            for (int k = 0; k < n; k++) t[off + k] = t[(long long)((r * k) % n) * (L / n)];
        }
    void *d = nullptr;
    if (cudaMallocAsync(&d, sizeof(spns::cx<T>) * total, st) != cudaSuccess) return nullptr;
    if (cudaMemcpyAsync(d, t.data(), sizeof(spns::cx<T>) * total, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
        cudaFreeAsync(d, st);
        return nullptr;
    }
    return d;
}

// Opt-in to the dynamic shared memory of a launch.  Set even below 48 KB: the
// kernel's static shared memory counts against the same 48 KB default limit.
template <class K> inline cudaError_t spns_set_smem(K kern, size_t bytes) {
    if (bytes <= 16 * 1024) return cudaSuccess;
    return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

// Precision-specific operations of a handle (spns_f64.cu, spns_f32.cu).
struct PrecOps {
    int (*step_once)(spns_handle *h);                         // one New_Fractional_Step_Method
    int (*run_velocity)(spns_handle *h, double *phys);        // inverse transform of u (CFL maxima)
    int (*shell_sums)(spns_handle *h);                        // E(K), Om(K) of u into h->bins
    int (*forcing_scale)(spns_handle *h, int last_eff, int nullify); // u *= FT[K]
    int (*conj_correction)(spns_handle *h);                   // kz=0 conjugate correction
    int (*seed_draw)(spns_handle *h, unsigned long long seed, int lim_x, int lim_y, int lim_z); // Philox field, unscaled
    int (*invariant_spectra)(spns_handle *h, double *out);    // 5 spectra of the gradient invariants
    int (*slab_phase)(spns_handle *h, int phase);             // one phase of a slab-decomposed step
    // one step of n members of h0's class in one launch per pass (device table `tab`), on stream st
    int (*batch_step)(spns_handle *h0, const spns::BatchMember *tab, int n, cudaStream_t st);
};

// Lengths with batched pass kernels (ensembles of small boxes).
#define SPNS_DISPATCH_BATCH(Lval, call)                                                     \
    switch (Lval) {                                                                          \
    case 48: { constexpr int LL = 48; call; } break;                                         \
    case 72: { constexpr int LL = 72; call; } break;                                         \
    case 96: { constexpr int LL = 96; call; } break;                                         \
    case 144: { constexpr int LL = 144; call; } break;                                       \
    case 192: { constexpr int LL = 192; call; } break;                                       \
    default: return spns_fail(h, SPNS_ERR_UNSUPPORTED_SIZE, "no batched kernels at FFT length %d", Lval); \
    }
inline bool spns_batch_length(int L) { return L == 48 || L == 72 || L == 96 || L == 144 || L == 192; }
extern const PrecOps spns_ops_f64;
extern const PrecOps spns_ops_f32;
inline const PrecOps &spns_ops(const spns_handle *h) { return h->prec == SPNS_FP64 ? spns_ops_f64 : spns_ops_f32; }
