// solver_kernels.cuh -- the five fused passes of one pseudospectral step and the
// small kernels around them (B200 / sm_100a, bandwidth-bound, no tensor cores).
//
// Data layout in HBM (complex elements, kz contiguous everywhere):
//   S0 compact spectral state   [iy][ix][kz]   Ky x Kx x Kz   (retained modes only)
//   S1 after the x transform    [iy][x][kz]    Ky x Mx x Kz
//   S2 after the y transform    [y][x][kz]     My x Mx x Kz
// Kx=2*hx+1 (kx=-hx..hx), Ky=2*hy+1, Kz=hz+1 (kz=0..hz) with h=N/2: the 3/2-rule
// box of the reference (src/HIT_LES.cpp:858-873, both +-N/2 kept for even N).
// Wavenumbers are k = s*m with s the length factor of the axis, so a non-cubic
// box of the reference (src/MAIN.cpp:216-260, src/HIT_LES.cpp:867-871) runs on
// its true grid (ActualM) instead of the expanded one.
//
// Pass plan of one step (DNS, advective form of the reference):
//   K1 inverse x : S0 u,v,w          -> S1 u,v,w, du/dx, dv/dx, dw/dx
//   K2 inverse y : S1 (6)            -> S2 + du/dy, dv/dy, dw/dy (9)
//   K3 z         : c2r of 12 fields (dz from u,v,w), conv = u_j d_j u_i (+ CFL
//                  maxima), r2c -> S2 conv_x, conv_y, conv_z
//   K4 forward y : S2 (3)            -> S1 (3)
//   K5 forward x : S1 (3)            -> S0 G (3)
//   K6 sweep     : G, u, R^{n-1} [, u^{n-1}] -> 1/M^3, R, Coriolis, forcing,
//                  AB2 or kappa-scheme predictor, projection -> u^{n+1}, R^n.
// The rotational form (opt-in) carries u and the vorticity instead (5, 6 and 6
// fields in K1, K2, K3).  LES (Smagorinsky) adds the SGS stress, whose
// divergence is folded into the forward passes (i kz t_i3 in K3, i ky t_i2 in
// K4, i kx t_i1 in K5).
#pragma once
#include "fft768.cuh"

namespace spns {

enum Mode { MODE_VEL = 0, MODE_ROT = 1, MODE_ADV = 2, MODE_LES = 3, MODE_INV = 4 };
// MODE_INV: velocity-gradient invariants (post-processing, not a step): the x/y
// passes form the gradients as in MODE_ADV, the z pass forms Q_G, Q_S, R_G, R_S, V^2
// on the grid and transforms them forward, the forward y/x passes carry 5 fields.

struct Geo {
    int Kx, Ky, Kz;   // retained mode counts (Ky: rows held, the slab's in a slab decomposition)
    int hx, hy, hz;   // half widths
    int Mx, My, Mz;   // true FFT grid (Mx: x planes held, the slab's in the y/z passes of a slab decomposition)
    int sx, sy, sz;   // wavenumber scale per axis (length factor)
    long long S0, S1, S2; // elements per field in each layout
    int y0, Kyg;      // first compact ky row held and the box's compact ky count (0 and Ky on one GPU)
};

// m2 (ky/sy) of compact row iy held by this geometry
__host__ __device__ __forceinline__ int ky_mode(const Geo &g, int iy) {
    const int r = g.y0 + iy;
    return r <= g.hy ? r : r - g.Kyg;
}

// Solver scalars living in device memory (read by kernels, updated by the
// finisher), so that a captured step stays valid while they change.
struct DevScalars {
    double dt, time, nu, kappa, alpha;
    double maxvel, phi0;
    double ek_tot, ok_tot, relambda;
    double sumsq_phys;                   // sum of u^2+v^2+w^2 over the grid (energy check)
    unsigned long long max_bits[4];      // max|u|, max|v|, max|w|, max(|u|/Ax+|v|/Ay+|w|/Az)
    long long iter;
    int nonfinite, domain_err;
    int wait_timeout;                    // a bounded wait of a staged pass gave up (SPNS_ERR_TIMEOUT)
    double ef;                           // slab decomposition: this slab's energy of the forced shells
};

struct StepConsts {
    double inv_norm;      // 1/(Mx*My*Mz) of the true grid
    double omega_x, omega_y, omega_z;
    double Ax, Ay, Az, inv_Ax, inv_Ay, inv_Az;
    double C_At, Ah, t1;
    double kopt_k[2], phi[3], c[14];
    double les_ct;        // (C_Smag*delta)^2
    double fixed_dt;
    int eps_on, eps_kmin, eps_kmax;
    int rotating, self_adaptive;
};

__device__ __forceinline__ int ffreq(int a, int M) { return a <= M / 2 ? a : a - M; }

// Blocks per SM the x/y passes are compiled for (their register budget), per
// pass (1 inverse x, 2 inverse y, 4 forward y, 5 forward x).
#ifndef SPNS_AX_MINB
#define SPNS_AX_MINB 2
#endif
#ifndef SPNS_K2_MINB
#define SPNS_K2_MINB SPNS_AX_MINB
#endif
#ifndef SPNS_K1_MINB
#define SPNS_K1_MINB SPNS_AX_MINB
#endif
#ifndef SPNS_K5_MINB
#define SPNS_K5_MINB SPNS_AX_MINB
#endif
#ifndef SPNS_F32_AX_MINB
#define SPNS_F32_AX_MINB 2
#endif
template <typename T, int PASS> struct AxisMinBlocks {
    static constexpr int N = sizeof(T) == 8 ? ((PASS == 2 || PASS == 4) ? SPNS_K2_MINB : PASS == 1 ? SPNS_K1_MINB : SPNS_K5_MINB)
                                            : SPNS_F32_AX_MINB;
};

// Field counts of the work buffers per mode.
template <int MODE> struct Fields {
    static constexpr int K1 = MODE == MODE_VEL ? 3 : 6;                          // S1 after the inverse x pass
    static constexpr int K2 = MODE == MODE_VEL ? 3 : MODE == MODE_ROT ? 6 : 9;  // S2 after the inverse y pass
    static constexpr int K4 = MODE == MODE_LES ? 6 : MODE == MODE_INV ? 5 : 3;  // S1 after the forward y pass
    static constexpr int NOUT = MODE == MODE_INV ? 5 : 3;                       // compact outputs of the forward x pass
};

// ===========================================================================
// K1: inverse transform along x.  Block = (kz chunk, iy).
//   VEL: u,v,w   ROT: u,v,w and the vorticity w_x=i(ky w-kz v), w_y=i(kz u-kx w),
//   w_z=i(kx v-ky u) (ky is the block's, kx the row's)   ADV/LES: u,v,w, du/dx, dv/dx, dw/dx
// ===========================================================================
template <typename T, int L, int E, int P, int MODE>
__device__ __forceinline__ void k1_inv_x_body(Geo g, const cx<T> *__restrict__ u, const cx<T> *__restrict__ v,
                                              const cx<T> *__restrict__ w, cx<T> *__restrict__ out, const cx<T> *__restrict__ tw) {
    extern __shared__ __align__(16) unsigned char smraw[];
    const int tid = threadIdx.x, p = tid % P, q = tid / P;
    const int iy = blockIdx.y, kz = blockIdx.x * P + p;
    const bool ok = kz < g.Kz;
    const T kzf = T(g.sz * kz);
    const T kyf = T(g.sy * ky_mode(g, iy));
    SmRowMajor<T, P> sm{reinterpret_cast<cx<T> *>(smraw), p};
    const long long rb = (long long)iy * g.Kx;
#pragma unroll 1
    for (int f = 0; f < Fields<MODE>::K1; f++) {
        cx<T> r[E];
#pragma unroll
        for (int e = 0; e < E; e++) {
            const int row = in_row<L, E, true>(q, e);
            const int m1 = ffreq(row, L);
            cx<T> val = zero<T>();
            if (ok && m1 <= g.hx && m1 >= -g.hx) {
                const long long idx = (rb + (m1 >= 0 ? m1 : m1 + g.Kx)) * g.Kz + kz;
                const T kx = T(g.sx * m1);
                if (f == 0) val = u[idx];
                else if (f == 1) val = v[idx];
                else if (f == 2) val = w[idx];
                else if (MODE == MODE_ROT) {
                    if (f == 3) { cx<T> b = v[idx], c = w[idx]; val = mul_i(mk<T>(kyf * c.x - kzf * b.x, kyf * c.y - kzf * b.y)); }
                    else if (f == 4) { cx<T> a = u[idx], c = w[idx]; val = mul_i(mk<T>(kzf * a.x - kx * c.x, kzf * a.y - kx * c.y)); }
                    else { cx<T> a = u[idx], b = v[idx]; val = mul_i(mk<T>(kx * b.x - kyf * a.x, kx * b.y - kyf * a.y)); }
                } else { // x-derivatives
                    const cx<T> *src = f == 3 ? u : f == 4 ? v : w;
                    val = mul_i(kx * src[idx]);
                }
            }
            r[e] = val;
        }
        fft<T, L, E, true>(r, sm, q, tw);
        if (ok) {
            cx<T> *o = out + (long long)f * g.S1 + (long long)iy * g.Mx * g.Kz + kz;
#pragma unroll
            for (int e = 0; e < E; e++) o[(long long)out_row<L, E, true>(q, e) * g.Kz] = r[e];
        }
    }
}

// ===========================================================================
// K2: inverse transform along y.  Block = (kz chunk, x).
//   ROT: u,v,w, w_x, w_y, w_z (formed by K1)
//   ADV/LES: u,v,w, du/dx,dv/dx,dw/dx, du/dy,dv/dy,dw/dy
// ===========================================================================
template <typename T, int L, int E, int P, int MODE>
__device__ __forceinline__ void k2_inv_y_body(Geo g, const cx<T> *__restrict__ in, cx<T> *__restrict__ out,
                                              const cx<T> *__restrict__ tw) {
    extern __shared__ __align__(16) unsigned char smraw[];
    const int tid = threadIdx.x, p = tid % P, q = tid / P;
    const int x = blockIdx.y, kz = blockIdx.x * P + p;
    const bool ok = kz < g.Kz;
    const T kzf = T(g.sz * kz);
    SmRowMajor<T, P> sm{reinterpret_cast<cx<T> *>(smraw), p};
    const long long col = (long long)x * g.Kz + kz;
#pragma unroll 1
    for (int f = 0; f < Fields<MODE>::K2; f++) {
        cx<T> r[E];
#pragma unroll
        for (int e = 0; e < E; e++) {
            const int row = in_row<L, E, true>(q, e);
            const int m2 = ffreq(row, L);
            cx<T> val = zero<T>();
            if (ok && m2 <= g.hy && m2 >= -g.hy) {
                const cx<T> *F = in + (long long)(m2 >= 0 ? m2 : m2 + g.Ky) * g.Mx * g.Kz + col;
                const T ky = T(g.sy * m2);
                if (MODE == MODE_VEL || MODE == MODE_ROT) {
                    val = F[(long long)f * g.S1];
                } else {
                    if (f < 6) val = F[(long long)f * g.S1];
                    else val = mul_i(ky * F[(long long)(f - 6) * g.S1]);
                }
            }
            r[e] = val;
        }
        fft<T, L, E, true>(r, sm, q, tw);
        if (ok) {
            cx<T> *o = out + (long long)f * g.S2 + col;
#pragma unroll
            for (int e = 0; e < E; e++) o[(long long)out_row<L, E, true>(q, e) * g.Mx * g.Kz] = r[e];
        }
    }
}

// ===========================================================================
// K3: along z.  c2r of two real fields per complex transform (a + i b with
// Hermitian extension; the kz=0 entries keep their real parts only, as a c2r of
// the reference does), pointwise products on the grid, r2c of the products
// (again two per transform) truncated to kz<=hz.  Block = P consecutive
// pencils; each thread keeps the values of its own grid rows in registers, so
// the inverse/forward hand-off needs no shared-memory round trip.
// ===========================================================================
// Loads the 2-for-1 spectrum Z = Xa + i Xb at the thread's input rows.
// ma/mb: multiply the field by i*kz (z derivative) first.
template <typename T, int L, int E>
__device__ __forceinline__ void k3_load_pair(cx<T> (&r)[E], const cx<T> *__restrict__ A, bool ma, const cx<T> *__restrict__ B,
                                             bool mb, int Kz, T sz, int q, bool ok) {
#pragma unroll
    for (int e = 0; e < E; e++) {
        const int row = in_row<L, E, true>(q, e);
        cx<T> z = zero<T>();
        if (ok) {
            const bool lo = row < Kz, hi = row > L - Kz;
            if (lo || hi) {
                const int kk = lo ? row : L - row;
                cx<T> a = A[kk], b = B ? B[kk] : zero<T>();
                if (ma) a = mul_i(T(kk) * sz * a);
                if (mb) b = mul_i(T(kk) * sz * b);
                if (row == 0) z = mk<T>(a.x, b.x);
                else if (lo) z = mk<T>(a.x - b.y, a.y + b.x);
                else z = mk<T>(a.x + b.y, b.x - a.y);
            }
        }
        r[e] = z;
    }
}

template <typename T> __device__ __forceinline__ void block_max4(const double (&v)[4], DevScalars *ds) {
    __shared__ double red[4][32];
    double m[4] = {v[0], v[1], v[2], v[3]};
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int i = 0; i < 4; i++) m[i] = fmax(m[i], __shfl_xor_sync(0xffffffffu, m[i], o));
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    if (lane == 0)
#pragma unroll
        for (int i = 0; i < 4; i++) red[i][wid] = m[i];
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int i = 0; i < 4; i++) m[i] = lane < nw ? red[i][lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
#pragma unroll
            for (int i = 0; i < 4; i++) m[i] = fmax(m[i], __shfl_xor_sync(0xffffffffu, m[i], o));
        if (lane == 0)
#pragma unroll
            for (int i = 0; i < 4; i++) {
                double x = m[i];
                if (!(x <= 1.7976931348623157e308)) atomicExch(&ds->nonfinite, 1); // NaN or Inf
                else atomicMax(&ds->max_bits[i], (unsigned long long)__double_as_longlong(x));
            }
    }
    __syncthreads();
}

__device__ __forceinline__ void block_sum(double v, double *dst) {
    __shared__ double red[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    if (lane == 0) red[wid] = v;
    __syncthreads();
    if (wid == 0) {
        v = lane < nw ? red[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) atomicAdd(dst, v);
    }
    __syncthreads();
}

// Block maximum of a non-negative double, folded into *dst (its bits order as the values do).
__device__ __forceinline__ void block_max_bits(double v, unsigned long long *dst) {
    __shared__ double red[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    if (lane == 0) red[wid] = v;
    __syncthreads();
    if (wid == 0) {
        v = lane < nw ? red[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (lane == 0) atomicMax(dst, (unsigned long long)__double_as_longlong(v));
    }
    __syncthreads();
}

// Forward transform of the register pair z = a + i b and extraction of both
// half spectra for kz < Kz:  Xa = (Z_k + conj Z_{L-k})/2, Xb = (Z_k - conj Z_{L-k})/(2i).
// With jz: Xa += i kz Xb (the z-derivative of b folded into a; SGS divergence).
template <typename T, int L, int E>
__device__ __forceinline__ void k3_store_pair(cx<T> (&r)[E], SmPencil<T, L, E> sm, int q, int Kz, cx<T> *A, cx<T> *B,
                                              bool fold_dz_b_into_a, T sz, bool ok, const cx<T> *__restrict__ tw) {
    constexpr int Q = L / E;
    pencil_fft<T, L, E, false, (32 % (L / E) == 0)>(r, sm, q, tw);
#pragma unroll
    for (int e = 0; e < E; e++) sm.at(out_row<L, E, false>(q, e)) = r[e];
    __syncthreads();
    if (ok) {
        const T h = T(0.5);
        for (int k = q; k < Kz; k += Q) {
            cx<T> zk = sm.at(k), zm = sm.at(k == 0 ? 0 : L - k);
            cx<T> xa = mk<T>(h * (zk.x + zm.x), h * (zk.y - zm.y));
            cx<T> xb = mk<T>(h * (zk.y + zm.y), h * (zm.x - zk.x));
            if (fold_dz_b_into_a) xa = xa + mul_i(T(k) * sz * xb);
            A[k] = xa;
            if (B) B[k] = xb;
        }
    }
    __syncthreads();
}

// Single real field: forward transform of (a + 0i), kz < Kz written directly.
template <typename T, int L, int E>
__device__ __forceinline__ void k3_store_single(cx<T> (&r)[E], SmPencil<T, L, E> sm, int q, int Kz, cx<T> *A, bool ok,
                                                const cx<T> *__restrict__ tw) {
    pencil_fft<T, L, E, false, (32 % (L / E) == 0)>(r, sm, q, tw);
    if (ok) {
#pragma unroll
        for (int e = 0; e < E; e++) {
            const int row = out_row<L, E, false>(q, e);
            if (row < Kz) A[row] = r[e];
        }
    }
}

// One forward job of the z pass: a pair (k3_store_pair) or, with `single`, a
// single real field (k3_store_single), behind one copy of the transform code.
template <typename T, int L, int E>
__device__ __forceinline__ void k3_store_job(cx<T> (&r)[E], SmPencil<T, L, E> sm, int q, int Kz, cx<T> *A, cx<T> *B, bool fold,
                                             bool single, T sz, bool ok, const cx<T> *__restrict__ tw) {
    constexpr int Q = L / E;
    pencil_fft<T, L, E, false, (32 % (L / E) == 0)>(r, sm, q, tw);
    if (single) {
        if (ok) {
#pragma unroll
            for (int e = 0; e < E; e++) {
                const int row = out_row<L, E, false>(q, e);
                if (row < Kz) A[row] = r[e];
            }
        }
        return;
    }
#pragma unroll
    for (int e = 0; e < E; e++) sm.at(out_row<L, E, false>(q, e)) = r[e];
    __syncthreads();
    if (ok) {
        const T h = T(0.5);
        for (int k = q; k < Kz; k += Q) {
            cx<T> zk = sm.at(k), zm = sm.at(k == 0 ? 0 : L - k);
            cx<T> xa = mk<T>(h * (zk.x + zm.x), h * (zk.y - zm.y));
            cx<T> xb = mk<T>(h * (zk.y + zm.y), h * (zm.x - zk.x));
            if (fold) xa = xa + mul_i(T(k) * sz * xb);
            A[k] = xa;
            if (B) B[k] = xb;
        }
    }
    __syncthreads();
}

// Running CFL maxima; a NaN or Inf velocity turns the maxima into +Inf (fmax
// alone would drop NaN), which the block reduction reports as non-finite.
template <typename T>
__device__ __forceinline__ void cfl_update(double (&mx)[4], double uu, double vv, double ww, const StepConsts &c) {
    const double au = fabs(uu), av = fabs(vv), aw = fabs(ww);
    const double s = au * c.inv_Ax + av * c.inv_Ay + aw * c.inv_Az;
    if (!(s <= 1.7976931348623157e308)) { mx[0] = mx[1] = mx[2] = mx[3] = __longlong_as_double(0x7ff0000000000000LL); return; }
    mx[0] = fmax(mx[0], au); mx[1] = fmax(mx[1], av); mx[2] = fmax(mx[2], aw);
    mx[3] = fmax(mx[3], s);
}

// Asynchronous global->shared copy of one complex element (LDGSTS; 16 B for
// double, 8 B for float), completed per thread by commit/wait groups.
template <typename T> __device__ __forceinline__ void cp_async_elem(cx<T> *smem_dst, const cx<T> *gsrc) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
    if constexpr (sizeof(cx<T>) == 16) asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gsrc) : "memory");
    else asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Shared-memory slots of physical fields kept per pencil (rows of this thread only).
// slots: 0 u, 1 v, 2 w, 3..5 conv_x,y,z, LES 6..11 a11, a12, a22, a13, a23, a33 (then t_ij)
template <int MODE> struct K3Phys { static constexpr int N = MODE == MODE_ADV ? 6 : MODE == MODE_LES ? 12 : MODE == MODE_INV ? 9 : 0; };
// The first slots live in registers (indexed by the thread's register slot e, not
// by row), the rest in shared memory: the twelve LES slots of a 384-pencil take
// 37 KB of shared memory in FP64, which alone would allow 4 pencils per SM.
#ifndef SPNS_K3_REG_SLOTS
#define SPNS_K3_REG_SLOTS 6
#endif
#ifndef SPNS_F32_K3_REG_SLOTS
#define SPNS_F32_K3_REG_SLOTS 9
#endif
#ifndef SPNS_Z_STAGE_PAIRS
#define SPNS_Z_STAGE_PAIRS 3      // double rotational z pass: input pairs staged in shared memory
#endif
#ifndef SPNS_F32_Z_STAGE_PAIRS
#define SPNS_F32_Z_STAGE_PAIRS 3
#endif
template <typename T> struct K3StagePairs { static constexpr int N = sizeof(T) == 8 ? SPNS_Z_STAGE_PAIRS : SPNS_F32_Z_STAGE_PAIRS; };
#ifndef SPNS_F32_Z_STAGE_LES
#define SPNS_F32_Z_STAGE_LES 1    // single-precision LES z pass: stage the nine input fields in shared memory
#endif
// Staging slot of S2 input field f (0 u, 1 v, 2 w, 3-5 d/dx, 6-8 d/dy) in the LES z pass:
// the order of first use by the pairs, 0 1 2 3 6 4 7 5 8.
__host__ __device__ constexpr int k3_stage_slot(int f) { return f <= 3 ? f : f == 6 ? 4 : f == 4 ? 5 : f == 7 ? 6 : f == 5 ? 7 : 8; }
template <typename T, int MODE, int E = 12> struct K3Reg {
    // with few values per thread (E <= 6) more slots fit in registers
    static constexpr int R = E <= 6 ? (sizeof(T) == 8 ? 8 : 12) : sizeof(T) == 8 ? SPNS_K3_REG_SLOTS : SPNS_F32_K3_REG_SLOTS;
    static constexpr int N = K3Phys<MODE>::N < R ? K3Phys<MODE>::N : R;   // slots in registers
    static constexpr int NSM = K3Phys<MODE>::N - N;                       // slots in shared memory
};
template <int S, int NREG, int L, typename T, int E>
__device__ __forceinline__ T &k3_slot(T (&rg)[NREG > 0 ? NREG : 1][E], T *ph, int e, int row) {
    if constexpr (S < NREG) return rg[S][e];
    else return ph[(S - NREG) * L + row];
}

// STAGE (rotational form): the six input fields of the block's pencils are
// copied into shared memory asynchronously at the start, in the order the
// three pairs use them, so the loads of the second and third pairs overlap the
// transforms of the first.  Dynamic shared memory then holds P*6*Kz extra
// complex values after the exchange buffers.
// Register budget of the z pass, as registers per thread (0: none), turned into
// the minimum resident blocks per SM of __launch_bounds__ for the block size
// at hand: single precision 128 for the velocity and rotational forms (16 warps
// per SM), 168 for the advective and LES forms (12 warps); double precision none.
#ifndef SPNS_K3_REGS_ROT
#define SPNS_K3_REGS_ROT 0
#endif
#ifndef SPNS_K3_REGS_ADV
#define SPNS_K3_REGS_ADV 0
#endif
#ifndef SPNS_F32_K3_REGS_ROT
#define SPNS_F32_K3_REGS_ROT 128
#endif
#ifndef SPNS_F32_K3_REGS_ADV
#define SPNS_F32_K3_REGS_ADV 168
#endif
template <typename T, int MODE, int THREADS> struct K3MinBlocks {
    static constexpr bool D = sizeof(T) == 8;
    static constexpr int REGS = (MODE == MODE_LES || MODE == MODE_ADV) ? (D ? SPNS_K3_REGS_ADV : SPNS_F32_K3_REGS_ADV)
                              : (MODE == MODE_ROT || MODE == MODE_VEL) ? (D ? SPNS_K3_REGS_ROT : SPNS_F32_K3_REGS_ROT) : 0;
    static constexpr int B = REGS > 0 ? 65536 / (REGS * THREADS) : 1;
    static constexpr int N = B < 1 ? 1 : B;
};
template <typename T, int L, int E, int P, int MODE, bool STAGE>
__device__ __forceinline__ void k3_z_body(Geo g, cx<T> *__restrict__ buf, const StepConsts &c, DevScalars *ds,
                                          double *__restrict__ phys, const cx<T> *__restrict__ tw) {
    extern __shared__ __align__(16) unsigned char smraw[];
    constexpr int Q = L / E;
    const int tid = threadIdx.x, p = tid / Q, q = tid % Q;
    const long long npen = (long long)g.Mx * g.My;
    const long long pen = (long long)blockIdx.x * P + p;
    const bool ok = pen < npen;
    const long long base = (ok ? pen : 0) * g.Kz;
    cx<T> *smc = reinterpret_cast<cx<T> *>(smraw);
    constexpr int PITCH = pencil_pitch<T, L, E>();
    SmPencil<T, L, E> sm{smc + p * PITCH};
    constexpr int NREG = K3Reg<T, MODE, E>::N;
    T *ph = reinterpret_cast<T *>(smc + P * PITCH) + (long long)p * K3Reg<T, MODE, E>::NSM * L;
    const T sz = T(g.sz);
    cx<T> *const B0 = buf + base;
#define F(i) (B0 + (long long)(i) * g.S2)
    double mx[4] = {0.0, 0.0, 0.0, 0.0};

    if constexpr (MODE == MODE_VEL) {
        cx<T> A[E], B[E];
        k3_load_pair<T, L, E>(A, F(0), false, F(1), false, g.Kz, sz, q, ok);
        pencil_fft<T, L, E, true, (32 % (L / E) == 0)>(A, sm, q, tw);
        k3_load_pair<T, L, E>(B, F(2), false, nullptr, false, g.Kz, sz, q, ok);
        pencil_fft<T, L, E, true, (32 % (L / E) == 0)>(B, sm, q, tw);
        double ss = 0.0;
#pragma unroll
        for (int e = 0; e < E; e++) {
            const double uu = A[e].x, vv = A[e].y, ww = B[e].x;
            cfl_update<T>(mx, uu, vv, ww, c);
            ss += uu * uu + vv * vv + ww * ww;
        }
        if (!ok) { mx[0] = mx[1] = mx[2] = mx[3] = 0.0; ss = 0.0; }
        if (phys && ok) {
            const int y = (int)(pen / g.Mx), x = (int)(pen % g.Mx);
            const long long n3 = (long long)g.Mx * g.My * g.Mz;
            double *o = phys + ((long long)x * g.My + y) * g.Mz;
#pragma unroll
            for (int e = 0; e < E; e++) {
                const int row = out_row<L, E, true>(q, e);
                o[row] = A[e].x; o[n3 + row] = A[e].y; o[2 * n3 + row] = B[e].x;
            }
        }
        block_max4<T>(mx, ds);
        block_sum(ss, &ds->sumsq_phys);
    } else if constexpr (MODE == MODE_ROT) {
        // pairs (u, w_x), (v, w_y), (w, w_z);  c = w x u  (= u.grad u + gradient)
        // STAGE: the input fields of the last NSP pairs are copied into shared memory
        // asynchronously at the start, in the order the pairs use them, so their loads
        // overlap the transforms of the earlier pairs.
        constexpr int NSP = STAGE ? K3StagePairs<T>::N : 0;
        constexpr int FIRST = 3 - NSP;
        cx<T> A[E];
        const cx<T> *src[6] = {F(0), F(1), F(2), F(3), F(4), F(5)};
        if constexpr (STAGE) {
            cx<T> *st = smc + P * PITCH + (long long)p * 2 * NSP * g.Kz;
#pragma unroll
            for (int gp = FIRST; gp < 3; gp++) {
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const int f = gp + 3 * h, slot = 2 * (gp - FIRST) + h;
                    if (ok)
                        for (int k = q; k < g.Kz; k += Q) cp_async_elem<T>(st + slot * g.Kz + k, src[f] + k);
                }
                cp_async_commit();
            }
#pragma unroll
            for (int gp = FIRST; gp < 3; gp++) {
                src[gp] = st + 2 * (gp - FIRST) * g.Kz;
                src[gp + 3] = st + (2 * (gp - FIRST) + 1) * g.Kz;
            }
        }
        // Physical values in register slots 0 u, 1 w_x, 2 v, 3 w_y, 4 c_z.  The pair
        // loop is unrolled (rolled, with slots written in one iteration and read in a
        // later one, it computed wrong products); the two forward jobs share one
        // transform body.  The slots are defined on entry all the same.
        T rs[5][E];
#pragma unroll
        for (int i = 0; i < 5; i++)
#pragma unroll
            for (int e = 0; e < E; e++) rs[i][e] = T(0);
#pragma unroll
        for (int pi = 0; pi < 3; pi++) {
            if constexpr (STAGE) {
                if (pi == FIRST) { cp_async_wait<NSP - 1>(); __syncthreads(); }
                else if (pi == FIRST + 1) { cp_async_wait<(NSP >= 2 ? NSP - 2 : 0)>(); __syncthreads(); }
                else if (pi == FIRST + 2) { cp_async_wait<0>(); __syncthreads(); }
            }
            k3_load_pair<T, L, E>(A, src[pi], false, src[pi + 3], false, g.Kz, sz, q, ok);
            pencil_fft<T, L, E, true, (32 % (L / E) == 0)>(A, sm, q, tw);
            if (pi == 0) {
#pragma unroll
                for (int e = 0; e < E; e++) { rs[0][e] = A[e].x; rs[1][e] = A[e].y; }
            } else if (pi == 1) {
#pragma unroll
                for (int e = 0; e < E; e++) { rs[2][e] = A[e].x; rs[3][e] = A[e].y; rs[4][e] = rs[1][e] * A[e].x - A[e].y * rs[0][e]; }
            }
        }
#pragma unroll
        for (int e = 0; e < E; e++) {
            const T uu = rs[0][e], ox = rs[1][e], vv = rs[2][e], oy = rs[3][e], ww = A[e].x, oz = A[e].y;
            cfl_update<T>(mx, uu, vv, ww, c);
            A[e] = mk<T>(oy * ww - oz * vv, oz * uu - ox * ww);
        }
        if (!ok) { mx[0] = mx[1] = mx[2] = mx[3] = 0.0; }
        block_max4<T>(mx, ds);
#pragma unroll 1
        for (int j = 0; j < 2; j++) {
            if (j == 1) {
#pragma unroll
                for (int e = 0; e < E; e++) A[e] = mk<T>(rs[4][e], T(0));
            }
            // c_z goes over w_x (field 3, consumed by the first pair): the forward y pass
            // reads the rotational nonlinear term from fields 0, 1 and 3 (k4_in_field)
            k3_store_job<T, L, E>(A, sm, q, g.Kz, j == 0 ? F(0) : F(3), j == 0 ? F(1) : nullptr, false, j == 1, sz, ok, tw);
        }
    } else if constexpr (MODE == MODE_INV) {
        // Velocity-gradient invariants (src/HIT_LES.cpp:1297-1319, definitions
        // src/tensor_algebra.cpp:165-306, 356-358) of G_ij = d_j u_i, and the
        // eddy-viscosity statistics of the grid: `phys` holds 3 accumulators here
        // (sum of nu_t, sum of nu_t^2, bits of the maximum nu_t).
        // S2 inputs as in the advective form: 0 u, 1 v, 2 w, 3 du/dx, 4 dv/dx, 5 dw/dx,
        // 6 du/dy, 7 dv/dy, 8 dw/dy; z-derivatives formed here.  Slots s = 3 i + j hold G_ij.
        // Outputs (S2 fields 0..4): Q_G, Q_S, R_G, R_S, V^2 forward-transformed, kz <= hz.
        double nut_sum = 0.0, nut_sq = 0.0, nut_max = 0.0;
        cx<T> A[E];
        T rg[NREG > 0 ? NREG : 1][E];
#pragma unroll
        for (int i = 0; i < (NREG > 0 ? NREG : 1); i++)
#pragma unroll
            for (int e = 0; e < E; e++) rg[i][e] = T(0);
#define PH(slot, row) k3_slot<(slot), NREG, L, T, E>(rg, ph, e, row)
        // pairs: (du/dx, du/dy), (dv/dx, dv/dy), (dw/dx, dw/dy), (du/dz, dv/dz), (dw/dz, -)
#pragma unroll 1
        for (int pi = 0; pi < 5; pi++) {
            const cx<T> *fa = pi < 3 ? F(3 + pi) : pi == 3 ? F(0) : F(2);
            const cx<T> *fb = pi < 3 ? F(6 + pi) : pi == 3 ? F(1) : nullptr;
            k3_load_pair<T, L, E>(A, fa, pi >= 3, fb, pi == 3, g.Kz, sz, q, ok);
            pencil_fft<T, L, E, true, (32 % (L / E) == 0)>(A, sm, q, tw);
            switch (pi) {
            case 0:
#pragma unroll
                for (int e = 0; e < E; e++) { const int row = out_row<L, E, true>(q, e); PH(0, row) = A[e].x; PH(1, row) = A[e].y; }
                break;
            case 1:
#pragma unroll
                for (int e = 0; e < E; e++) { const int row = out_row<L, E, true>(q, e); PH(3, row) = A[e].x; PH(4, row) = A[e].y; }
                break;
            case 2:
#pragma unroll
                for (int e = 0; e < E; e++) { const int row = out_row<L, E, true>(q, e); PH(6, row) = A[e].x; PH(7, row) = A[e].y; }
                break;
            case 3:
#pragma unroll
                for (int e = 0; e < E; e++) { const int row = out_row<L, E, true>(q, e); PH(2, row) = A[e].x; PH(5, row) = A[e].y; }
                break;
            default:
#pragma unroll
                for (int e = 0; e < E; e++) { const int row = out_row<L, E, true>(q, e); PH(8, row) = A[e].x; }
                break;
            }
        }
        // invariants per grid row, written over slots 0..4
#pragma unroll
        for (int e = 0; e < E; e++) {
            const int row = out_row<L, E, true>(q, e);
            double G[3][3], S[3][3], O[3][3], S2[3][3], O2[3][3];
            G[0][0] = PH(0, row); G[0][1] = PH(1, row); G[0][2] = PH(2, row);
            G[1][0] = PH(3, row); G[1][1] = PH(4, row); G[1][2] = PH(5, row);
            G[2][0] = PH(6, row); G[2][1] = PH(7, row); G[2][2] = PH(8, row);
#pragma unroll
            for (int i = 0; i < 3; i++)
#pragma unroll
                for (int j = 0; j < 3; j++) { S[i][j] = 0.5 * G[i][j] + 0.5 * G[j][i]; O[i][j] = G[i][j] - S[i][j]; }
            double trG = G[0][0] + G[1][1] + G[2][2], trS = S[0][0] + S[1][1] + S[2][2], trGG = 0.0, trSS = 0.0, trS2O2 = 0.0;
#pragma unroll
            for (int i = 0; i < 3; i++)
#pragma unroll
                for (int j = 0; j < 3; j++) {
                    trGG += G[i][j] * G[j][i];
                    trSS += S[i][j] * S[j][i];
                    double s2 = 0.0, o2 = 0.0;
#pragma unroll
                    for (int k = 0; k < 3; k++) { s2 += S[i][k] * S[k][j]; o2 += O[i][k] * O[k][j]; }
                    S2[i][j] = s2; O2[i][j] = o2;
                }
#pragma unroll
            for (int i = 0; i < 3; i++)
#pragma unroll
                for (int k = 0; k < 3; k++) trS2O2 += S2[i][k] * O2[k][i];
            auto det3 = [](const double (&t)[3][3]) {
                double d = 0.0;
                d += t[0][0] * t[1][1] * t[2][2];
                d += t[0][1] * t[1][2] * t[2][0];
                d += t[0][2] * t[1][0] * t[2][1];
                d -= t[0][2] * t[1][1] * t[2][0];
                d -= t[0][1] * t[1][0] * t[2][2];
                d -= t[0][0] * t[1][2] * t[2][1];
                return d;
            };
            const double QG = 0.5 * (trG * trG - trGG), QS = 0.5 * (trS * trS - trSS);
            // eddy viscosity of this grid point (src/HIT_LES.cpp:130-142, same expression order)
            {
                double ne = 2.0 * G[0][0] * G[0][0];
                ne += 2.0 * G[1][1] * G[1][1];
                ne += 2.0 * G[2][2] * G[2][2];
                ne += (G[0][1] + G[1][0]) * (G[0][1] + G[1][0]);
                ne += (G[0][2] + G[2][0]) * (G[0][2] + G[2][0]);
                ne += (G[1][2] + G[2][1]) * (G[1][2] + G[2][1]);
                const double nt = ok ? c.les_ct * sqrt(ne) : 0.0;
                nut_sum += nt; nut_sq += nt * nt; nut_max = fmax(nut_max, nt);
            }
            PH(0, row) = T(QG);
            PH(1, row) = T(QS);
            PH(2, row) = T(det3(G));
            PH(3, row) = T(det3(S));
            PH(4, row) = T(4.0 * (trS2O2 - 2.0 * QS * (QG - QS)));
        }
        if (phys) {
            block_sum(nut_sum, phys);
            block_sum(nut_sq, phys + 1);
            block_max_bits(nut_max, reinterpret_cast<unsigned long long *>(phys + 2));
        }
#pragma unroll 1
        for (int j = 0; j < 3; j++) {
            if (j == 0) {
#pragma unroll
                for (int e = 0; e < E; e++) { const int row = out_row<L, E, true>(q, e); A[e] = mk<T>(PH(0, row), PH(1, row)); }
            } else if (j == 1) {
#pragma unroll
                for (int e = 0; e < E; e++) { const int row = out_row<L, E, true>(q, e); A[e] = mk<T>(PH(2, row), PH(3, row)); }
            } else {
#pragma unroll
                for (int e = 0; e < E; e++) { const int row = out_row<L, E, true>(q, e); A[e] = mk<T>(PH(4, row), T(0)); }
            }
            k3_store_job<T, L, E>(A, sm, q, g.Kz, F(2 * j), j < 2 ? F(2 * j + 1) : nullptr, false, j == 2, sz, ok, tw);
        }
        (void)mx;
#undef PH
    } else {
        // Advective form of the reference (src/HIT_LES.cpp:74-125): conv_i = u_j d_j u_i.
        // S2 inputs: 0 u, 1 v, 2 w, 3 du/dx, 4 dv/dx, 5 dw/dx, 6 du/dy, 7 dv/dy, 8 dw/dy;
        // z-derivatives are formed here from u, v, w.  Physical values of the
        // thread's own rows are kept in per-thread slots, the first K3Reg::N in
        // registers and the rest in shared memory (own rows only: no barrier needed).
        // LES (src/HIT_LES.cpp:130-171): strain combinations a_ij accumulate in further slots.
        // The transforms run in two loops (inverse pairs, forward jobs) around one
        // copy of the transform code each: unrolled one after another, the eleven
        // LES transforms overflow the instruction cache.
        cx<T> A[E];
        T rg[NREG > 0 ? NREG : 1][E];
        // slots are written in one iteration of the pair loop and read in later ones:
        // define them on entry (a rolled loop over partly defined registers miscompiled)
#pragma unroll
        for (int i = 0; i < (NREG > 0 ? NREG : 1); i++)
#pragma unroll
            for (int e = 0; e < E; e++) rg[i][e] = T(0);
#define PH(slot, row) k3_slot<(slot), NREG, L, T, E>(rg, ph, e, row)
        // inverse pairs: (u, v), (w, du/dz), (du/dx, du/dy), (dv/dx, dv/dy), (dw/dx, dw/dy), (dv/dz, dw/dz)
        // STAGE (single-precision LES): the nine input fields of the block's pencils are
        // copied into shared memory asynchronously at the start, in five groups in the
        // order the pairs first use them ({u, v}, {w}, {du/dx, du/dy}, {dv/dx, dv/dy},
        // {dw/dx, dw/dy}), so later pairs' loads overlap the earlier transforms.
        // Field f sits in staging slot K3StageSlot(f) of its pencil.
        cx<T> *const st = reinterpret_cast<cx<T> *>(reinterpret_cast<T *>(smc + P * PITCH) +
                                                    (long long)P * K3Reg<T, MODE, E>::NSM * L) + (long long)p * 9 * g.Kz;
        if constexpr (STAGE) {
#pragma unroll
            for (int grp = 0; grp < 5; grp++) {
#pragma unroll
                for (int h2 = 0; h2 < 2; h2++) {
                    const int f = grp == 0 ? h2 : grp == 1 ? (h2 == 0 ? 2 : -1) : (h2 == 0 ? grp + 1 : grp + 4);
                    if (f >= 0 && ok)
                        for (int k = q; k < g.Kz; k += Q) cp_async_elem<T>(st + k3_stage_slot(f) * g.Kz + k, F(f) + k);
                }
                cp_async_commit();
            }
        }
#pragma unroll 1
        for (int pi = 0; pi < 6; pi++) {
            const int fa = pi == 0 ? 0 : pi == 1 ? 2 : pi == 5 ? 1 : pi + 1;
            const int fb = pi == 0 ? 1 : pi == 1 ? 0 : pi == 5 ? 2 : pi + 4;
            if constexpr (STAGE) {
                switch (pi) {
                case 0: cp_async_wait<4>(); break;
                case 1: cp_async_wait<3>(); break;
                case 2: cp_async_wait<2>(); break;
                case 3: cp_async_wait<1>(); break;
                default: cp_async_wait<0>(); break;
                }
                __syncthreads();
                k3_load_pair<T, L, E>(A, st + k3_stage_slot(fa) * g.Kz, pi == 5, st + k3_stage_slot(fb) * g.Kz, pi == 1 || pi == 5,
                                      g.Kz, sz, q, ok);
            } else {
                k3_load_pair<T, L, E>(A, F(fa), pi == 5, F(fb), pi == 1 || pi == 5, g.Kz, sz, q, ok);
            }
            pencil_fft<T, L, E, true, (32 % (L / E) == 0)>(A, sm, q, tw);
            switch (pi) {
            case 0:
#pragma unroll
                for (int e = 0; e < E; e++) { const int row = out_row<L, E, true>(q, e); PH(0, row) = A[e].x; PH(1, row) = A[e].y; }
                break;
            case 1:
#pragma unroll
                for (int e = 0; e < E; e++) {
                    const int row = out_row<L, E, true>(q, e);
                    const T ww = A[e].x;
                    PH(2, row) = ww;
                    cfl_update<T>(mx, PH(0, row), PH(1, row), ww, c);
                    PH(3, row) = ww * A[e].y;
                    if (MODE == MODE_LES) PH(9, row) = A[e].y; // a13 = du/dz (+ dw/dx below)
                }
                break;
            case 2:
#pragma unroll
                for (int e = 0; e < E; e++) {
                    const int row = out_row<L, E, true>(q, e);
                    PH(3, row) = PH(0, row) * A[e].x + PH(1, row) * A[e].y + PH(3, row);
                    if (MODE == MODE_LES) { PH(6, row) = A[e].x; PH(7, row) = A[e].y; } // a11, a12 (partial)
                }
                break;
            case 3:
#pragma unroll
                for (int e = 0; e < E; e++) {
                    const int row = out_row<L, E, true>(q, e);
                    PH(4, row) = PH(0, row) * A[e].x + PH(1, row) * A[e].y;
                    if (MODE == MODE_LES) { PH(7, row) = PH(7, row) + A[e].x; PH(8, row) = A[e].y; } // a12, a22
                }
                break;
            case 4:
#pragma unroll
                for (int e = 0; e < E; e++) {
                    const int row = out_row<L, E, true>(q, e);
                    PH(5, row) = PH(0, row) * A[e].x + PH(1, row) * A[e].y;
                    if (MODE == MODE_LES) { PH(9, row) = PH(9, row) + A[e].x; PH(10, row) = A[e].y; } // a13, a23 (partial)
                }
                break;
            default:
#pragma unroll
                for (int e = 0; e < E; e++) {
                    const int row = out_row<L, E, true>(q, e);
                    const T ww = PH(2, row);
                    PH(4, row) = PH(4, row) + ww * A[e].x;
                    PH(5, row) = PH(5, row) + ww * A[e].y;
                    if (MODE == MODE_LES) { PH(10, row) = PH(10, row) + A[e].x; PH(11, row) = A[e].y; } // a23, a33
                }
                break;
            }
        }
        if (!ok) { mx[0] = mx[1] = mx[2] = mx[3] = 0.0; }
        block_max4<T>(mx, ds);
        if constexpr (MODE == MODE_LES) {
            // eddy viscosity and SGS stress (src/HIT_LES.cpp:130-154), written over the a_ij slots:
            // slot 6 t11, 7 t12, 8 t22, 9 t13, 10 t23, 11 t33
            const T ct = T(c.les_ct);
#pragma unroll
            for (int e = 0; e < E; e++) {
                const int row = out_row<L, E, true>(q, e);
                const T a11 = PH(6, row), a12 = PH(7, row), a22 = PH(8, row), a13 = PH(9, row), a23 = PH(10, row), a33 = PH(11, row);
                T ne = T(2.0) * a11 * a11;
                ne += T(2.0) * a22 * a22;
                ne += T(2.0) * a33 * a33;
                ne += a12 * a12;
                ne += a13 * a13;
                ne += a23 * a23;
                ne = ct * sqrt(ne);
                PH(6, row) = T(-2.0) * ne * a11;
                PH(7, row) = T(-1.0) * ne * a12;
                PH(8, row) = T(-2.0) * ne * a22;
                PH(9, row) = T(-1.0) * ne * a13;
                PH(10, row) = T(-1.0) * ne * a23;
                PH(11, row) = T(-2.0) * ne * a33;
            }
        }
        // forward jobs.  ADV: (conv_x, conv_y) -> 0, 1; conv_z -> 2.
        // LES outputs: 0 G_x = conv_x + i kz t13, 1 G_y, 2 G_z, 3 t11, 4 t12, 5 t13, 6 t22, 7 t23
        constexpr int NJOB = MODE == MODE_LES ? 5 : 2;
#pragma unroll 1
        for (int j = 0; j < NJOB; j++) {
            cx<T> *oa, *ob = nullptr;
            bool fold = false, single = false;
            if (MODE == MODE_ADV) {
                if (j == 0) {
#pragma unroll
                    for (int e = 0; e < E; e++) { const int row = out_row<L, E, true>(q, e); A[e] = mk<T>(PH(3, row), PH(4, row)); }
                    oa = F(0); ob = F(1);
                } else {
#pragma unroll
                    for (int e = 0; e < E; e++) { const int row = out_row<L, E, true>(q, e); A[e] = mk<T>(PH(5, row), T(0)); }
                    oa = F(2); single = true;
                }
            } else {
                switch (j) {
                case 0:
#pragma unroll
                    for (int e = 0; e < E; e++) { const int row = out_row<L, E, true>(q, e); A[e] = mk<T>(PH(3, row), PH(9, row)); }
                    oa = F(0); ob = F(5); fold = true;
                    break;
                case 1:
#pragma unroll
                    for (int e = 0; e < E; e++) { const int row = out_row<L, E, true>(q, e); A[e] = mk<T>(PH(4, row), PH(10, row)); }
                    oa = F(1); ob = F(7); fold = true;
                    break;
                case 2:
#pragma unroll
                    for (int e = 0; e < E; e++) { const int row = out_row<L, E, true>(q, e); A[e] = mk<T>(PH(5, row), PH(11, row)); }
                    oa = F(2); fold = true;
                    break;
                case 3:
#pragma unroll
                    for (int e = 0; e < E; e++) { const int row = out_row<L, E, true>(q, e); A[e] = mk<T>(PH(6, row), PH(7, row)); }
                    oa = F(3); ob = F(4);
                    break;
                default:
#pragma unroll
                    for (int e = 0; e < E; e++) { const int row = out_row<L, E, true>(q, e); A[e] = mk<T>(PH(8, row), T(0)); }
                    oa = F(6); single = true;
                    break;
                }
            }
            k3_store_job<T, L, E>(A, sm, q, g.Kz, oa, ob, fold, single, sz, ok, tw);
        }
#undef PH
    }
#undef F
}

// S2 field holding component f of the nonlinear term after the z pass: the
// rotational form writes c_z over w_x (field 3), the others in order.
template <int MODE> __host__ __device__ constexpr int k4_in_field(int f) { return (MODE == MODE_ROT && f == 2) ? 3 : f; }

// ===========================================================================
// K4: forward transform along y with ky truncation.  Block = (kz chunk, x).
// LES: G_i += i ky t_i2 (SGS divergence, y part).
// ===========================================================================
template <typename T, int L, int E, int P, int MODE>
__device__ __forceinline__ void k4_fwd_y_body(Geo g, const cx<T> *__restrict__ in, cx<T> *__restrict__ out,
                                              const cx<T> *__restrict__ tw) {
    extern __shared__ __align__(16) unsigned char smraw[];
    const int tid = threadIdx.x, p = tid % P, q = tid / P;
    const int x = blockIdx.y, kz = blockIdx.x * P + p;
    const bool ok = kz < g.Kz;
    SmRowMajor<T, P> sm{reinterpret_cast<cx<T> *>(smraw), p};
    const long long col = (long long)x * g.Kz + kz;
    auto load_fft = [&](cx<T>(&r)[E], int f) {
        const cx<T> *src = in + (long long)f * g.S2 + col;
#pragma unroll
        for (int e = 0; e < E; e++) r[e] = ok ? src[(long long)in_row<L, E, false>(q, e) * g.Mx * g.Kz] : zero<T>();
        fft<T, L, E, false>(r, sm, q, tw);
    };
    auto store = [&](const cx<T>(&r)[E], int f, const cx<T> *add, bool use_add) {
        if (!ok) return;
        cx<T> *o = out + (long long)f * g.S1 + col;
#pragma unroll
        for (int e = 0; e < E; e++) {
            const int m2 = ffreq(out_row<L, E, false>(q, e), L);
            if (m2 <= g.hy && m2 >= -g.hy) {
                cx<T> val = r[e];
                if (use_add) val = val + mul_i(T(g.sy * m2) * add[e]);
                o[(long long)(m2 >= 0 ? m2 : m2 + g.Ky) * g.Mx * g.Kz] = val;
            }
        }
    };
    if constexpr (MODE != MODE_LES) {
#pragma unroll 1
        for (int f = 0; f < Fields<MODE>::NOUT; f++) {
            cx<T> r[E];
            load_fft(r, k4_in_field<MODE>(f));
            store(r, f, r, false);
        }
    } else {
        // in (S2): 0 G_x, 1 G_y, 2 G_z, 3 t11, 4 t12, 5 t13, 6 t22, 7 t23
        // out (S1): 0 G_x + i ky t12, 1 G_y + i ky t22, 2 G_z + i ky t23, 3 t11, 4 t12, 5 t13
        const int gi[3] = {0, 1, 2}, ti[3] = {4, 6, 7};
#pragma unroll 1
        for (int i = 0; i < 3; i++) {
            cx<T> r[E], t[E];
            load_fft(r, gi[i]);
            load_fft(t, ti[i]);
            store(r, i, t, true);
            if (i == 0) store(t, 4, t, false);
        }
#pragma unroll 1
        for (int f = 3; f <= 5; f += 2) {
            cx<T> r[E];
            load_fft(r, f);
            store(r, f, r, false);
        }
    }
}

// ===========================================================================
// K5: forward transform along x with kx truncation into the compact layout
// (S0).  Block = (kz chunk, iy).  LES: G_i += i kx t_i1 (SGS divergence, x part).
// ===========================================================================
template <typename T, int L, int E, int P, int MODE>
__device__ __forceinline__ void k5_fwd_x_body(Geo g, const cx<T> *__restrict__ in, cx<T> *__restrict__ G,
                                              const cx<T> *__restrict__ tw) {
    extern __shared__ __align__(16) unsigned char smraw[];
    const int tid = threadIdx.x, p = tid % P, q = tid / P;
    const int iy = blockIdx.y, kz = blockIdx.x * P + p;
    const bool ok = kz < g.Kz;
    SmRowMajor<T, P> sm{reinterpret_cast<cx<T> *>(smraw), p};
    const long long col = (long long)iy * g.Mx * g.Kz + kz;
    auto load_fft = [&](cx<T>(&r)[E], int f) {
        const cx<T> *src = in + (long long)f * g.S1 + col;
#pragma unroll
        for (int e = 0; e < E; e++) r[e] = ok ? src[(long long)in_row<L, E, false>(q, e) * g.Kz] : zero<T>();
        fft<T, L, E, false>(r, sm, q, tw);
    };
#pragma unroll 1
    for (int f = 0; f < Fields<MODE>::NOUT; f++) {
        cx<T> r[E];
        load_fft(r, f);
        if constexpr (MODE == MODE_LES) {
            cx<T> t[E];
            load_fft(t, 3 + f); // t11, t21=t12, t31=t13
#pragma unroll
            for (int e = 0; e < E; e++) {
                const int m1 = ffreq(out_row<L, E, false>(q, e), L);
                r[e] = r[e] + mul_i(T(g.sx * m1) * t[e]);
            }
        }
        if (ok) {
            cx<T> *o = G + (long long)f * g.S0 + (long long)iy * g.Kx * g.Kz + kz;
#pragma unroll
            for (int e = 0; e < E; e++) {
                const int m1 = ffreq(out_row<L, E, false>(q, e), L);
                if (m1 <= g.hx && m1 >= -g.hx) o[(long long)(m1 >= 0 ? m1 : m1 + g.Kx) * g.Kz] = r[e];
            }
        }
    }
}

// ===========================================================================
// K6: the spectral sweep of the step over the compact state (streaming; every
// load of a mode is issued before any store):
//   src/HIT_LES.cpp:196-242  R = -conv (0 at k=0) - nu k^2 u [- div tau] [+ Coriolis]
//   src/HIT_LES.cpp:243-278  constant-power forcing (when enabled)
//   src/HIT_LES.cpp:295-339  predictor: AB2, or the kappa scheme
//   src/HIT_LES.cpp:346-359  projection  u -= k (k.u)/k^2
// G holds the un-normalised nonlinear term (x1/M^3 here).  Kappa scheme: the
// new state is written over the u^{n-1} buffer Un1 and the caller swaps U/Un1.
// Single precision (T = float) is the compensated form: the states u^n, u^{n-1}
// and u^{n+1} are pairs hi + lo of floats (about 48 significant bits) that this
// sweep combines and splits in double, so the small increments dt*R are not
// rounded away; G and R are plain floats.  In double precision the lo pointers
// are unused (null).
// ===========================================================================
template <typename T, bool SELF>
__device__ __forceinline__ void k6_sweep_body(Geo g, const cx<T> *__restrict__ G, const cx<T> *U, const cx<T> *Ulo, cx<T> *R,
                                              cx<T> *Uout, cx<T> *Uoutlo, const cx<T> *Un1, const cx<T> *Un1lo, const StepConsts &c,
                                              const DevScalars *__restrict__ ds) {
    constexpr bool HILO = sizeof(T) == 4;
    const int iy = blockIdx.y;
    const int n = g.Kx * g.Kz;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int ix = t / g.Kz, kz = t - ix * g.Kz;
    const long long idx = (long long)iy * n + t;
    const long long S0 = g.S0;
    // loads first
    cx<T> gg[3], uu[3], r0[3], up[3], ul[3], upl[3];
#pragma unroll
    for (int i = 0; i < 3; i++) { gg[i] = G[i * S0 + idx]; uu[i] = U[i * S0 + idx]; r0[i] = R[i * S0 + idx]; }
    if constexpr (HILO) {
#pragma unroll
        for (int i = 0; i < 3; i++) ul[i] = Ulo[i * S0 + idx];
    }
    const double nu = ds->nu, dt = ds->dt, kap = ds->kappa, alpha = ds->alpha;
    const bool first = ds->iter == 0;
    if (SELF) {
#pragma unroll
        for (int i = 0; i < 3; i++) up[i] = first ? uu[i] : Un1[i * S0 + idx];
        if constexpr (HILO) {
#pragma unroll
            for (int i = 0; i < 3; i++) upl[i] = first ? ul[i] : Un1lo[i * S0 + idx];
        }
    }
    const int m1 = ix <= g.hx ? ix : ix - g.Kx, m2 = ky_mode(g, iy);
    const long long k1 = (long long)g.sx * m1, k2 = (long long)g.sy * m2, k3 = (long long)g.sz * kz;
    const double rad2 = (double)(k1 * k1 + k2 * k2 + k3 * k3);
    const bool mean = !(rad2 > 0.0);
    const double ct = nu * rad2;
    double ur[3], ui[3], rr[3], ri[3];
#pragma unroll
    for (int i = 0; i < 3; i++) {
        ur[i] = uu[i].x; ui[i] = uu[i].y;
        if constexpr (HILO) { ur[i] += (double)ul[i].x; ui[i] += (double)ul[i].y; }
        const double gr = mean ? 0.0 : (double)gg[i].x * c.inv_norm;
        const double gi = mean ? 0.0 : (double)gg[i].y * c.inv_norm;
        rr[i] = -gr - ct * ur[i];
        ri[i] = -gi - ct * ui[i];
    }
    if (c.rotating) {
        rr[0] += 2 * (c.omega_z * ur[1] - c.omega_y * ur[2]); ri[0] += 2 * (c.omega_z * ui[1] - c.omega_y * ui[2]);
        rr[1] += 2 * (c.omega_x * ur[2] - c.omega_z * ur[0]); ri[1] += 2 * (c.omega_x * ui[2] - c.omega_z * ui[0]);
        rr[2] += 2 * (c.omega_y * ur[0] - c.omega_x * ur[1]); ri[2] += 2 * (c.omega_y * ui[0] - c.omega_x * ui[1]);
    }
    if (c.eps_on) {
        const int K = (int)round(sqrt(rad2));
        if (c.eps_kmin <= K && K <= c.eps_kmax) {
#pragma unroll
            for (int i = 0; i < 3; i++) { rr[i] += alpha * ur[i]; ri[i] += alpha * ui[i]; }
        } else if (K == 0) {
#pragma unroll
            for (int i = 0; i < 3; i++) { rr[i] = 0.0; ri[i] = 0.0; }
        }
    }
    double sr[3], si[3];
    const double k05 = SELF ? 1.0 / (kap + 0.5) : 0.0;
#pragma unroll
    for (int i = 0; i < 3; i++) {
        if (SELF) {
            double pr = (double)up[i].x, pi = (double)up[i].y;
            if constexpr (HILO) { pr += (double)upl[i].x; pi += (double)upl[i].y; }
            sr[i] = k05 * (2.0 * kap * ur[i] + dt * ((1.0 + kap) * rr[i] - kap * (double)r0[i].x) - (kap - 0.5) * pr);
            si[i] = k05 * (2.0 * kap * ui[i] + dt * ((1.0 + kap) * ri[i] - kap * (double)r0[i].y) - (kap - 0.5) * pi);
        } else {
            sr[i] = ur[i] + dt * (1.5 * rr[i] - 0.5 * (double)r0[i].x);
            si[i] = ui[i] + dt * (1.5 * ri[i] - 0.5 * (double)r0[i].y);
        }
    }
    if (rad2 > 0.0) {
        const double kk[3] = {(double)k1, (double)k2, (double)k3};
        const double inv = 1.0 / rad2;
        const double ar = (kk[0] * sr[0] + kk[1] * sr[1] + kk[2] * sr[2]) * inv;
        const double ai = (kk[0] * si[0] + kk[1] * si[1] + kk[2] * si[2]) * inv;
#pragma unroll
        for (int i = 0; i < 3; i++) { sr[i] -= ar * kk[i]; si[i] -= ai * kk[i]; }
    }
#pragma unroll
    for (int i = 0; i < 3; i++) {
        R[i * S0 + idx] = mk<T>(T(rr[i]), T(ri[i]));
        const T hr = T(sr[i]), hi = T(si[i]);
        Uout[i * S0 + idx] = mk<T>(hr, hi);
        if constexpr (HILO) Uoutlo[i * S0 + idx] = mk<T>(T(sr[i] - (double)hr), T(si[i] - (double)hi));
    }
}

// ===========================================================================
// Small kernels
// ===========================================================================
__device__ __forceinline__ double Topt_d(const StepConsts &c, double phi0, int *err) {
    const double PI_ = 3.141592653589793238462643;
    auto FuL = [](double x, double x0, double x1, double f0, double f1) { return f0 + (x - x0) * (f1 - f0) / (x1 - x0); };
    auto FuG = [&](double x, double a, double b, double cc, double x0, double x1, double f0, double f1) {
        return (a * x * x + b * x + cc) * ((x - x0) * (x - x1)) + FuL(x, x0, x1, f0, f1);
    };
    if (phi0 >= 0.0 && phi0 < c.phi[0]) return FuG(phi0, 0.0, c.c[0], c.c[1], 0.0, c.phi[0], 4.0 / 3.0, c.t1);
    if (phi0 >= c.phi[0] && phi0 <= PI_ / 2.0) return FuG(phi0, c.c[2], c.c[3], c.c[4], c.phi[0], PI_ / 2.0, c.t1, 1.0);
    *err = 1;
    return 0.0;
}
__device__ __forceinline__ double Kopt_d(const StepConsts &c, double phi0, int *err) {
    const double PI_ = 3.141592653589793238462643;
    auto FuL = [](double x, double x0, double x1, double f0, double f1) { return f0 + (x - x0) * (f1 - f0) / (x1 - x0); };
    auto FuG = [&](double x, double a, double b, double cc, double x0, double x1, double f0, double f1) {
        return (a * x * x + b * x + cc) * ((x - x0) * (x - x1)) + FuL(x, x0, x1, f0, f1);
    };
    if (phi0 >= 0.0 && phi0 <= c.phi[0]) return 1.0;
    if (phi0 > c.phi[0] && phi0 <= c.phi[1]) return FuG(phi0, c.c[5], c.c[6], c.c[7], c.phi[0], c.phi[1], 1.0, c.kopt_k[0]);
    if (phi0 > c.phi[1] && phi0 <= c.phi[2]) return FuG(phi0, c.c[8], c.c[9], c.c[10], c.phi[1], c.phi[2], c.kopt_k[0], c.kopt_k[1]);
    if (phi0 > c.phi[2] && phi0 <= PI_ / 2.0) return FuG(phi0, c.c[11], c.c[12], c.c[13], c.phi[2], PI_ / 2.0, c.kopt_k[1], 0.0);
    *err = 1;
    return 0.0;
}

// src/HIT_LES.cpp:365-403, from the maxima gathered by the last inverse transform.
__device__ __forceinline__ void recalc_dt(const StepConsts &c, DevScalars *ds) {
    if (c.fixed_dt > 0.0) { ds->dt = c.fixed_dt; return; }
    const double nu = ds->nu;
    if (c.self_adaptive) {
        const double MaxVel = __longlong_as_double((long long)ds->max_bits[3]);
        ds->maxvel = MaxVel;
        const double Ah = c.Ah;
        const double phi0 = atan(MaxVel * Ah * Ah / (0.35 * nu * 12.0));
        ds->phi0 = phi0;
        int err = 0;
        double At = Topt_d(c, phi0, &err) / sqrt((MaxVel * MaxVel) / (0.35 * 0.35) + (144.0 * nu * nu / (Ah * Ah * Ah * Ah)));
        ds->kappa = Kopt_d(c, phi0, &err);
        if (err) ds->domain_err = 1;
        ds->dt = c.C_At * At;
    } else {
        const double mu = __longlong_as_double((long long)ds->max_bits[0]);
        const double mv = __longlong_as_double((long long)ds->max_bits[1]);
        const double mw = __longlong_as_double((long long)ds->max_bits[2]);
        const double MaxVel = fmax(mu / c.Ax, fmax(mv / c.Ay, mw / c.Az));
        ds->maxvel = MaxVel;
        const double C_visc = 0.2 * fmin(c.Ax * c.Ax, fmin(c.Ay * c.Ay, c.Az * c.Az)) / nu;
        const double C_conv = 0.35 / MaxVel;
        ds->dt = c.C_At * fmin(C_visc, C_conv);
    }
}

static __global__ void k_recalc_dt(StepConsts c, DevScalars *ds) { recalc_dt(c, ds); }

// End of New_Fractional_Step_Method (src/HIT_LES.cpp:19-24).
static __global__ void k_finish_step(StepConsts c, DevScalars *ds) {
    recalc_dt(c, ds);
    ds->time = ds->time + ds->dt;
    ds->iter += 1;
}

static __global__ void k_reset_max(DevScalars *ds) {
    for (int i = 0; i < 4; i++) ds->max_bits[i] = 0ull;
    ds->sumsq_phys = 0.0;
}

// Shell sums of the spectral state (src/HIT_LES.cpp:1137-1214 with the
// KineticEnergy and Enstrophy integrands of :991-1003).  Modes with kz>0 carry
// their conjugate (weight 2).  Ek[K], Om[K] for K=round(|k|) <= Kmax.
// State value hi (+ lo when the compensated single-precision form passes one) in double.
template <typename T> __device__ __forceinline__ cx<double> load_state(const cx<T> *hi, const cx<T> *lo, long long i) {
    const cx<T> a = hi[i];
    cx<double> r = mk<double>((double)a.x, (double)a.y);
    if (lo) { const cx<T> b = lo[i]; r.x += (double)b.x; r.y += (double)b.y; }
    return r;
}

// Adds each lane's e (and o, when hO is given) to the bins hE[K] (hO[K]) in shared
// memory, K < 0 adding nothing.  Called by all 32 lanes with K non-decreasing in the
// lane (consecutive kz of one row): the lanes of one shell are then contiguous,
// a segmented scan over the runs of equal K (five shuffle steps) leaves each run's
// sum in its last lane, and those lanes add to distinct bins in one atomic
// instruction.  (Consecutive kz fall in different shells about every other mode,
// so per-lane atomics would collide on few bins and a loop over the warp's shells
// would run about twenty rounds.)  Lanes out of order only cost extra atomics.
__device__ __forceinline__ void warp_shell_add(int K, double e, double o, double *hE, double *hO) {
    const int lane = threadIdx.x & 31;
    const int Kprev = __shfl_up_sync(0xffffffffu, K, 1);
    const unsigned heads = __ballot_sync(0xffffffffu, lane == 0 || Kprev != K);
    const int start = 31 - __clz(heads & (0xffffffffu >> (31 - lane)));   // first lane of this lane's run
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const double te = __shfl_up_sync(0xffffffffu, e, off);
        const double to = hO ? __shfl_up_sync(0xffffffffu, o, off) : 0.0;
        if (lane - off >= start) { e += te; o += to; }
    }
    const bool tail = lane == 31 || ((heads >> (lane + 1)) & 1u);
    if (tail && K >= 0) {
        atomicAdd(&hE[K], e);
        if (hO) atomicAdd(&hO[K], o);
    }
}

// Walks this warp's share of the compact modes 32 at a time: a contiguous run of whole
// rows (iy, ix), flattened, so that every round but the last is 32 consecutive modes
// (coalesced loads, no idle lanes at the end of a row of Kz modes).  Calls
// f(valid, idx, kz, r12) on all 32 lanes each round, r12 = (sx m1)^2 + (sy m2)^2 of
// the lane's row (recomputed only when the lane enters a new row).  Along a row K
// grows with kz, so a round's lanes form runs of equal K, as warp_shell_add wants.
template <typename F> __device__ __forceinline__ void warp_mode_rounds(const Geo &g, F &&f) {
    const int lane = threadIdx.x & 31;
    const int rows = g.Ky * g.Kx;
    const int nw = (gridDim.x * blockDim.x) >> 5, wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int per = (rows + nw - 1) / nw;
    const int r0 = (int)min((long long)wid * per, (long long)rows), r1 = min(rows, r0 + per);
    const long long end = (long long)r1 * g.Kz;
    int row = r0, kz = lane;
    while (kz >= g.Kz) { kz -= g.Kz; row++; }
    int crow = -1;
    long long r12 = 0;
    for (long long base = (long long)r0 * g.Kz; base < end; base += 32) {
        const long long idx = base + lane;
        const bool valid = idx < end;
        if (valid && row != crow) {
            crow = row;
            const int ix = row % g.Kx, iy = row / g.Kx;
            const long long k1 = (long long)g.sx * (ix <= g.hx ? ix : ix - g.Kx);
            const long long k2 = (long long)g.sy * ky_mode(g, iy);
            r12 = k1 * k1 + k2 * k2;
        }
        f(valid, idx, kz, r12);
        kz += 32;
        while (kz >= g.Kz) { kz -= g.Kz; row++; }
    }
}

// Shell-sum kernels: 256 threads, at most 42 registers, so six blocks fill an SM
// and a grid of SHELL_BLOCKS_PER_SM blocks per SM is one wave.
constexpr int SHELL_BLOCKS_PER_SM = 6;

template <typename T>
__global__ void __launch_bounds__(256, SHELL_BLOCKS_PER_SM) k_shell_sums(Geo g, const cx<T> *__restrict__ u, const cx<T> *__restrict__ v, const cx<T> *__restrict__ w,
                             const cx<T> *__restrict__ ulo, const cx<T> *__restrict__ vlo, const cx<T> *__restrict__ wlo,
                             int Kmax, double *__restrict__ Ek, double *__restrict__ Om) {
    extern __shared__ double hist[];
    double *hE = hist, *hO = hist + (Kmax + 1);
    for (int i = threadIdx.x; i < 2 * (Kmax + 1); i += blockDim.x) hist[i] = 0.0;
    __syncthreads();
    warp_mode_rounds(g, [&](bool valid, long long idx, int kz, long long r12) {
        int K = -1;
        double e = 0.0, o = 0.0;
        if (valid) {
            const long long k3 = (long long)g.sz * kz;
            const double rad2 = (double)(r12 + k3 * k3);
            K = (int)round(sqrt(rad2));
            if (K <= Kmax) {
                const cx<double> a = load_state(u, ulo, idx), b = load_state(v, vlo, idx), cc = load_state(w, wlo, idx);
                e = 0.5 * (a.x * a.x + a.y * a.y + b.x * b.x + b.y * b.y + cc.x * cc.x + cc.y * cc.y);
                if (kz != 0) e *= 2.0;
                o = 2.0 * rad2 * e;
            } else {
                K = -1;
            }
        }
        warp_shell_add(K, e, o, hE, hO);
    });
    __syncthreads();
    for (int i = threadIdx.x; i <= Kmax; i += blockDim.x) {
        if (hE[i] != 0.0) atomicAdd(&Ek[i], hE[i]);
        if (hO[i] != 0.0) atomicAdd(&Om[i], hO[i]);
    }
}

// Shell sums of |F|^2 (conjugate weight 2 for kz>0), scaled by `scale`: the
// spectrum of one scalar field (src/HIT_LES.cpp:1137-1214 with the integrands of
// the invariant spectra, :1006-1025).
template <typename T>
__global__ void __launch_bounds__(256, SHELL_BLOCKS_PER_SM) k_shell_sums_scalar(Geo g, const cx<T> *__restrict__ F, double scale, int Kmax, double *__restrict__ out) {
    extern __shared__ double hist[];
    for (int i = threadIdx.x; i <= Kmax; i += blockDim.x) hist[i] = 0.0;
    __syncthreads();
    warp_mode_rounds(g, [&](bool valid, long long idx, int kz, long long r12) {
        int K = -1;
        double e = 0.0;
        if (valid) {
            const long long k3 = (long long)g.sz * kz;
            K = (int)round(sqrt((double)(r12 + k3 * k3)));
            if (K <= Kmax) {
                const cx<T> a = F[idx];
                e = scale * ((double)a.x * a.x + (double)a.y * a.y);
                if (kz != 0) e *= 2.0;
            } else {
                K = -1;
            }
        }
        warp_shell_add(K, e, 0.0, hist, nullptr);
    });
    __syncthreads();
    for (int i = threadIdx.x; i <= Kmax; i += blockDim.x)
        if (hist[i] != 0.0) atomicAdd(&out[i], hist[i]);
}

// Totals of the shell sums: Ek_Tot over K=0..Kmax, Ok_Tot over K=1..Kmax.
// what: 0 energy only, 1 energy+enstrophy (+ReLambda), 2 Forcing_Reynolds_Lambda.
static __global__ void k_totals(const double *Ek, const double *Om, int Kmax, DevScalars *ds, int what, double relambda) {
    double e = 0.0, o = 0.0;
    for (int K = 0; K <= Kmax; K++) e += Ek[K];
    for (int K = 1; K <= Kmax; K++) o += Om[K];
    ds->ek_tot = e;
    if (what >= 1) ds->ok_tot = o;
    if (what == 1) ds->relambda = e / ds->nu * sqrt(20.0 / 3.0 / o);
    if (what == 2) ds->nu = e / relambda * sqrt(20.0 / 3.0 / o);
}

// Constant-power forcing coefficient alpha = eps/(2 E_f), E_f the energy of
// shells [kmin,kmax] of the current state (src/HIT_LES.cpp:250-256).
// Constant-power forcing amplitude (the disabled block of src/HIT_LES.cpp:243-278,
// with eps as a parameter): alpha = eps / (2 Ef), Ef the energy of the
// shells kmin..kmax of the state (the sum over those shells of the E(K) of k_shell_sums).
// Only modes with |s m| <= kmax + 1 on every axis can round into those shells,
// so one block visits that sub-box directly, in a fixed order with a fixed
// reduction tree: alpha does not depend on timing.  EPS_BAND_THREADS threads.
constexpr int EPS_BAND_THREADS = 256;
// partial (slab decomposition): only the rows this geometry holds are summed and the
// sum goes to ds->ef, for the caller to add up over the slabs and k_eps_alpha to use.
template <typename T>
__global__ void __launch_bounds__(EPS_BAND_THREADS) k_eps_band(Geo g, const cx<T> *__restrict__ u, const cx<T> *__restrict__ v,
                                                               const cx<T> *__restrict__ w, const cx<T> *__restrict__ ulo,
                                                               const cx<T> *__restrict__ vlo, const cx<T> *__restrict__ wlo,
                                                               int kmin, int kmax, double eps, DevScalars *ds, int partial = 0) {
    __shared__ double red[EPS_BAND_THREADS];
    const int mx = min(g.hx, (kmax + 1) / g.sx), my = min(g.hy, (kmax + 1) / g.sy), mz = min(g.hz, (kmax + 1) / g.sz);
    const int nx = 2 * mx + 1, ny = 2 * my + 1, nz = mz + 1;
    const int count = nx * ny * nz;
    double acc = 0.0;
    for (int c = threadIdx.x; c < count; c += EPS_BAND_THREADS) {
        const int kz = c % nz, t = c / nz;
        const int m1 = t % nx - mx, m2 = t / nx - my;
        const int ix = m1 >= 0 ? m1 : m1 + g.Kx, iy = (m2 >= 0 ? m2 : m2 + g.Kyg) - g.y0;
        if (iy < 0 || iy >= g.Ky) continue;   // row held by another slab
        const long long k1 = (long long)g.sx * m1, k2 = (long long)g.sy * m2, k3 = (long long)g.sz * kz;
        const int K = (int)round(sqrt((double)(k1 * k1 + k2 * k2 + k3 * k3)));
        if (K < kmin || K > kmax) continue;
        const long long idx = ((long long)iy * g.Kx + ix) * g.Kz + kz;
        const cx<double> a = load_state(u, ulo, idx), b = load_state(v, vlo, idx), cc = load_state(w, wlo, idx);
        double e = 0.5 * (a.x * a.x + a.y * a.y + b.x * b.x + b.y * b.y + cc.x * cc.x + cc.y * cc.y);
        if (kz != 0) e *= 2.0;
        acc += e;
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int o = EPS_BAND_THREADS / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double Ef = red[0];
        if (partial) ds->ef = Ef;
        else ds->alpha = Ef > 1e-30 ? eps / (2.0 * Ef) : 0.0;
    }
}

// alpha from the forced shells' energy summed over the slabs (ds->ef)
static __global__ void k_eps_alpha(double eps, DevScalars *ds) {
    const double Ef = ds->ef;
    ds->alpha = Ef > 1e-30 ? eps / (2.0 * Ef) : 0.0;
}


// src/HIT_LES.cpp:417-419: FT[K] = sqrt(Forced_Ek[K]/Ek[K]).
static __global__ void k_forcing_factors(const double *Ek, const double *Forced, int last_eff, double *FT) {
    for (int K = threadIdx.x; K <= last_eff; K += blockDim.x) FT[K] = Ek[K] > 0.0 ? sqrt(Forced[K] / Ek[K]) : 0.0;
}

// src/HIT_LES.cpp:421-438: scale shells K<=last_eff, optionally zero the rest.
// With lo parts (compensated single precision) the product is formed in double
// and split again into hi + lo.
template <typename T>
__global__ void k_forcing_scale(Geo g, cx<T> *u, cx<T> *v, cx<T> *w, cx<T> *ulo, cx<T> *vlo, cx<T> *wlo, const double *FT,
                                int last_eff, int nullify) {
    const long long n = g.S0;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += (long long)gridDim.x * blockDim.x) {
        const int kz = (int)(idx % g.Kz);
        const long long t = idx / g.Kz;
        const int ix = (int)(t % g.Kx), iy = (int)(t / g.Kx);
        const long long k1 = (long long)g.sx * (ix <= g.hx ? ix : ix - g.Kx);
        const long long k2 = (long long)g.sy * ky_mode(g, iy);
        const long long k3 = (long long)g.sz * kz;
        const int K = (int)round(sqrt((double)(k1 * k1 + k2 * k2 + k3 * k3)));
        if (K <= last_eff) {
            if (ulo) {
                cx<T> *hs[3] = {u, v, w}, *ls[3] = {ulo, vlo, wlo};
                for (int i = 0; i < 3; i++) {
                    const cx<double> x = load_state<T>(hs[i], ls[i], idx);
                    const double xr = FT[K] * x.x, xi = FT[K] * x.y;
                    const T hr = T(xr), hi = T(xi);
                    hs[i][idx] = mk<T>(hr, hi);
                    ls[i][idx] = mk<T>(T(xr - (double)hr), T(xi - (double)hi));
                }
            } else {
                const T f = T(FT[K]);
                u[idx] = f * u[idx]; v[idx] = f * v[idx]; w[idx] = f * w[idx];
            }
        } else if (nullify) {
            u[idx] = zero<T>(); v[idx] = zero<T>(); w[idx] = zero<T>();
            if (ulo) { ulo[idx] = zero<T>(); vlo[idx] = zero<T>(); wlo[idx] = zero<T>(); }
        }
    }
}

// src/HIT_LES.cpp:446-476 on the kz=0 plane: u(k1<0 or k1=0,k2<0) = conj(u(-k)).
// The written and the read halves are disjoint, so no staging copy is needed.
template <typename T>
__global__ void k_conj_correction(Geo g, cx<T> *u, cx<T> *v, cx<T> *w, cx<T> *ulo, cx<T> *vlo, cx<T> *wlo) {
    const int n = g.Kx * g.Ky;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const int ix = t % g.Kx, iy = t / g.Kx;
        const int m1 = ix <= g.hx ? ix : ix - g.Kx, m2 = iy <= g.hy ? iy : iy - g.Ky;
        if (m1 < 0 || (m1 == 0 && m2 < 0)) {
            const int jx = -m1, jy = -m2 >= 0 ? -m2 : -m2 + g.Ky;
            const long long dst = ((long long)iy * g.Kx + ix) * g.Kz, src = ((long long)jy * g.Kx + jx) * g.Kz;
            u[dst] = conj(u[src]); v[dst] = conj(v[src]); w[dst] = conj(w[src]);
            if (ulo) { ulo[dst] = conj(ulo[src]); vlo[dst] = conj(vlo[src]); wlo[dst] = conj(wlo[src]); }
        }
    }
}

// ===========================================================================
// Slab decomposition: reorder of a [nf][n1][n2][Kz] array into per-rank blocks
// [s][f][n1_s][n2_s][Kz] split along axis 1 (rows n1) or 2 (n2) by the ranks'
// block ranges (FFTW-MPI's default block: ceil(n/ranks) per rank), and back.
// Block s starts at off[s] of the staging array; a rank's outgoing blocks are
// contiguous there, in rank order, as an all-to-all sends them.
// ===========================================================================
#define SPNS_SLAB_MAX_RANKS 64
struct SlabRanges {
    int n, blk;                          // ranks, block size of the split axis
    int start[SPNS_SLAB_MAX_RANKS], count[SPNS_SLAB_MAX_RANKS];
    long long off[SPNS_SLAB_MAX_RANKS];  // element offset of rank s's block in the staging array
};
template <typename T>
__global__ void k_slab_pack(cx<T> *__restrict__ full, cx<T> *__restrict__ stage, int nf, int n1, int n2, int Kz, SlabRanges r, int axis,
                            int unpack) {
    const long long n = (long long)nf * n1 * n2 * Kz;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += (long long)gridDim.x * blockDim.x) {
        const int kz = (int)(idx % Kz);
        long long t = idx / Kz;
        const int i2 = (int)(t % n2);
        t /= n2;
        const int i1 = (int)(t % n1), f = (int)(t / n1);
        const int a = axis == 1 ? i1 : i2;
        const int s = a / r.blk;
        const int loc = a - r.start[s];
        const int n1s = axis == 1 ? r.count[s] : n1, n2s = axis == 1 ? n2 : r.count[s];
        const long long st = r.off[s] + (((long long)f * n1s + (axis == 1 ? loc : i1)) * n2s + (axis == 1 ? i2 : loc)) * Kz + kz;
        if (unpack) full[idx] = stage[st];
        else stage[st] = full[idx];
    }
}

// ===========================================================================
// Seeded initial field on the device (no reference counterpart: the reference
// starts from its K41 draw or a file).  Philox4x32-10 (Salmon, Moraes, Dror and
// Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC'11), key = seed,
// counter = (compact mode index, draw number), so every mode draws its own
// numbers and the field does not depend on the launch shape.
// ===========================================================================
struct Philox4 { unsigned x, y, z, w; };
__host__ __device__ __forceinline__ Philox4 philox4x32_10(Philox4 c, unsigned k0, unsigned k1) {
#pragma unroll
    for (int r = 0; r < 10; r++) {
        const unsigned long long p0 = 0xD2511F53ull * c.x, p1 = 0xCD9E8D57ull * c.z;
        Philox4 n;
        n.x = (unsigned)(p1 >> 32) ^ c.y ^ k0;
        n.y = (unsigned)p1;
        n.z = (unsigned)(p0 >> 32) ^ c.w ^ k1;
        n.w = (unsigned)p0;
        c = n;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return c;
}

// Two standard normals from one Philox block: two 53-bit uniforms, Box-Muller.
__device__ __forceinline__ void philox_normal2(unsigned long long idx, unsigned draw, unsigned long long seed, double &z0, double &z1) {
    Philox4 c{(unsigned)idx, (unsigned)(idx >> 32), draw, 0u};
    const Philox4 r = philox4x32_10(c, (unsigned)seed, (unsigned)(seed >> 32));
    const double u0 = (double)(((unsigned long long)(r.x >> 5) << 26) | (r.y >> 6)) * 0x1.0p-53;
    const double u1 = (double)(((unsigned long long)(r.z >> 5) << 26) | (r.w >> 6)) * 0x1.0p-53;
    const double rad = sqrt(-2.0 * log(1.0 - u0));
    double sn, cs;
    sincospi(2.0 * u1, &sn, &cs);
    z0 = rad * cs;
    z1 = rad * sn;
}

// Complex Gaussian velocity of every retained mode, projected onto k-perp;
// zero outside |m_i| <= lim_i and at k=0; on kz=0 the half with m1<0 (or
// m1=0, m2<0) is the conjugate of its partner's draw.  Written as the state
// (hi + lo split when lo is given).
template <typename T>
__global__ void k_seed_draw(Geo g, unsigned long long seed, int lim_x, int lim_y, int lim_z, cx<T> *u, cx<T> *v, cx<T> *w,
                            cx<T> *ulo, cx<T> *vlo, cx<T> *wlo) {
    const long long n = g.S0;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += (long long)gridDim.x * blockDim.x) {
        const int kz = (int)(idx % g.Kz);
        const long long t = idx / g.Kz;
        const int ix = (int)(t % g.Kx), iy = (int)(t / g.Kx);
        int m1 = ix <= g.hx ? ix : ix - g.Kx, m2 = iy <= g.hy ? iy : iy - g.Ky;
        const double k1 = (double)g.sx * m1, k2 = (double)g.sy * m2, k3 = (double)g.sz * kz;
        const double k2s = k1 * k1 + k2 * k2 + k3 * k3;
        const bool keep = (m1 <= lim_x && -m1 <= lim_x && m2 <= lim_y && -m2 <= lim_y && kz <= lim_z && k2s > 0.0);
        double re[3] = {0.0, 0.0, 0.0}, im[3] = {0.0, 0.0, 0.0};
        if (keep) {
            const bool mirror = kz == 0 && (m1 < 0 || (m1 == 0 && m2 < 0));
            long long src = idx;
            if (mirror) {
                const int p1 = -m1, p2 = -m2;
                src = ((long long)(p2 >= 0 ? p2 : p2 + g.Ky) * g.Kx + (p1 >= 0 ? p1 : p1 + g.Kx)) * g.Kz;
            }
            for (int c = 0; c < 3; c++) philox_normal2((unsigned long long)src, (unsigned)c, seed, re[c], im[c]);
            const double kk[3] = {mirror ? -k1 : k1, mirror ? -k2 : k2, k3};
            const double dr = (kk[0] * re[0] + kk[1] * re[1] + kk[2] * re[2]) / k2s;
            const double di = (kk[0] * im[0] + kk[1] * im[1] + kk[2] * im[2]) / k2s;
            for (int c = 0; c < 3; c++) { re[c] -= dr * kk[c]; im[c] -= di * kk[c]; }
            if (mirror) for (int c = 0; c < 3; c++) im[c] = -im[c];
        }
        cx<T> *hs[3] = {u, v, w}, *ls[3] = {ulo, vlo, wlo};
        for (int c = 0; c < 3; c++) {
            const T hr = T(re[c]), hi = T(im[c]);
            hs[c][idx] = mk<T>(hr, hi);
            if (ulo) ls[c][idx] = mk<T>(T(re[c] - (double)hr), T(im[c] - (double)hi));
        }
    }
}

// Shell factors of the seeded field: target(K) = K^4 exp(-2 (K/kp)^2) on the
// non-empty shells K >= 1, normalised to total energy 3/2 urms^2;
// FT[K] = sqrt(target(K) / E(K)).  One block.
static __global__ void k_seed_factors(const double *Ek, int Kmax, double kp, double urms, double *FT) {
    __shared__ double tot;
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int K = 1; K <= Kmax; K++)
            if (Ek[K] > 0.0) { const double x = (double)K / kp; s += (double)K * K * K * K * exp(-2.0 * x * x); }
        tot = s;
    }
    __syncthreads();
    for (int K = threadIdx.x; K <= Kmax; K += blockDim.x) {
        double f = 0.0;
        if (K >= 1 && Ek[K] > 0.0 && tot > 0.0) {
            const double x = (double)K / kp;
            const double target = (double)K * K * K * K * exp(-2.0 * x * x) * (1.5 * urms * urms) / tot;
            f = sqrt(target / Ek[K]);
        }
        FT[K] = f;
    }
}

// Direct DFT along one axis (initial-field transform of the input file; init only).
// in: complex lines, out: complex lines; out[o][k] = sum_n in[o][n] * w^(k*n mod N).
// Line l of `nl` lines starts at (l / inner)*outer_stride + (l % inner), element stride `es`.
static __global__ void k_dft_axis(const double2 *__restrict__ in, double2 *__restrict__ out, int N, int nk, const int *__restrict__ kidx,
                           long long nl, long long inner, long long in_outer, long long out_outer, long long es_in,
                           long long es_out, const double2 *__restrict__ twN) {
    const long long tot = nl * nk;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += (long long)gridDim.x * blockDim.x) {
        const int kk = (int)(t % nk);
        const long long l = t / nk;
        const long long ib = (l / inner) * in_outer + (l % inner), ob = (l / inner) * out_outer + (l % inner);
        const int k = kidx[kk];
        double sr = 0.0, si = 0.0;
        long long m = 0;
        for (int n = 0; n < N; n++) {
            const double2 a = in[ib + n * es_in], wv = twN[m];
            sr += a.x * wv.x - a.y * wv.y;
            si += a.x * wv.y + a.y * wv.x;
            m += k; if (m >= N) m -= N;
        }
        out[ob + (long long)kk * es_out] = make_double2(sr, si);
    }
}

// ===========================================================================
// Kernels of the passes, for one box and for a batch of boxes of the same
// geometry and launch shape.  A batch runs one launch per pass for all its
// members: blockIdx.z selects the member, whose buffers, scalars and constants
// come from a device table (BatchMember).  The arithmetic is the one-box kernel's.
// ===========================================================================
template <typename T, int L, int E, int P, int MODE>
__global__ void __launch_bounds__(P *(L / E), AxisMinBlocks<T, 1>::N) k1_inv_x(Geo g, const cx<T> *__restrict__ u, const cx<T> *__restrict__ v,
                                                                           const cx<T> *__restrict__ w, cx<T> *__restrict__ out,
                                                                           const cx<T> *__restrict__ tw) {
    k1_inv_x_body<T, L, E, P, MODE>(g, u, v, w, out, tw);
}
template <typename T, int L, int E, int P, int MODE>
__global__ void __launch_bounds__(P *(L / E), AxisMinBlocks<T, 2>::N) k2_inv_y(Geo g, const cx<T> *__restrict__ in, cx<T> *__restrict__ out,
                                                                           const cx<T> *__restrict__ tw) {
    k2_inv_y_body<T, L, E, P, MODE>(g, in, out, tw);
}
template <typename T, int L, int E, int P, int MODE, bool STAGE = false>
__global__ void __launch_bounds__(P *(L / E), K3MinBlocks<T, MODE, P *(L / E)>::N) k3_z(Geo g, cx<T> *__restrict__ buf, StepConsts c,
                                                                                        DevScalars *ds, double *__restrict__ phys,
                                                                                        const cx<T> *__restrict__ tw) {
    k3_z_body<T, L, E, P, MODE, STAGE>(g, buf, c, ds, phys, tw);
}
template <typename T, int L, int E, int P, int MODE>
__global__ void __launch_bounds__(P *(L / E), AxisMinBlocks<T, 4>::N) k4_fwd_y(Geo g, const cx<T> *__restrict__ in, cx<T> *__restrict__ out,
                                                                           const cx<T> *__restrict__ tw) {
    k4_fwd_y_body<T, L, E, P, MODE>(g, in, out, tw);
}
template <typename T, int L, int E, int P, int MODE>
__global__ void __launch_bounds__(P *(L / E), AxisMinBlocks<T, 5>::N) k5_fwd_x(Geo g, const cx<T> *__restrict__ in, cx<T> *__restrict__ G,
                                                                           const cx<T> *__restrict__ tw) {
    k5_fwd_x_body<T, L, E, P, MODE>(g, in, G, tw);
}
template <typename T, bool SELF>
__global__ void __launch_bounds__(256) k6_sweep(Geo g, const cx<T> *__restrict__ G, const cx<T> *U, const cx<T> *Ulo, cx<T> *R, cx<T> *Uout,
                                                cx<T> *Uoutlo, const cx<T> *Un1, const cx<T> *Un1lo, StepConsts c,
                                                const DevScalars *__restrict__ ds) {
    k6_sweep_body<T, SELF>(g, G, U, Ulo, R, Uout, Uoutlo, Un1, Un1lo, c, ds);
}

// One member of a batched launch.  The state is [3][S0] (hi parts; Ulo the
// compensated form's lo parts, else null), R the previous right-hand side, B1/B2
// the S1/S2 work buffers (B2 also holds the nonlinear term after the x pass).
struct BatchMember {
    void *U, *Ulo, *R, *B1, *B2;
    DevScalars *ds;
    StepConsts c;
};
template <typename T, int L, int E, int P, int MODE>
__global__ void __launch_bounds__(P *(L / E), AxisMinBlocks<T, 1>::N) k1_inv_x_batch(Geo g, const BatchMember *__restrict__ tab,
                                                                                 const cx<T> *__restrict__ tw) {
    const BatchMember &m = tab[blockIdx.z];
    const cx<T> *U = static_cast<const cx<T> *>(m.U);
    k1_inv_x_body<T, L, E, P, MODE>(g, U, U + g.S0, U + 2 * g.S0, static_cast<cx<T> *>(m.B1), tw);
}
template <typename T, int L, int E, int P, int MODE>
__global__ void __launch_bounds__(P *(L / E), AxisMinBlocks<T, 2>::N) k2_inv_y_batch(Geo g, const BatchMember *__restrict__ tab,
                                                                                 const cx<T> *__restrict__ tw) {
    const BatchMember &m = tab[blockIdx.z];
    k2_inv_y_body<T, L, E, P, MODE>(g, static_cast<const cx<T> *>(m.B1), static_cast<cx<T> *>(m.B2), tw);
}
template <typename T, int L, int E, int P, int MODE, bool STAGE = false>
__global__ void __launch_bounds__(P *(L / E), K3MinBlocks<T, MODE, P *(L / E)>::N) k3_z_batch(Geo g, const BatchMember *__restrict__ tab,
                                                                                              const cx<T> *__restrict__ tw) {
    const BatchMember &m = tab[blockIdx.z];
    k3_z_body<T, L, E, P, MODE, STAGE>(g, static_cast<cx<T> *>(m.B2), m.c, m.ds, nullptr, tw);
}
template <typename T, int L, int E, int P, int MODE>
__global__ void __launch_bounds__(P *(L / E), AxisMinBlocks<T, 4>::N) k4_fwd_y_batch(Geo g, const BatchMember *__restrict__ tab,
                                                                                 const cx<T> *__restrict__ tw) {
    const BatchMember &m = tab[blockIdx.z];
    k4_fwd_y_body<T, L, E, P, MODE>(g, static_cast<const cx<T> *>(m.B2), static_cast<cx<T> *>(m.B1), tw);
}
template <typename T, int L, int E, int P, int MODE>
__global__ void __launch_bounds__(P *(L / E), AxisMinBlocks<T, 5>::N) k5_fwd_x_batch(Geo g, const BatchMember *__restrict__ tab,
                                                                                 const cx<T> *__restrict__ tw) {
    const BatchMember &m = tab[blockIdx.z];
    k5_fwd_x_body<T, L, E, P, MODE>(g, static_cast<const cx<T> *>(m.B1), static_cast<cx<T> *>(m.B2), tw);
}
// Adams-Bashforth members only (the kappa scheme swaps state buffers every step).
template <typename T>
__global__ void __launch_bounds__(256) k6_sweep_batch(Geo g, const BatchMember *__restrict__ tab) {
    const BatchMember &m = tab[blockIdx.z];
    cx<T> *U = static_cast<cx<T> *>(m.U), *Ulo = static_cast<cx<T> *>(m.Ulo);
    k6_sweep_body<T, false>(g, static_cast<const cx<T> *>(m.B2), U, Ulo, static_cast<cx<T> *>(m.R), U, Ulo, nullptr, nullptr, m.c, m.ds);
}
static __global__ void k_reset_max_batch(const BatchMember *__restrict__ tab) {
    DevScalars *ds = tab[blockIdx.x].ds;
    for (int i = 0; i < 4; i++) ds->max_bits[i] = 0ull;
    ds->sumsq_phys = 0.0;
}
static __global__ void k_finish_step_batch(const BatchMember *__restrict__ tab) {
    const BatchMember &m = tab[blockIdx.x];
    recalc_dt(m.c, m.ds);
    m.ds->time = m.ds->time + m.ds->dt;
    m.ds->iter += 1;
}

} // namespace spns
