// fft_core.cuh -- register/shared-memory Stockham FFT engine for sm_100a.
//
// One pencil of length L is processed by Q = L/E threads, each holding E
// complex values in registers.  A stage of radix R performs E/R butterflies
// per thread; between stages the values are exchanged through shared memory
// (one buffer, two barriers per stage; warp barriers when a pencil lives in
// one warp).  The first stage reads its inputs from registers filled by the
// caller at rows  j + r*(L/R_first)  and the last stage leaves its outputs in
// registers at rows  j + r*(L/R_last)  (j = q + Q*m), so callers load pencils
// straight from global memory and store results straight back (or keep them
// in registers for fused pointwise work).
//
// Stockham autosort, stage (R, Ns): butterfly j, k = j mod Ns,
//   inputs  x_r = in[j + r*L/R],  x_r *= w_L^{r*k*L/(Ns*R)},  y = DFT_R(x),
//   outputs out[(j/Ns)*Ns*R + k + r*Ns] = y_r.
// Radices 2, 3, 4, 6, 8, 12: the composite ones with a factor 3 use the
// prime-factor (Good-Thomas) split 2x3 / 4x3, which needs no inner twiddles.
// Twiddles: w^1 of a butterfly is read from a table w_L^m = exp(-2 pi i m/L)
// computed on the host in extended precision.  Stage (R, Ns) needs w_L^{r k L/(Ns R)}
// = w_n^{r k} with n = Ns R and k = j mod Ns; the table carries, after its L base
// entries, a copy w_n^m of the base values for every divisor n < L of L
// (tw_sub_offset), so the lanes of a warp (consecutive k) read consecutive
// entries instead of entries L/n apart: one or two L1 wavefronts per warp load
// instead of up to 32 lines.  The values are the same table entries, so results
// do not change.  In double precision its powers
// w^r are formed by repeated complex multiplication (one table read per
// butterfly instead of R-1: the table reads contend with the shared-memory
// exchange for the load/store pipe); in single precision, where a chain of up
// to 10 products would add ~1e-6 relative error, the powers of two are read
// from the table and every other power is one or two products of them
// (twiddle_powers).  The inverse uses the conjugates.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "fft_layouts.h"

namespace spns {

template <typename T> struct alignas(2 * sizeof(T)) cx { T x, y; };

template <typename T> __device__ __forceinline__ cx<T> mk(T a, T b) { cx<T> r; r.x = a; r.y = b; return r; }
template <typename T> __device__ __forceinline__ cx<T> operator+(cx<T> a, cx<T> b) { return mk<T>(a.x + b.x, a.y + b.y); }
template <typename T> __device__ __forceinline__ cx<T> operator-(cx<T> a, cx<T> b) { return mk<T>(a.x - b.x, a.y - b.y); }
template <typename T> __device__ __forceinline__ cx<T> operator*(T s, cx<T> a) { return mk<T>(s * a.x, s * a.y); }
template <typename T> __device__ __forceinline__ cx<T> cmul(cx<T> a, cx<T> b) { return mk<T>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
template <typename T> __device__ __forceinline__ cx<T> cmulc(cx<T> a, cx<T> b) { return mk<T>(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y); }
template <typename T> __device__ __forceinline__ cx<T> conj(cx<T> a) { return mk<T>(a.x, -a.y); }
// i*a
template <typename T> __device__ __forceinline__ cx<T> mul_i(cx<T> a) { return mk<T>(-a.y, a.x); }
template <typename T> __device__ __forceinline__ cx<T> zero() { return mk<T>(T(0), T(0)); }

// ---------------------------------------------------------------------------
// Radix plan: greedy factors of L from {12, 8, 6, 4, 3, 2}, each dividing E.
// Forward order = greedy order, inverse order = reversed, so the last radix of
// an inverse transform equals the first radix of a forward one (the register
// hand-off between them needs the same row mapping).
// ---------------------------------------------------------------------------
__host__ __device__ constexpr int pick_radix(int rem, int E) {
    return (rem % 12 == 0 && E % 12 == 0) ? 12
         : (rem % 8 == 0 && E % 8 == 0) ? 8
         : (rem % 6 == 0 && E % 6 == 0) ? 6
         : (rem % 4 == 0 && E % 4 == 0) ? 4
         : (rem % 3 == 0 && E % 3 == 0) ? 3
         : (rem % 2 == 0 && E % 2 == 0) ? 2 : 0;
}
__host__ __device__ constexpr int n_stages(int L, int E) {
    int n = 0, rem = L;
    while (rem > 1) { int r = pick_radix(rem, E); if (r == 0) return -1; rem /= r; n++; }
    return n;
}
__host__ __device__ constexpr int greedy_radix(int L, int E, int s) {
    int rem = L;
    for (int i = 0; i < s; i++) rem /= pick_radix(rem, E);
    return pick_radix(rem, E);
}
template <int L, int E, bool INV> struct Plan {
    static constexpr int NST = n_stages(L, E);
    static_assert(NST > 0, "length not factorable with radices dividing E");
    static_assert(L % E == 0, "E must divide L");
    static constexpr int Q = L / E;
    __host__ __device__ static constexpr int radix(int s) { return INV ? greedy_radix(L, E, NST - 1 - s) : greedy_radix(L, E, s); }
    __host__ __device__ static constexpr int ns(int s) { int p = 1; for (int i = 0; i < s; i++) p *= radix(i); return p; }
    static constexpr int R_first = radix(0);
    static constexpr int R_last = radix(NST - 1);
};

// ---------------------------------------------------------------------------
// Small DFTs (in place); INV selects exp(+2*pi*i/R).
// ---------------------------------------------------------------------------
template <typename T, bool INV> __device__ __forceinline__ void dft2(cx<T> *x) {
    cx<T> a = x[0], b = x[1];
    x[0] = a + b; x[1] = a - b;
}
template <typename T, bool INV> __device__ __forceinline__ void dft3(cx<T> *x) {
    const T c3 = T(-0.5);
    const T s3 = INV ? T(0.86602540378443864676372317075294) : T(-0.86602540378443864676372317075294);
    cx<T> s = x[1] + x[2], d = x[1] - x[2];
    cx<T> y0 = x[0] + s;
    cx<T> m = mk<T>(x[0].x + c3 * s.x, x[0].y + c3 * s.y);
    cx<T> e = mk<T>(-s3 * d.y, s3 * d.x);
    x[0] = y0; x[1] = m + e; x[2] = m - e;
}
template <typename T, bool INV> __device__ __forceinline__ void dft4(cx<T> *x) {
    cx<T> t0 = x[0] + x[2], t1 = x[0] - x[2], t2 = x[1] + x[3], t3 = x[1] - x[3];
    cx<T> u = INV ? mk<T>(-t3.y, t3.x) : mk<T>(t3.y, -t3.x); // (+/-i)*t3
    x[0] = t0 + t2; x[2] = t0 - t2; x[1] = t1 + u; x[3] = t1 - u;
}
template <typename T, bool INV> __device__ __forceinline__ void dft8(cx<T> *x) {
    const T h = T(0.70710678118654752440084436210485);
    cx<T> e[4] = {x[0], x[2], x[4], x[6]}, o[4] = {x[1], x[3], x[5], x[7]};
    dft4<T, INV>(e); dft4<T, INV>(o);
    // w8^k for k=1..3: forward exp(-i*pi*k/4)
    cx<T> o1 = INV ? mk<T>(h * (o[1].x - o[1].y), h * (o[1].x + o[1].y)) : mk<T>(h * (o[1].x + o[1].y), h * (o[1].y - o[1].x));
    cx<T> o2 = INV ? mk<T>(-o[2].y, o[2].x) : mk<T>(o[2].y, -o[2].x);
    cx<T> o3 = INV ? mk<T>(-h * (o[3].x + o[3].y), h * (o[3].x - o[3].y)) : mk<T>(h * (o[3].y - o[3].x), -h * (o[3].x + o[3].y));
    x[0] = e[0] + o[0]; x[4] = e[0] - o[0];
    x[1] = e[1] + o1;   x[5] = e[1] - o1;
    x[2] = e[2] + o2;   x[6] = e[2] - o2;
    x[3] = e[3] + o3;   x[7] = e[3] - o3;
}
// Good-Thomas split of R = A*B (gcd 1): input n = (B a + A b) mod R, output
// k with k = ka (mod A), k = kb (mod B); DFT_A over a, then DFT_B over b.
template <int A, int B> struct PFA {
    static constexpr int R = A * B;
    __host__ __device__ static constexpr int in(int a, int b) { return (B * a + A * b) % R; }
    __host__ __device__ static constexpr int out(int ka, int kb) {
        int invB = 1;
        while ((B * invB) % A != 1 % A) invB++;
        int invA = 1;
        while ((A * invA) % B != 1 % B) invA++;
        return (ka * B * invB + kb * A * invA) % R;
    }
};
template <typename T, bool INV, int A, int B> __device__ __forceinline__ void dft_pfa(cx<T> *x) {
    using P = PFA<A, B>;
    cx<T> t[A * B];
#pragma unroll
    for (int b = 0; b < B; b++) {
        cx<T> col[A];
#pragma unroll
        for (int a = 0; a < A; a++) col[a] = x[P::in(a, b)];
        if constexpr (A == 2) dft2<T, INV>(col);
        else if constexpr (A == 4) dft4<T, INV>(col);
        else dft8<T, INV>(col);
#pragma unroll
        for (int a = 0; a < A; a++) t[a * B + b] = col[a];
    }
#pragma unroll
    for (int ka = 0; ka < A; ka++) {
        cx<T> row[B];
#pragma unroll
        for (int b = 0; b < B; b++) row[b] = t[ka * B + b];
        dft3<T, INV>(row);
#pragma unroll
        for (int kb = 0; kb < B; kb++) x[P::out(ka, kb)] = row[kb];
    }
}
template <typename T, int R, bool INV> __device__ __forceinline__ void dft(cx<T> *x) {
    if constexpr (R == 2) dft2<T, INV>(x);
    else if constexpr (R == 3) dft3<T, INV>(x);
    else if constexpr (R == 4) dft4<T, INV>(x);
    else if constexpr (R == 6) dft_pfa<T, INV, 2, 3>(x);
    else if constexpr (R == 8) dft8<T, INV>(x);
    else if constexpr (R == 12) dft_pfa<T, INV, 4, 3>(x);
}

// ---------------------------------------------------------------------------
// Stage engine.  SM is a shared-memory accessor:  cx<T>& SM::at(int row).
// v[m*R + r] holds the input (before the stage) / output (after) of butterfly
// j = q + Q*m, leg r.  WARP: the threads of a pencil exchange within one warp.
// ---------------------------------------------------------------------------
template <class SM, class = void> struct SmPadded { static constexpr bool value = false; };
template <class SM> struct SmPadded<SM, decltype((void)SM::PADDED)> { static constexpr bool value = SM::PADDED; };
// layout of exchange S of a padded accessor (pad >= 0, or -1 for the XOR swizzle); 0 for the others
template <class SM, bool INV, int S> __host__ __device__ constexpr int ex_pad() {
    if constexpr (SmPadded<SM>::value) return SM::template Ex<INV, S>::PAD;
    else return 0;
}

// Offset of the sub-table w_n^m (m < n) in a twiddle table of length L: 0 for
// n = L (the base table), else L plus the sizes of the sub-tables of the divisors
// of L below n (spns_make_twiddles lays them out in increasing n).
__host__ __device__ constexpr int tw_sub_offset(int L, int n) {
    if (n >= L) return 0;
    int off = L;
    for (int d = 2; d < n; d++)
        if (L % d == 0) off += d;
    return off;
}
// Entries of a twiddle table of length L with all its sub-tables.
__host__ __device__ constexpr int tw_table_size(int L) {
    int s = L;
    for (int d = 2; d < L; d++)
        if (L % d == 0) s += d;
    return s;
}
// Single precision reads the powers of two of a butterfly's twiddle; w_n^{r k} for
// r = 2, 4, 8 sits in a power table of its own (n entries, k contiguous) so that those
// reads are contiguous across a warp too.  Three power tables follow the sub-tables,
// each holding every divisor n >= 2 of L (L included) in increasing n.
__host__ __device__ constexpr int tw_pow_offset(int L, int n, int r) {
    const int ri = r == 2 ? 0 : r == 4 ? 1 : 2;
    int off = tw_table_size(L) * (1 + ri);
    for (int d = 2; d < n; d++)
        if (L % d == 0) off += d;
    return off;
}
__host__ __device__ constexpr int tw_full_size(int L) { return 4 * tw_table_size(L); }

template <bool WARP> __device__ __forceinline__ void stage_barrier() {
    if constexpr (WARP) __syncwarp(); else __syncthreads();
}

// Single precision: the powers w^r of a butterfly's twiddle.  With SPNS_F32_TW_POW the
// powers of two come from the table and the others are one or two products of
// them (w^3 = w^2 w, w^7 = w^4 w^3, ...; about 2e-7 relative error at most), which
// reads 4 instead of 11 table entries for a radix-12 butterfly; without it every
// power is read.  At N=512 the single-precision z pass took 10.31 ms against 11.89.
#ifndef SPNS_F32_TW_POW
#define SPNS_F32_TW_POW 1
#endif
template <typename T, int R>
__device__ __forceinline__ void twiddle_powers(cx<T> (&wp)[R], const cx<T> *__restrict__ tw, int step) {
#pragma unroll
    for (int r = 1; r < R; r++) {
        if (!SPNS_F32_TW_POW || (r & (r - 1)) == 0) {
            wp[r] = tw[r * step];
        } else {
            int hb = 1;
            while (hb * 2 <= r) hb *= 2;
            wp[r] = cmul(wp[hb], wp[r - hb]);
        }
    }
}

template <typename T, int L, int E, bool INV, bool WARP, int S, class SM>
__device__ __forceinline__ void fft_run(cx<T> (&v)[E], SM sm, int q, const cx<T> *__restrict__ tw) {
    using PL = Plan<L, E, INV>;
    constexpr int R = PL::radix(S);
    constexpr int Ns = PL::ns(S);
    constexpr int Q = PL::Q;
    constexpr int MB = E / R;
#pragma unroll
    for (int m = 0; m < MB; m++) {
        if constexpr (Ns > 1) {
            const int j = q + Q * m;
            const int k = j % Ns;                  // w^r = w_n^{r k}, n = Ns R, r k < n
            constexpr int TWO = tw_sub_offset(L, Ns * R);
            const cx<T> *__restrict__ twn = tw + TWO;
            if constexpr (sizeof(T) == 4) {
                cx<T> wp[R];
                if constexpr (SPNS_F32_TW_POW) {
                    constexpr int P2 = tw_pow_offset(L, Ns * R, 2), P4 = tw_pow_offset(L, Ns * R, 4),
                                  P8 = tw_pow_offset(L, Ns * R, 8);
                    wp[1] = twn[k];
#pragma unroll
                    for (int r = 2; r < R; r++) {
                        if (r == 2) wp[r] = tw[P2 + k];
                        else if (r == 4) wp[r] = tw[P4 + k];
                        else if (r == 8) wp[r] = tw[P8 + k];
                        else {
                            int hb = 1;
                            while (hb * 2 <= r) hb *= 2;
                            wp[r] = cmul(wp[hb], wp[r - hb]);
                        }
                    }
                } else {
                    twiddle_powers<T, R>(wp, twn, k);
                }
#pragma unroll
                for (int r = 1; r < R; r++) v[m * R + r] = INV ? cmulc(v[m * R + r], wp[r]) : cmul(v[m * R + r], wp[r]);
            } else {
                const cx<T> w1 = twn[k];
                cx<T> w = w1;
#pragma unroll
                for (int r = 1; r < R; r++) {
                    v[m * R + r] = INV ? cmulc(v[m * R + r], w) : cmul(v[m * R + r], w);
                    if (r + 1 < R) w = cmul(w, w1);
                }
            }
        }
        dft<T, R, INV>(&v[m * R]);
    }
    if constexpr (S + 1 < PL::NST) {
        constexpr int R2 = PL::radix(S + 1);
        constexpr int MB2 = E / R2;
        if constexpr (ex_pad<SM, INV, S>() < 0) {
            // XOR-swizzled layout (fewer bank conflicts for this exchange)
#pragma unroll
            for (int m = 0; m < MB; m++) {
                const int j = q + Q * m;
                const int base = (j / Ns) * Ns * R + (j % Ns);
#pragma unroll
                for (int r = 0; r < R; r++) sm.xr(base + r * Ns) = v[m * R + r];
            }
            stage_barrier<WARP>();
#pragma unroll
            for (int m = 0; m < MB2; m++) {
                const int j = q + Q * m;
#pragma unroll
                for (int r = 0; r < R2; r++) v[m * R2 + r] = sm.xr(j + r * (L / R2));
            }
            stage_barrier<WARP>();
        } else if constexpr (SmPadded<SM>::value) {
            // padded layout: one base address per butterfly group, offsets in the instructions
            constexpr int X = Ns * R, PAD = SM::template Ex<INV, S>::PAD, XP = X + PAD;
            cx<T> *const b = sm.base;
#pragma unroll
            for (int m = 0; m < MB; m++) {
                cx<T> *w;
                if constexpr (Q % Ns == 0) {
                    w = b + (q / Ns) * XP + (q % Ns) + m * (Q / Ns) * XP;
                } else {
                    const int j = q + Q * m, hi = j / Ns;
                    w = b + hi * XP + (j - hi * Ns);
                }
#pragma unroll
                for (int r = 0; r < R; r++) w[r * Ns] = v[m * R + r];
            }
            stage_barrier<WARP>();
            constexpr int STEP = L / R2, PSTEP = STEP + (STEP / X) * PAD;
            static_assert(STEP % X == 0, "exchange read stride must be a multiple of the pad block");
#pragma unroll
            for (int m = 0; m < MB2; m++) {
                const cx<T> *rd;
                if constexpr (Q % X == 0) {
                    rd = b + q + (q / X) * PAD + m * (Q + (Q / X) * PAD);
                } else {
                    const int row = q + Q * m;
                    rd = b + row + (row / X) * PAD;
                }
#pragma unroll
                for (int r = 0; r < R2; r++) v[m * R2 + r] = rd[r * PSTEP];
            }
            stage_barrier<WARP>();
        } else {
#pragma unroll
            for (int m = 0; m < MB; m++) {
                const int j = q + Q * m;
                const int base = (j / Ns) * Ns * R + (j % Ns);
#pragma unroll
                for (int r = 0; r < R; r++) sm.at(base + r * Ns) = v[m * R + r];
            }
            stage_barrier<WARP>();
#pragma unroll
            for (int m = 0; m < MB2; m++) {
                const int j = q + Q * m;
#pragma unroll
                for (int r = 0; r < R2; r++) v[m * R2 + r] = sm.at(j + r * (L / R2));
            }
            stage_barrier<WARP>();
        }
        fft_run<T, L, E, INV, WARP, S + 1, SM>(v, sm, q, tw);
    }
}

// Row of register slot e before the first stage (inputs) / after the last stage (outputs).
template <int L, int E, bool INV> __device__ __forceinline__ int in_row(int q, int e) {
    using PL = Plan<L, E, INV>;
    constexpr int R = PL::R_first;
    return q + PL::Q * (e / R) + (e % R) * (L / R);
}
template <int L, int E, bool INV> __device__ __forceinline__ int out_row(int q, int e) {
    using PL = Plan<L, E, INV>;
    constexpr int R = PL::R_last;
    return q + PL::Q * (e / R) + (e % R) * (L / R);
}

// The thread index goes through an opaque move so that the shared-memory
// addresses of the stages are recomputed per transform instead of being kept
// live across every transform of a kernel (which exhausts the register file).
// WARP=true only where each pencil's threads lie in one warp (Q divides 32 in a
// pencil-major thread layout).
template <typename T, int L, int E, bool INV, class SM, bool WARP = false>
__device__ __forceinline__ void fft(cx<T> (&v)[E], SM sm, int q, const cx<T> *__restrict__ tw) {
    int qq;
    asm volatile("mov.b32 %0, %1;" : "=r"(qq) : "r"(q));
    fft_run<T, L, E, INV, WARP, 0, SM>(v, sm, qq, tw);
}

// Accessor: tile of P pencils stored row-major [row][P] (pencil index fastest).
template <typename T, int P> struct SmRowMajor {
    cx<T> *base; int p;
    __device__ __forceinline__ cx<T> &at(int row) const { return base[row * P + p]; }
};
// Accessor: pencil-major [p][PITCH], rows stored in order (post-processing
// reads rows k and L-k of consecutive k: conflict-free as is).  The Stockham
// exchanges of fft_run use their own padded layouts inside the same buffer
// (PencilLayout below), so `at` is only for accesses outside the transform.
template <typename T, int L, int E> struct SmPencil;

// ---------------------------------------------------------------------------
// Padded exchange layouts of the pencil-major buffer.
//
// Exchange S (written by stage S: radix R, span Ns; read by stage S+1: radix
// R2) stores row r at  r + (r / X) * PAD  with X = Ns*R.  A butterfly's R
// writes  (j/Ns)*X + j%Ns + r*Ns  all lie in one block of X rows, and the
// reads  q + Q*m + r2*(L/R2)  step by multiples of X (L/R2 = X * the radices
// after S+1), so every access of a thread is one base address plus
// compile-time offsets: no per-access index arithmetic.  PAD per exchange and
// the pencil pitch come from fft_layouts.h, generated by gen_layouts.py, which
// counts the shared-memory wavefronts of each exchange's writes and reads; where
// the XOR swizzle below has fewer, the table selects it (PAD = -1) and that
// exchange pays per-access index arithmetic instead.
// ---------------------------------------------------------------------------
template <typename T, int L, int E> struct SmPencil {
    cx<T> *base;
    static constexpr bool PADDED = true;
    static constexpr int WPL = (int)(sizeof(cx<T>) / 4);
    static constexpr int PITCH = exch::table_pitch(WPL, L, E);
    static_assert(PITCH >= L, "no exchange layout generated for this length and E (gen_layouts.py)");
    static constexpr int G = WPL == 4 ? 8 : 16;   // rows of one 128-byte bank line
    // layout of exchange S of the inverse (INV) or forward plan: pad >= 0, or -1 for the XOR swizzle
    template <bool INV, int S> struct Ex {
#ifdef SPNS_EXCH_XOR_ONLY
        static constexpr int PAD = -1;
#else
        static constexpr int PAD = exch::table_pad(WPL, L, E, INV, S);
#endif
        static_assert(PAD >= -1, "no exchange layout generated for this stage (gen_layouts.py)");
        static_assert((PAD < 0 ? (L + G - 1) / G * G : L + (L / (Plan<L, E, INV>::ns(S) * Plan<L, E, INV>::radix(S))) * PAD) <= PITCH,
                      "exchange layout exceeds the pencil pitch");
    };
    __device__ __forceinline__ cx<T> &at(int row) const { return base[row]; }
    // XOR swizzle of the low row bits by the bits two places up; maps each aligned block of G rows onto itself
    __device__ __forceinline__ cx<T> &xr(int row) const { return base[row ^ ((row >> 2) & (G - 1))]; }
};

} // namespace spns
