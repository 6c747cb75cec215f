// fft768.cuh -- a length-768 pencil transform with two shared-memory exchanges
// instead of three, for 64 threads holding 12 values each.
//
// The generic engine (fft_core.cuh) needs every radix to divide the values per
// thread, so E = 12 gives 768 = 12 x 4 x 4 x 4: three exchanges of the whole
// pencil per transform.  Here the middle stage is radix 16 on 48 of the 64
// threads (16 values each; the other 16 threads only take part in the
// barriers): 768 = 12 x 16 x 4 forward, 4 x 16 x 12 inverse.  The first stage
// reads and the last stage leaves the values in the same registers and rows as
// the generic plans with the same first and last radices (rows q + 64 e for a
// radix-12 end, q + 64 (e/4) + 192 (e%4) for a radix-4 end), so the two are
// interchangeable at the call site.
//
// Stockham stages as in fft_core.cuh: stage (R, Ns), butterfly j, k = j mod Ns,
// inputs x_r = in[j + r L/R] times w_L^{r k L/(Ns R)}, outputs
// out[(j/Ns) Ns R + k + r Ns].  The exchanges are padded so that the 16-byte
// accesses of every phase of a warp hit distinct banks:
//   forward  12 -> 16: p + p/12,          16 -> 4: p + 4 (p/192)
//   inverse   4 -> 16: p + p/4,           16 -> 12: p + 4 (p/64)
// which needs FFT768_PITCH complex values of shared memory per pencil.
#pragma once
#include "fft_core.cuh"

namespace spns {

constexpr int FFT768_PITCH = 960;

// 16-point DFT as 4 x 4 with the inner twiddles w16^(n2 k1), in place with the
// output transposed: X[k1 + 4 k2] is left in x[4 k1 + k2] (dft16_out gives the
// position of output r).  INV selects exp(+2 pi i/16).
__host__ __device__ constexpr int dft16_out(int r) { return 4 * (r % 4) + r / 4; }
template <typename T, bool INV> __device__ __forceinline__ void dft16(cx<T> *x) {
    const T c1 = T(0.92387953251128675612818318939679);   // cos(pi/8)
    const T s1 = T(0.38268343236508977172845998403040);   // sin(pi/8)
    const T h = T(0.70710678118654752440084436210485);
    const T sg = INV ? T(1) : T(-1);                      // sign of the sine of w16
#pragma unroll
    for (int n2 = 0; n2 < 4; n2++) {                      // x[4 k1 + n2] = DFT4 over n1 of x[4 n1 + n2]
        cx<T> c[4] = {x[n2], x[4 + n2], x[8 + n2], x[12 + n2]};
        dft4<T, INV>(c);
#pragma unroll
        for (int k1 = 0; k1 < 4; k1++) x[4 * k1 + n2] = c[k1];
    }
    // x[4 k1 + n2] *= w16^(n2 k1), w16^m = cos(m pi/8) + i sg sin(m pi/8)
#define SPNS_TW16(i, cr, si)                                                        \
    { const cx<T> a = x[i]; x[i] = mk<T>((cr) * a.x - sg * (si) * a.y, (cr) * a.y + sg * (si) * a.x); }
    SPNS_TW16(5, c1, s1)                 // m = 1
    SPNS_TW16(6, h, h)                   // m = 2
    SPNS_TW16(7, s1, c1)                 // m = 3
    SPNS_TW16(9, h, h)                   // m = 2
    { const cx<T> a = x[10]; x[10] = mk<T>(-sg * a.y, sg * a.x); }   // m = 4
    SPNS_TW16(11, -h, h)                 // m = 6
    SPNS_TW16(13, s1, c1)                // m = 3
    SPNS_TW16(14, -h, h)                 // m = 6
    SPNS_TW16(15, -c1, -s1)              // m = 9
#undef SPNS_TW16
#pragma unroll
    for (int k1 = 0; k1 < 4; k1++) dft4<T, INV>(&x[4 * k1]);   // x[4 k1 + k2] = X[k1 + 4 k2]
}

// x_r *= w^r (r = 1..R-1) for w = tw[step]; double: repeated products, single: the
// powers of two from the table and the others as products (fft_core.cuh).
template <typename T, int R, bool INV>
__device__ __forceinline__ void twiddle_apply(cx<T> *x, const cx<T> *__restrict__ tw, int step) {
    if constexpr (sizeof(T) == 4) {
        cx<T> wp[R];
        twiddle_powers<T, R>(wp, tw, step);
#pragma unroll
        for (int r = 1; r < R; r++) x[r] = INV ? cmulc(x[r], wp[r]) : cmul(x[r], wp[r]);
    } else {
        const cx<T> w1 = tw[step];
        cx<T> w = w1;
#pragma unroll
        for (int r = 1; r < R; r++) {
            x[r] = INV ? cmulc(x[r], w) : cmul(x[r], w);
            if (r + 1 < R) w = cmul(w, w1);
        }
    }
}

__device__ __forceinline__ int f768_padA(int p) { return p + p / 12; }
__device__ __forceinline__ int f768_padB(int p) { return p + 4 * (p / 192); }
__device__ __forceinline__ int i768_padA(int p) { return p + p / 4; }
__device__ __forceinline__ int i768_padB(int p) { return p + 4 * (p / 64); }

// One pencil of 768 values: 64 threads (q = 0..63) with v[12] each; `buf` is the
// pencil's shared buffer (FFT768_PITCH values); the 64 threads of a pencil are two
// warps of one block, synchronised with __syncthreads.
template <typename T, bool INV>
__device__ __forceinline__ void fft768_q64(cx<T> (&v)[12], cx<T> *buf, int q_in, const cx<T> *__restrict__ tw) {
    int q;
    asm volatile("mov.b32 %0, %1;" : "=r"(q) : "r"(q_in));
    if constexpr (!INV) {
        // stage 1: radix 12, Ns = 1 (no twiddles); inputs rows q + 64 r
        dft<T, 12, false>(v);
        {
            cx<T> *w = buf + 13 * q;                      // f768_padA(12 q + r) = 13 q + r
#pragma unroll
            for (int r = 0; r < 12; r++) w[r] = v[r];
        }
        __syncthreads();
        // stage 2: radix 16, Ns = 12, on threads q < 48
        cx<T> x[16];
        if (q < 48) {
#pragma unroll
            for (int r = 0; r < 16; r++) x[r] = buf[f768_padA(q + 48 * r)];
        }
        __syncthreads();
        if (q < 48) {
            const int k = q % 12;
            if (k) twiddle_apply<T, 16, false>(x, tw, 4 * k);
            dft16<T, false>(x);
            cx<T> *w = buf + (q / 12) * 196 + k;          // f768_padB((q/12) 192 + k + 12 r)
#pragma unroll
            for (int r = 0; r < 16; r++) w[12 * r] = x[dft16_out(r)];
        }
        __syncthreads();
        // stage 3: radix 4, Ns = 192: butterflies j = q + 64 m, outputs rows j + 192 r
#pragma unroll
        for (int m = 0; m < 3; m++) {
            const int j = q + 64 * m;
            cx<T> *x4 = &v[4 * m];
#pragma unroll
            for (int r = 0; r < 4; r++) x4[r] = buf[j + 196 * r];   // f768_padB(j + 192 r)
            twiddle_apply<T, 4, false>(x4, tw, j);
            dft<T, 4, false>(x4);
        }
        __syncthreads();
    } else {
        // stage 1: radix 4, Ns = 1: butterflies j = q + 64 m on rows j + 192 r
#pragma unroll
        for (int m = 0; m < 3; m++) {
            dft<T, 4, true>(&v[4 * m]);
            cx<T> *w = buf + i768_padA(4 * (q + 64 * m));
#pragma unroll
            for (int r = 0; r < 4; r++) w[r] = v[4 * m + r];   // 4 j + r, pad p/4 = j
        }
        __syncthreads();
        // stage 2: radix 16, Ns = 4, on threads q < 48
        cx<T> x[16];
        if (q < 48) {
#pragma unroll
            for (int r = 0; r < 16; r++) x[r] = buf[i768_padA(q + 48 * r)];
        }
        __syncthreads();
        if (q < 48) {
            const int k = q % 4;
            if (k) twiddle_apply<T, 16, true>(x, tw, 12 * k);
            dft16<T, true>(x);
            cx<T> *w = buf + (q / 4) * 68 + k;            // i768_padB((q/4) 64 + k + 4 r)
#pragma unroll
            for (int r = 0; r < 16; r++) w[4 * r] = x[dft16_out(r)];
        }
        __syncthreads();
        // stage 3: radix 12, Ns = 64: butterfly j = q, inputs q + 64 r, outputs rows q + 64 r
#pragma unroll
        for (int r = 0; r < 12; r++) v[r] = buf[q + 68 * r];          // i768_padB(q + 64 r)
        if (q) twiddle_apply<T, 12, true>(v, tw, q);
        dft<T, 12, true>(v);
        __syncthreads();
    }
}

} // namespace spns

namespace spns {

// Off by default: parity-tested (the length-768 tests pass with it on), but at
// N=512 the z pass took 14.68 ms with it against 14.64 ms with the three-exchange
// plan in double precision, 10.74 against 10.28 ms in single, and the persistent
// double z pass spilled with it (23.7 ms).  The exchanges are not what bounds the
// pass.  Build with -DSPNS_FFT768=1 to use it.
#ifndef SPNS_FFT768
#define SPNS_FFT768 0
#endif

// Pencil-major transform of one pencil (SmPencil buffer): fft768_q64 where it
// applies, the generic engine elsewhere.
template <typename T, int L, int E, bool INV, bool WARP>
__device__ __forceinline__ void pencil_fft(cx<T> (&v)[E], SmPencil<T, L, E> sm, int q, const cx<T> *__restrict__ tw) {
    if constexpr (SPNS_FFT768 && L == 768 && E == 12 && !WARP) {
        fft768_q64<T, INV>(v, sm.base, q, tw);
    } else {
        fft<T, L, E, INV, SmPencil<T, L, E>, WARP>(v, sm, q, tw);
    }
}

// Shared-memory values per pencil of a pencil-major z-pass buffer.
template <typename T, int L, int E> __host__ __device__ constexpr int pencil_pitch() {
    return (SPNS_FFT768 && L == 768 && E == 12 && SmPencil<T, L, E>::PITCH < FFT768_PITCH) ? FFT768_PITCH : SmPencil<T, L, E>::PITCH;
}

} // namespace spns
