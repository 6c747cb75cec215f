// edge_kernels.cuh -- exact aliasing correction that makes the rotational form
// of the nonlinear term equal to the reference's advective form.
//
// With the 3/2 rule and both +-N/2 kept (even N, M=3h per axis, h=N/2), the
// products of two modes on a plane p_i = -s*h alias onto the kept plane
// k_i = s*h.  The advective term u_j d_j u_i and the rotational term
// (w x u)_i differ by u_j d_i u_j = d_i(|u|^2/2) =: d_i q pointwise, and the DFT
// of the grid samples of d_i q equals i k_i Q(k) (removed by the projection)
// plus, on the planes k_i = s*h only,
//     C_i(k) = i (-s L_i M_i) M_i Phi(k_perp),
// where Phi is the unnormalised 2-D forward DFT over the two other axes of
// phi = 1/2 sum_j V_j^2, V_j the unnormalised 2-D inverse DFT of the
// coefficients of u_j on the source plane p_i = -s*h (all p_perp, the p_z<0
// half taken from the Hermitian partner).  Adding C to the rotational term
// reproduces the advective term after the projection, mode by mode.
// Planes: x (s=+-1, 2-D over y,z), y (s=+-1, over x,z), z (s=+1 only: the
// half spectrum keeps kz=+h, its source plane is p_z=-h).
#pragma once
#include "fft_core.cuh"
#include "solver_kernels.cuh"

namespace spns {

// A set of axes whose plane groups share the 2-D transform size R x C (all
// three for a cubic box), corrected together so that each phase is one launch.
// Planes are numbered over the set: axis slot k owns planes first[k] ..
// first[k+1]-1 (2 for x and y, s = +1 then -1; 1 for z).  Buffers:
//   V   [plane][comp][R][C]   source-plane velocities, then their 2-D inverse DFT
//   Phi [plane][R][C]         phi = 1/2 sum_j V_j^2, then its 2-D forward DFT
struct EdgeSet {
    int naxes;
    int axis[3];     // 0 x, 1 y, 2 z
    int first[4];
    int R, C;        // FFT grid of the two other axes (rows strided, columns contiguous)
};

__device__ __forceinline__ int edge_slot(const EdgeSet &es, int plane) {
    int k = 0;
    while (k + 1 < es.naxes && plane >= es.first[k + 1]) k++;
    return k;
}

// Source-plane coefficients of the three velocity components, zero padded to
// the R x C grid.
template <typename T>
__global__ void k_edge_build(Geo g, const cx<T> *__restrict__ U, EdgeSet es, cx<T> *__restrict__ out) {
    const long long n = (long long)es.R * es.C;
    const long long tot = n * 3 * es.first[es.naxes];
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += (long long)gridDim.x * blockDim.x) {
        const long long rc = t % n;
        const int comp = (int)((t / n) % 3), plane = (int)(t / (n * 3));
        const int k = edge_slot(es, plane), axis = es.axis[k], pl = plane - es.first[k];
        const int r = (int)(rc / es.C), c = (int)(rc % es.C);
        const int s = axis == 2 ? 1 : (pl == 0 ? 1 : -1);  // destination sign
        const int pr = ffreq(r, es.R), pc = ffreq(c, es.C);
        // source mode (px, py, pz) on plane p_axis = -s*h
        int px, py, pz;
        if (axis == 0) { px = -s * g.hx; py = pr; pz = pc; }
        else if (axis == 1) { px = pr; py = -s * g.hy; pz = pc; }
        else { px = pr; py = pc; pz = -g.hz; }
        cx<T> val = zero<T>();
        if (px >= -g.hx && px <= g.hx && py >= -g.hy && py <= g.hy && pz >= -g.hz && pz <= g.hz) {
            const bool cj = pz < 0;
            const int qx = cj ? -px : px, qy = cj ? -py : py, qz = cj ? -pz : pz;
            const long long idx = ((long long)(qy >= 0 ? qy : qy + g.Ky) * g.Kx + (qx >= 0 ? qx : qx + g.Kx)) * g.Kz + qz;
            val = U[(long long)comp * g.S0 + idx];
            if (cj) val = conj(val);
        }
        out[t] = val;
    }
}

// phi = 1/2 sum_j V_j^2 per plane: in [plane][comp][R][C] -> out [plane][R][C].
template <typename T>
__global__ void k_edge_square(const cx<T> *__restrict__ V, long long n, int nplanes, cx<T> *__restrict__ phi) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n * nplanes; t += (long long)gridDim.x * blockDim.x) {
        const long long pl = t / n, rc = t % n;
        const cx<T> *v = V + pl * 3 * n + rc;
        cx<T> a = v[0], b = v[n], c = v[2 * n];
        const T re = a.x * a.x - a.y * a.y + b.x * b.x - b.y * b.y + c.x * c.x - c.y * c.y;
        const T im = T(2) * (a.x * a.y + b.x * b.y + c.x * c.y);
        phi[t] = mk<T>(T(0.5) * re, T(0.5) * im);
    }
}

// G_axis(k) += i (-s L M) M Phi(k_perp) on the kept modes of the destination
// planes.  blockIdx.y = axis slot of the set.
template <typename T>
__global__ void k_edge_apply(Geo g, cx<T> *__restrict__ G, EdgeSet es, const cx<T> *__restrict__ Phi) {
    const int k = blockIdx.y;
    if (k >= es.naxes) return;
    const int axis = es.axis[k], nplanes = es.first[k + 1] - es.first[k];
    const long long n = (long long)es.R * es.C;
    int A, B;  // kept extents of the two other axes: (ky, kz), (kx, kz), (kx, ky)
    if (axis == 0) { A = g.Ky; B = g.Kz; } else if (axis == 1) { A = g.Kx; B = g.Kz; } else { A = g.Kx; B = g.Ky; }
    const long long tot = (long long)A * B * nplanes;
    const double M = axis == 0 ? g.Mx : axis == 1 ? g.My : g.Mz;
    const double Ls = axis == 0 ? g.sx : axis == 1 ? g.sy : g.sz;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += (long long)gridDim.x * blockDim.x) {
        const int pl = (int)(t / ((long long)A * B));
        const int ab = (int)(t % ((long long)A * B));
        const int ia = ab / B, ib = ab % B;
        const int s = axis == 2 ? 1 : (pl == 0 ? 1 : -1);
        int ix, iy, kz, r, c;
        if (axis == 0) {
            const int my = ia <= g.hy ? ia : ia - g.Ky;
            ix = s > 0 ? g.hx : g.Kx - g.hx; iy = ia; kz = ib;
            r = my >= 0 ? my : my + es.R; c = kz;
        } else if (axis == 1) {
            const int mx = ia <= g.hx ? ia : ia - g.Kx;
            ix = ia; iy = s > 0 ? g.hy : g.Ky - g.hy; kz = ib;
            r = mx >= 0 ? mx : mx + es.R; c = kz;
        } else {
            const int mx = ia <= g.hx ? ia : ia - g.Kx, my = ib <= g.hy ? ib : ib - g.Ky;
            ix = ia; iy = ib; kz = g.hz;
            r = mx >= 0 ? mx : mx + es.R; c = my >= 0 ? my : my + es.C;
        }
        const cx<T> ph = Phi[(long long)(es.first[k] + pl) * n + (long long)r * es.C + c];
        const T f = T(-(double)s * Ls * M * M);  // i * f * Phi
        const long long idx = ((long long)iy * g.Kx + ix) * g.Kz + kz;
        cx<T> *dst = G + (long long)axis * g.S0 + idx;
        *dst = *dst + mul_i(f * ph);
    }
}

// Batched 1-D FFTs of contiguous lines of length L (line stride L).
template <typename T, int L, int E, int P, bool INV>
__global__ void __launch_bounds__(P *(L / E)) k_lines(cx<T> *__restrict__ data, long long batch, const cx<T> *__restrict__ tw) {
    extern __shared__ __align__(16) unsigned char smraw[];
    constexpr int Q = L / E;
    const int tid = threadIdx.x, p = tid / Q, q = tid % Q;
    const long long line = (long long)blockIdx.x * P + p;
    const bool ok = line < batch;
    cx<T> *d = data + (ok ? line : 0) * L;
    SmPencil<T, L, E> sm{reinterpret_cast<cx<T> *>(smraw) + p * SmPencil<T, L, E>::PITCH};
    cx<T> r[E];
#pragma unroll
    for (int e = 0; e < E; e++) r[e] = ok ? d[in_row<L, E, INV>(q, e)] : zero<T>();
    fft<T, L, E, INV, SmPencil<T, L, E>, (32 % (L / E) == 0)>(r, sm, q, tw);
    if (ok)
#pragma unroll
        for (int e = 0; e < E; e++) d[out_row<L, E, INV>(q, e)] = r[e];
}

// Batched 1-D FFTs along the strided axis of [batch][L][ncols] arrays (P columns per block).
template <typename T, int L, int E, int P, bool INV>
__global__ void __launch_bounds__(P *(L / E)) k_cols(cx<T> *__restrict__ data, int ncols, const cx<T> *__restrict__ tw) {
    extern __shared__ __align__(16) unsigned char smraw[];
    const int tid = threadIdx.x, p = tid % P, q = tid / P;
    const int col = blockIdx.x * P + p;
    const bool ok = col < ncols;
    cx<T> *d = data + (long long)blockIdx.y * L * ncols + (ok ? col : 0);
    SmRowMajor<T, P> sm{reinterpret_cast<cx<T> *>(smraw), p};
    cx<T> r[E];
#pragma unroll
    for (int e = 0; e < E; e++) r[e] = ok ? d[(long long)in_row<L, E, INV>(q, e) * ncols] : zero<T>();
    fft<T, L, E, INV>(r, sm, q, tw);
    if (ok)
#pragma unroll
        for (int e = 0; e < E; e++) d[(long long)out_row<L, E, INV>(q, e) * ncols] = r[e];
}

} // namespace spns
