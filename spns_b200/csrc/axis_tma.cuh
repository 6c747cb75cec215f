// axis_tma.cuh -- x/y passes with their pencil tiles moved by the Tensor Memory
// Accelerator (sm_90+ cp.async.bulk.tensor, tile mode, no multicast).
//
// A pass transforms NOUT fields along one axis for P consecutive kz (one row of
// P complex values per grid point of the axis) at every "line" position of the
// other axis.  The tile of one field -- R-row boxes of a 4-D tensor map
// {2*Kz doubles, rows, lines, fields} over the pass's input buffer -- lands in
// shared memory in the row-major [row][P] order of the Stockham exchange, so the
// buffer a tile arrives in is also the exchange buffer of that field's
// transform.  Two buffers alternate: while field f is transformed in one, the
// other is being filled with the tile of field f+1, issued as soon as the
// transform of field f-1 released that buffer.  Blocks are
// persistent over (kz chunk, line) work items, so the pipeline runs across item
// boundaries and the HBM reads never stop for a transform.
//
//   inverse (INV): compact input rows m = -h..h (stored 0..h, Kc-h..Kc-1) are
//     placed at FFT rows 0..h and L-h..L-1; the rows between are read as zero.
//     Output: all L rows.  Optional y-derivative: outputs f >= DERIV_FROM are
//     i*s*m times the input (src/HIT_LES.cpp:34-58 on this axis).
//   forward: all L input rows; output rows truncated to |m| <= h in compact order.
//
// Every mbarrier wait is bounded (see zpass_staged.cuh); a wait that gives up
// records wait_timeout in the solver scalars and the block stops.
#pragma once
#include "zpass_staged.cuh"
#include <cuda.h>

namespace spns {

struct AxisArgs {
    int h;              // half width of the compact axis (inverse input / forward output)
    int Kc;             // compact rows 2h+1
    int lines;          // line positions (blockIdx-equivalent second index)
    int Kz;             // retained kz
    int nout;           // fields transformed
    unsigned long long src;   // tensor-map field of output f in bits 4f..4f+3
    int deriv_from;     // outputs f >= deriv_from are multiplied by i*s*m (inverse only)
    int s;              // wavenumber scale of the axis
    long long o_row, o_line, o_field;   // output strides (complex elements)
    int rbox;           // rows per TMA box
};

__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, int c0, int c1, int c2, int c3, unsigned long long *bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];\n" ::"r"(
            smem_addr(dst)),
        "l"(reinterpret_cast<unsigned long long>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_addr(bar))
        : "memory");
}

// Boxes of one tile: (global row, shared row) pairs.  Inverse: ceil((h+1)/R) boxes
// from row 0 and ceil(h/R) boxes ending at the last compact row, placed so that
// the last one ends at FFT row L-1; forward: L/R boxes.
template <int L, bool INV> __host__ __device__ __forceinline__ int axis_boxes(int h, int R) {
    return INV ? (h + 1 + R - 1) / R + (h + R - 1) / R : L / R;
}
template <int L, bool INV>
__device__ __forceinline__ void axis_box(int b, int h, int Kc, int R, int &grow, int &srow) {
    if (!INV) { grow = srow = b * R; return; }
    const int npos = (h + 1 + R - 1) / R;
    if (b < npos) { grow = srow = b * R; return; }
    const int nneg = (h + R - 1) / R, k = b - npos;
    grow = Kc - (nneg - k) * R;
    srow = L - (nneg - k) * R;
}

template <typename T, int L, int E, int P, bool INV>
__global__ void __launch_bounds__(P *(L / E), 1) k_axis_tma(const __grid_constant__ CUtensorMap tin, AxisArgs a, cx<T> *__restrict__ out,
                                                            const cx<T> *__restrict__ tw, DevScalars *ds) {
    constexpr int Q = L / E, THREADS = P * Q;
    constexpr size_t BUF = (size_t)L * P * sizeof(cx<T>);
    extern __shared__ __align__(128) unsigned char smraw_axis[];
    unsigned char *base = reinterpret_cast<unsigned char *>((reinterpret_cast<size_t>(smraw_axis) + 127) & ~(size_t)127);
    cx<T> *const buf0 = reinterpret_cast<cx<T> *>(base);
    unsigned long long *const bars = reinterpret_cast<unsigned long long *>(base + 2 * BUF);
    const int tid = threadIdx.x, p = tid % P, q = tid / P;
    const int R = a.rbox;
    const int nbox = axis_boxes<L, INV>(a.h, R);
    const unsigned tile_bytes = (unsigned)(nbox * R * P * sizeof(cx<T>));
    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        fence_mbar_init();
    }
    __syncthreads();

    const int nchunk = (a.Kz + P - 1) / P;
    const long long nitems = (long long)nchunk * a.lines;
    // this block's sequence of (item, field) tiles: item = blockIdx.x + k*gridDim.x
    const long long my_items = nitems > blockIdx.x ? (nitems - 1 - blockIdx.x) / gridDim.x + 1 : 0;
    const long long nseq = my_items * a.nout;
    auto issue = [&](long long s) {   // tile of sequence index s into buffer s&1 (thread 0)
        const long long it = blockIdx.x + (s / a.nout) * gridDim.x;
        const int f = (int)(s % a.nout);
        const int chunk = (int)(it % nchunk), line = (int)(it / nchunk);
        cx<T> *dst = buf0 + (s & 1) * (long long)L * P;
        unsigned long long *bar = &bars[s & 1];
        fence_proxy_async_smem();
        mbar_arrive_expect_tx(bar, tile_bytes);
        for (int b = 0; b < nbox; b++) {
            int grow, srow;
            axis_box<L, INV>(b, a.h, a.Kc, R, grow, srow);
            tma_load_4d(dst + (long long)srow * P, &tin, 2 * chunk * P, grow, line, (int)((a.src >> (4 * f)) & 15ull), bar);
        }
    };
    if (tid == 0) {
        if (nseq > 0) issue(0);
        if (nseq > 1) issue(1);
    }
    unsigned par0 = 0u, par1 = 0u;   // phase parity of each buffer's barrier
    for (long long s = 0; s < nseq; s++) {
        const long long it = blockIdx.x + (s / a.nout) * gridDim.x;
        const int f = (int)(s % a.nout);
        const int chunk = (int)(it % nchunk), line = (int)(it / nchunk);
        const int kz = chunk * P + p;
        const int b = (int)(s & 1);
        cx<T> *const tile = buf0 + b * (long long)L * P;
        const bool arrived = mbar_wait_bounded(&bars[b], b ? par1 : par0, ZS_WAIT_LIMIT);
        if (b) par1 ^= 1u; else par0 ^= 1u;
        if (!__syncthreads_and(arrived ? 1 : 0)) {
            if (tid == 0) atomicExch(&ds->wait_timeout, 1);
            break;
        }
        cx<T> r[E];
        const bool deriv = INV && f >= a.deriv_from;
#pragma unroll
        for (int e = 0; e < E; e++) {
            const int row = in_row<L, E, INV>(q, e);
            cx<T> v = zero<T>();
            if (!INV || row <= a.h || row >= L - a.h) {
                v = tile[row * P + p];
                if (deriv) v = mul_i(T(a.s * ffreq(row, L)) * v);
            }
            r[e] = v;
        }
        __syncthreads();   // the tile is read: its buffer becomes the exchange buffer
        fft<T, L, E, INV>(r, SmRowMajor<T, P>{tile, p}, q, tw);
        if (kz < a.Kz) {
            cx<T> *o = out + (long long)f * a.o_field + (long long)line * a.o_line + kz;
#pragma unroll
            for (int e = 0; e < E; e++) {
                const int row = out_row<L, E, INV>(q, e);
                if (INV) {
                    o[(long long)row * a.o_row] = r[e];
                } else {
                    const int m = ffreq(row, L);
                    if (m <= a.h && m >= -a.h) o[(long long)(m >= 0 ? m : m + a.Kc) * a.o_row] = r[e];
                }
            }
        }
        // fft() ends with a barrier after its last exchange reads: the buffer is free
        if (tid == 0 && s + 2 < nseq) issue(s + 2);
    }
    (void)THREADS;
}

} // namespace spns
