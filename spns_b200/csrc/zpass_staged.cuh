// zpass_staged.cuh -- the rotational-form z pass, persistent over the grid, with
// its input pairs staged by bulk asynchronous copies.
//
// Same arithmetic as k3_z<MODE_ROT> (solver_kernels.cuh): c2r of the six real
// fields u, v, w, w_x, w_y, w_z as three 2-for-1 complex transforms, the
// product c = w x u and the CFL maxima on the grid, r2c of c truncated to
// kz <= hz (src/HIT_LES.cpp:74-125 up to the gradient the projection removes).
// What differs is the schedule:
//   * A block of PB pencils (Q = L/E threads each) is persistent: it walks the
//     groups of PB consecutive pencils with a stride of the grid.  Only the two
//     fields of the next input pair are staged in shared memory, by
//     cp.async.bulk (TMA bulk copies global -> shared, completion counted in
//     bytes on an mbarrier), while the current pair is transformed; the first
//     pair of the next group is fetched during the two forward transforms.  The
//     staging takes 2*PB*Kz complex values instead of 6*PB*Kz, so more blocks fit
//     an SM.  In single precision a group of pencils need not start on 16 bytes
//     (Kz is odd), so there the staging uses per-lane cp.async instead.
//   * Working set per thread: four physical slots (u, v, w_x, w_y; the last
//     SLOTS_SM of them in shared memory, own rows only) and one complex register
//     array.  c_z
//     is transformed as soon as it is known (after the second pair) and written
//     over the w_x field of the same pencil (S2 field 3, consumed at the first
//     pair), so the forward y pass reads the nonlinear term from fields 0, 1, 3.
//   * Pencils of Q <= 32 threads exchange within their warp (__syncwarp).
//   * CFL maxima accumulate per thread over all pencils and are reduced once per
//     block at the end.
// Every mbarrier wait is bounded; a wait that gives up records wait_timeout in
// the solver scalars (reported as SPNS_ERR_TIMEOUT by the host) and the block
// skips its remaining pencils; no copy is left in flight.
#pragma once
#include "solver_kernels.cuh"

namespace spns {

__device__ __forceinline__ unsigned smem_addr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
// makes the barrier initialisation visible to the asynchronous (TMA) proxy
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
// orders earlier generic-proxy accesses of shared memory before later async-proxy ones
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}
// bulk copy of `bytes` (multiple of 16, both addresses 16-byte aligned) from global to shared memory
__device__ __forceinline__ void bulk_copy_g2s(void *dst, const void *src, unsigned bytes, unsigned long long *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n"
        ".reg .pred p;\n"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        "selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Polls the barrier phase `parity` at most `limit` times (each poll may suspend the
// thread for a short, hardware-defined time); false if it did not complete.
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long *bar, unsigned parity, int limit) {
    for (int i = 0; i < limit; i++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

constexpr int ZS_WAIT_LIMIT = 1 << 22;

// Shared memory of one block: PB exchange buffers, 2 staging fields of PB pencils
// (stride KS complex values per field), SLOTS_SM physical slots of L reals per
// pencil, then the block's mbarrier.
template <typename T, int L, int E, int PB, int SLOTS_SM> struct ZStagedLayout {
    static constexpr int Q = L / E;
    static constexpr int PITCH = pencil_pitch<T, L, E>();
    static constexpr long long SLOT_ELEMS = ((long long)SLOTS_SM * PB * L * (long long)sizeof(T) + (long long)sizeof(cx<T>) - 1) / (long long)sizeof(cx<T>);
    // staging stride of one field: PB*Kz rounded up to 16 bytes
    __host__ __device__ static int stage_stride(int Kz) {
        const int per16 = 16 / (int)sizeof(cx<T>);
        return (PB * Kz + per16 - 1) / per16 * per16;
    }
    __host__ __device__ static long long elems(int Kz) { return (long long)PB * PITCH + 2LL * stage_stride(Kz) + SLOT_ELEMS; }
    __host__ __device__ static size_t smem_bytes(int Kz) { return (size_t)elems(Kz) * sizeof(cx<T>) + 16; }
};

// Physical slot S (0 u, 1 v, 2 w_x, 3 w_y) of register slot e (grid row `row`):
// the first NREG in registers, the rest in shared memory (stride `pitch` reals).
template <int S, int NREG, typename T, int E>
__device__ __forceinline__ T &zs_slot(T (&rg)[NREG > 0 ? NREG : 1][E], T *sm_slots, int pitch, int e, int row) {
    if constexpr (S < NREG) return rg[S][e];
    else return sm_slots[(S - NREG) * pitch + row];
}

// Opaque copy of the thread index: the row and address arithmetic that depends on
// it is recomputed where it is used instead of being hoisted out of the pencil
// loop and kept live in registers for every register slot.
__device__ __forceinline__ int zs_opaque(int q) {
    int r;
    asm volatile("mov.b32 %0, %1;" : "=r"(r) : "r"(q));
    return r;
}

template <typename T, int L, int E, int PB, int SLOTS_SM, int MINB>
__global__ void __launch_bounds__(PB *(L / E), MINB) k3_rot_staged(Geo g, cx<T> *__restrict__ buf, StepConsts c, DevScalars *ds,
                                                                   const cx<T> *__restrict__ tw) {
    using LY = ZStagedLayout<T, L, E, PB, SLOTS_SM>;
    constexpr int Q = LY::Q, THREADS = PB * Q;
    static_assert(SLOTS_SM >= 0 && SLOTS_SM <= 4, "zero to four slots in shared memory");
    constexpr bool WARP = (32 % Q == 0);                      // a pencil never leaves its warp
    constexpr bool BULK = sizeof(cx<T>) == 16;                // double: 16-byte elements, bulk copies
    extern __shared__ __align__(128) unsigned char smraw_zs[];
    const int tid = threadIdx.x, sub = tid / Q, q0 = tid % Q;
    const int Kz = g.Kz;
    const int KS = LY::stage_stride(Kz);
    cx<T> *const smc = reinterpret_cast<cx<T> *>(smraw_zs);
    SmPencil<T, L, E> sm{smc + sub * LY::PITCH};
    cx<T> *const stA = smc + PB * LY::PITCH;                  // staging: field a of the pair
    cx<T> *const stB = stA + KS;                              // field b
    T *const slot_sm = reinterpret_cast<T *>(stB + KS) + sub * L;   // slot j of this pencil at slot_sm[j*PB*L + row]
    unsigned long long *const bar = reinterpret_cast<unsigned long long *>(smc + LY::elems(Kz));
    if (tid == 0) {
        mbar_init(bar, 1);
        fence_mbar_init();
    }
    __syncthreads();

    const long long npen = (long long)g.Mx * g.My;
    const long long ngrp = (npen + PB - 1) / PB;
    const T sz = T(g.sz);
    unsigned parity = 0;
    bool bad = false;
    double mx[4] = {0.0, 0.0, 0.0, 0.0};

    // stage fields fa, fb of pencil group grp (its valid pencils are contiguous in each field)
    auto issue = [&](long long grp, int fa, int fb) {
        const long long p0 = grp * PB;
        const int np = (int)(npen - p0 < PB ? npen - p0 : PB);
        const cx<T> *A = buf + (long long)fa * g.S2 + p0 * Kz, *B = buf + (long long)fb * g.S2 + p0 * Kz;
        if constexpr (BULK) {
            if (tid == 0) {
                const unsigned bytes = (unsigned)(np * Kz * sizeof(cx<T>));
                fence_proxy_async_smem();
                mbar_arrive_expect_tx(bar, 2 * bytes);
                bulk_copy_g2s(stA, A, bytes, bar);
                bulk_copy_g2s(stB, B, bytes, bar);
            }
        } else {
            for (int k = tid; k < np * Kz; k += THREADS) {
                cp_async_elem<T>(stA + k, A + k);
                cp_async_elem<T>(stB + k, B + k);
            }
            cp_async_commit();
        }
    };
    // the staged pair is complete and visible to every thread of the block
    auto wait_stage = [&]() -> bool {
        bool ok = true;
        if constexpr (BULK) {
            ok = mbar_wait_bounded(bar, parity, ZS_WAIT_LIMIT);
            parity ^= 1u;
        } else {
            cp_async_wait<0>();
        }
        return __syncthreads_and(ok ? 1 : 0) != 0;
    };

    long long grp = blockIdx.x;
    if (grp < ngrp) issue(grp, 0, 3);
    for (; grp < ngrp; grp += gridDim.x) {
        const int q = zs_opaque(q0);
        const long long pen = grp * PB + sub;
        const bool ok = pen < npen;
        cx<T> *const B0 = buf + (ok ? pen : 0) * Kz;
#define FZ(i) (B0 + (long long)(i) * g.S2)
        const cx<T> *sa = stA + sub * Kz, *sb = stB + sub * Kz;
        cx<T> A[E];
        constexpr int NREG = 4 - SLOTS_SM;
        T r_sl[NREG > 0 ? NREG : 1][E];
        // physical slot j (0 u, 1 v, 2 w_x, 3 w_y) of register slot e
#define SL(j, e) zs_slot<(j), NREG, T, E>(r_sl, slot_sm, PB * L, (e), out_row<L, E, true>(q, (e)))
        // pair 0: u + i w_x
        if (!wait_stage()) { bad = true; break; }
        k3_load_pair<T, L, E>(A, sa, false, sb, false, Kz, sz, q, ok);
        __syncthreads();
        issue(grp, 1, 4);
        pencil_fft<T, L, E, true, WARP>(A, sm, q, tw);
#pragma unroll
        for (int e = 0; e < E; e++) { SL(0, e) = A[e].x; SL(2, e) = A[e].y; }
        // pair 1: v + i w_y; then c_z = w_x v - w_y u, transformed and written over w_x (field 3)
        if (!wait_stage()) { bad = true; break; }
        k3_load_pair<T, L, E>(A, sa, false, sb, false, Kz, sz, q, ok);
        __syncthreads();
        issue(grp, 2, 5);
        pencil_fft<T, L, E, true, WARP>(A, sm, q, tw);
#pragma unroll
        for (int e = 0; e < E; e++) {
            const T vv = A[e].x, oy = A[e].y;
            SL(1, e) = vv; SL(3, e) = oy;
            A[e] = mk<T>(SL(2, e) * vv - oy * SL(0, e), T(0));
        }
        pencil_fft<T, L, E, false, WARP>(A, sm, q, tw);
        if (ok) {
            cx<T> *o = FZ(3);
#pragma unroll
            for (int e = 0; e < E; e++) {
                const int row = out_row<L, E, false>(q, e);
                if (row < Kz) o[row] = A[e];
            }
        }
        // pair 2: w + i w_z; then (c_x, c_y) and the CFL maxima
        if (!wait_stage()) { bad = true; break; }
        k3_load_pair<T, L, E>(A, sa, false, sb, false, Kz, sz, q, ok);
        __syncthreads();
        if (grp + gridDim.x < ngrp) issue(grp + gridDim.x, 0, 3);
        pencil_fft<T, L, E, true, WARP>(A, sm, q, tw);
#pragma unroll
        for (int e = 0; e < E; e++) {
            const T ww = A[e].x, oz = A[e].y, uu = SL(0, e), vv = SL(1, e);
            if (ok) cfl_update<T>(mx, uu, vv, ww, c);
            A[e] = mk<T>(SL(3, e) * ww - oz * vv, oz * uu - SL(2, e) * ww);
        }
        // forward transform of c_x + i c_y and extraction of both half spectra, kz < Kz
        pencil_fft<T, L, E, false, WARP>(A, sm, q, tw);
#pragma unroll
        for (int e = 0; e < E; e++) sm.at(out_row<L, E, false>(q, e)) = A[e];
        stage_barrier<WARP>();
        if (ok) {
            const T h = T(0.5);
            cx<T> *oa = FZ(0), *ob = FZ(1);
            for (int k = q; k < Kz; k += Q) {
                const cx<T> zk = sm.at(k), zm = sm.at(k == 0 ? 0 : L - k);
                oa[k] = mk<T>(h * (zk.x + zm.x), h * (zk.y - zm.y));
                ob[k] = mk<T>(h * (zk.y + zm.y), h * (zm.x - zk.x));
            }
        }
        stage_barrier<WARP>();
#undef SL
#undef FZ
    }
    if (bad && tid == 0) atomicExch(&ds->wait_timeout, 1);
    block_max4<T>(mx, ds);
}

} // namespace spns
