// passes.cuh -- launch code of one step, templated on the arithmetic type T of
// the transforms (double: FP64 form; float: compensated FP32 hi/lo form).
// Included by exactly one translation unit per precision (spns_f64.cu,
// spns_f32.cu), which exports the PrecOps table of that precision.
#pragma once
#include "handle.h"

#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

template <typename T> struct Passes {
    using C = spns::cx<T>;
    static constexpr bool HILO = sizeof(T) == 4;

    static C *U(spns_handle *h, int f = 0) { return (C *)h->U + (long long)f * h->g.S0; }
    static C *Ulo(spns_handle *h, int f = 0) { return HILO ? (C *)h->Ulo + (long long)f * h->g.S0 : nullptr; }
    static const C *tw(spns_handle *h, int L) { return (const C *)h->tw[L]; }

    template <int L, int MODE, int ALT = 0> static cudaError_t launch_k1(spns_handle *h) {
        using S = ShapeK1A<T, L, ALT>;
        auto kern = spns::k1_inv_x<T, L, S::E, S::P, MODE>;
        cudaError_t e = spns_set_smem(kern, S::SMEM_ROW);
        if (e != cudaSuccess) return e;
        dim3 grid((h->g.Kz + S::P - 1) / S::P, h->g.Ky);
        kern<<<grid, S::THREADS, S::SMEM_ROW, h->st>>>(h->g, U(h, 0), U(h, 1), U(h, 2), (C *)h->B1, tw(h, L));
        return cudaGetLastError();
    }
    // ---- x/y passes with TMA-moved tiles (double precision, axis_tma.cuh) ----
    // Tensor map {2*Kz doubles, rows, lines, fields} over an input buffer, cached per
    // (pass, buffer) in the handle.  Box {2P, R, 1, 1}.
    static cudaError_t axis_map(spns_handle *h, int pass, const void *in, int rows, int lines, int fields, long long row_stride,
                                long long line_stride, long long field_stride, int P, int R, const CUtensorMap **out) {
        const auto key = std::make_pair(pass, in);
        auto it = h->tmaps.find(key);
        if (it == h->tmaps.end()) {
            static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
            if (!encode) {
                void *fn = nullptr;
                cudaDriverEntryPointQueryResult q;
                cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
                if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn) return e != cudaSuccess ? e : cudaErrorNotSupported;
                encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
            }
            const size_t cs = sizeof(C);
            cuuint64_t dims[4] = {(cuuint64_t)(2 * h->g.Kz), (cuuint64_t)rows, (cuuint64_t)lines, (cuuint64_t)fields};
            cuuint64_t strides[3] = {(cuuint64_t)(row_stride * cs), (cuuint64_t)(line_stride * cs), (cuuint64_t)(field_stride * cs)};
            cuuint32_t box[4] = {(cuuint32_t)(2 * P), (cuuint32_t)R, 1u, 1u};
            cuuint32_t estr[4] = {1u, 1u, 1u, 1u};
            CUtensorMap m;
            CUresult r = encode(&m, sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4,
                                const_cast<void *>(in), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
            if (r != CUDA_SUCCESS) return cudaErrorInvalidValue;
            it = h->tmaps.emplace(key, m).first;
        }
        *out = &it->second;
        return cudaSuccess;
    }
    // Persistent launch of k_axis_tma: one wave of blocks (one per SM at this shared memory).
    template <int L, bool INV>
    static cudaError_t launch_axis_tma(spns_handle *h, const CUtensorMap *map, const spns::AxisArgs &a, C *out) {
        using S = AxisTmaShape<T, L>;
        auto kern = spns::k_axis_tma<T, L, S::E, S::P, INV>;
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::SMEM);
        if (e != cudaSuccess) return e;
        constexpr int THREADS = S::P * (L / S::E);
        int per_sm = 0;
        if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, THREADS, S::SMEM)) != cudaSuccess) return e;
        if (per_sm < 1) return cudaErrorInvalidConfiguration;
        const long long items = (long long)((a.Kz + S::P - 1) / S::P) * a.lines;
        const long long blocks = std::min<long long>(items, (long long)h->sms * per_sm);
        kern<<<(unsigned)blocks, THREADS, S::SMEM, h->st>>>(*map, a, out, tw(h, L), h->ds);
        return cudaGetLastError();
    }
    // Shared-memory placement of an inverse tile needs the boxes from both ends not to overlap.
    template <int L> static bool axis_tma_fits(int hh) {
        const int R = SPNS_AX_TMA_R;
        const int npos = (hh + R) / R, nneg = (hh + R - 1) / R;
        return hh >= 1 && 2 * hh + 1 <= L && L - nneg * R >= npos * R;
    }
    template <int L, int MODE> static cudaError_t launch_k2_tma(spns_handle *h) {
        using S = AxisTmaShape<T, L>;
        const spns::Geo &g = h->g;
        const int nin = (h->B1 == h->inv_B1 || MODE == spns::MODE_INV) ? 6 : h->nB1;
        const CUtensorMap *map = nullptr;
        cudaError_t e = axis_map(h, 2, h->B1, g.Ky, g.Mx, nin, (long long)g.Mx * g.Kz, g.Kz, g.S1, S::P, SPNS_AX_TMA_R, &map);
        if (e != cudaSuccess) return e;
        spns::AxisArgs a{};
        a.h = g.hy; a.Kc = g.Ky; a.lines = g.Mx; a.Kz = g.Kz; a.nout = spns::Fields<MODE>::K2;
        for (int f = 0; f < a.nout; f++) a.src |= (unsigned long long)(f < 6 ? f : f - 6) << (4 * f);
        a.deriv_from = (MODE == spns::MODE_VEL || MODE == spns::MODE_ROT) ? 99 : 6;
        a.s = g.sy; a.o_row = (long long)g.Mx * g.Kz; a.o_line = g.Kz; a.o_field = g.S2; a.rbox = SPNS_AX_TMA_R;
        return launch_axis_tma<L, true>(h, map, a, (C *)h->B2);
    }
    template <int L, int MODE> static cudaError_t launch_k4_tma(spns_handle *h) {
        using S = AxisTmaShape<T, L>;
        const spns::Geo &g = h->g;
        const int nin = MODE == spns::MODE_INV ? 9 : h->nB2;
        const CUtensorMap *map = nullptr;
        cudaError_t e = axis_map(h, 4, h->B2, g.My, g.Mx, nin, (long long)g.Mx * g.Kz, g.Kz, g.S2, S::P, SPNS_AX_TMA_R, &map);
        if (e != cudaSuccess) return e;
        spns::AxisArgs a{};
        a.h = g.hy; a.Kc = g.Ky; a.lines = g.Mx; a.Kz = g.Kz; a.nout = spns::Fields<MODE>::NOUT;
        for (int f = 0; f < a.nout; f++) a.src |= (unsigned long long)spns::k4_in_field<MODE>(f) << (4 * f);
        a.deriv_from = 99;
        a.s = g.sy; a.o_row = (long long)g.Mx * g.Kz; a.o_line = g.Kz; a.o_field = g.S1; a.rbox = SPNS_AX_TMA_R;
        return launch_axis_tma<L, false>(h, map, a, (C *)h->B1);
    }
    template <int L, int MODE> static cudaError_t launch_k5_tma(spns_handle *h) {
        using S = AxisTmaShape<T, L>;
        const spns::Geo &g = h->g;
        const int nin = MODE == spns::MODE_INV ? 6 : h->nB1;
        const CUtensorMap *map = nullptr;
        cudaError_t e = axis_map(h, 5, h->B1, g.Mx, g.Ky, nin, g.Kz, (long long)g.Mx * g.Kz, g.S1, S::P, SPNS_AX_TMA_R, &map);
        if (e != cudaSuccess) return e;
        spns::AxisArgs a{};
        a.h = g.hx; a.Kc = g.Kx; a.lines = g.Ky; a.Kz = g.Kz; a.nout = spns::Fields<MODE>::NOUT;
        for (int f = 0; f < a.nout; f++) a.src |= (unsigned long long)f << (4 * f);
        a.deriv_from = 99;
        a.s = g.sx; a.o_row = g.Kz; a.o_line = (long long)g.Kx * g.Kz; a.o_field = g.S0; a.rbox = SPNS_AX_TMA_R;
        return launch_axis_tma<L, false>(h, map, a, (C *)h->B2);
    }

    template <int L, int MODE, int ALT = 0> static cudaError_t launch_k2(spns_handle *h) {
        if constexpr (AxisTmaShape<T, L>::ON && ALT == 0)
            if (axis_tma_fits<L>(h->g.hy)) return launch_k2_tma<L, MODE>(h);
        using S = ShapeK2A<T, L, ALT>;
        auto kern = spns::k2_inv_y<T, L, S::E, S::P, MODE>;
        cudaError_t e = spns_set_smem(kern, S::SMEM_ROW);
        if (e != cudaSuccess) return e;
        dim3 grid((h->g.Kz + S::P - 1) / S::P, h->g.Mx);
        kern<<<grid, S::THREADS, S::SMEM_ROW, h->st>>>(h->g, (const C *)h->B1, (C *)h->B2, tw(h, L));
        return cudaGetLastError();
    }
    // Rotational z pass staged pair by pair with bulk copies (zpass_staged.cuh),
    // persistent: one wave of blocks over the SMs.
    template <int L> static cudaError_t launch_k3_staged(spns_handle *h) {
        using ZS = ZStagedShape<T, L>;
        using LY = spns::ZStagedLayout<T, L, ZS::E, ZS::PB, ZS::SLOTS>;
        auto kern = spns::k3_rot_staged<T, L, ZS::E, ZS::PB, ZS::SLOTS, ZS::MINB>;
        const size_t smem = LY::smem_bytes(h->g.Kz);
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        constexpr int THREADS = ZS::PB * LY::Q;
        int dev = 0, sms = 0, per_sm = 0;
        if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
        if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
        if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, THREADS, smem)) != cudaSuccess) return e;
        if (per_sm < 1) return cudaErrorInvalidConfiguration;
        const long long groups = ((long long)h->g.Mx * h->g.My + ZS::PB - 1) / ZS::PB;
        long long blocks = (long long)sms * per_sm;
        if (blocks > groups) blocks = groups;
        kern<<<(unsigned)blocks, THREADS, smem, h->st>>>(h->g, (C *)h->B2, h->c, h->ds, tw(h, L));
        return cudaGetLastError();
    }
    template <int L, int MODE, int ALT = 0> static cudaError_t launch_k3(spns_handle *h, double *phys) {
        if constexpr (MODE == spns::MODE_ROT && ALT == 0 && ZStagedShape<T, L>::ON) return launch_k3_staged<L>(h);
        using S3 = Shape3<T, L, MODE, ALT>;
        constexpr bool STAGE_ROT = MODE == spns::MODE_ROT && ShapeSel<T>::Z_STAGE;
        constexpr bool STAGE_LES = MODE == spns::MODE_LES && sizeof(T) == 4 && SPNS_F32_Z_STAGE_LES;
        constexpr bool STAGE = STAGE_ROT || STAGE_LES;
        auto kern = spns::k3_z<T, L, S3::E, S3::P, MODE, STAGE>;
        constexpr size_t stage_fields = STAGE_ROT ? 2 * spns::K3StagePairs<T>::N : STAGE_LES ? 9 : 0;
        // the staging is sized by Kz at run time: at most L/2+1 values per field and pencil
        static_assert(S3::SMEM + (size_t)S3::P * stage_fields * (L / 2 + 1) * sizeof(C) <= 227 * 1024,
                      "z-pass shared memory (exchange, physical slots and staging) exceeds 227 KB for this shape");
        const size_t smem = S3::SMEM + (size_t)S3::P * stage_fields * h->g.Kz * sizeof(C);
        cudaError_t e = spns_set_smem(kern, smem);
        if (e != cudaSuccess) return e;
        const long long npen = (long long)h->g.Mx * h->g.My;
        dim3 grid((unsigned)((npen + S3::P - 1) / S3::P));
        kern<<<grid, S3::THREADS, smem, h->st>>>(h->g, (C *)h->B2, h->c, h->ds, phys, tw(h, L));
        return cudaGetLastError();
    }
    template <int L, int MODE, int ALT = 0> static cudaError_t launch_k4(spns_handle *h) {
        if constexpr (AxisTmaShape<T, L>::ON && ALT == 0 && MODE != spns::MODE_LES)
            if (2 * h->g.hy + 1 <= L) return launch_k4_tma<L, MODE>(h);
        using S = ShapeK2A<T, L, ALT>;
        auto kern = spns::k4_fwd_y<T, L, S::E, S::P, MODE>;
        cudaError_t e = spns_set_smem(kern, S::SMEM_ROW);
        if (e != cudaSuccess) return e;
        dim3 grid((h->g.Kz + S::P - 1) / S::P, h->g.Mx);
        kern<<<grid, S::THREADS, S::SMEM_ROW, h->st>>>(h->g, (const C *)h->B2, (C *)h->B1, tw(h, L));
        return cudaGetLastError();
    }
    template <int L, int MODE, int ALT = 0> static cudaError_t launch_k5(spns_handle *h) {
        if constexpr (AxisTmaShape<T, L>::ON && ALT == 0 && MODE != spns::MODE_LES)
            if (2 * h->g.hx + 1 <= L) return launch_k5_tma<L, MODE>(h);
        using S = ShapeK5A<T, L, ALT>;
        auto kern = spns::k5_fwd_x<T, L, S::E, S::P, MODE>;
        cudaError_t e = spns_set_smem(kern, S::SMEM_ROW);
        if (e != cudaSuccess) return e;
        dim3 grid((h->g.Kz + S::P - 1) / S::P, h->g.Ky);
        kern<<<grid, S::THREADS, S::SMEM_ROW, h->st>>>(h->g, (const C *)h->B1, (C *)h->B2, tw(h, L));
        return cudaGetLastError();
    }
    // Launch of pass K1..K5 in the shape the handle selected (shape_alt).
#define SPNS_SELECT(name, idx, ...)                                                              \
    template <int L, int MODE> static cudaError_t sel_##name(spns_handle *h) {                    \
        if constexpr (shape_alt_ok<L, MODE>())                                                    \
            if (h->shape_alt[idx]) return launch_##name<L, MODE, 1>(h __VA_ARGS__);               \
        return launch_##name<L, MODE, 0>(h __VA_ARGS__);                                          \
    }
    SPNS_SELECT(k1, 1)
    SPNS_SELECT(k2, 2)
    SPNS_SELECT(k3, 3, , nullptr)
    SPNS_SELECT(k4, 4)
    SPNS_SELECT(k5, 5)
#undef SPNS_SELECT

    // Spectral sweep; with the kappa scheme the new state goes into the u^{n-1}
    // buffers and the state buffers are swapped after the launch.
    static cudaError_t launch_k6(spns_handle *h) {
        const int n = h->g.Kx * h->g.Kz;
        dim3 grid((n + 255) / 256, h->g.Ky);
        const C *G = (const C *)h->B2;
        if (h->a.isSelfAdaptive) {
            spns::k6_sweep<T, true><<<grid, 256, 0, h->st>>>(h->g, G, U(h), Ulo(h), (C *)h->R, (C *)h->Up, (C *)h->Uplo,
                                                              (const C *)h->Up, (const C *)h->Uplo, h->c, h->ds);
            std::swap(h->U, h->Up);
            std::swap(h->Ulo, h->Uplo);
        } else {
            spns::k6_sweep<T, false><<<grid, 256, 0, h->st>>>(h->g, G, U(h), Ulo(h), (C *)h->R, U(h), Ulo(h), nullptr, nullptr,
                                                               h->c, h->ds);
        }
        return cudaGetLastError();
    }

    // Batched 1-D FFTs for the 2-D edge planes.
    template <int L, bool INV> static cudaError_t launch_lines(spns_handle *h, C *data, long long batch) {
        using S = Shape<T, L>;
        auto kern = spns::k_lines<T, L, S::E, S::P, INV>;
        cudaError_t e = spns_set_smem(kern, S::SMEM_PEN);
        if (e != cudaSuccess) return e;
        kern<<<(unsigned)((batch + S::P - 1) / S::P), S::THREADS, S::SMEM_PEN, h->st>>>(data, batch, tw(h, L));
        return cudaGetLastError();
    }
    template <int L, bool INV> static cudaError_t launch_cols(spns_handle *h, C *data, int ncols, int nbatch) {
        using S = Shape<T, L>;
        auto kern = spns::k_cols<T, L, S::E, S::P, INV>;
        cudaError_t e = spns_set_smem(kern, S::SMEM_ROW);
        if (e != cudaSuccess) return e;
        dim3 grid((ncols + S::P - 1) / S::P, nbatch);
        kern<<<grid, S::THREADS, S::SMEM_ROW, h->st>>>(data, ncols, tw(h, L));
        return cudaGetLastError();
    }

    // Inverse transform of the velocity only (Recalculate_Velocity_Antitransform):
    // refreshes the CFL maxima and, if phys != NULL, writes u,v,w on the grid.
    static int run_velocity(spns_handle *h, double *phys) {
        spns::k_reset_max<<<1, 1, 0, h->st>>>(h->ds);
        CKL();
        DISPATCH(h->g.Mx, LAUNCH((launch_k1<LL, spns::MODE_VEL>(h))));
        DISPATCH(h->g.My, LAUNCH((launch_k2<LL, spns::MODE_VEL>(h))));
        DISPATCH(h->g.Mz, LAUNCH((launch_k3<LL, spns::MODE_VEL>(h, phys))));
        return SPNS_OK;
    }

    // E(K), Om(K) of the state into h->bins.
    static int shell_sums(spns_handle *h) {
        const int nb = h->last_rad_max + 1;
        CK(cudaMemsetAsync(h->bins, 0, sizeof(double) * 2 * nb, h->st));
        const long long n = h->g.S0;
        const int blocks = (int)std::min<long long>((n + 255) / 256, (long long)spns::SHELL_BLOCKS_PER_SM * h->sms);
        spns::k_shell_sums<T><<<blocks, 256, sizeof(double) * 2 * nb, h->st>>>(h->g, U(h, 0), U(h, 1), U(h, 2), Ulo(h, 0), Ulo(h, 1),
                                                                              Ulo(h, 2), h->last_rad_max, h->bins, h->bins + nb);
        CKL();
        return SPNS_OK;
    }

    static int forcing_scale(spns_handle *h, int last_eff, int nullify) {
        const long long n = h->g.S0;
        const int blocks = (int)std::min<long long>((n + 255) / 256, 16LL * h->sms);
        spns::k_forcing_scale<T><<<blocks, 256, 0, h->st>>>(h->g, U(h, 0), U(h, 1), U(h, 2), Ulo(h, 0), Ulo(h, 1), Ulo(h, 2), h->FT,
                                                           last_eff, nullify);
        CKL();
        return SPNS_OK;
    }

    static int conj_correction(spns_handle *h) {
        spns::k_conj_correction<T><<<64, 256, 0, h->st>>>(h->g, U(h, 0), U(h, 1), U(h, 2), Ulo(h, 0), Ulo(h, 1), Ulo(h, 2));
        CKL();
        return SPNS_OK;
    }

    static int seed_draw(spns_handle *h, unsigned long long seed, int lim_x, int lim_y, int lim_z) {
        const long long n = h->g.S0;
        const int blocks = (int)std::min<long long>((n + 255) / 256, 16LL * h->sms);
        spns::k_seed_draw<T><<<blocks, 256, 0, h->st>>>(h->g, seed, lim_x, lim_y, lim_z, U(h, 0), U(h, 1), U(h, 2), Ulo(h, 0),
                                                       Ulo(h, 1), Ulo(h, 2));
        CKL();
        return SPNS_OK;
    }

    // Spectra of the velocity-gradient invariants Q_G, Q_S, R_G, R_S, V^2 of the
    // current state (Recalculate_Invariants_Distribution, src/HIT_LES.cpp:1297-1319):
    // the five passes in MODE_INV on work buffers of the advective size (allocated
    // on first use and kept; the step's own buffers and graphs are not touched),
    // then shell sums of |F|^2 / (Mx My Mz)^2.  out[c*(last_rad_max+1) + K] on the host.
    static int invariant_spectra(spns_handle *h, double *out) {
        const spns::Geo &g = h->g;
        const int nb = h->last_rad_max + 1;
        if (!h->inv_B1) {
            CK(cudaMallocAsync(&h->inv_B1, sizeof(C) * 6 * (size_t)g.S1, h->st));
            CK(cudaMallocAsync(&h->inv_B2, sizeof(C) * 9 * (size_t)g.S2, h->st));
            CK(cudaMallocAsync((void **)&h->inv_bins, sizeof(double) * (5 * nb + 3), h->st));
        }
        double *nut = h->inv_bins + 5 * nb;               // nu_t sum, sum of squares, max bits
        CK(cudaMemsetAsync(nut, 0, sizeof(double) * 3, h->st));
        std::swap(h->B1, h->inv_B1);
        std::swap(h->B2, h->inv_B2);
        auto passes = [&]() -> int {
            DISPATCH(g.Mx, LAUNCH((launch_k1<LL, spns::MODE_INV>(h))));
            DISPATCH(g.My, LAUNCH((launch_k2<LL, spns::MODE_INV>(h))));
            DISPATCH(g.Mz, LAUNCH((launch_k3<LL, spns::MODE_INV>(h, nut))));
            DISPATCH(g.My, LAUNCH((launch_k4<LL, spns::MODE_INV>(h))));
            DISPATCH(g.Mx, LAUNCH((launch_k5<LL, spns::MODE_INV>(h))));
            return SPNS_OK;
        };
        const int r = passes();
        std::swap(h->B1, h->inv_B1);
        std::swap(h->B2, h->inv_B2);
        if (r) return r;
        CK(cudaMemsetAsync(h->inv_bins, 0, sizeof(double) * 5 * nb, h->st));
        const double scale = h->c.inv_norm * h->c.inv_norm;
        const int blocks = (int)std::min<long long>((g.S0 + 255) / 256, (long long)spns::SHELL_BLOCKS_PER_SM * h->sms);
        for (int c = 0; c < 5; c++) {
            spns::k_shell_sums_scalar<T><<<blocks, 256, sizeof(double) * nb, h->st>>>(
                g, (const C *)h->inv_B2 + (long long)c * g.S0, scale, h->last_rad_max, h->inv_bins + (long long)c * nb);
            CKL();
        }
        std::vector<double> host((size_t)5 * nb + 3);
        CK(cudaMemcpyAsync(host.data(), h->inv_bins, sizeof(double) * host.size(), cudaMemcpyDeviceToHost, h->st));
        CK(cudaStreamSynchronize(h->st));
        if (out) std::copy(host.begin(), host.begin() + 5 * nb, out);
        const double npts = (double)g.Mx * g.My * g.Mz;
        unsigned long long mb;
        std::memcpy(&mb, &host[5 * nb + 2], sizeof(mb));
        double mx;
        std::memcpy(&mx, &mb, sizeof(mx));
        h->nut_stats[0] = host[5 * nb] / npts;
        h->nut_stats[1] = std::sqrt(host[5 * nb + 1] / npts);
        h->nut_stats[2] = mx;
        return SPNS_OK;
    }

    // Exact aliasing correction of the rotational form on the +-N/2 planes
    // (edge_kernels.cuh), added to the compact nonlinear term G held in B2.
    static int edge_correction(spns_handle *h) {
        const spns::Geo &g = h->g;
        // group the aliasing axes by the size of their 2-D transforms (one group for a cubic box)
        int RC[3][2] = {{g.My, g.Mz}, {g.Mx, g.Mz}, {g.Mx, g.My}};
        bool done[3] = {false, false, false};
        for (int a0 = 0; a0 < 3; a0++) {
            if (!h->edge_axis[a0] || done[a0]) continue;
            spns::EdgeSet es;
            es.naxes = 0;
            es.R = RC[a0][0];
            es.C = RC[a0][1];
            es.first[0] = 0;
            for (int a = a0; a < 3; a++) {
                if (!h->edge_axis[a] || done[a] || RC[a][0] != es.R || RC[a][1] != es.C) continue;
                done[a] = true;
                es.axis[es.naxes] = a;
                es.first[es.naxes + 1] = es.first[es.naxes] + (a == 2 ? 1 : 2);
                es.naxes++;
            }
            const int np = es.first[es.naxes];
            const long long n = (long long)es.R * es.C;
            C *V = (C *)h->edge, *Phi = V + 3 * (long long)np * n;
            const long long nb = n * 3 * np;
            const int blocks = (int)std::min<long long>((nb + 255) / 256, 16LL * h->sms);
            spns::k_edge_build<T><<<blocks, 256, 0, h->st>>>(g, U(h), es, V);
            CKL();
            DISPATCH(es.C, LAUNCH((launch_lines<LL, true>(h, V, (long long)es.R * 3 * np))));
            DISPATCH(es.R, LAUNCH((launch_cols<LL, true>(h, V, es.C, 3 * np))));
            spns::k_edge_square<T><<<blocks, 256, 0, h->st>>>(V, n, np, Phi);
            CKL();
            DISPATCH(es.C, LAUNCH((launch_lines<LL, false>(h, Phi, (long long)es.R * np))));
            DISPATCH(es.R, LAUNCH((launch_cols<LL, false>(h, Phi, es.C, np))));
            const int ablocks = (int)std::min<long long>((n * 2 + 255) / 256, 8LL * h->sms);
            spns::k_edge_apply<T><<<dim3(ablocks, es.naxes), 256, 0, h->st>>>(g, (C *)h->B2, es, Phi);
            CKL();
            h->edge_launches += 7;
        }
        return SPNS_OK;
    }

    // Records an event before the next kernel of a profiled step.
    static void prof_mark(spns_handle *h, int slot, const char *name) {
        if (h->prof_steps >= h->prof_cap_steps) return;
        if (slot >= 16) return;
        if (h->prof_steps == 0 && (int)h->prof_names.size() <= slot) h->prof_names.push_back(name ? name : "");
        cudaEventRecord(h->prof_ev[(size_t)h->prof_steps * 16 + slot], h->st);
    }

    // One New_Fractional_Step_Method (src/HIT_LES.cpp:9-25).
    static int step_once(spns_handle *h) {
        int nk = 0;
        h->edge_launches = 0;
        int slot = 0;
        const bool prof = h->prof_steps < h->prof_cap_steps;
#define MARK(name) do { if (prof) prof_mark(h, slot++, name); } while (0)
        if (h->a.eps_forcing > 0.0) {
            MARK("eps_band");
            spns::k_eps_band<T><<<1, spns::EPS_BAND_THREADS, 0, h->st>>>(h->g, U(h, 0), U(h, 1), U(h, 2), Ulo(h, 0), Ulo(h, 1), Ulo(h, 2),
                                                                      h->a.eps_kmin, h->a.eps_kmax, h->a.eps_forcing, h->ds);
            CKL();
            nk += 1;
        }
        const int mode = h->a.isLES ? spns::MODE_LES : h->a.nonlinear_form == 2 ? spns::MODE_ADV : spns::MODE_ROT;
#define STEP_PASSES(MD)                                                                       \
        MARK("k1_inv_x");                                                                     \
        DISPATCH(h->g.Mx, LAUNCH((sel_k1<LL, MD>(h))));                                    \
        MARK("k2_inv_y");                                                                     \
        DISPATCH(h->g.My, LAUNCH((sel_k2<LL, MD>(h))));                                    \
        MARK("reset_max");                                                                    \
        spns::k_reset_max<<<1, 1, 0, h->st>>>(h->ds);                                         \
        CKL();                                                                                \
        MARK("k3_z");                                                                         \
        DISPATCH(h->g.Mz, LAUNCH((sel_k3<LL, MD>(h))));                           \
        MARK("k4_fwd_y");                                                                     \
        DISPATCH(h->g.My, LAUNCH((sel_k4<LL, MD>(h))));                                    \
        MARK("k5_fwd_x");                                                                     \
        DISPATCH(h->g.Mx, LAUNCH((sel_k5<LL, MD>(h))));                                    \
        if (MD == spns::MODE_ROT && h->edge) {                                                \
            MARK("edge_correction");                                                          \
            int r_ = edge_correction(h);                                                      \
            if (r_) return r_;                                                                \
        }                                                                                     \
        MARK("k6_sweep");                                                                     \
        LAUNCH(launch_k6(h));
        if (mode == spns::MODE_LES) { STEP_PASSES(spns::MODE_LES) }
        else if (mode == spns::MODE_ROT) { STEP_PASSES(spns::MODE_ROT) }
        else { STEP_PASSES(spns::MODE_ADV) }
#undef STEP_PASSES
        MARK("finish_step");
        spns::k_finish_step<<<1, 1, 0, h->st>>>(h->c, h->ds);
        CKL();
        MARK(nullptr);
        if (prof) { if (h->prof_steps == 0) h->prof_nk = slot - 1; h->prof_steps++; }
        if (mode == spns::MODE_ROT && h->edge) nk += h->edge_launches;             // build, 2+2 line FFTs, square, apply per group
        h->kernels_per_step = nk + 8;
        return SPNS_OK;
#undef MARK
    }

    // ---- slab decomposition (spns_slab_phase) ----
    // Reorder between a [nf][n1][n2][Kz] array and the all-to-all staging blocks.
    static cudaError_t slab_pack(spns_handle *h, void *full, void *stage, int nf, int n1, int n2, const spns::SlabRanges &r, int axis,
                                 int unpack) {
        const long long n = (long long)nf * n1 * n2 * h->g.Kz;
        const int blocks = (int)std::min<long long>((n + 255) / 256, 16LL * h->sms);
        spns::k_slab_pack<T><<<blocks, 256, 0, h->st>>>((C *)full, (C *)stage, nf, n1, n2, h->g.Kz, r, axis, unpack);
        return cudaGetLastError();
    }
    // Offsets of the staging blocks: block s holds nf * (axis 1: count_s * n2, axis 2: n1 * count_s) * Kz.
    static spns::SlabRanges slab_offsets(const spns::SlabRanges &r0, int nf, int n1, int n2, int Kz, int axis) {
        spns::SlabRanges r = r0;
        long long o = 0;
        for (int s = 0; s < r.n; s++) {
            r.off[s] = o;
            o += (long long)nf * (axis == 1 ? (long long)r.count[s] * n2 : (long long)n1 * r.count[s]) * Kz;
        }
        return r;
    }
    // The y and z passes run on this rank's x planes: swap the x-slab geometry and S1 buffer in.
    static void slab_swap(spns_handle *h) {
        std::swap(h->g, h->gx);
        std::swap(h->B1, h->B1x);
    }
    // Phases of one step (advective arithmetic or LES; the caller exchanges the
    // staging arrays and reduces the scalars between phases, see include/spns.h):
    //   VEL_A  inverse x pass of u, v, w on this rank's ky rows; pack for the exchange
    //   VEL_B  unpack; inverse y pass and z pass of u, v, w on this rank's x planes (CFL maxima)
    //   DT     time step from the maxima reduced over the ranks
    //   A      [forced shells' energy of this slab]; inverse x pass; pack
    //   B      unpack; [forcing amplitude]; inverse y, z and forward y passes; pack back
    //   C      unpack; forward x pass; spectral sweep; end of the step
    static int slab_phase(spns_handle *h, int phase) {
        const spns::Geo gy = h->g, gx = h->gx;
        const int ny = gy.Ky, Mx = gy.Mx, Ky = gx.Ky, nx = gx.Mx, Kz = gy.Kz;
        const bool les = h->a.isLES;
        const int nf1 = spns::Fields<spns::MODE_ADV>::K1;                        // 6 (advective and LES)
        const int nf4 = les ? spns::Fields<spns::MODE_LES>::K4 : spns::Fields<spns::MODE_ADV>::K4;
        const spns::SlabRanges fwd_pack3 = slab_offsets(h->xr, 3, ny, Mx, Kz, 2), fwd_unpack3 = slab_offsets(h->yr, 3, Ky, nx, Kz, 1);
        const spns::SlabRanges fwd_pack = slab_offsets(h->xr, nf1, ny, Mx, Kz, 2), fwd_unpack = slab_offsets(h->yr, nf1, Ky, nx, Kz, 1);
        const spns::SlabRanges back_pack = slab_offsets(h->yr, nf4, Ky, nx, Kz, 1), back_unpack = slab_offsets(h->xr, nf4, ny, Mx, Kz, 2);
        int r = SPNS_OK;
        auto xpasses = [&](auto body) -> int {
            slab_swap(h);
            const int rr = body();
            slab_swap(h);
            return rr;
        };
        switch (phase) {
        case SPNS_SLAB_VEL_A:
            DISPATCH(gy.Mx, LAUNCH((launch_k1<LL, spns::MODE_VEL>(h))));
            LAUNCH(slab_pack(h, h->B1, h->XS, 3, ny, Mx, fwd_pack3, 2, 0));
            return SPNS_OK;
        case SPNS_SLAB_VEL_B:
            LAUNCH(slab_pack(h, h->B1x, h->XR, 3, Ky, nx, fwd_unpack3, 1, 1));
            r = xpasses([&]() -> int {
                spns::k_reset_max<<<1, 1, 0, h->st>>>(h->ds);
                CKL();
                DISPATCH(gx.My, LAUNCH((launch_k2<LL, spns::MODE_VEL>(h))));
                DISPATCH(gx.Mz, LAUNCH((launch_k3<LL, spns::MODE_VEL>(h, nullptr))));
                return SPNS_OK;
            });
            return r;
        case SPNS_SLAB_DT:
            spns::k_recalc_dt<<<1, 1, 0, h->st>>>(h->c, h->ds);
            CKL();
            return SPNS_OK;
        case SPNS_SLAB_A:
            if (h->a.eps_forcing > 0.0) {
                spns::k_eps_band<T><<<1, spns::EPS_BAND_THREADS, 0, h->st>>>(gy, U(h, 0), U(h, 1), U(h, 2), Ulo(h, 0), Ulo(h, 1), Ulo(h, 2),
                                                                          h->a.eps_kmin, h->a.eps_kmax, h->a.eps_forcing, h->ds, 1);
                CKL();
            }
            if (les) { DISPATCH(gy.Mx, LAUNCH((launch_k1<LL, spns::MODE_LES>(h)))); }
            else { DISPATCH(gy.Mx, LAUNCH((launch_k1<LL, spns::MODE_ADV>(h)))); }
            LAUNCH(slab_pack(h, h->B1, h->XS, nf1, ny, Mx, fwd_pack, 2, 0));
            return SPNS_OK;
        case SPNS_SLAB_B:
            LAUNCH(slab_pack(h, h->B1x, h->XR, nf1, Ky, nx, fwd_unpack, 1, 1));
            if (h->a.eps_forcing > 0.0) {
                spns::k_eps_alpha<<<1, 1, 0, h->st>>>(h->a.eps_forcing, h->ds);
                CKL();
            }
            r = xpasses([&]() -> int {
#define SLAB_YZ(MD)                                                                    \
                DISPATCH(gx.My, LAUNCH((launch_k2<LL, MD>(h))));                      \
                spns::k_reset_max<<<1, 1, 0, h->st>>>(h->ds);                          \
                CKL();                                                                 \
                DISPATCH(gx.Mz, LAUNCH((launch_k3<LL, MD>(h, nullptr))));             \
                DISPATCH(gx.My, LAUNCH((launch_k4<LL, MD>(h))));
                if (les) { SLAB_YZ(spns::MODE_LES) } else { SLAB_YZ(spns::MODE_ADV) }
#undef SLAB_YZ
                return SPNS_OK;
            });
            if (r) return r;
            LAUNCH(slab_pack(h, h->B1x, h->XS, nf4, Ky, nx, back_pack, 1, 0));
            return SPNS_OK;
        case SPNS_SLAB_C:
            LAUNCH(slab_pack(h, h->B1, h->XR, nf4, ny, Mx, back_unpack, 2, 1));
            if (les) { DISPATCH(gy.Mx, LAUNCH((launch_k5<LL, spns::MODE_LES>(h)))); }
            else { DISPATCH(gy.Mx, LAUNCH((launch_k5<LL, spns::MODE_ADV>(h)))); }
            LAUNCH(launch_k6(h));
            spns::k_finish_step<<<1, 1, 0, h->st>>>(h->c, h->ds);
            CKL();
            return SPNS_OK;
        default:
            return spns_fail(h, SPNS_ERR_INVALID_ARGUMENT, "unknown slab phase %d", phase);
        }
    }

    // ---- batched step of same-class boxes (ensembles) ----
    // Every member of the table has h0's geometry, form, launch shapes and the
    // Adams-Bashforth scheme without constant-power forcing or edge correction.
    template <int L, int MODE, int ALT> static cudaError_t launch_k1b(spns_handle *h, const spns::BatchMember *tab, int n, cudaStream_t st) {
        using S = ShapeK1A<T, L, ALT>;
        auto kern = spns::k1_inv_x_batch<T, L, S::E, S::P, MODE>;
        cudaError_t e = spns_set_smem(kern, S::SMEM_ROW);
        if (e != cudaSuccess) return e;
        kern<<<dim3((h->g.Kz + S::P - 1) / S::P, h->g.Ky, n), S::THREADS, S::SMEM_ROW, st>>>(h->g, tab, tw(h, L));
        return cudaGetLastError();
    }
    template <int L, int MODE, int ALT> static cudaError_t launch_k2b(spns_handle *h, const spns::BatchMember *tab, int n, cudaStream_t st) {
        using S = ShapeK2A<T, L, ALT>;
        auto kern = spns::k2_inv_y_batch<T, L, S::E, S::P, MODE>;
        cudaError_t e = spns_set_smem(kern, S::SMEM_ROW);
        if (e != cudaSuccess) return e;
        kern<<<dim3((h->g.Kz + S::P - 1) / S::P, h->g.Mx, n), S::THREADS, S::SMEM_ROW, st>>>(h->g, tab, tw(h, L));
        return cudaGetLastError();
    }
    template <int L, int MODE, int ALT> static cudaError_t launch_k3b(spns_handle *h, const spns::BatchMember *tab, int n, cudaStream_t st) {
        using S3 = Shape3<T, L, MODE, ALT>;
        constexpr bool STAGE = MODE == spns::MODE_LES && sizeof(T) == 4 && SPNS_F32_Z_STAGE_LES;
        auto kern = spns::k3_z_batch<T, L, S3::E, S3::P, MODE, STAGE>;
        const size_t smem = S3::SMEM + (size_t)S3::P * (STAGE ? 9 : 0) * h->g.Kz * sizeof(C);
        cudaError_t e = spns_set_smem(kern, smem);
        if (e != cudaSuccess) return e;
        const long long npen = (long long)h->g.Mx * h->g.My;
        kern<<<dim3((unsigned)((npen + S3::P - 1) / S3::P), 1, n), S3::THREADS, smem, st>>>(h->g, tab, tw(h, L));
        return cudaGetLastError();
    }
    template <int L, int MODE, int ALT> static cudaError_t launch_k4b(spns_handle *h, const spns::BatchMember *tab, int n, cudaStream_t st) {
        using S = ShapeK2A<T, L, ALT>;
        auto kern = spns::k4_fwd_y_batch<T, L, S::E, S::P, MODE>;
        cudaError_t e = spns_set_smem(kern, S::SMEM_ROW);
        if (e != cudaSuccess) return e;
        kern<<<dim3((h->g.Kz + S::P - 1) / S::P, h->g.Mx, n), S::THREADS, S::SMEM_ROW, st>>>(h->g, tab, tw(h, L));
        return cudaGetLastError();
    }
    template <int L, int MODE, int ALT> static cudaError_t launch_k5b(spns_handle *h, const spns::BatchMember *tab, int n, cudaStream_t st) {
        using S = ShapeK5A<T, L, ALT>;
        auto kern = spns::k5_fwd_x_batch<T, L, S::E, S::P, MODE>;
        cudaError_t e = spns_set_smem(kern, S::SMEM_ROW);
        if (e != cudaSuccess) return e;
        kern<<<dim3((h->g.Kz + S::P - 1) / S::P, h->g.Ky, n), S::THREADS, S::SMEM_ROW, st>>>(h->g, tab, tw(h, L));
        return cudaGetLastError();
    }
#define SPNS_SELECT_B(name, idx)                                                                                       \
    template <int L, int MODE> static cudaError_t sel_##name(spns_handle *h, const spns::BatchMember *tab, int n, cudaStream_t st) { \
        if constexpr (shape_alt_ok<L, MODE>())                                                                         \
            if (h->shape_alt[idx]) return launch_##name<L, MODE, 1>(h, tab, n, st);                                    \
        return launch_##name<L, MODE, 0>(h, tab, n, st);                                                               \
    }
    SPNS_SELECT_B(k1b, 1)
    SPNS_SELECT_B(k2b, 2)
    SPNS_SELECT_B(k3b, 3)
    SPNS_SELECT_B(k4b, 4)
    SPNS_SELECT_B(k5b, 5)
#undef SPNS_SELECT_B
    static int batch_step(spns_handle *h, const spns::BatchMember *tab, int n, cudaStream_t st) {
        const int mode = h->a.isLES ? spns::MODE_LES : spns::MODE_ADV;
        spns::k_reset_max_batch<<<n, 1, 0, st>>>(tab);
        CKL();
#define BATCH_PASSES(MD)                                                                  \
        SPNS_DISPATCH_BATCH(h->g.Mx, LAUNCH((sel_k1b<LL, MD>(h, tab, n, st))));           \
        SPNS_DISPATCH_BATCH(h->g.My, LAUNCH((sel_k2b<LL, MD>(h, tab, n, st))));           \
        SPNS_DISPATCH_BATCH(h->g.Mz, LAUNCH((sel_k3b<LL, MD>(h, tab, n, st))));           \
        SPNS_DISPATCH_BATCH(h->g.My, LAUNCH((sel_k4b<LL, MD>(h, tab, n, st))));           \
        SPNS_DISPATCH_BATCH(h->g.Mx, LAUNCH((sel_k5b<LL, MD>(h, tab, n, st))));
        if (mode == spns::MODE_LES) { BATCH_PASSES(spns::MODE_LES) }
        else { BATCH_PASSES(spns::MODE_ADV) }
#undef BATCH_PASSES
        {
            const int nk = h->g.Kx * h->g.Kz;
            spns::k6_sweep_batch<T><<<dim3((nk + 255) / 256, h->g.Ky, n), 256, 0, st>>>(h->g, tab);
            CKL();
        }
        spns::k_finish_step_batch<<<n, 1, 0, st>>>(tab);
        CKL();
        return SPNS_OK;
    }

    static constexpr PrecOps ops() {
        return PrecOps{&step_once, &run_velocity, &shell_sums, &forcing_scale, &conj_correction, &seed_draw, &invariant_spectra,
                       &slab_phase, &batch_step};
    }
};
