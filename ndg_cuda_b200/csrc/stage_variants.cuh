// Candidate tiles of the fused stage kernels for the autotuner: every order
// N is instantiated with E = 2, 4, 8 and 16 elements per CTA (powers of two:
// whole element lines per shared-memory wavefront, which the bank-conflict-
// free layout needs) where the tile fits 512 threads and 113 KB of shared
// memory (two CTAs per SM).
// stage_variants_fp64.cu and stage_variants_fp32.cu instantiate these
// templates for the FP64 (default rounding) and the FP32 form.
#pragma once

#include "stage_templates.cuh"

#include <cuda_runtime.h>

#include <type_traits>

namespace ndg {
namespace dev {

constexpr int kTileChoices[] = {2, 4, 8, 16};

// Orders with tensor-core variants (the contraction passes on the tensor
// cores pay once the lines are long: N >= 6).
constexpr int kTensorMinOrder = 6;

template <bool F32, int N, int E, bool TC = false>
struct Variant {
    using T = std::conditional_t<F32, TileF<N, E>, Tile<N, E>>;
    static constexpr bool feasible = T::kThreads <= 512 && T::kBytes <= 113 * 1024 && (!TC || (E <= 8 && N >= kTensorMinOrder));
};

template <int N>
Coeffs<N> variant_coeffs() {
    Coeffs<N> c;
    host_coefficients(N, c.dhat, c.xn, c.lm, c.lp, c.w, c.iw);
    c.fill_even_odd();
    return c;
}

template <int N>
CoeffsF<N> variant_coeffs_f() {
    const Coeffs<N> d = variant_coeffs<N>();
    CoeffsF<N> c;
    for (int i = 0; i < (N + 1) * (N + 1); ++i) c.dhat[i] = static_cast<float>(d.dhat[i]);
    for (int i = 0; i <= N; ++i) {
        c.xn[i] = static_cast<float>(d.xn[i]);
        c.lm[i] = static_cast<float>(d.lm[i]);
        c.lp[i] = static_cast<float>(d.lp[i]);
        c.w[i] = static_cast<float>(d.w[i]);
        c.iw[i] = static_cast<float>(d.iw[i]);
    }
    even_odd_halves(N + 1, d.dhat, c.ea, c.so);
    return c;
}

template <bool F32, int N, int E, bool TC>
cudaError_t variant_prepare() {
    if constexpr (Variant<F32, N, E, TC>::feasible) {
        using T = typename Variant<F32, N, E, TC>::T;
        if constexpr (F32)
            return cudaFuncSetAttribute(stage_kernel_f32<N, E, TC>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(T::kBytes));
        else
            return cudaFuncSetAttribute(stage_kernel<N, false, E, TC>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(T::kBytes));
    } else {
        return cudaErrorInvalidValue;
    }
}

template <bool F32, int N, int E, bool TC>
cudaError_t variant_launch(const StageArgs& a, cudaStream_t stream) {
    if constexpr (Variant<F32, N, E, TC>::feasible) {
        using T = typename Variant<F32, N, E, TC>::T;
        const dim3 grid(static_cast<unsigned>((a.n_elements + T::EPB - 1) / T::EPB), static_cast<unsigned>(a.n_instances));
        if constexpr (F32)
            stage_kernel_f32<N, E, TC><<<grid, T::kThreads, T::kBytes, stream>>>(a, variant_coeffs_f<N>());
        else
            stage_kernel<N, false, E, TC><<<grid, T::kThreads, T::kBytes, stream>>>(a, variant_coeffs<N>());
        return cudaGetLastError();
    } else {
        return cudaErrorInvalidValue;
    }
}

// Tile codes of order N: E for the SIMT passes, kTensorTile + E for the
// tensor-core passes (TC true), each where feasible.
template <bool F32, int N, bool TC>
int variant_candidates(int* out, int max) {
    const bool ok[] = {Variant<F32, N, 2, TC>::feasible, Variant<F32, N, 4, TC>::feasible, Variant<F32, N, 8, TC>::feasible,
                       Variant<F32, N, 16, TC>::feasible};
    int count = 0;
    for (int i = 0; i < 4; ++i)
        if (ok[i] && count < max) out[count++] = kTileChoices[i] + (TC ? kTensorTile : 0);
    return count;
}

#define NDG_VARIANT_TILES(FN, F32_, N_, TC_, ...)            \
    switch (epb) {                                            \
        case 2: return FN<F32_, N_, 2, TC_>(__VA_ARGS__);     \
        case 4: return FN<F32_, N_, 4, TC_>(__VA_ARGS__);     \
        case 8: return FN<F32_, N_, 8, TC_>(__VA_ARGS__);     \
        case 16: return FN<F32_, N_, 16, TC_>(__VA_ARGS__);   \
        default: return cudaErrorInvalidValue;                \
    }

template <bool F32, int N, bool TC>
cudaError_t variant_prepare_n(int epb) {
    NDG_VARIANT_TILES(variant_prepare, F32, N, TC)
}

template <bool F32, int N, bool TC>
cudaError_t variant_launch_n(int epb, const StageArgs& a, cudaStream_t stream) {
    NDG_VARIANT_TILES(variant_launch, F32, N, TC, a, stream)
}

#define NDG_VARIANT_ORDERS(CALL)  \
    switch (N) {                  \
        case 1: CALL(1);          \
        case 2: CALL(2);          \
        case 3: CALL(3);          \
        case 4: CALL(4);          \
        case 5: CALL(5);          \
        case 6: CALL(6);          \
        case 7: CALL(7);          \
        case 8: CALL(8);          \
        case 9: CALL(9);          \
        case 10: CALL(10);        \
        case 11: CALL(11);        \
        case 12: CALL(12);        \
        case 13: CALL(13);        \
        case 14: CALL(14);        \
        case 15: CALL(15);        \
        case 16: CALL(16);        \
        default: break;           \
    }

}  // namespace dev
}  // namespace ndg
