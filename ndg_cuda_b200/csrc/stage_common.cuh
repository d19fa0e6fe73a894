// Device arithmetic shared by the stage kernels of uniform meshes
// (stage_kernels.cu), of mixed-order meshes (general_kernels.cu) and by the
// variable-speed and adjoint kernels (adjoint_kernels.cu): rounding
// helpers, metrics, the bulk-copy/mbarrier primitives, the tile layout of
// the fused stage and the by-value coefficient block.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace ndg {
namespace dev {

// ---------------------------------------------------------------------------
// Arithmetic with selectable rounding: S (strict, FP64 only) rounds every
// operation on its own in the written order; otherwise the compiler may
// contract, and R may be float (the FP32 forms).
template <bool S, typename R>
__device__ __forceinline__ R mul(R a, R b) {
    if constexpr (S) {
        static_assert(sizeof(R) == 8, "strict rounding is FP64");
        return __dmul_rn(a, b);
    } else {
        return a * b;
    }
}
template <bool S, typename R>
__device__ __forceinline__ R add(R a, R b) {
    if constexpr (S) {
        static_assert(sizeof(R) == 8, "strict rounding is FP64");
        return __dadd_rn(a, b);
    } else {
        return a + b;
    }
}
template <bool S, typename R>
__device__ __forceinline__ R sub(R a, R b) {
    if constexpr (S) {
        static_assert(sizeof(R) == 8, "strict rounding is FP64");
        return __dsub_rn(a, b);
    } else {
        return a - b;
    }
}
// s + a*b: two roundings in strict mode, one FMA otherwise.
template <bool S, typename R>
__device__ __forceinline__ R madd(R s, R a, R b) {
    if constexpr (S) {
        static_assert(sizeof(R) == 8, "strict rounding is FP64");
        return __dadd_rn(s, __dmul_rn(a, b));
    } else {
        return fma(a, b, s);
    }
}
// a / b: the IEEE quotient in strict mode (and for FP32), a * (1/b) allowed otherwise by the caller.
template <bool S, typename R>
__device__ __forceinline__ R div(R a, R b) {
    if constexpr (S) {
        static_assert(sizeof(R) == 8, "strict rounding is FP64");
        return __ddiv_rn(a, b);
    } else {
        return a / b;
    }
}

// The reference plane wave g(x, t) (include/functions/analytical_solution.tpp:4-10,
// constants of include/helpers/constants.h:15-18).
__device__ __forceinline__ void plane_wave(double x, double y, double t, double& p, double& u, double& v) {
    const double kx = 0.707106781186548, ky = 0.707106781186548, d = 0.120112240878645;
    const double a = __dsub_rn(__dadd_rn(__dmul_rn(kx, __dsub_rn(x, -0.2)), __dmul_rn(ky, __dsub_rn(y, -0.2))), t);
    p = exp(__ddiv_rn(__dmul_rn(-a, a), __dmul_rn(d, d)));
    u = __dmul_rn(p, kx);
    v = __dmul_rn(p, ky);
}

// Bilinear metric term ((1 - t) a + (1 + t) b) / 4 of quad_metrics.
template <bool S, typename R = double>
__device__ __forceinline__ R metric(R t, R a, R b) {
    return mul<S>(add<S>(mul<S>(sub<S>(R(1), t), a), mul<S>(add<S>(R(1), t), b)), R(0.25));
}

// Linear-in-t metric term of quad_metrics: ((1 - t) d0 + (1 + t) d1) / 4.
// Strict mode evaluates the reference's expression; the default mode the
// equivalent fma(t, (d1 - d0) / 4, (d0 + d1) / 4).
template <bool S, typename R = double>
struct MetricLine {
    R d0, d1, a, b;
    __device__ __forceinline__ MetricLine(R d0_, R d1_) : d0(d0_), d1(d1_), a(R(0.25) * (d0_ + d1_)), b(R(0.25) * (d1_ - d0_)) {}
    __device__ __forceinline__ R operator()(R t) const { return S ? metric<S, R>(t, d0, d1) : fma(t, b, a); }
};

// ---------------------------------------------------------------------------
// TMA bulk copy and mbarrier (PTX ISA: cp.async.bulk, mbarrier).
__device__ __forceinline__ uint32_t smem_addr(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}
__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Waits for phase 0 of an mbarrier, giving up after `limit_ns`: the error
// word is then set and false returned so that the CTA stops.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned* error, uint64_t limit_ns) {
    const uint32_t a = smem_addr(bar);
    uint32_t done = 0;
    const uint64_t t0 = global_ns();
    while (true) {
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n selp.u32 %0, 1, 0, p;\n}"
            : "=r"(done)
            : "r"(a)
            : "memory");
        if (done) return true;
        if (global_ns() - t0 > limit_ns) {
            atomicOr(error, 1u);
            return false;
        }
    }
}

constexpr uint64_t kWaitLimitNs = 2000000000ull;  // 2 s

// ---------------------------------------------------------------------------
// Tile of the fused stage: E elements per CTA (E even), or for E = 0 the
// default: as many as fit ~60 KB of shared memory (several CTAs per SM) and
// 256 threads.
template <int N, int E = 0>
struct Tile {
    static constexpr int n = N + 1;
    static constexpr int NN = n * n;
    static constexpr int per_element_doubles = 2 * 3 * NN + 2 * 3 * 4 * n + NN + 4;
    static constexpr int by_smem = (60 * 1024 / 8) / per_element_doubles;
    static constexpr int by_threads = 256 / (3 * n);
    static constexpr int raw = by_smem < by_threads ? by_smem : by_threads;
    static constexpr int EPB = E > 0 ? E : (raw >= 2 ? (raw & ~1) : 2);
    static_assert(EPB % 2 == 0, "tiles hold an even number of elements (aligned bulk copies)");
    static constexpr int kThreads = (3 * EPB * n + 31) / 32 * 32;
    // Node-wise work per thread in the RK phase: ceil(3 EPB NN / threads).
    static constexpr int kNodeIters = (3 * EPB * NN + kThreads - 1) / kThreads;
    // shared memory layout (doubles); the bulk-copied q tile first
    static constexpr int kQ = 0;                         // [3][EPB][NN] q, then q of the next stage
    static constexpr int kG = kQ + 3 * EPB * NN;         // [3][EPB][NN] time derivative G
    static constexpr int kOwn = kG + 3 * EPB * NN;       // [3][EPB][4][n] own side traces
    static constexpr int kFar = kOwn + 3 * EPB * 4 * n;  // [3][EPB][4][n] far side traces, then side fluxes
    static constexpr int kJ = kFar + 3 * EPB * 4 * n;    // [EPB][NN] 1/J (J in strict mode)
    static constexpr int kS = kJ + EPB * NN;             // [EPB][4] edge metric per side
    static constexpr int kZ = kS + EPB * 4;              // [NN] zeros: the absent flux component
    static constexpr int kBar = kZ + NN;                 // mbarrier (8 bytes)
    static constexpr int kDoubles = kBar + 2;
    static constexpr size_t kBytes = sizeof(double) * kDoubles;
};

// Coefficients of order N, passed by value as a kernel parameter so that
// every use is a constant-bank operand with a compile-time offset.
template <int N>
struct Coeffs {
    double dhat[(N + 1) * (N + 1)];
    double xn[N + 1], lm[N + 1], lp[N + 1], w[N + 1], iw[N + 1];
};

}  // namespace dev
}  // namespace ndg
