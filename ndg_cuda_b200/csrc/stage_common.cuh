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

// Polls phase 0 of an mbarrier until it completes or `limit_ns` has passed;
// true when it completed.
__device__ __forceinline__ bool mbar_poll(uint64_t* bar, uint64_t limit_ns) {
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
        if (global_ns() - t0 > limit_ns) return false;
    }
}

// Waits for phase 0 of an mbarrier with a CTA-wide decision; every thread of
// the CTA calls it (it is also a __syncthreads), after a barrier that orders
// the mbarrier's initialisation before every poll. Each thread polls with the
// time limit, then the CTA gives up together if any thread timed out: the
// error word is set, thread 0 waits once more (bounded) so that a copy that
// was about to land is not left writing into an exited CTA, and false is
// returned to every thread so that the CTA stops as one.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned* error, uint64_t limit_ns) {
    const bool ok = mbar_poll(bar, limit_ns);
    if (!__syncthreads_or(!ok)) return true;
    if (threadIdx.x == 0) {
        atomicOr(error, 1u);
        mbar_poll(bar, limit_ns);
    }
    __syncthreads();
    return false;
}

constexpr uint64_t kWaitLimitNs = 2000000000ull;  // 2 s

// 8-byte asynchronous copy global -> shared (cp.async, no register staging)
// and the wait for all of this thread's copies.
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async4(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
// An L2 policy that makes the lines it touches the first to go
// (createpolicy), and the 8-byte copy under it: for the state a stage reads
// once and rewrites (q, k), so that it does not push out of L2 the traces
// and plan arrays every stage gathers from again.
__device__ __forceinline__ uint64_t evict_first_policy() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ void cp_async8_stream(void* dst, const void* src, uint64_t policy) {
    asm volatile("cp.async.ca.shared.global.L2::cache_hint [%0], [%1], 8, %2;" ::"r"(smem_addr(dst)), "l"(src), "l"(policy) : "memory");
}
// Hint: bring the 128-byte line holding p into L2 (prefetch.global.L2).
__device__ __forceinline__ void prefetch_l2(const void* p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

// ---------------------------------------------------------------------------
// Warp-level tensor-core products (PTX ISA: mma.sync). Fragments, with
// g = lane / 4 and t = lane % 4:
//   f64 m16n8k4:  A rows g, g + 8 at column t (a0, a1); B row t, column g
//                 (b0); C rows g, g + 8 at columns 2t, 2t + 1 (c0 c1, c2 c3).
//   tf32 m16n8k8: A (g, t), (g + 8, t), (g, t + 4), (g + 8, t + 4); B (t, g),
//                 (t + 4, g); C as for f64.
__device__ __forceinline__ void dmma_16x8x4(double (&c)[4], double a0, double a1, double b0) {
    asm("mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0, %1, %2, %3}, {%4, %5}, {%6}, {%0, %1, %2, %3};"
        : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
        : "d"(a0), "d"(a1), "d"(b0));
}
__device__ __forceinline__ void tf32mma_16x8x8(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, {%0, %1, %2, %3};"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}
// Round to TF32 (nearest, ties away from zero), kept in a 32-bit register.
__device__ __forceinline__ uint32_t to_tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}

// Per-lane tables of the tensor-core contraction passes of order N, built
// on the host (tc_lane_table_fp64 / _fp32) and read once per CTA, coalesced:
// lane-dependent entries would otherwise be divergent constant loads.
//   FP64 (m16n8k4): B[s][u][lane] = Dhat[8u + g][4s + t] (0 outside n x n);
//     LPW[u][h][lane], LMW[u][h][lane] = l(+1)[i] / w[i], l(-1)[i] / w[i] at
//     i = 8u + 2t + h (0 for i >= n); XK[s][lane] = node 4s + t (0 beyond).
//   FP32 (3xTF32 m16n8k8): B[s][u][lane][4] = TF32 high and low parts of
//     Dhat[8u + g][8s + t] and Dhat[8u + g][8s + t + 4]; LPW, LMW as FP64's
//     in float; XK[s][lane][2] = nodes 8s + t and 8s + t + 4.
template <int N>
struct TcTable64 {
    static constexpr int n = N + 1;
    static constexpr int KS = (n + 3) / 4;  // k-steps of 4
    static constexpr int NT = (n + 7) / 8;  // n-tiles of 8 output nodes
    static constexpr int kB = 0, kLPW = KS * NT * 32, kLMW = kLPW + NT * 64, kXK = kLMW + NT * 64, kSize = kXK + KS * 32;
};
template <int N>
struct TcTable32 {
    static constexpr int n = N + 1;
    static constexpr int KS = (n + 7) / 8;  // k-steps of 8
    static constexpr int NT = (n + 7) / 8;
    static constexpr int kB = 0, kLPW = KS * NT * 128, kLMW = kLPW + NT * 64, kXK = kLMW + NT * 64, kSize = kXK + KS * 64;
};

// ---------------------------------------------------------------------------
// Shared-memory placement of the uniform-order stage tiles without bank
// conflicts.
//
// The stage kernels order their line threads as (field f, line m, element
// e) with e fastest, so one shared-memory wavefront's group of G threads
// (G = 16 for 8-byte values, 32 for 4-byte values: 128 bytes either way)
// holds G / EPB consecutive lines of every element of the tile. A row sweep
// reads node (m, j) of each thread's element and a column sweep node
// (j, m), with j in lockstep. Node (i, j) of element e of field f sits at
// f QS + e ES + i P + j, and two threads of a group conflict when their
// addresses differ by a nonzero multiple of G. So:
//   P       the row pitch, odd: n, or n + 1 when n is even;
//   ES      the element stride: the first value in [n P, n P + G) with the
//           fewest wavefronts of the row and column sweeps over the groups
//           that lie in one field;
//   QS, Z   the field stride, in [EPB ES, EPB ES + G), and the residue of
//           the zero array's offset, for the groups that straddle two
//           fields (own-field sweeps and the flux-line reads of the other
//           fields and of the zero array);
//   SE, FS  element and field strides of the side arrays (4 n values per
//           element, value m of side s at s n + m), the same way.
// Every candidate's wavefront count is evaluated exactly, group by group,
// at compile time. EPB must divide G (whole lines per group). The search
// also serves kernels that order their threads (field, element, line), line
// fastest (element_fast = false); there an odd row pitch and an element
// stride that puts consecutive elements half a group apart make both sweeps
// conflict-free when n divides G.
namespace bank {

struct Strides {
    int P, ES, QS, Z, SE, FS;
};

enum Pattern : int { kRowOwn, kColOwn, kRowX, kColX, kRowY, kColY, kSideOwn, kSideFlux0, kSideFlux1, kSideFlux2 };

// Address (in values) read by thread (f, e, m) in one instruction of a
// pattern. The flux lines take X = u, p, 0 and Y = v, 0, p for f = 0, 1, 2;
// the zero array starts at Z.
constexpr int address(int pat, const Strides& L, int n, int f, int e, int m) {
    switch (pat) {
        case kRowOwn: return f * L.QS + e * L.ES + m * L.P;
        case kColOwn: return f * L.QS + e * L.ES + m;
        case kRowX: return f == 0 ? L.QS + e * L.ES + m * L.P : (f == 1 ? e * L.ES + m * L.P : L.Z + m * L.P);
        case kColX: return f == 0 ? L.QS + e * L.ES + m : (f == 1 ? e * L.ES + m : L.Z + m);
        case kRowY: return f == 0 ? 2 * L.QS + e * L.ES + m * L.P : (f == 1 ? L.Z + m * L.P : e * L.ES + m * L.P);
        case kColY: return f == 0 ? 2 * L.QS + e * L.ES + m : (f == 1 ? L.Z + m : e * L.ES + m);
        case kSideOwn: return f * L.FS + e * L.SE + m;
        default: return (pat - kSideFlux0) * L.FS + e * L.SE + f * n + m;  // all threads read field pat - kSideFlux0 of side f
    }
}

// Wavefronts of one instruction in the group of threads [g0, g0 + G): the
// most distinct addresses that share a bank. Zero-array reads of a line
// already read by another element of the group repeat its address (a
// broadcast) and are skipped.
constexpr int group_wavefronts(int pat, const Strides& L, int n, int EPB, int G, int g0, bool element_fast) {
    int bank[32] = {};
    bool seen_zero[32] = {};
    int worst = 0;
    for (int t = g0; t < g0 + G; ++t) {
        const int f = t / (EPB * n);
        if (f >= 3) break;
        const int rr = t - f * EPB * n;
        const int m = element_fast ? rr / EPB : rr - (rr / n) * n;
        const int e = element_fast ? rr - m * EPB : rr / n;
        const bool zero = (pat == kRowX || pat == kColX) ? f == 2 : ((pat == kRowY || pat == kColY) ? f == 1 : false);
        if (zero) {
            if (seen_zero[m]) continue;  // another element's read of this line: a broadcast
            seen_zero[m] = true;
        }
        const int b = address(pat, L, n, f, e, m) % G;
        if (++bank[b] > worst) worst = bank[b];
    }
    return worst;
}

// Sum over the groups within one field (straddling = false) or over the (at
// most two) groups that hold a field boundary (straddling = true).
constexpr int wavefronts(int pat, const Strides& L, int n, int EPB, int G, bool straddling, bool element_fast) {
    const int field = EPB * n;
    const int b1 = field / G * G, b2 = 2 * field / G * G;
    const bool s1 = field % G != 0, s2 = (2 * field) % G != 0;
    if (straddling)
        return (s1 ? group_wavefronts(pat, L, n, EPB, G, b1, element_fast) : 0) +
               (s2 && b2 != b1 ? group_wavefronts(pat, L, n, EPB, G, b2, element_fast) : 0);
    int total = 0;
    for (int g0 = 0; g0 < 3 * field; g0 += G)
        if (!((s1 && g0 == b1) || (s2 && g0 == b2))) total += group_wavefronts(pat, L, n, EPB, G, g0, element_fast);
    return total;
}

constexpr int straddling_q_cost(const Strides& L, int n, int EPB, int G, bool ef) {
    int c = 0;
    for (int p = kRowOwn; p <= kColOwn; ++p) c += 2 * wavefronts(p, L, n, EPB, G, true, ef);  // traces and G sweeps
    for (int p = kRowX; p <= kColY; ++p) c += wavefronts(p, L, n, EPB, G, true, ef);
    return c;
}

constexpr Strides search(int N, int EPB, int G, bool ef = true) {
    const int n = N + 1;
    Strides L{n % 2 ? n : n + 1, 0, 0, 0, 0, 0};
    int best = 1 << 30;
    for (int s = n * L.P; s < n * L.P + G; ++s) {
        Strides T = L;
        T.ES = s;
        T.QS = EPB * s;
        const int c = wavefronts(kRowOwn, T, n, EPB, G, false, ef) + wavefronts(kColOwn, T, n, EPB, G, false, ef);
        if (c < best) best = c, L.ES = s;
    }
    best = 1 << 30;
    for (int s = 4 * n; s < 4 * n + G; ++s) {
        Strides T = L;
        T.SE = s;
        T.FS = EPB * s;
        const int c = wavefronts(kSideOwn, T, n, EPB, G, false, ef);
        if (c < best) best = c, L.SE = s;
    }
    best = 1 << 30;
    for (int s = EPB * L.ES; s < EPB * L.ES + G; ++s) {
        Strides T = L;
        T.QS = s;
        T.Z = 0;
        const int c = straddling_q_cost(T, n, EPB, G, ef);
        if (c < best) best = c, L.QS = s;
    }
    best = 1 << 30;
    for (int z = 0; z < G; ++z) {
        Strides T = L;
        T.Z = z;
        const int c = straddling_q_cost(T, n, EPB, G, ef);
        if (c < best) best = c, L.Z = z;
    }
    best = 1 << 30;
    for (int s = EPB * L.SE; s < EPB * L.SE + G; ++s) {
        Strides T = L;
        T.FS = s;
        int c = wavefronts(kSideOwn, T, n, EPB, G, true, ef);
        for (int p = kSideFlux0; p <= kSideFlux2; ++p) c += wavefronts(p, T, n, EPB, G, true, ef);
        if (c < best) best = c, L.FS = s;
    }
    return L;
}

// First offset >= at whose residue modulo G is z.
constexpr int place(int at, int z, int G) { return at + ((z - at % G) % G + G) % G; }

constexpr int pow2_floor(int v) {
    int p = 1;
    while (2 * p <= v) p *= 2;
    return p;
}

}  // namespace bank

// ---------------------------------------------------------------------------
// D-hat times a line by the even-odd decomposition (A. Solomonoff, "A fast
// algorithm for spectral differentiation", J. Comput. Phys. 98, 1992). The
// nodes are symmetric about 0, so D-hat is centro-antisymmetric:
// dhat[n-1-i][n-1-j] = -dhat[i][j]. With e_j = x_j + x_{n-1-j} and
// o_j = x_j - x_{n-1-j} (j < H = n / 2), and e_H = x_H for odd n, the part
// of y = dhat x that is odd under reversal is A_i = sum_j ea[i][j] e_j
// (i < H) and the even part S_i = sum_j so[i][j] o_j (i < HO = n - H); then
// y_i = S_i + A_i and y_{n-1-i} = S_i - A_i (y_H = S_H for odd n). That is
// H HO + HO H multiply-adds (40 at n = 9) instead of n^2 (81), and half the
// coefficient loads. The sums round differently from the plain product, so
// the strict form keeps the plain one. `out(i, y_i)` takes each output; the
// pairs go in chunks of up to 5, so at most 10 accumulators are live.
template <int n, typename R, typename Out>
__device__ __forceinline__ void dhat_even_odd(const R* ea, const R* so, const R (&x)[n], Out&& out) {
    constexpr int H = n / 2, HO = n - H, C = HO < 5 ? HO : 5;
    R e[HO], o[H];
#pragma unroll
    for (int j = 0; j < H; ++j) {
        e[j] = x[j] + x[n - 1 - j];
        o[j] = x[j] - x[n - 1 - j];
    }
    if constexpr (HO > H) e[H] = x[H];
#pragma unroll
    for (int i0 = 0; i0 < HO; i0 += C) {
        R A[C], Sv[C];
#pragma unroll
        for (int c = 0; c < C; ++c) {
            if (i0 + c < H) A[c] = ea[(i0 + c) * HO] * e[0];
            if (i0 + c < HO) Sv[c] = so[(i0 + c) * H] * o[0];
        }
#pragma unroll
        for (int j = 1; j < HO; ++j)
#pragma unroll
            for (int c = 0; c < C; ++c) {
                if (i0 + c < H) A[c] = fma(ea[(i0 + c) * HO + j], e[j], A[c]);
                if (i0 + c < HO && j < H) Sv[c] = fma(so[(i0 + c) * H + j], o[j], Sv[c]);
            }
#pragma unroll
        for (int c = 0; c < C; ++c) {
            const int i = i0 + c;
            if (i < H) {
                out(i, Sv[c] + A[c]);
                out(n - 1 - i, Sv[c] - A[c]);
            } else if (i < HO) {
                out(i, Sv[c]);
            }
        }
    }
}

// Lowest orders at which the stage kernels contract by dhat_even_odd,
// measured per order on 256 x 256 meshes (best tile of each, against the
// plain product). FP32 form: N = 7 to 16 gain 2-10% per launch (N = 8:
// 135.7 -> 129.2 us), N <= 5 are even, N = 6 loses 3%. FP64 (not strict):
// N = 11 to 16 gain 2-5%, N <= 9 are even (the FP64 kernel there is bound by
// shared-memory traffic, not by its multiply-adds) and N = 10 loses 4.6%.
constexpr int kEvenOddMinOrder64 = 11;
constexpr int kEvenOddMinOrder32 = 7;

// Host: the even-odd halves of an n x n D-hat (dhat_even_odd), rounded to R.
template <typename R>
inline void even_odd_halves(int n, const double* dhat, R* ea, R* so) {
    const int H = n / 2, HO = n - H;
    for (int i = 0; i < H; ++i)
        for (int j = 0; j < HO; ++j)
            ea[i * HO + j] = static_cast<R>(j < H ? 0.5 * (dhat[i * n + j] + dhat[i * n + n - 1 - j]) : dhat[i * n + j]);
    for (int i = 0; i < HO; ++i)
        for (int j = 0; j < H; ++j) so[i * H + j] = static_cast<R>(0.5 * (dhat[i * n + j] - dhat[i * n + n - 1 - j]));
}

// ---------------------------------------------------------------------------
// Occupancy of the fused stage tiles. The target is as many CTAs per SM as
// fit in 200 KB of shared memory (the rest of the SM's 256 KB stays L1 for
// the side plan, corner and RK-register loads) and in `min_regs` registers
// per thread, at most 32. ptxas gives these kernels about 72 registers when
// it is free to choose; the target becomes a launch bound (bound_blocks)
// only where its register budget (allocated in steps of 8) is below that,
// i.e. where it raises the CTAs per SM. Measured on 256 x 256 meshes (best
// tile per order, against the free choice everywhere): FP64 N = 4 and 6
// 2.9% and 1.9% faster per launch, the FP32 form N = 6 7.6% and N = 10 1.2%;
// N = 8 and 12 keep their allocation. A bound everywhere (a budget of 80
// registers at the same 5 CTAs per SM for FP64 N = 10) lost 2.4% there.
constexpr int occupancy_target(size_t bytes, int threads, int min_regs) {
    const int by_smem = static_cast<int>(204800 / (bytes + 1024));
    const int by_regs = 65536 / (min_regs * threads);
    const int t = by_smem < by_regs ? by_smem : by_regs;
    return t < 1 ? 1 : (t > 32 ? 32 : t);
}
constexpr int register_budget(int blocks, int threads) { return 65536 / (blocks * threads) / 8 * 8; }
// The launch bound's CTAs per SM, or 0 (no bound: a zero minimum leaves
// ptxas its free choice).
constexpr int bound_blocks(size_t bytes, int threads, int min_regs) {
    const int t = occupancy_target(bytes, threads, min_regs);
    return register_budget(t, threads) < 72 ? t : 0;
}

// ---------------------------------------------------------------------------
// Tile of the fused stage: E elements per CTA (2, 4, 8 or 16), or for E = 0
// the default: 4 elements up to order 10, 2 above (the autotuner's choice
// on 256 x 256 meshes at N = 4, 6, 8 and at N = 12).
template <int N, int E = 0>
struct Tile {
    static constexpr int n = N + 1;
    static constexpr int NN = n * n;
    static constexpr int EPB = E > 0 ? E : (N <= 10 ? 4 : 2);
    static_assert(EPB == 2 || EPB == 4 || EPB == 8 || EPB == 16, "tiles hold 2, 4, 8 or 16 elements (whole lines per wavefront group)");
    static constexpr int kThreads = (3 * EPB * n + 31) / 32 * 32;
    // Node-wise phases of the stage kernels (tile copy, RK update): warp w
    // takes the (field, element) blocks w, w + kWarps, ... and its lanes the
    // nodes of a block, so no per-node division is needed.
    static constexpr int kWarps = kThreads / 32;
    static constexpr int kBlockIters = (3 * EPB + kWarps - 1) / kWarps;
    static constexpr int kLaneIters = (NN + 31) / 32;
    static constexpr bank::Strides L = bank::search(N, EPB, 16);
    static constexpr int P = L.P, ES = L.ES, QS = L.QS, SE = L.SE, FS = L.FS;
    // shared memory layout (doubles)
    static constexpr int kQ = 0;                        // [3][QS] q, then q of the next stage
    static constexpr int kG = kQ + 3 * QS;              // [3][QS] time derivative G
    static constexpr int kOwn = kG + 3 * QS;            // [3][FS] own side traces
    static constexpr int kFar = kOwn + 3 * FS;          // [3][FS] far side traces, then side fluxes
    static constexpr int kJ = kFar + 3 * FS;            // [EPB][ES] 1/J (J in strict mode)
    static constexpr int kS = kJ + EPB * ES;            // [EPB][4] edge metric per side
    static constexpr int kZ = bank::place(kS + EPB * 4, L.Z, 16);  // [n P] zeros: the absent flux component
    static constexpr int kDoubles = kZ + n * P;
    static constexpr size_t kBytes = sizeof(double) * kDoubles;
    // CTAs per SM of the kernel's launch bound (occupancy_target; 0: none).
    static constexpr int kMinBlocks = bound_blocks(kBytes, kThreads, 64);
    // Offset within an element of node nd = i n + j.
    __device__ static __forceinline__ int node(int nd) {
        if constexpr (P == n) {
            return nd;
        } else {
            const int i = nd / n;
            return i * P + (nd - i * n);
        }
    }
};

// Coefficients of order N, passed by value as a kernel parameter so that
// every use is a constant-bank operand with a compile-time offset.
template <int N>
struct Coeffs {
    static constexpr int n = N + 1, H = n / 2, HO = n - n / 2;
    double dhat[n * n];
    double xn[n], lm[n], lp[n], w[n], iw[n];
    double ea[H * HO], so[HO * H];  // even-odd halves of dhat (fill_even_odd)
    // The even-odd halves of dhat used by dhat_even_odd: ea[i][j] =
    // (dhat[i][j] + dhat[i][n-1-j]) / 2 for i < H, j < H, and ea[i][H] =
    // dhat[i][H] for odd n; so[i][j] = (dhat[i][j] - dhat[i][n-1-j]) / 2 for
    // i < HO, j < H.
    void fill_even_odd() { even_odd_halves(n, dhat, ea, so); }
};

}  // namespace dev
}  // namespace ndg
