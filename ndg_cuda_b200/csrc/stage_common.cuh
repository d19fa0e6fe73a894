// Device arithmetic shared by the stage kernels of uniform meshes
// (stage_kernels.cu) and of mixed-order meshes (general_kernels.cu).
#pragma once

#include <cuda_runtime.h>

namespace ndg {
namespace dev {

// ---------------------------------------------------------------------------
// Arithmetic with selectable rounding.
template <bool S> __device__ __forceinline__ double mul(double a, double b) { return S ? __dmul_rn(a, b) : a * b; }
template <bool S> __device__ __forceinline__ double add(double a, double b) { return S ? __dadd_rn(a, b) : a + b; }
template <bool S> __device__ __forceinline__ double sub(double a, double b) { return S ? __dsub_rn(a, b) : a - b; }
// s + a*b: two roundings in strict mode, one FMA otherwise.
template <bool S> __device__ __forceinline__ double madd(double s, double a, double b) { return S ? __dadd_rn(s, __dmul_rn(a, b)) : fma(a, b, s); }

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
template <bool S>
__device__ __forceinline__ double metric(double t, double a, double b) {
    return mul<S>(add<S>(mul<S>(sub<S>(1.0, t), a), mul<S>(add<S>(1.0, t), b)), 0.25);
}

// Linear-in-t metric term of quad_metrics: ((1 - t) d0 + (1 + t) d1) / 4.
// Strict mode evaluates the reference's expression; the default mode the
// equivalent fma(t, (d1 - d0) / 4, (d0 + d1) / 4).
template <bool S>
struct MetricLine {
    double d0, d1, a, b;
    __device__ __forceinline__ MetricLine(double d0_, double d1_) : d0(d0_), d1(d1_), a(0.25 * (d0_ + d1_)), b(0.25 * (d1_ - d0_)) {}
    __device__ __forceinline__ double operator()(double t) const { return S ? metric<S>(t, d0, d1) : fma(t, b, a); }
};

}  // namespace dev
}  // namespace ndg
