// Legendre-coefficient-decay error estimator on the device
// (Element2D_t::estimate_p_error and exponential_decay,
// src/entities/Element2D_t.cpp:274-343; called by Mesh2D_t::estimate_error,
// src/meshes/Mesh2D_t.cpp:4008-4012).
//
// For the last min(N+1, 4) modal orders p of the pressure, the spectrum is
// the sum over i < p of |p^_{i,p}| + |p^_{p,i}| plus |p^_{p,p}|, with modal
// coefficients p^ = sum_k sum_l P[k][l] L_i(x_k) w_k (2i+1)/2 L_p(x_l) ...
// A least-squares line through log(spectrum) against p gives the decay rate
// sigma and C; the error is sqrt(s_last^2 + C^2 / (2 sigma) exp(-2 sigma (N+1))).
//
// Every product and sum is rounded on its own (__dmul_rn/__dadd_rn) in the
// reference's order, so the spectrum and the fit are those of the
// reference's CPU build; log and exp are CUDA's, within one ulp of the host
// library's. Refine/coarsen flags therefore match the reference except for
// an error within an ulp of a tolerance.
//
// One thread per element and instance: the whole estimate is ~10^4 FP64
// operations per element, run once per adaptivity interval.
#include "ndg_internal.hpp"
#include "estimator.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

namespace ndg {
namespace dev {

namespace {
constexpr int kMaxPoly = kMaxOrder;
constexpr int kPolyTotal = (kMaxPoly + 1) * (kMaxPoly + 2) * (2 * kMaxPoly + 3) / 6;
__host__ __device__ constexpr int poly_offset(int N) { return N * (N + 1) * (2 * N + 1) / 6; }
}  // namespace

// Modal projection rows P_i(x_j) w_j (2i+1)/2 per order (NDG_t::polynomials_).
__constant__ double c_poly[kPolyTotal];

__global__ void estimate_error_kernel(EstimatorArgs a) {
    const int N = a.N, n = N + 1, NN = n * n;
    const int64_t total = a.count * a.n_instances;
    const double* poly = c_poly + poly_offset(N);
    const int npl = (N + 1 < 4) ? N + 1 : 4;  // n_points_least_squares_max (include/helpers/constants.h:19)
    for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < total; idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t inst = idx / a.count;
        const int64_t le = idx - inst * a.count;
        const int64_t e = a.ids ? a.ids[le] : le;
        const double* P = a.q + inst * 3 * a.block + (a.off2 ? a.off2[e] : e * NN);
        const int64_t out = inst * a.n_elements + e;
        double spectrum[4];
        for (int ni = 0; ni < npl; ++ni) {
            const int p = N + ni + 1 - npl;
            double s = 0.0;
            for (int i = 0; i < p; ++i) {
                double lx = 0.0, ly = 0.0;
                for (int kk = 0; kk < n; ++kk)
                    for (int l = 0; l < n; ++l) {
                        const double v = P[kk * n + l];
                        lx = __dadd_rn(lx, __dmul_rn(__dmul_rn(v, poly[i * n + kk]), poly[p * n + l]));
                        ly = __dadd_rn(ly, __dmul_rn(__dmul_rn(v, poly[p * n + kk]), poly[i * n + l]));
                    }
                s = __dadd_rn(s, __dadd_rn(fabs(lx), fabs(ly)));
            }
            double lx = 0.0;
            for (int kk = 0; kk < n; ++kk)
                for (int l = 0; l < n; ++l) lx = __dadd_rn(lx, __dmul_rn(__dmul_rn(P[kk * n + l], poly[p * n + kk]), poly[p * n + l]));
            spectrum[ni] = __dadd_rn(s, fabs(lx));
        }
        // Least-squares fit of log(spectrum) against p (exponential_decay).
        double x_avg = 0.0, y_avg = 0.0;
        for (int i = 0; i < npl; ++i) {
            x_avg = __dadd_rn(x_avg, static_cast<double>(N + i + 1 - npl));
            y_avg = __dadd_rn(y_avg, log(spectrum[i]));
        }
        x_avg = __ddiv_rn(x_avg, static_cast<double>(npl));
        y_avg = __ddiv_rn(y_avg, static_cast<double>(npl));
        double num = 0.0, den = 0.0;
        for (int i = 0; i < npl; ++i) {
            const double dp = __dsub_rn(static_cast<double>(N + i + 1 - npl), x_avg);
            num = __dadd_rn(num, __dmul_rn(dp, __dsub_rn(log(spectrum[i]), y_avg)));
            den = __dadd_rn(den, __dmul_rn(dp, dp));
        }
        const double sigma_signed = __ddiv_rn(num, den);
        const double C = exp(__dsub_rn(y_avg, __dmul_rn(sigma_signed, x_avg)));
        const double sigma = fabs(sigma_signed);
        const double tail = __dmul_rn(__ddiv_rn(__dmul_rn(__dmul_rn(C, C), 0.5), sigma), exp(__dmul_rn(__dmul_rn(-2.0, sigma), static_cast<double>(N + 1))));
        const double last = spectrum[npl - 1];
        const double err = __dsqrt_rn(__dadd_rn(__dmul_rn(last, last), tail));
        a.p_error[out] = err;
        a.p_sigma[out] = sigma;
        a.refine[out] = err > a.tolerance_min ? 1 : 0;
        a.coarsen[out] = err < a.tolerance_max ? 1 : 0;
    }
}

cudaError_t upload_polynomials(const Tables& t) {
    std::vector<double> poly(kPolyTotal, 0.0);
    for (int N = 0; N <= std::min(t.N_max, kMaxPoly); ++N) {
        const auto& v = t.get(NDG_TABLE_POLYNOMIALS, N);
        std::copy(v.begin(), v.end(), poly.begin() + poly_offset(N));
    }
    return cudaMemcpyToSymbol(c_poly, poly.data(), sizeof(double) * kPolyTotal);
}

cudaError_t launch_estimate_error(const EstimatorArgs& a, cudaStream_t stream) {
    if (a.N < 0 || a.N > kMaxPoly) return cudaErrorInvalidValue;
    const int64_t total = a.count * a.n_instances;
    if (total == 0) return cudaSuccess;
    const int blocks = static_cast<int>(std::min<int64_t>((total + 127) / 128, 148 * 16));
    estimate_error_kernel<<<blocks, 128, 0, stream>>>(a);
    return cudaGetLastError();
}

}  // namespace dev
}  // namespace ndg
