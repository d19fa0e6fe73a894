// Output interpolation of the solution (Mesh2D_t::get_solution and
// get_complete_solution, src/meshes/Mesh2D_t.cpp:4237-4296, which call
// Element2D_t::interpolate_solution and interpolate_complete_solution,
// src/entities/Element2D_t.cpp:580-646), on the device.
//
// For every domain element and every point (i, j) of an n x n grid of
// equispaced reference coordinates xi_i = i / (n - 1) * 2 - 1 (likewise
// eta_j): the physical coordinates through the bilinear map
// (include/functions/quad_map.tpp:2-7), the fields p, u, v and their time
// derivatives interpolated with the order's interpolation matrix I,
//     p_ij = sum_m sum_n p_mn I_im I_jn,
// and the analytic error sum_m sum_n |g(x_mn, t) - p_mn| I_im I_jn, with g
// the reference plane wave at the element's Gauss nodes. Every operation is
// rounded on its own in the reference's order, so x, y, the fields and the
// derivatives equal the reference's CPU output bit for bit; the analytic
// error differs only through the exponential of the plane wave (CUDA's exp
// against the host's).
//
// One block per element (grid-stride): the element's nodal values and the
// node-wise |g - q| (evaluated once per node rather than once per output
// point; the values are the same) are staged in shared memory, then the
// block's threads take the output points.
//
// Also here: the L2 error against the plane wave (l2_error_kernel), per
// element in a fixed reduction order; the host adds the elements in order.
#include "output.cuh"
#include "stage_common.cuh"

namespace ndg {
namespace dev {

namespace {

// quad_map in the reference's operation order.
__device__ __forceinline__ void quad_map(const double* c, double xi, double eta, double& gx, double& gy) {
    const double a = __dsub_rn(1.0, xi), b = __dadd_rn(xi, 1.0), cc = __dsub_rn(1.0, eta), d = __dadd_rn(eta, 1.0);
    gx = __dmul_rn(__dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(__dmul_rn(c[0], a), cc), __dmul_rn(__dmul_rn(c[2], b), cc)), __dmul_rn(__dmul_rn(c[4], b), d)),
                             __dmul_rn(__dmul_rn(c[6], a), d)),
                   0.25);
    gy = __dmul_rn(__dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(__dmul_rn(c[1], a), cc), __dmul_rn(__dmul_rn(c[3], b), cc)), __dmul_rn(__dmul_rn(c[5], b), d)),
                             __dmul_rn(__dmul_rn(c[7], a), d)),
                   0.25);
}

__global__ void __launch_bounds__(128) output_kernel(OutputArgs a) {
    extern __shared__ double sm[];  // [9][(N + 1)^2]: p, u, v, dp, du, dv, |g - p|, |g - u|, |g - v|
    const bool want_q = a.p || a.u || a.v;
    const bool want_g = a.G && (a.dp_dt || a.du_dt || a.dv_dt);
    const bool want_e = a.p_err || a.u_err || a.v_err;
    const int P = a.n_interp;
    const int PP = P * P;
    const double span = static_cast<double>(P - 1);
    for (int64_t e = blockIdx.x; e < a.K; e += gridDim.x) {
        const int N = a.N[e], n = N + 1, NN = n * n;
        const double* c = a.corners + 8 * e;
        const double* nodes = a.nodes + a.nodes_off[N];
        const double* I = a.interp + a.interp_off[N];
        const int64_t o2 = a.off2[e];
        for (int t = threadIdx.x; t < NN; t += blockDim.x) {
            double q[3];
#pragma unroll
            for (int f = 0; f < 3; ++f) q[f] = a.q[f * a.block + o2 + t];
            if (want_q)
#pragma unroll
                for (int f = 0; f < 3; ++f) sm[f * NN + t] = q[f];
            if (want_g)
#pragma unroll
                for (int f = 0; f < 3; ++f) sm[(3 + f) * NN + t] = a.G[f * a.block + o2 + t];
            if (want_e) {
                const int m = t / n, nn = t - m * n;
                double gx, gy, g[3];
                quad_map(c, nodes[m], nodes[nn], gx, gy);
                plane_wave(gx, gy, a.time, g[0], g[1], g[2]);
#pragma unroll
                for (int f = 0; f < 3; ++f) sm[(6 + f) * NN + t] = fabs(__dsub_rn(g[f], q[f]));
            }
        }
        __syncthreads();
        for (int t = threadIdx.x; t < PP; t += blockDim.x) {
            const int i = t / P, j = t - i * P;
            const int64_t out = e * PP + t;
            if (a.x || a.y) {
                const double xi = __dsub_rn(__dmul_rn(__ddiv_rn(static_cast<double>(i), span), 2.0), 1.0);
                const double eta = __dsub_rn(__dmul_rn(__ddiv_rn(static_cast<double>(j), span), 2.0), 1.0);
                double gx, gy;
                quad_map(c, xi, eta, gx, gy);
                if (a.x) a.x[out] = gx;
                if (a.y) a.y[out] = gy;
            }
            double acc[9] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
            for (int m = 0; m < n; ++m) {
                const double im = I[i * n + m];
                for (int nn = 0; nn < n; ++nn) {
                    const double jn = I[j * n + nn];
                    const int k = m * n + nn;
                    if (want_q)
#pragma unroll
                        for (int f = 0; f < 3; ++f) acc[f] = __dadd_rn(acc[f], __dmul_rn(__dmul_rn(sm[f * NN + k], im), jn));
                    if (want_g)
#pragma unroll
                        for (int f = 3; f < 6; ++f) acc[f] = __dadd_rn(acc[f], __dmul_rn(__dmul_rn(sm[f * NN + k], im), jn));
                    if (want_e)
#pragma unroll
                        for (int f = 6; f < 9; ++f) acc[f] = __dadd_rn(acc[f], __dmul_rn(__dmul_rn(sm[f * NN + k], im), jn));
                }
            }
            double* dst[9] = {a.p, a.u, a.v, a.dp_dt, a.du_dt, a.dv_dt, a.p_err, a.u_err, a.v_err};
#pragma unroll
            for (int f = 0; f < 9; ++f)
                if (dst[f] && (f < 3 || (f < 6 && want_g) || f >= 6)) dst[f][out] = acc[f];
        }
        __syncthreads();
    }
}

// Per element: sum over nodes of w_i w_j J_ij (q - g)^2 for p, u, v, with
// J = x_xi y_eta - x_eta y_xi of the bilinear map in the reference's
// expression (Element2D_t.cpp:743-777) and g the reference plane wave.
__global__ void __launch_bounds__(128) l2_error_kernel(L2Args a) {
    __shared__ double red[3][128];
    for (int64_t e = blockIdx.x; e < a.K; e += gridDim.x) {
        const int N = a.N[e], n = N + 1, NN = n * n;
        const double* c = a.corners + 8 * e;
        const double* xn = a.nodes + a.vec_off[N];
        const double* w = a.weights + a.vec_off[N];
        const int64_t o2 = a.off2[e];
        double s[3] = {0.0, 0.0, 0.0};
        for (int t = threadIdx.x; t < NN; t += blockDim.x) {
            const int i = t / n, j = t - i * n;
            const double xi = xn[i], eta = xn[j];
            const double m00 = metric<true>(eta, __dsub_rn(c[2], c[0]), __dsub_rn(c[4], c[6]));
            const double m01 = metric<true>(xi, __dsub_rn(c[6], c[0]), __dsub_rn(c[4], c[2]));
            const double m10 = metric<true>(eta, __dsub_rn(c[3], c[1]), __dsub_rn(c[5], c[7]));
            const double m11 = metric<true>(xi, __dsub_rn(c[7], c[1]), __dsub_rn(c[5], c[3]));
            const double J = __dsub_rn(__dmul_rn(m00, m11), __dmul_rn(m01, m10));
            double gx, gy, g[3];
            quad_map(c, xi, eta, gx, gy);
            plane_wave(gx, gy, a.time, g[0], g[1], g[2]);
            const double ww = __dmul_rn(__dmul_rn(w[i], w[j]), J);
#pragma unroll
            for (int f = 0; f < 3; ++f) {
                const double d = __dsub_rn(a.q[f * a.block + o2 + t], g[f]);
                s[f] = fma(ww * d, d, s[f]);
            }
        }
#pragma unroll
        for (int f = 0; f < 3; ++f) red[f][threadIdx.x] = s[f];
        __syncthreads();
        for (int h = blockDim.x / 2; h > 0; h >>= 1) {
            if (threadIdx.x < h)
#pragma unroll
                for (int f = 0; f < 3; ++f) red[f][threadIdx.x] += red[f][threadIdx.x + h];
            __syncthreads();
        }
        if (threadIdx.x == 0)
#pragma unroll
            for (int f = 0; f < 3; ++f) a.partial[3 * e + f] = red[f][0];
        __syncthreads();
    }
}

}  // namespace

cudaError_t launch_l2_error(const L2Args& a, cudaStream_t stream) {
    if (a.K == 0) return cudaSuccess;
    const int blocks = static_cast<int>(a.K < 148 * 16 ? a.K : 148 * 16);
    l2_error_kernel<<<blocks, 128, 0, stream>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_output(const OutputArgs& a, int max_N, cudaStream_t stream) {
    if (a.K == 0) return cudaSuccess;
    const size_t smem = sizeof(double) * 9 * static_cast<size_t>(max_N + 1) * static_cast<size_t>(max_N + 1);
    const int blocks = static_cast<int>(a.K < 148 * 16 ? a.K : 148 * 16);
    output_kernel<<<blocks, 128, smem, stream>>>(a);
    return cudaGetLastError();
}

}  // namespace dev
}  // namespace ndg
