// Fused DG stage kernels for sm_100a (B200), uniform order N, conforming faces.
//
// One launch performs one low-storage RK3 stage for every element of every
// instance: the reference's seven stage calls (interpolate_to_boundaries,
// boundary_conditions, project_to_faces, calculate_wave_fluxes,
// project_to_elements, compute_dg_wave_derivative, rk3_step;
// include/solvers/Solver2D_t.tcu:46-70) become the passes of one CTA that
// owns a tile of EPB consecutive elements:
//
//   prologue  8-byte asynchronous copies (cp.async) place the tile's
//             q = (p, u, v) in shared memory, in a padded layout free of
//             bank conflicts (Tile, stage_common.cuh), and the far-side
//             traces of its sides (the neighbours' traces of the previous
//             stage, which they wrote into this element's far slots);
//             meanwhile all threads build J and edge metrics from the four
//             corners
//   rows      bottom/top own traces
//   columns   xi-direction flux lines (kept in registers), right/left own traces
//   flux      upwind flux of every side node, times the edge metric
//   xi pass   Dhat . line + lift                       -> G (columns)
//   eta pass  eta-direction flux lines, Dhat . line + lift, then /J -> G (rows)
//   RK        k = a k + G, q += g dt k in FP64, node by node, coalesced
//   traces    four side traces of the new q for the next stage, written
//             into the far slots of the neighbour across each interior side
//
// Work is spread as one thread per (field, line, element), 3 EPB (N+1)
// threads per CTA, the element index fastest; shared memory carries only the
// q tile, G, J and the side data. HBM traffic per
// element and stage: q and k read and written (the algorithmic 32 B per
// degree of freedom), one trace write (into the neighbours' far slots) and
// one contiguous far-trace read of 4(N+1) values per field, and 8 corner
// coordinates. Metrics are recomputed in
// registers: on straight-sided quads x_xi, y_xi depend only on eta and
// x_eta, y_eta only on xi (quad_metrics, include/functions/quad_metrics.tpp:2-7).
//
// Field blocks hold an even number of elements (one unused element when K is
// odd) and tiles start on even elements, so the FP32 form's bulk copy of the
// FP64 tile (cp.async.bulk + mbarrier) starts on a 16-byte boundary and
// moves a multiple of 16 bytes.
//
// STRICT instantiations round every operation in the reference's order
// (__dmul_rn/__dadd_rn, true divisions) and reproduce its CPU results bit
// for bit; the default instantiations contract to FMAs and multiply by
// reciprocals.
#include "ndg_internal.hpp"
#include "stage_common.cuh"
#include "stage_kernels.cuh"
#include "stage_templates.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <vector>

namespace ndg {
namespace dev {

// Tables per order, packed as the reference's device NDG_t packs them:
// order N starts at N(N+1)/2 (vectors) and N(N+1)(2N+1)/6 (matrices).
constexpr int kVecTotal = (kMaxOrder + 1) * (kMaxOrder + 2) / 2;
constexpr int kMatTotal = (kMaxOrder + 1) * (kMaxOrder + 2) * (2 * kMaxOrder + 3) / 6;
__host__ __device__ constexpr int vec_offset(int N) { return N * (N + 1) / 2; }
__host__ __device__ constexpr int mat_offset(int N) { return N * (N + 1) * (2 * N + 1) / 6; }

__constant__ double c_nodes[kVecTotal];
__constant__ double c_weights[kVecTotal];
__constant__ double c_inv_weights[kVecTotal];
__constant__ double c_lagrange_left[kVecTotal];
__constant__ double c_lagrange_right[kVecTotal];
__constant__ double c_dhat[kMatTotal];

// Side trace of one field: value m of side s (reference order: bottom and
// right run with the element axes, top and left reversed;
// src/entities/Element2D_t.cpp:86-125).
template <int N, bool S>
__device__ __forceinline__ double side_trace(const double* __restrict__ q, int s, int m) {
    constexpr int n = N + 1;
    const double* l = (s == 0 || s == 3) ? c_lagrange_left + vec_offset(N) : c_lagrange_right + vec_offset(N);
    const int line = (s < 2) ? m : N - m;
    const int base = (s == 0 || s == 2) ? line * n : line;
    const int stride = (s == 0 || s == 2) ? 1 : n;
    double acc = 0.0;
#pragma unroll
    for (int j = 0; j < n; ++j) acc = madd<S>(acc, l[j], q[base + j * stride]);
    return acc;
}

// Side traces in FP32 (start of a run, or after the host changed q).
template <int N>
__global__ void __launch_bounds__(256) trace_kernel_f32(TraceArgs a) {
    constexpr int n = N + 1, NN = n * n;
    const int64_t K = a.n_elements, Kp = a.field_stride;
    const int64_t total = static_cast<int64_t>(a.n_instances) * 3 * K * 4 * n;
    const double* lm = c_lagrange_left + vec_offset(N);
    const double* lp = c_lagrange_right + vec_offset(N);
    for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < total; idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int m = static_cast<int>(idx % n);
        const int s = static_cast<int>((idx / n) % 4);
        const int64_t e = (idx / (4 * n)) % K;
        const int64_t fi = idx / (4 * n * K);
        const double* qe = a.q + (fi * Kp + e) * NN;
        const double* l = (s == 0 || s == 3) ? lm : lp;
        const int line = (s < 2) ? m : N - m;
        const int base = (s == 0 || s == 2) ? line * n : line;
        const int stride = (s == 0 || s == 2) ? 1 : n;
        float acc = 0.0f;
        for (int j = 0; j < n; ++j) acc = fmaf(static_cast<float>(l[j]), static_cast<float>(qe[base + j * stride]), acc);
        if (a.link) {
            const int2 lk = a.link[4 * e + s];
            if (((lk.y >> 2) & 7) == kInterior) a.trace_out_f[((fi * Kp + lk.x) * 4 + (lk.y & 3)) * n + (N - m)] = acc;
        } else {
            a.trace_out_f[((fi * Kp + e) * 4 + s) * n + m] = acc;
        }
    }
}

// Side traces only (start of a run, or after the host changed q).
template <int N, bool S>
__global__ void __launch_bounds__(256) trace_kernel(TraceArgs a) {
    constexpr int n = N + 1, NN = n * n;
    const int64_t K = a.n_elements, Kp = a.field_stride;
    const int64_t total = static_cast<int64_t>(a.n_instances) * 3 * K * 4 * n;
    for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < total; idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int m = static_cast<int>(idx % n);
        const int s = static_cast<int>((idx / n) % 4);
        const int64_t e = (idx / (4 * n)) % K;
        const int64_t fi = idx / (4 * n * K);  // instance * 3 + field
        const double* qf = a.q + (fi * Kp + e) * NN;
        const double v = side_trace<N, S>(qf, s, m);
        if (a.link) {
            const int2 lk = a.link[4 * e + s];
            if (((lk.y >> 2) & 7) == kInterior) a.trace_out[((fi * Kp + lk.x) * 4 + (lk.y & 3)) * n + (N - m)] = v;
        } else {
            a.trace_out[((fi * Kp + e) * 4 + s) * n + m] = v;
        }
    }
}

// Reference plane-wave initial condition (Mesh2D_t.cpp:1192-1216) on every
// node of every instance, through the bilinear map of
// include/functions/quad_map.tpp:2-7 in the reference's operation order.
__global__ void initial_condition_kernel(double* q, double* k, const double* corners, int N, int64_t K, int64_t Kp, int n_instances) {
    const int n = N + 1, NN = n * n;
    const int64_t total = K * NN;
    const double* xn = c_nodes + vec_offset(N);
    for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < total; idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t e = idx / NN;
        const int node = static_cast<int>(idx - e * NN);
        const int i = node / n, j = node - (node / n) * n;
        const double* c = corners + 8 * e;
        const double xi = xn[i], eta = xn[j];
        const double a = __dsub_rn(1.0, xi), b = __dadd_rn(xi, 1.0), cc = __dsub_rn(1.0, eta), d = __dadd_rn(eta, 1.0);
        const double gx = __dmul_rn(__dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(__dmul_rn(c[0], a), cc), __dmul_rn(__dmul_rn(c[2], b), cc)), __dmul_rn(__dmul_rn(c[4], b), d)),
                                              __dmul_rn(__dmul_rn(c[6], a), d)),
                                    0.25);
        const double gy = __dmul_rn(__dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(__dmul_rn(c[1], a), cc), __dmul_rn(__dmul_rn(c[3], b), cc)), __dmul_rn(__dmul_rn(c[5], b), d)),
                                              __dmul_rn(__dmul_rn(c[7], a), d)),
                                    0.25);
        double p, u, v;
        plane_wave(gx, gy, 0.0, p, u, v);
        for (int inst = 0; inst < n_instances; ++inst) {
            double* qi = q + static_cast<int64_t>(inst) * 3 * Kp * NN;
            double* ki = k + static_cast<int64_t>(inst) * 3 * Kp * NN;
            qi[idx] = p;
            qi[Kp * NN + idx] = u;
            qi[2 * Kp * NN + idx] = v;
            ki[idx] = 0.0;
            ki[Kp * NN + idx] = 0.0;
            ki[2 * Kp * NN + idx] = 0.0;
        }
    }
}

// CFL time step: min over elements of CFL * delta_xy_min / (N^2 c)
// (Solver2D_t.cpp:19-29), one block, deterministic tree reduction.
__global__ void delta_t_kernel(const double* delta_xy_min, const int* elem_N, int64_t K, double cfl, double* out) {
    __shared__ double red[1024];
    double v = __longlong_as_double(0x7FF0000000000000ll);  // +inf
    for (int64_t e = threadIdx.x; e < K; e += blockDim.x) {
        const int Ne = elem_N[e];
        v = fmin(v, __ddiv_rn(__dmul_rn(cfl, delta_xy_min[e]), static_cast<double>(Ne * Ne)));
    }
    red[threadIdx.x] = v;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w /= 2) {
        if (threadIdx.x < w) red[threadIdx.x] = fmin(red[threadIdx.x], red[threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = red[0];
}

// Time update of the reference's loop (Solver2D_t.tcu:37-42, 72) with
// step = {time, dt, dt_mesh, t_end}: advance, then the next step's dt,
// shortened to land on t_end.
__global__ void end_step_kernel(double* step) {
    const double time = step[0] + step[1];
    step[0] = time;
    step[1] = (time + step[2] > step[3]) ? step[3] - time : step[2];
}

// ---------------------------------------------------------------------------
// Host copies of the packed tables (set by upload_tables): the stage kernels
// take their order's coefficients as a by-value parameter.
namespace {
std::vector<double> h_nodes(kVecTotal), h_weights(kVecTotal), h_inv_weights(kVecTotal), h_ll(kVecTotal), h_lr(kVecTotal), h_dhat(kMatTotal);
}

template <int N>
Coeffs<N> make_coeffs() {
    Coeffs<N> c;
    constexpr int n = N + 1;
    for (int i = 0; i < n; ++i) {
        c.xn[i] = h_nodes[static_cast<size_t>(vec_offset(N) + i)];
        c.lm[i] = h_ll[static_cast<size_t>(vec_offset(N) + i)];
        c.lp[i] = h_lr[static_cast<size_t>(vec_offset(N) + i)];
        c.w[i] = h_weights[static_cast<size_t>(vec_offset(N) + i)];
        c.iw[i] = h_inv_weights[static_cast<size_t>(vec_offset(N) + i)];
    }
    for (int i = 0; i < n * n; ++i) c.dhat[i] = h_dhat[static_cast<size_t>(mat_offset(N) + i)];
    c.fill_even_odd();
    return c;
}

void host_coefficients(int N, double* dhat, double* xn, double* lm, double* lp, double* w, double* iw) {
    const int n = N + 1;
    for (int i = 0; i < n; ++i) {
        xn[i] = h_nodes[static_cast<size_t>(vec_offset(N) + i)];
        lm[i] = h_ll[static_cast<size_t>(vec_offset(N) + i)];
        lp[i] = h_lr[static_cast<size_t>(vec_offset(N) + i)];
        w[i] = h_weights[static_cast<size_t>(vec_offset(N) + i)];
        iw[i] = h_inv_weights[static_cast<size_t>(vec_offset(N) + i)];
    }
    for (int i = 0; i < n * n; ++i) dhat[i] = h_dhat[static_cast<size_t>(mat_offset(N) + i)];
}

std::vector<double> tc_lane_table_fp64(int N) {
    const int n = N + 1, KS = (n + 3) / 4, NT = (n + 7) / 8;
    const int kLPW = KS * NT * 32, kLMW = kLPW + NT * 64, kXK = kLMW + NT * 64, kSize = kXK + KS * 32;
    std::vector<double> dh(static_cast<size_t>(n * n)), xn(n), lm(n), lp(n), w(n), iw(n);
    host_coefficients(N, dh.data(), xn.data(), lm.data(), lp.data(), w.data(), iw.data());
    std::vector<double> t(static_cast<size_t>(kSize), 0.0);
    for (int lane = 0; lane < 32; ++lane) {
        const int g = lane >> 2, tt = lane & 3;
        for (int s = 0; s < KS; ++s)
            for (int u = 0; u < NT; ++u) {
                const int i = 8 * u + g, k = 4 * s + tt;
                t[static_cast<size_t>((s * NT + u) * 32 + lane)] = (i < n && k < n) ? dh[static_cast<size_t>(i * n + k)] : 0.0;
            }
        for (int u = 0; u < NT; ++u)
            for (int h = 0; h < 2; ++h) {
                const int i = 8 * u + 2 * tt + h;
                t[static_cast<size_t>(kLPW + (u * 2 + h) * 32 + lane)] = i < n ? lp[static_cast<size_t>(i)] * iw[static_cast<size_t>(i)] : 0.0;
                t[static_cast<size_t>(kLMW + (u * 2 + h) * 32 + lane)] = i < n ? lm[static_cast<size_t>(i)] * iw[static_cast<size_t>(i)] : 0.0;
            }
        for (int s = 0; s < KS; ++s) {
            const int k = 4 * s + tt;
            t[static_cast<size_t>(kXK + s * 32 + lane)] = k < n ? xn[static_cast<size_t>(k)] : 0.0;
        }
    }
    return t;
}

namespace {
// TF32 rounding of the host (nearest, ties away from zero on the magnitude:
// cvt.rna.tf32.f32), as a float whose low 13 mantissa bits are zero.
float tf32_round(float x) {
    uint32_t b;
    std::memcpy(&b, &x, sizeof b);
    if ((b & 0x7f800000u) != 0x7f800000u) b = (b + 0x1000u) & 0xffffe000u;
    float r;
    std::memcpy(&r, &b, sizeof r);
    return r;
}
}  // namespace

std::vector<float> tc_lane_table_fp32(int N) {
    const int n = N + 1, KS = (n + 7) / 8, NT = (n + 7) / 8;
    const int kLPW = KS * NT * 128, kLMW = kLPW + NT * 64, kXK = kLMW + NT * 64, kSize = kXK + KS * 64;
    std::vector<double> dh(static_cast<size_t>(n * n)), xn(n), lm(n), lp(n), w(n), iw(n);
    host_coefficients(N, dh.data(), xn.data(), lm.data(), lp.data(), w.data(), iw.data());
    std::vector<float> t(static_cast<size_t>(kSize), 0.0f);
    for (int lane = 0; lane < 32; ++lane) {
        const int g = lane >> 2, tt = lane & 3;
        for (int s = 0; s < KS; ++s)
            for (int u = 0; u < NT; ++u)
                for (int r = 0; r < 2; ++r) {
                    const int i = 8 * u + g, k = 8 * s + tt + 4 * r;
                    const float v = (i < n && k < n) ? static_cast<float>(dh[static_cast<size_t>(i * n + k)]) : 0.0f;
                    const float hi = tf32_round(v), lo = tf32_round(v - hi);
                    t[static_cast<size_t>(((s * NT + u) * 32 + lane) * 4 + r)] = hi;
                    t[static_cast<size_t>(((s * NT + u) * 32 + lane) * 4 + 2 + r)] = lo;
                }
        for (int u = 0; u < NT; ++u)
            for (int h = 0; h < 2; ++h) {
                const int i = 8 * u + 2 * tt + h;
                t[static_cast<size_t>(kLPW + (u * 2 + h) * 32 + lane)] = i < n ? static_cast<float>(lp[static_cast<size_t>(i)] * iw[static_cast<size_t>(i)]) : 0.0f;
                t[static_cast<size_t>(kLMW + (u * 2 + h) * 32 + lane)] = i < n ? static_cast<float>(lm[static_cast<size_t>(i)] * iw[static_cast<size_t>(i)]) : 0.0f;
            }
        for (int s = 0; s < KS; ++s)
            for (int r = 0; r < 2; ++r) {
                const int k = 8 * s + tt + 4 * r;
                t[static_cast<size_t>(kXK + (s * 32 + lane) * 2 + r)] = k < n ? static_cast<float>(xn[static_cast<size_t>(k)]) : 0.0f;
            }
    }
    return t;
}

// ---------------------------------------------------------------------------
// Host launchers.

template <int N, bool S>
static cudaError_t launch_stage_t(const StageArgs& a, cudaStream_t stream) {
    using T = Tile<N>;
    const dim3 grid(static_cast<unsigned>((a.n_elements + T::EPB - 1) / T::EPB), static_cast<unsigned>(a.n_instances));
    stage_kernel<N, S, 0><<<grid, T::kThreads, T::kBytes, stream>>>(a, make_coeffs<N>());
    return cudaGetLastError();
}

template <int N, bool S>
static cudaError_t launch_trace_t(const TraceArgs& a, cudaStream_t stream) {
    const int64_t total = static_cast<int64_t>(a.n_instances) * 3 * a.n_elements * 4 * (N + 1);
    const int blocks = static_cast<int>(std::min<int64_t>((total + 255) / 256, 148 * 32));
    trace_kernel<N, S><<<blocks, 256, 0, stream>>>(a);
    return cudaGetLastError();
}

// Opts the stage kernel of one order into more than 48 KB of dynamic shared
// memory on the current device. Called once per device and order, before
// any launch or stream capture.
template <int N, bool S>
static cudaError_t prepare_t() {
    return cudaFuncSetAttribute(stage_kernel<N, S, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(Tile<N>::kBytes));
}

template <int N, bool S>
static int epb_t() {
    return Tile<N>::EPB;
}

#define NDG_DISPATCH_ORDER(FN, N_, STRICT_, ...)                                          \
    switch (N_) {                                                                         \
        case 1: return STRICT_ ? FN<1, true>(__VA_ARGS__) : FN<1, false>(__VA_ARGS__);    \
        case 2: return STRICT_ ? FN<2, true>(__VA_ARGS__) : FN<2, false>(__VA_ARGS__);    \
        case 3: return STRICT_ ? FN<3, true>(__VA_ARGS__) : FN<3, false>(__VA_ARGS__);    \
        case 4: return STRICT_ ? FN<4, true>(__VA_ARGS__) : FN<4, false>(__VA_ARGS__);    \
        case 5: return STRICT_ ? FN<5, true>(__VA_ARGS__) : FN<5, false>(__VA_ARGS__);    \
        case 6: return STRICT_ ? FN<6, true>(__VA_ARGS__) : FN<6, false>(__VA_ARGS__);    \
        case 7: return STRICT_ ? FN<7, true>(__VA_ARGS__) : FN<7, false>(__VA_ARGS__);    \
        case 8: return STRICT_ ? FN<8, true>(__VA_ARGS__) : FN<8, false>(__VA_ARGS__);    \
        case 9: return STRICT_ ? FN<9, true>(__VA_ARGS__) : FN<9, false>(__VA_ARGS__);    \
        case 10: return STRICT_ ? FN<10, true>(__VA_ARGS__) : FN<10, false>(__VA_ARGS__); \
        case 11: return STRICT_ ? FN<11, true>(__VA_ARGS__) : FN<11, false>(__VA_ARGS__); \
        case 12: return STRICT_ ? FN<12, true>(__VA_ARGS__) : FN<12, false>(__VA_ARGS__); \
        case 13: return STRICT_ ? FN<13, true>(__VA_ARGS__) : FN<13, false>(__VA_ARGS__); \
        case 14: return STRICT_ ? FN<14, true>(__VA_ARGS__) : FN<14, false>(__VA_ARGS__); \
        case 15: return STRICT_ ? FN<15, true>(__VA_ARGS__) : FN<15, false>(__VA_ARGS__); \
        case 16: return STRICT_ ? FN<16, true>(__VA_ARGS__) : FN<16, false>(__VA_ARGS__); \
        default: break;                                                                   \
    }

template <int N>
static CoeffsF<N> make_coeffs_f() {
    const Coeffs<N> d = make_coeffs<N>();
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

template <int N, bool Unused>
static cudaError_t prepare_f32_t() {
    return cudaFuncSetAttribute(stage_kernel_f32<N, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(TileF<N, 0>::kBytes));
}

template <int N, bool Unused>
static cudaError_t launch_stage_f32_t(const StageArgs& a, cudaStream_t stream) {
    using T = TileF<N, 0>;
    const dim3 grid(static_cast<unsigned>((a.n_elements + T::EPB - 1) / T::EPB), static_cast<unsigned>(a.n_instances));
    stage_kernel_f32<N, 0><<<grid, T::kThreads, T::kBytes, stream>>>(a, make_coeffs_f<N>());
    return cudaGetLastError();
}

template <int N, bool Unused>
static cudaError_t launch_trace_f32_t(const TraceArgs& a, cudaStream_t stream) {
    const int64_t total = static_cast<int64_t>(a.n_instances) * 3 * a.n_elements * 4 * (N + 1);
    const int blocks = static_cast<int>(std::min<int64_t>((total + 255) / 256, 148 * 32));
    trace_kernel_f32<N><<<blocks, 256, 0, stream>>>(a);
    return cudaGetLastError();
}

cudaError_t prepare_kernels(int N, bool strict) {
    NDG_DISPATCH_ORDER(prepare_t, N, strict)
    return cudaErrorInvalidValue;
}

cudaError_t launch_stage(int N, bool strict, const StageArgs& a, cudaStream_t stream) {
    NDG_DISPATCH_ORDER(launch_stage_t, N, strict, a, stream)
    return cudaErrorInvalidValue;
}

cudaError_t launch_traces(int N, bool strict, const TraceArgs& a, cudaStream_t stream) {
    NDG_DISPATCH_ORDER(launch_trace_t, N, strict, a, stream)
    return cudaErrorInvalidValue;
}

cudaError_t prepare_kernels_f32(int N) {
    NDG_DISPATCH_ORDER(prepare_f32_t, N, false)
    return cudaErrorInvalidValue;
}

cudaError_t launch_stage_f32(int N, const StageArgs& a, cudaStream_t stream) {
    NDG_DISPATCH_ORDER(launch_stage_f32_t, N, false, a, stream)
    return cudaErrorInvalidValue;
}

cudaError_t launch_traces_f32(int N, const TraceArgs& a, cudaStream_t stream) {
    NDG_DISPATCH_ORDER(launch_trace_f32_t, N, false, a, stream)
    return cudaErrorInvalidValue;
}

int elements_per_block(int N) {
    NDG_DISPATCH_ORDER(epb_t, N, false)
    return 0;
}

cudaError_t launch_initial_conditions(double* q, double* k, const double* corners, int N, int64_t K, int64_t Kp, int n_instances, cudaStream_t stream) {
    const int64_t total = K * (N + 1) * (N + 1);
    const int blocks = static_cast<int>(std::min<int64_t>((total + 255) / 256, 148 * 16));
    initial_condition_kernel<<<blocks, 256, 0, stream>>>(q, k, corners, N, K, Kp, n_instances);
    return cudaGetLastError();
}

cudaError_t launch_delta_t(const double* delta_xy_min, const int* elem_N, int64_t K, double cfl, double* out, cudaStream_t stream) {
    delta_t_kernel<<<1, 1024, 0, stream>>>(delta_xy_min, elem_N, K, cfl, out);
    return cudaGetLastError();
}

cudaError_t launch_end_step(double* step, cudaStream_t stream) {
    end_step_kernel<<<1, 1, 0, stream>>>(step);
    return cudaGetLastError();
}

cudaError_t upload_tables(const Tables& t) {
    if (t.N_max < 1) return cudaSuccess;
    std::vector<double> nodes(kVecTotal, 0.0), weights(kVecTotal, 0.0), inv_w(kVecTotal, 0.0), ll(kVecTotal, 0.0), lr(kVecTotal, 0.0);
    std::vector<double> dhat(kMatTotal, 0.0);
    for (int N = 0; N <= std::min(t.N_max, kMaxOrder); ++N) {
        const int n = N + 1;
        for (int i = 0; i < n; ++i) {
            const size_t at = static_cast<size_t>(vec_offset(N) + i);
            nodes[at] = t.get(NDG_TABLE_NODES, N)[static_cast<size_t>(i)];
            weights[at] = t.get(NDG_TABLE_WEIGHTS, N)[static_cast<size_t>(i)];
            inv_w[at] = 1.0 / t.get(NDG_TABLE_WEIGHTS, N)[static_cast<size_t>(i)];
            ll[at] = t.get(NDG_TABLE_LAGRANGE_LEFT, N)[static_cast<size_t>(i)];
            lr[at] = t.get(NDG_TABLE_LAGRANGE_RIGHT, N)[static_cast<size_t>(i)];
        }
        for (int i = 0; i < n * n; ++i) dhat[static_cast<size_t>(mat_offset(N) + i)] = t.get(NDG_TABLE_DERIVATIVE_MATRICES_HAT, N)[static_cast<size_t>(i)];
    }
    h_nodes = nodes;
    h_weights = weights;
    h_inv_weights = inv_w;
    h_ll = ll;
    h_lr = lr;
    h_dhat = dhat;
    cudaError_t err;
    if ((err = cudaMemcpyToSymbol(c_nodes, nodes.data(), sizeof(double) * kVecTotal)) != cudaSuccess) return err;
    if ((err = cudaMemcpyToSymbol(c_weights, weights.data(), sizeof(double) * kVecTotal)) != cudaSuccess) return err;
    if ((err = cudaMemcpyToSymbol(c_inv_weights, inv_w.data(), sizeof(double) * kVecTotal)) != cudaSuccess) return err;
    if ((err = cudaMemcpyToSymbol(c_lagrange_left, ll.data(), sizeof(double) * kVecTotal)) != cudaSuccess) return err;
    if ((err = cudaMemcpyToSymbol(c_lagrange_right, lr.data(), sizeof(double) * kVecTotal)) != cudaSuccess) return err;
    return cudaMemcpyToSymbol(c_dhat, dhat.data(), sizeof(double) * kMatTotal);
}

}  // namespace dev
}  // namespace ndg
