// Fused DG stage kernels for sm_100a (B200), uniform order N, conforming faces.
//
// One launch performs one low-storage RK3 stage for every element of every
// instance: the reference's seven stage calls (interpolate_to_boundaries,
// boundary_conditions, project_to_faces, calculate_wave_fluxes,
// project_to_elements, compute_dg_wave_derivative, rk3_step;
// include/solvers/Solver2D_t.tcu:46-70) become the phases of one CTA that
// holds a tile of EPB elements in shared memory:
//
//   P1  stream q = (p, u, v) of the tile into shared memory (coalesced);
//       build the per-element metric vectors from the four corners
//   P2  per element side node: own trace (l(+-1) . q line), the far-side
//       trace (neighbour's stored trace or a boundary rule), upwind flux,
//       times the side's edge metric -> element side flux
//   P3  xi lines:  Dhat . (y_eta F - x_eta G) + lift           -> G
//   P4  eta lines: Dhat . (-y_xi F + x_xi G) + lift, then /J   -> G
//   P5  k = a k + G, q += g dt k (FP64), streamed back to HBM
//   P6  side traces of the new q -> trace buffer for the next stage
//
// HBM traffic per element and stage: q and k read and written (the
// algorithmic 32 B per degree of freedom) plus one trace write and one
// neighbour-trace read of 4(N+1) values per field. Geometry is 8 corner
// coordinates per element; metrics, Jacobians and edge metrics are
// recomputed in registers, because on straight-sided quads x_xi, y_xi depend
// only on eta and x_eta, y_eta only on xi (quad_metrics,
// include/functions/quad_metrics.tpp:2-7).
//
// STRICT instantiations round every operation in the reference's order
// (__dmul_rn/__dadd_rn, true divisions) and reproduce its CPU results bit
// for bit; the default instantiations contract to FMAs and multiply by
// reciprocal weights.
#include "ndg_internal.hpp"
#include "stage_kernels.cuh"

#include <cuda_runtime.h>

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

// ---------------------------------------------------------------------------
// Arithmetic with selectable rounding.
template <bool S> __device__ __forceinline__ double mul(double a, double b) { return S ? __dmul_rn(a, b) : a * b; }
template <bool S> __device__ __forceinline__ double add(double a, double b) { return S ? __dadd_rn(a, b) : a + b; }
template <bool S> __device__ __forceinline__ double sub(double a, double b) { return S ? __dsub_rn(a, b) : a - b; }
// s + a*b: two roundings in strict mode, one FMA otherwise.
template <bool S> __device__ __forceinline__ double madd(double s, double a, double b) { return S ? __dadd_rn(s, __dmul_rn(a, b)) : fma(a, b, s); }

template <int N>
struct Tile {
    static constexpr int n = N + 1;
    static constexpr int NN = n * n;
    static constexpr int kThreads = 256;
    static constexpr int EPB = (kThreads / (3 * n)) > 0 ? (kThreads / (3 * n)) : 1;
    // shared memory layout, in doubles
    static constexpr int kQ = 0;                        // [3][EPB][NN]
    static constexpr int kG = kQ + 3 * EPB * NN;        // [3][EPB][NN]
    static constexpr int kF = kG + 3 * EPB * NN;        // [3][EPB][4][n] element side fluxes
    static constexpr int kM = kF + 3 * EPB * 4 * n;     // [EPB][4][n] x_xi(eta), y_xi(eta), x_eta(xi), y_eta(xi)
    static constexpr int kS = kM + EPB * 4 * n;         // [EPB][4] edge metric per side
    static constexpr int kDoubles = kS + EPB * 4;
    static constexpr size_t kBytes = sizeof(double) * kDoubles;
};

// Side trace of one field: value m of side s (reference order: bottom and
// right run with the element axes, top and left reversed;
// src/entities/Element2D_t.cpp:86-125).
template <int N, bool S>
__device__ __forceinline__ double side_trace(const double* __restrict__ q, int s, int m) {
    constexpr int n = N + 1;
    const double* lm = c_lagrange_left + vec_offset(N);
    const double* lp = c_lagrange_right + vec_offset(N);
    const int line = (s < 2) ? m : N - m;
    double acc = 0.0;
    if (s == 0) {
#pragma unroll
        for (int j = 0; j < n; ++j) acc = madd<S>(acc, lm[j], q[line * n + j]);
    } else if (s == 2) {
#pragma unroll
        for (int j = 0; j < n; ++j) acc = madd<S>(acc, lp[j], q[line * n + j]);
    } else if (s == 1) {
#pragma unroll
        for (int j = 0; j < n; ++j) acc = madd<S>(acc, lp[j], q[j * n + line]);
    } else {
#pragma unroll
        for (int j = 0; j < n; ++j) acc = madd<S>(acc, lm[j], q[j * n + line]);
    }
    return acc;
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

template <int N, bool S>
__global__ void __launch_bounds__(256) stage_kernel(StageArgs a) {
    using T = Tile<N>;
    constexpr int n = T::n, NN = T::NN, EPB = T::EPB;
    extern __shared__ double smem[];
    double* qs = smem + T::kQ;
    double* gs = smem + T::kG;
    double* fs = smem + T::kF;
    double* ms = smem + T::kM;
    double* ss = smem + T::kS;

    const int tid = threadIdx.x;
    const int64_t K = a.n_elements;
    const int64_t e0 = static_cast<int64_t>(blockIdx.x) * EPB;
    const int ne = static_cast<int>((K - e0) < EPB ? (K - e0) : EPB);
    const int64_t inst = blockIdx.y;
    double* q = a.q + inst * 3 * K * NN;
    double* k = a.k + inst * 3 * K * NN;
    const double* tr_in = a.trace_in + inst * 3 * K * 4 * n;
    double* tr_out = a.trace_out + inst * 3 * K * 4 * n;
    const double* xn = c_nodes + vec_offset(N);
    const double time = a.step[0];
    const double dt = a.step[1];

    // P1: q tile and metric vectors.
    const int tile_vals = ne * NN;
    for (int idx = tid; idx < 3 * tile_vals; idx += T::kThreads) {
        const int f = idx / tile_vals;
        const int r = idx - f * tile_vals;
        qs[f * EPB * NN + r] = q[(f * K + e0) * NN + r];
    }
    for (int idx = tid; idx < ne * n; idx += T::kThreads) {
        const int e = idx / n, i = idx - e * n;
        const double* c = a.corners + 8 * (e0 + e);
        const double x0 = c[0], y0 = c[1], x1 = c[2], y1 = c[3], x2 = c[4], y2 = c[5], x3 = c[6], y3 = c[7];
        const double t = xn[i];
        const double lo = sub<S>(1.0, t), hi = add<S>(1.0, t);
        double* m = ms + e * 4 * n;
        m[0 * n + i] = mul<S>(add<S>(mul<S>(lo, sub<S>(x1, x0)), mul<S>(hi, sub<S>(x2, x3))), 0.25);  // x_xi at eta = t
        m[1 * n + i] = mul<S>(add<S>(mul<S>(lo, sub<S>(y1, y0)), mul<S>(hi, sub<S>(y2, y3))), 0.25);  // y_xi at eta = t
        m[2 * n + i] = mul<S>(add<S>(mul<S>(lo, sub<S>(x3, x0)), mul<S>(hi, sub<S>(x2, x1))), 0.25);  // x_eta at xi = t
        m[3 * n + i] = mul<S>(add<S>(mul<S>(lo, sub<S>(y3, y0)), mul<S>(hi, sub<S>(y2, y1))), 0.25);  // y_eta at xi = t
    }
    for (int idx = tid; idx < ne * 4; idx += T::kThreads) {
        // Edge metric of side s, constant along a straight side
        // (Element2D_t.cpp:756-769): |d(x,y)/dxi| at eta = -1, +1 for sides
        // 0, 2 and |d(x,y)/deta| at xi = +1, -1 for sides 1, 3.
        const int e = idx >> 2, sd = idx & 3;
        const double* c = a.corners + 8 * (e0 + e);
        const double x0 = c[0], y0 = c[1], x1 = c[2], y1 = c[3], x2 = c[4], y2 = c[5], x3 = c[6], y3 = c[7];
        const double at = (sd == 0 || sd == 3) ? -1.0 : 1.0;
        const double l2 = sub<S>(1.0, at), h2 = add<S>(1.0, at);
        double dx, dy;
        if (sd == 0 || sd == 2) {
            dx = mul<S>(add<S>(mul<S>(l2, sub<S>(x1, x0)), mul<S>(h2, sub<S>(x2, x3))), 0.25);
            dy = mul<S>(add<S>(mul<S>(l2, sub<S>(y1, y0)), mul<S>(h2, sub<S>(y2, y3))), 0.25);
        } else {
            dx = mul<S>(add<S>(mul<S>(l2, sub<S>(x3, x0)), mul<S>(h2, sub<S>(x2, x1))), 0.25);
            dy = mul<S>(add<S>(mul<S>(l2, sub<S>(y3, y0)), mul<S>(h2, sub<S>(y2, y1))), 0.25);
        }
        ss[idx] = sqrt(add<S>(mul<S>(dx, dx), mul<S>(dy, dy)));
    }
    __syncthreads();

    // P2: element side fluxes.
    for (int idx = tid; idx < ne * 4 * n; idx += T::kThreads) {
        const int e = idx / (4 * n);
        const int s = (idx / n) & 3;
        const int m = idx - (idx / n) * n;
        const int64_t ge = e0 + e;
        double own[3], far[3];
#pragma unroll
        for (int f = 0; f < 3; ++f) own[f] = side_trace<N, S>(qs + (f * EPB + e) * NN, s, m);
        const int2 link = a.link[4 * ge + s];
        const double2 nrm = a.normal[4 * ge + s];
        const int kind = (link.y >> 2) & 7;
        const int role = (link.y >> 5) & 1;
        if (kind == kInterior) {
            const int nb_side = link.y & 3;
#pragma unroll
            for (int f = 0; f < 3; ++f) far[f] = tr_in[((f * K + link.x) * 4 + nb_side) * n + (N - m)];
        } else if (kind == kMirror || kind == kCopy) {
            // Ghost trace: the element's own trace reversed and scaled by the
            // ghost's edge metric; walls and symmetry planes then mirror the
            // normal velocity (Mesh2D_t.cpp:4366-4434, 4601-4710).
            const double gsc = a.gscale[4 * ge + s];
            far[0] = mul<S>(own[0], gsc);
            const double gu = mul<S>(own[1], gsc), gv = mul<S>(own[2], gsc);
            if (kind == kMirror) {
                const double tx = -nrm.y, ty = nrm.x;
                const double l0 = -add<S>(mul<S>(gu, nrm.x), mul<S>(gv, nrm.y));
                const double l1 = add<S>(mul<S>(gu, tx), mul<S>(gv, ty));
                far[1] = add<S>(mul<S>(nrm.x, l0), mul<S>(tx, l1));
                far[2] = add<S>(mul<S>(nrm.y, l0), mul<S>(ty, l1));
            } else {
                far[1] = gu;
                far[2] = gv;
            }
        } else if (kind == kAnalytic) {
            // Inflow: the analytic wave on the ghost edge at the stage time
            // (Mesh2D_t.cpp:4575-4599); the face reads ghost node N - m.
            const double4 g = a.inflow[4 * ge + s];
            const double r = mul<S>(add<S>(xn[N - m], 1.0), 0.5);
            const double gx = add<S>(mul<S>(g.z, r), mul<S>(g.x, sub<S>(1.0, r)));
            const double gy = add<S>(mul<S>(g.w, r), mul<S>(g.y, sub<S>(1.0, r)));
            plane_wave(gx, gy, add<S>(time, mul<S>(a.rk_b, dt)), far[0], far[1], far[2]);
        } else {
            far[0] = far[1] = far[2] = 0.0;
        }
        // Upwind flux of the face (Solver2D_t.cpp:48-63) with the face's own
        // left/right order, then the element's view of it
        // (Mesh2D_t.cpp:3895-3929): scaled by the edge metric, and negated
        // for the face's right element.
        const double Lp = role ? far[0] : own[0], Lu = role ? far[1] : own[1], Lv = role ? far[2] : own[2];
        const double Rp = role ? own[0] : far[0], Ru = role ? own[1] : far[1], Rv = role ? own[2] : far[2];
        const double wL = add<S>(Lp, add<S>(mul<S>(Lu, nrm.x), mul<S>(Lv, nrm.y)));
        const double wR = sub<S>(Rp, add<S>(mul<S>(Ru, nrm.x), mul<S>(Rv, nrm.y)));
        const double fp = mul<S>(sub<S>(wL, wR), 0.5);
        const double sum = add<S>(wL, wR);
        const double fu = mul<S>(mul<S>(nrm.x, sum), 0.5);
        const double fv = mul<S>(mul<S>(nrm.y, sum), 0.5);
        const double sf = ss[e * 4 + s];
        fs[((0 * EPB + e) * 4 + s) * n + m] = mul<S>(role ? -fp : fp, sf);
        fs[((1 * EPB + e) * 4 + s) * n + m] = mul<S>(role ? -fu : fu, sf);
        fs[((2 * EPB + e) * 4 + s) * n + m] = mul<S>(role ? -fv : fv, sf);
    }
    __syncthreads();

    const double* Dh = c_dhat + mat_offset(N);
    const double* lm = c_lagrange_left + vec_offset(N);
    const double* lp = c_lagrange_right + vec_offset(N);
    const double* w = c_weights + vec_offset(N);
    const double* iw = c_inv_weights + vec_offset(N);

    // P3: xi lines (fixed eta index j), Solver2D_t.cpp:71-101.
    for (int idx = tid; idx < 3 * ne * n; idx += T::kThreads) {
        const int f = idx / (ne * n);
        const int r = idx - f * ne * n;
        const int e = r / n, j = r - (r / n) * n;
        const double* P = qs + (0 * EPB + e) * NN;
        const double* U = qs + (1 * EPB + e) * NN;
        const double* V = qs + (2 * EPB + e) * NN;
        const double* m = ms + e * 4 * n;
        double fl[n];
#pragma unroll
        for (int i = 0; i < n; ++i) {
            const double x_eta = m[2 * n + i], y_eta = m[3 * n + i];
            if (f == 0) fl[i] = sub<S>(mul<S>(y_eta, U[i * n + j]), mul<S>(x_eta, V[i * n + j]));
            else if (f == 1) fl[i] = mul<S>(y_eta, P[i * n + j]);
            else fl[i] = -mul<S>(x_eta, P[i * n + j]);
        }
        const double fr = fs[((f * EPB + e) * 4 + 1) * n + j];
        const double fl3 = fs[((f * EPB + e) * 4 + 3) * n + (N - j)];
        double* G = gs + (f * EPB + e) * NN;
#pragma unroll
        for (int i = 0; i < n; ++i) {
            double acc = 0.0;
#pragma unroll
            for (int mm = 0; mm < n; ++mm) acc = madd<S>(acc, Dh[i * n + mm], fl[mm]);
            const double lift = S ? __ddiv_rn(add<S>(mul<S>(fr, lp[i]), mul<S>(fl3, lm[i])), w[i])
                                  : (fr * lp[i] + fl3 * lm[i]) * iw[i];
            G[i * n + j] = -add<S>(acc, lift);
        }
    }
    __syncthreads();

    // P4: eta lines (fixed xi index i), Solver2D_t.cpp:103-134, then /J.
    for (int idx = tid; idx < 3 * ne * n; idx += T::kThreads) {
        const int f = idx / (ne * n);
        const int r = idx - f * ne * n;
        const int e = r / n, i = r - (r / n) * n;
        const double* P = qs + (0 * EPB + e) * NN + i * n;
        const double* U = qs + (1 * EPB + e) * NN + i * n;
        const double* V = qs + (2 * EPB + e) * NN + i * n;
        const double* m = ms + e * 4 * n;
        double fl[n];
#pragma unroll
        for (int j = 0; j < n; ++j) {
            const double x_xi = m[0 * n + j], y_xi = m[1 * n + j];
            if (f == 0) fl[j] = add<S>(mul<S>(-y_xi, U[j]), mul<S>(x_xi, V[j]));
            else if (f == 1) fl[j] = mul<S>(-y_xi, P[j]);
            else fl[j] = mul<S>(x_xi, P[j]);
        }
        const double ft = fs[((f * EPB + e) * 4 + 2) * n + (N - i)];
        const double fb = fs[((f * EPB + e) * 4 + 0) * n + i];
        const double x_eta = m[2 * n + i], y_eta = m[3 * n + i];
        double* G = gs + (f * EPB + e) * NN + i * n;
#pragma unroll
        for (int j = 0; j < n; ++j) {
            double acc = 0.0;
#pragma unroll
            for (int mm = 0; mm < n; ++mm) acc = madd<S>(acc, Dh[j * n + mm], fl[mm]);
            const double lift = S ? __ddiv_rn(add<S>(mul<S>(ft, lp[j]), mul<S>(fb, lm[j])), w[j])
                                  : (ft * lp[j] + fb * lm[j]) * iw[j];
            const double jac = sub<S>(mul<S>(m[0 * n + j], y_eta), mul<S>(x_eta, m[1 * n + j]));
            const double num = sub<S>(G[j], add<S>(acc, lift));
            G[j] = S ? __ddiv_rn(num, jac) : num * __drcp_rn(jac);
        }
    }
    __syncthreads();

    // P5: low-storage RK3 update (Solver2D_t.cpp:138-172), FP64.
    const double gdt = mul<S>(a.rk_g, dt);
    for (int idx = tid; idx < 3 * tile_vals; idx += T::kThreads) {
        const int f = idx / tile_vals;
        const int r = idx - f * tile_vals;
        const int64_t gi = (f * K + e0) * NN + r;
        const double G = gs[f * EPB * NN + r];
        const double kn = a.first ? G : add<S>(mul<S>(a.rk_a, k[gi]), G);
        const double qn = add<S>(qs[f * EPB * NN + r], mul<S>(gdt, kn));
        k[gi] = kn;
        q[gi] = qn;
        qs[f * EPB * NN + r] = qn;
        if (a.G_out) a.G_out[inst * 3 * K * NN + gi] = G;
    }
    __syncthreads();

    // P6: side traces of the new solution for the next stage.
    for (int idx = tid; idx < ne * 4 * n; idx += T::kThreads) {
        const int e = idx / (4 * n);
        const int s = (idx / n) & 3;
        const int m = idx - (idx / n) * n;
#pragma unroll
        for (int f = 0; f < 3; ++f) tr_out[((f * K + e0 + e) * 4 + s) * n + m] = side_trace<N, S>(qs + (f * EPB + e) * NN, s, m);
    }
}

// Side traces only (start of a run, or after the host changed q).
template <int N, bool S>
__global__ void __launch_bounds__(256) trace_kernel(TraceArgs a) {
    using T = Tile<N>;
    constexpr int n = T::n, NN = T::NN, EPB = T::EPB;
    extern __shared__ double smem[];
    const int64_t K = a.n_elements;
    const int64_t e0 = static_cast<int64_t>(blockIdx.x) * EPB;
    const int ne = static_cast<int>((K - e0) < EPB ? (K - e0) : EPB);
    const int64_t inst = blockIdx.y;
    const double* q = a.q + inst * 3 * K * NN;
    double* tr_out = a.trace_out + inst * 3 * K * 4 * n;
    const int tile_vals = ne * NN;
    for (int idx = threadIdx.x; idx < 3 * tile_vals; idx += T::kThreads) {
        const int f = idx / tile_vals;
        const int r = idx - f * tile_vals;
        smem[f * EPB * NN + r] = q[(f * K + e0) * NN + r];
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < ne * 4 * n; idx += T::kThreads) {
        const int e = idx / (4 * n);
        const int s = (idx / n) & 3;
        const int m = idx - (idx / n) * n;
#pragma unroll
        for (int f = 0; f < 3; ++f) tr_out[((f * K + e0 + e) * 4 + s) * n + m] = side_trace<N, S>(smem + (f * EPB + e) * NN, s, m);
    }
}

// Reference plane-wave initial condition (Mesh2D_t.cpp:1192-1216) on every
// node of every instance, bilinear map of include/functions/quad_map.tpp:2-7.
__global__ void initial_condition_kernel(double* q, double* k, const double* corners, int N, int64_t K, int n_instances) {
    const int n = N + 1, NN = n * n;
    const int64_t total = K * NN;
    const double* xn = c_nodes + vec_offset(N);
    for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < total; idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t e = idx / NN;
        const int node = static_cast<int>(idx - e * NN);
        const int i = node / n, j = node - (node / n) * n;
        const double* c = corners + 8 * e;
        const double xi = xn[i], eta = xn[j];
        const double gx = __dmul_rn(__dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(__dmul_rn(c[0], __dsub_rn(1.0, xi)), __dsub_rn(1.0, eta)),
                                                                  __dmul_rn(__dmul_rn(c[2], __dadd_rn(xi, 1.0)), __dsub_rn(1.0, eta))),
                                                        __dmul_rn(__dmul_rn(c[4], __dadd_rn(xi, 1.0)), __dadd_rn(eta, 1.0))),
                                              __dmul_rn(__dmul_rn(c[6], __dsub_rn(1.0, xi)), __dadd_rn(eta, 1.0))),
                                    0.25);
        const double gy = __dmul_rn(__dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(__dmul_rn(c[1], __dsub_rn(1.0, xi)), __dsub_rn(1.0, eta)),
                                                                  __dmul_rn(__dmul_rn(c[3], __dadd_rn(xi, 1.0)), __dsub_rn(1.0, eta))),
                                                        __dmul_rn(__dmul_rn(c[5], __dadd_rn(xi, 1.0)), __dadd_rn(eta, 1.0))),
                                              __dmul_rn(__dmul_rn(c[7], __dsub_rn(1.0, xi)), __dadd_rn(eta, 1.0))),
                                    0.25);
        double p, u, v;
        plane_wave(gx, gy, 0.0, p, u, v);
        for (int inst = 0; inst < n_instances; ++inst) {
            double* qi = q + static_cast<int64_t>(inst) * 3 * total;
            double* ki = k + static_cast<int64_t>(inst) * 3 * total;
            qi[idx] = p;
            qi[total + idx] = u;
            qi[2 * total + idx] = v;
            ki[idx] = 0.0;
            ki[total + idx] = 0.0;
            ki[2 * total + idx] = 0.0;
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

// Step bookkeeping of the reference's time loop (Solver2D_t.tcu:37-42, 72):
// step = {time, dt, dt_mesh, t_end}.
__global__ void begin_step_kernel(double* step) {
    const double time = step[0], dt_mesh = step[2], t_end = step[3];
    step[1] = (time + dt_mesh > t_end) ? t_end - time : dt_mesh;
}
__global__ void end_step_kernel(double* step) {
    const double time = step[0] + step[1];
    step[0] = time;
    step[1] = (time + step[2] > step[3]) ? step[3] - time : step[2];
}

// ---------------------------------------------------------------------------
// Host launchers.

template <int N, bool S>
static cudaError_t launch_stage_t(const StageArgs& a, cudaStream_t stream) {
    using T = Tile<N>;
    const dim3 grid(static_cast<unsigned>((a.n_elements + T::EPB - 1) / T::EPB), static_cast<unsigned>(a.n_instances));
    stage_kernel<N, S><<<grid, T::kThreads, T::kBytes, stream>>>(a);
    return cudaGetLastError();
}

template <int N, bool S>
static cudaError_t launch_trace_t(const TraceArgs& a, cudaStream_t stream) {
    using T = Tile<N>;
    const size_t bytes = sizeof(double) * 3 * T::EPB * T::NN;
    const dim3 grid(static_cast<unsigned>((a.n_elements + T::EPB - 1) / T::EPB), static_cast<unsigned>(a.n_instances));
    trace_kernel<N, S><<<grid, T::kThreads, bytes, stream>>>(a);
    return cudaGetLastError();
}

// Opts the kernels of one order into more than 48 KB of dynamic shared memory
// on the current device. Called once per device and order, before any launch
// or stream capture.
template <int N, bool S>
static cudaError_t prepare_t() {
    using T = Tile<N>;
    cudaError_t err = cudaFuncSetAttribute(stage_kernel<N, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(T::kBytes));
    if (err != cudaSuccess) return err;
    return cudaFuncSetAttribute(trace_kernel<N, S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(sizeof(double) * 3 * T::EPB * T::NN));
}

#define NDG_DISPATCH_ORDER(FN, N_, STRICT_, ...)                  \
    switch (N_) {                                                 \
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
        default: return cudaErrorInvalidValue;                    \
    }

cudaError_t prepare_kernels(int N, bool strict) {
    NDG_DISPATCH_ORDER(prepare_t, N, strict)
}

cudaError_t launch_stage(int N, bool strict, const StageArgs& a, cudaStream_t stream) {
    NDG_DISPATCH_ORDER(launch_stage_t, N, strict, a, stream)
}

cudaError_t launch_traces(int N, bool strict, const TraceArgs& a, cudaStream_t stream) {
    NDG_DISPATCH_ORDER(launch_trace_t, N, strict, a, stream)
}

int elements_per_block(int N) {
    const int n = N + 1;
    return (256 / (3 * n)) > 0 ? 256 / (3 * n) : 1;
}

cudaError_t launch_initial_conditions(double* q, double* k, const double* corners, int N, int64_t K, int n_instances, cudaStream_t stream) {
    const int64_t total = K * (N + 1) * (N + 1);
    const int blocks = static_cast<int>(std::min<int64_t>((total + 255) / 256, 148 * 16));
    initial_condition_kernel<<<blocks, 256, 0, stream>>>(q, k, corners, N, K, n_instances);
    return cudaGetLastError();
}

cudaError_t launch_delta_t(const double* delta_xy_min, const int* elem_N, int64_t K, double cfl, double* out, cudaStream_t stream) {
    delta_t_kernel<<<1, 1024, 0, stream>>>(delta_xy_min, elem_N, K, cfl, out);
    return cudaGetLastError();
}

cudaError_t launch_begin_step(double* step, cudaStream_t stream) {
    begin_step_kernel<<<1, 1, 0, stream>>>(step);
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
            nodes[static_cast<size_t>(vec_offset(N) + i)] = t.get(NDG_TABLE_NODES, N)[static_cast<size_t>(i)];
            weights[static_cast<size_t>(vec_offset(N) + i)] = t.get(NDG_TABLE_WEIGHTS, N)[static_cast<size_t>(i)];
            inv_w[static_cast<size_t>(vec_offset(N) + i)] = 1.0 / t.get(NDG_TABLE_WEIGHTS, N)[static_cast<size_t>(i)];
            ll[static_cast<size_t>(vec_offset(N) + i)] = t.get(NDG_TABLE_LAGRANGE_LEFT, N)[static_cast<size_t>(i)];
            lr[static_cast<size_t>(vec_offset(N) + i)] = t.get(NDG_TABLE_LAGRANGE_RIGHT, N)[static_cast<size_t>(i)];
        }
        for (int i = 0; i < n * n; ++i) dhat[static_cast<size_t>(mat_offset(N) + i)] = t.get(NDG_TABLE_DERIVATIVE_MATRICES_HAT, N)[static_cast<size_t>(i)];
    }
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
