// Fused DG stage kernels for sm_100a (B200), uniform order N, conforming faces.
//
// One launch performs one low-storage RK3 stage for every element of every
// instance: the reference's seven stage calls (interpolate_to_boundaries,
// boundary_conditions, project_to_faces, calculate_wave_fluxes,
// project_to_elements, compute_dg_wave_derivative, rk3_step;
// include/solvers/Solver2D_t.tcu:46-70) become the passes of one CTA that
// owns a tile of EPB consecutive elements:
//
//   prologue  one thread starts a TMA bulk copy (cp.async.bulk + mbarrier)
//             of the tile's q = (p, u, v) into shared memory; meanwhile all
//             threads prefetch the far-side traces of their side nodes (the
//             neighbours' traces of the previous stage) and build J and edge
//             metrics from the four corners
//   rows      bottom/top own traces
//   columns   xi-direction flux lines (kept in registers), right/left own traces
//   flux      upwind flux of every side node, times the edge metric
//   xi pass   Dhat . line + lift                       -> G (columns)
//   eta pass  eta-direction flux lines, Dhat . line + lift, then /J -> G (rows)
//   RK        k = a k + G, q += g dt k in FP64, node by node, coalesced
//   traces    four side traces of the new q for the next stage
//
// Work is spread as one thread per (field, element, line), 3 EPB (N+1)
// threads per CTA; shared memory carries only the q tile, G, J and the side
// data. HBM traffic per
// element and stage: q and k read and written (the algorithmic 32 B per
// degree of freedom), one trace write and one neighbour-trace read of 4(N+1)
// values per field, and 8 corner coordinates. Metrics are recomputed in
// registers: on straight-sided quads x_xi, y_xi depend only on eta and
// x_eta, y_eta only on xi (quad_metrics, include/functions/quad_metrics.tpp:2-7).
//
// Field blocks hold an even number of elements (one unused element when K is
// odd) and tiles start on even elements, so every tile copy starts on a
// 16-byte boundary and moves a multiple of 16 bytes, as cp.async.bulk needs.
//
// STRICT instantiations round every operation in the reference's order
// (__dmul_rn/__dadd_rn, true divisions) and reproduce its CPU results bit
// for bit; the default instantiations contract to FMAs and multiply by
// reciprocals.
#include "ndg_internal.hpp"
#include "stage_common.cuh"
#include "stage_kernels.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
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

template <int N, bool S>
__global__ void __launch_bounds__(Tile<N>::kThreads) stage_kernel(StageArgs a, const __grid_constant__ Coeffs<N> cf) {
    using T = Tile<N>;
    constexpr int n = T::n, NN = T::NN, EPB = T::EPB;
    extern __shared__ __align__(128) double smem[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + T::kBar);
    double* qs = smem + T::kQ;
    double* gs = smem + T::kG;
    double* own_s = smem + T::kOwn;
    double* far_s = smem + T::kFar;  // far traces, then element side fluxes in place
    double* js = smem + T::kJ;
    double* ss = smem + T::kS;
    double* zs = smem + T::kZ;
    constexpr int FS = EPB * 4 * n;  // field stride of own_s / far_s

    const int tid = threadIdx.x;
    const int64_t K = a.n_elements;
    const int64_t Kp = a.field_stride;  // elements per field block (K rounded up to even)
    const int64_t e0 = static_cast<int64_t>(blockIdx.x) * EPB;
    const int ne = static_cast<int>((K - e0) < EPB ? (K - e0) : EPB);
    const int ne_copy = (ne + 1) & ~1;  // the tile copy moves an even number of elements
    const int64_t inst = blockIdx.y;
    double* q = a.q + inst * 3 * Kp * NN;
    double* k = a.k + inst * 3 * Kp * NN;
    const double* tr_in = a.trace_in + inst * 3 * Kp * 4 * n;
    double* tr_out = a.trace_out + inst * 3 * Kp * 4 * n;
    const double* xn = cf.xn;
    const double* lm = cf.lm;
    const double* lp = cf.lp;
    const double time = a.step[0];
    const double dt = a.step[1];

    // Line threads: (field f, element e of the tile, line or node index m).
    const int f = tid / (EPB * n);
    const int rr = tid - f * (EPB * n);
    const int e = rr / n;
    const int m = rr - e * n;
    const bool active = f < 3 && e < ne;
    const int64_t ge = e0 + e;

    // Prologue: one bulk copy per field brings the q tile into shared memory.
    if (tid == 0) {
        mbar_init(bar, 1);
        mbar_fence_init();
        const uint32_t bytes = static_cast<uint32_t>(ne_copy * NN * sizeof(double));
        mbar_expect_tx(bar, 3 * bytes);
        for (int ff = 0; ff < 3; ++ff) bulk_load(qs + ff * EPB * NN, q + (ff * Kp + e0) * NN, bytes, bar);
    }
    for (int i = tid; i < NN; i += T::kThreads) zs[i] = 0.0;
    // Far traces of this thread's field at node m of the four sides (the
    // neighbour's trace of the previous stage), element metrics, edge
    // metrics and J.
    double x0 = 0, y0 = 0, x1 = 0, y1 = 0, x2 = 0, y2 = 0, x3 = 0, y3 = 0;
    if (active) {
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            const int2 lk = a.link[4 * ge + s];
            const double v = (((lk.y >> 2) & 7) == kInterior) ? tr_in[((f * Kp + lk.x) * 4 + (lk.y & 3)) * n + (N - m)] : 0.0;
            far_s[f * FS + (e * 4 + s) * n + m] = v;
        }
        const double* c = a.corners + 8 * ge;
        x0 = c[0]; y0 = c[1]; x1 = c[2]; y1 = c[3]; x2 = c[4]; y2 = c[5]; x3 = c[6]; y3 = c[7];
    }
    // x_xi, y_xi are functions of eta; x_eta, y_eta functions of xi.
    const MetricLine<S> x_xi(sub<S>(x1, x0), sub<S>(x2, x3)), y_xi(sub<S>(y1, y0), sub<S>(y2, y3));
    const MetricLine<S> x_eta(sub<S>(x3, x0), sub<S>(x2, x1)), y_eta(sub<S>(y3, y0), sub<S>(y2, y1));
    if (active) {
        const double tm = xn[m];
        if (f == 2) {
            // Edge metric of side sd, constant along a straight side
            // (Element2D_t.cpp:756-769): |d(x,y)/dxi| at eta = -1, +1 for
            // sides 0, 2 and |d(x,y)/deta| at xi = +1, -1 for sides 1, 3.
            for (int sd = m; sd < 4; sd += n) {
                const double at = (sd == 0 || sd == 3) ? -1.0 : 1.0;
                const double dx = (sd == 0 || sd == 2) ? metric<S>(at, x_xi.d0, x_xi.d1) : metric<S>(at, x_eta.d0, x_eta.d1);
                const double dy = (sd == 0 || sd == 2) ? metric<S>(at, y_xi.d0, y_xi.d1) : metric<S>(at, y_eta.d0, y_eta.d1);
                ss[e * 4 + sd] = sqrt(add<S>(mul<S>(dx, dx), mul<S>(dy, dy)));
            }
        }
        // J at nodes (m, j), j = f, f + 3, ...: x_xi(eta_j) y_eta(xi_m) - x_eta(xi_m) y_xi(eta_j)
        // (Element2D_t.cpp:752).
        const double xe = x_eta(tm), ye = y_eta(tm);
        for (int j = f; j < n; j += 3) {
            const double tj = xn[j];
            const double jac = sub<S>(mul<S>(x_xi(tj), ye), mul<S>(xe, y_xi(tj)));
            js[e * NN + m * n + j] = S ? jac : __drcp_rn(jac);
        }
    }
    __syncthreads();  // mbarrier init, zeros, far traces, edge metrics, J
    if (!mbar_wait(bar, a.error, kWaitLimitNs)) return;

    // Own side traces of this thread's field (Element2D_t.cpp:86-125):
    // bottom and top from row m, right and left from column m.
    // The flux lines take (X, Y) = (u, v), (p, 0), (0, p) for f = 0, 1, 2:
    // x_flux = (c u, p, 0), y_flux = (c v, 0, p) (Solver2D_t.cpp:31-37).
    const double* Qe = qs + e * NN;
    const double* Xe = f == 0 ? Qe + 1 * EPB * NN : (f == 1 ? Qe : zs);
    const double* Ye = f == 0 ? Qe + 2 * EPB * NN : (f == 1 ? zs : Qe);
    if (active) {
        const double* Qf = Qe + f * EPB * NN;
        double b = 0.0, t = 0.0, r = 0.0, l = 0.0;
#pragma unroll
        for (int j = 0; j < n; ++j) {
            const double qr = Qf[m * n + j], qc = Qf[j * n + m];
            b = madd<S>(b, lm[j], qr);
            t = madd<S>(t, lp[j], qr);
            r = madd<S>(r, lp[j], qc);
            l = madd<S>(l, lm[j], qc);
        }
        double* o = own_s + f * FS + e * 4 * n;
        o[0 * n + m] = b;
        o[2 * n + (N - m)] = t;
        o[1 * n + m] = r;
        o[3 * n + (N - m)] = l;
    }
    __syncthreads();

    // Flux pass: side nodes m of side f, and of side 3 for f = 0. Far traces
    // of boundary sides, the upwind flux (Solver2D_t.cpp:48-63) in the face's
    // own left/right order, then the element's view of it
    // (Mesh2D_t.cpp:3895-3929): times the edge metric, negated for the face's
    // right element.
    if (active) {
        for (int pass = 0; pass < 2; ++pass) {
            if (pass == 1 && f != 0) break;
            const int s = pass == 0 ? f : 3;
            const int2 lk = a.link[4 * ge + s];
            const int kind = (lk.y >> 2) & 7;
            const int role = (lk.y >> 5) & 1;
            const double2 nv = a.normal[4 * ge + s];
            const int o = (e * 4 + s) * n + m;
            const double op = own_s[o], ou = own_s[FS + o], ov = own_s[2 * FS + o];
            double fp_, fu_, fv_;
            if (kind == kInterior) {
                fp_ = far_s[o];
                fu_ = far_s[FS + o];
                fv_ = far_s[2 * FS + o];
            } else if (kind == kMirror || kind == kCopy) {
                // Ghost trace: the own trace reversed and scaled by the ghost's
                // edge metric; walls and symmetry planes then mirror the normal
                // velocity (Mesh2D_t.cpp:4366-4434, 4601-4710).
                const double gsc = a.gscale[4 * ge + s];
                fp_ = mul<S>(op, gsc);
                const double gu = mul<S>(ou, gsc), gv = mul<S>(ov, gsc);
                if (kind == kMirror) {
                    const double tx = -nv.y, ty = nv.x;
                    const double l0 = -add<S>(mul<S>(gu, nv.x), mul<S>(gv, nv.y));
                    const double l1 = add<S>(mul<S>(gu, tx), mul<S>(gv, ty));
                    fu_ = add<S>(mul<S>(nv.x, l0), mul<S>(tx, l1));
                    fv_ = add<S>(mul<S>(nv.y, l0), mul<S>(ty, l1));
                } else {
                    fu_ = gu;
                    fv_ = gv;
                }
            } else if (kind == kAnalytic) {
                // Inflow: the analytic wave on the ghost edge at the stage time
                // (Mesh2D_t.cpp:4575-4599); the face reads ghost node N - m.
                const double4 gq = a.inflow[4 * ge + s];
                const double r = mul<S>(add<S>(xn[N - m], 1.0), 0.5);
                const double gx = add<S>(mul<S>(gq.z, r), mul<S>(gq.x, sub<S>(1.0, r)));
                const double gy = add<S>(mul<S>(gq.w, r), mul<S>(gq.y, sub<S>(1.0, r)));
                plane_wave(gx, gy, add<S>(time, mul<S>(a.rk_b, dt)), fp_, fu_, fv_);
            } else {
                fp_ = fu_ = fv_ = 0.0;
            }
            const double Lp = role ? fp_ : op, Lu = role ? fu_ : ou, Lv = role ? fv_ : ov;
            const double Rp = role ? op : fp_, Ru = role ? ou : fu_, Rv = role ? ov : fv_;
            const double wL = add<S>(Lp, add<S>(mul<S>(Lu, nv.x), mul<S>(Lv, nv.y)));
            const double wR = sub<S>(Rp, add<S>(mul<S>(Ru, nv.x), mul<S>(Rv, nv.y)));
            const double flp = mul<S>(sub<S>(wL, wR), 0.5);
            const double sum = add<S>(wL, wR);
            const double flu = mul<S>(mul<S>(nv.x, sum), 0.5);
            const double flv = mul<S>(mul<S>(nv.y, sum), 0.5);
            const double sf = ss[e * 4 + s];
            far_s[o] = mul<S>(role ? -flp : flp, sf);
            far_s[FS + o] = mul<S>(role ? -flu : flu, sf);
            far_s[2 * FS + o] = mul<S>(role ? -flv : flv, sf);
        }
    }
    __syncthreads();

    const double* Dh = cf.dhat;
    const double* w = cf.w;
    const double* iw = cf.iw;
    const double* F = far_s + f * FS + e * 4 * n;  // this thread's field, element side fluxes

    // xi pass (eta index j = m): contravariant flux line eta_y X - eta_x Y
    // (Solver2D_t.cpp:72-80), Dhat . line + lift, G = -(...) (:82-101); G column j.
    if (active) {
        const int j = m;
        double col[n];
#pragma unroll
        for (int i = 0; i < n; ++i) col[i] = sub<S>(mul<S>(y_eta(xn[i]), Xe[i * n + j]), mul<S>(x_eta(xn[i]), Ye[i * n + j]));
        const double fr = F[1 * n + j], fl3 = F[3 * n + (N - j)];
        double* G = gs + (f * EPB + e) * NN + j;
#pragma unroll
        for (int i = 0; i < n; ++i) {
            double acc = 0.0;
#pragma unroll
            for (int mm = 0; mm < n; ++mm) acc = madd<S>(acc, Dh[i * n + mm], col[mm]);
            const double lift = S ? __ddiv_rn(add<S>(mul<S>(fr, lp[i]), mul<S>(fl3, lm[i])), w[i]) : (fr * lp[i] + fl3 * lm[i]) * iw[i];
            G[i * n] = -add<S>(acc, lift);
        }
    }
    __syncthreads();

    // eta pass (xi index i = m): line -xi_y X + xi_x Y (Solver2D_t.cpp:103-113),
    // G = (G - (Dhat . line + lift)) / J (:114-133); G row i.
    if (active) {
        const int i = m;
        double line[n];
#pragma unroll
        for (int j = 0; j < n; ++j) line[j] = add<S>(mul<S>(-y_xi(xn[j]), Xe[i * n + j]), mul<S>(x_xi(xn[j]), Ye[i * n + j]));
        const double ft = F[2 * n + (N - i)], fb = F[0 * n + i];
        double* G = gs + (f * EPB + e) * NN + i * n;
        const double* jrow = js + e * NN + i * n;
#pragma unroll
        for (int j = 0; j < n; ++j) {
            double acc = 0.0;
#pragma unroll
            for (int mm = 0; mm < n; ++mm) acc = madd<S>(acc, Dh[j * n + mm], line[mm]);
            const double lift = S ? __ddiv_rn(add<S>(mul<S>(ft, lp[j]), mul<S>(fb, lm[j])), w[j]) : (ft * lp[j] + fb * lm[j]) * iw[j];
            const double num = sub<S>(G[j], add<S>(acc, lift));
            G[j] = S ? __ddiv_rn(num, jrow[j]) : num * jrow[j];
        }
    }
    __syncthreads();

    // Low-storage RK3 update (Solver2D_t.cpp:138-172), node by node:
    // coalesced reads of k (prefetched) and writes of k and q.
    const double gdt = mul<S>(a.rk_g, dt);
    double kold[T::kNodeIters];
#pragma unroll
    for (int c = 0; c < T::kNodeIters; ++c) {
        const int idx = tid + c * T::kThreads;
        const int ff = idx / (EPB * NN), r = idx - ff * (EPB * NN);
        kold[c] = (!a.first && ff < 3 && r < ne * NN) ? k[(ff * Kp + e0) * NN + r] : 0.0;
    }
#pragma unroll
    for (int c = 0; c < T::kNodeIters; ++c) {
        const int idx = tid + c * T::kThreads;
        const int ff = idx / (EPB * NN), r = idx - ff * (EPB * NN);
        if (ff < 3 && r < ne * NN) {
            const double G = gs[ff * EPB * NN + r];
            const double kn = a.first ? G : add<S>(mul<S>(a.rk_a, kold[c]), G);
            const double qn = add<S>(qs[ff * EPB * NN + r], mul<S>(gdt, kn));
            const int64_t gi = (ff * Kp + e0) * NN + r;
            k[gi] = kn;
            q[gi] = qn;
            qs[ff * EPB * NN + r] = qn;
            if (a.G_out) a.G_out[inst * 3 * Kp * NN + gi] = G;
        }
    }
    __syncthreads();

    // Side traces of the new solution for the next stage: bottom/top from
    // row m, right/left from column m (Element2D_t.cpp:86-125).
    if (active) {
        const double* row = qs + (f * EPB + e) * NN + m * n;
        const double* cl = qs + (f * EPB + e) * NN + m;
        double b = 0.0, t = 0.0, r = 0.0, l = 0.0;
#pragma unroll
        for (int j = 0; j < n; ++j) {
            b = madd<S>(b, lm[j], row[j]);
            t = madd<S>(t, lp[j], row[j]);
            r = madd<S>(r, lp[j], cl[j * n]);
            l = madd<S>(l, lm[j], cl[j * n]);
        }
        double* to = tr_out + (f * Kp + ge) * 4 * n;
        to[0 * n + m] = b;
        to[2 * n + (N - m)] = t;
        to[1 * n + m] = r;
        to[3 * n + (N - m)] = l;
    }
}

// ---------------------------------------------------------------------------
// FP32 form of the stage (uniform order, conforming faces): traces, fluxes,
// metrics and the volume term in FP32 with FMA contraction; q and k stay
// FP64 in HBM and the RK update runs in FP64, so only the stage's time
// derivative G carries FP32 rounding. Traces are stored in FP32, halving
// their traffic.
template <int N>
struct CoeffsF {
    float dhat[(N + 1) * (N + 1)];
    float xn[N + 1], lm[N + 1], lp[N + 1], w[N + 1], iw[N + 1];
};

template <int N>
struct TileF {
    static constexpr int n = N + 1;
    static constexpr int NN = n * n;
    static constexpr int EPB = Tile<N>::EPB;
    static constexpr int kThreads = Tile<N>::kThreads;
    static constexpr int kNodeIters = Tile<N>::kNodeIters;
    // the bulk-copied FP64 q tile, then FP32 arrays (offsets in floats past it)
    static constexpr int kQd = 3 * EPB * NN;             // doubles
    static constexpr int kQf = 0;                        // [3][EPB][NN] q in FP32
    static constexpr int kG = kQf + 3 * EPB * NN;        // [3][EPB][NN]
    static constexpr int kOwn = kG + 3 * EPB * NN;       // [3][EPB][4][n]
    static constexpr int kFar = kOwn + 3 * EPB * 4 * n;  // [3][EPB][4][n] far traces, then side fluxes
    static constexpr int kJ = kFar + 3 * EPB * 4 * n;    // [EPB][NN] 1/J
    static constexpr int kS = kJ + EPB * NN;             // [EPB][4]
    static constexpr int kZ = kS + EPB * 4;              // [NN] zeros
    static constexpr int kFloats = (kZ + NN + 3) / 4 * 4;  // keeps the mbarrier 16-byte aligned
    static constexpr size_t kBytes = sizeof(double) * kQd + sizeof(float) * kFloats + 16;
};

// ((1 - t) d0 + (1 + t) d1) / 4 as fma(t, (d1 - d0) / 4, (d0 + d1) / 4) in FP32.
struct MetricLineF {
    float a, b;
    __device__ __forceinline__ MetricLineF(float d0, float d1) : a(0.25f * (d0 + d1)), b(0.25f * (d1 - d0)) {}
    __device__ __forceinline__ float operator()(float t) const { return fmaf(t, b, a); }
};

template <int N>
__global__ void __launch_bounds__(TileF<N>::kThreads) stage_kernel_f32(StageArgs a, const __grid_constant__ CoeffsF<N> cf) {
    using T = TileF<N>;
    constexpr int n = T::n, NN = T::NN, EPB = T::EPB;
    extern __shared__ __align__(128) double smem[];
    double* qs = smem;
    float* fsm = reinterpret_cast<float*>(smem + T::kQd);
    float* qf = fsm + T::kQf;
    float* gs = fsm + T::kG;
    float* own_s = fsm + T::kOwn;
    float* far_s = fsm + T::kFar;
    float* js = fsm + T::kJ;
    float* ss = fsm + T::kS;
    float* zs = fsm + T::kZ;
    uint64_t* bar = reinterpret_cast<uint64_t*>(fsm + T::kFloats);
    constexpr int FS = EPB * 4 * n;

    const int tid = threadIdx.x;
    const int64_t K = a.n_elements;
    const int64_t Kp = a.field_stride;
    const int64_t e0 = static_cast<int64_t>(blockIdx.x) * EPB;
    const int ne = static_cast<int>((K - e0) < EPB ? (K - e0) : EPB);
    const int ne_copy = (ne + 1) & ~1;
    const int64_t inst = blockIdx.y;
    double* q = a.q + inst * 3 * Kp * NN;
    double* k = a.k + inst * 3 * Kp * NN;
    const float* tr_in = a.trace_in_f + inst * 3 * Kp * 4 * n;
    float* tr_out = a.trace_out_f + inst * 3 * Kp * 4 * n;
    const float* xn = cf.xn;
    const float* lm = cf.lm;
    const float* lp = cf.lp;
    const double time = a.step[0];
    const double dt = a.step[1];

    const int f = tid / (EPB * n);
    const int rr = tid - f * (EPB * n);
    const int e = rr / n;
    const int m = rr - e * n;
    const bool active = f < 3 && e < ne;
    const int64_t ge = e0 + e;

    if (tid == 0) {
        mbar_init(bar, 1);
        mbar_fence_init();
        const uint32_t bytes = static_cast<uint32_t>(ne_copy * NN * sizeof(double));
        mbar_expect_tx(bar, 3 * bytes);
        for (int ff = 0; ff < 3; ++ff) bulk_load(qs + ff * EPB * NN, q + (ff * Kp + e0) * NN, bytes, bar);
    }
    for (int i = tid; i < NN; i += T::kThreads) zs[i] = 0.0f;
    float x0 = 0, y0 = 0, x1 = 0, y1 = 0, x2 = 0, y2 = 0, x3 = 0, y3 = 0;
    if (active) {
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            const int2 lk = a.link[4 * ge + s];
            const float v = (((lk.y >> 2) & 7) == kInterior) ? tr_in[((f * Kp + lk.x) * 4 + (lk.y & 3)) * n + (N - m)] : 0.0f;
            far_s[f * FS + (e * 4 + s) * n + m] = v;
        }
        const double* c = a.corners + 8 * ge;
        x0 = static_cast<float>(c[0]); y0 = static_cast<float>(c[1]); x1 = static_cast<float>(c[2]); y1 = static_cast<float>(c[3]);
        x2 = static_cast<float>(c[4]); y2 = static_cast<float>(c[5]); x3 = static_cast<float>(c[6]); y3 = static_cast<float>(c[7]);
    }
    const MetricLineF x_xi(x1 - x0, x2 - x3), y_xi(y1 - y0, y2 - y3);
    const MetricLineF x_eta(x3 - x0, x2 - x1), y_eta(y3 - y0, y2 - y1);
    if (active) {
        const float tm = xn[m];
        if (f == 2) {
            for (int sd = m; sd < 4; sd += n) {
                const float at = (sd == 0 || sd == 3) ? -1.0f : 1.0f;
                const float dx = (sd == 0 || sd == 2) ? x_xi(at) : x_eta(at);
                const float dy = (sd == 0 || sd == 2) ? y_xi(at) : y_eta(at);
                ss[e * 4 + sd] = sqrtf(dx * dx + dy * dy);
            }
        }
        const float xe = x_eta(tm), ye = y_eta(tm);
        for (int j = f; j < n; j += 3) {
            const float tj = xn[j];
            js[e * NN + m * n + j] = __frcp_rn(x_xi(tj) * ye - xe * y_xi(tj));
        }
    }
    __syncthreads();
    if (!mbar_wait(bar, a.error, kWaitLimitNs)) return;
    for (int i = tid; i < 3 * EPB * NN; i += T::kThreads) qf[i] = static_cast<float>(qs[i]);
    __syncthreads();

    const float* Qe = qf + e * NN;
    const float* Xe = f == 0 ? Qe + 1 * EPB * NN : (f == 1 ? Qe : zs);
    const float* Ye = f == 0 ? Qe + 2 * EPB * NN : (f == 1 ? zs : Qe);
    if (active) {
        const float* Qf = Qe + f * EPB * NN;
        float b = 0.0f, t = 0.0f, r = 0.0f, l = 0.0f;
#pragma unroll
        for (int j = 0; j < n; ++j) {
            const float qr = Qf[m * n + j], qc = Qf[j * n + m];
            b = fmaf(lm[j], qr, b);
            t = fmaf(lp[j], qr, t);
            r = fmaf(lp[j], qc, r);
            l = fmaf(lm[j], qc, l);
        }
        float* o = own_s + f * FS + e * 4 * n;
        o[0 * n + m] = b;
        o[2 * n + (N - m)] = t;
        o[1 * n + m] = r;
        o[3 * n + (N - m)] = l;
    }
    __syncthreads();

    if (active) {
        for (int pass = 0; pass < 2; ++pass) {
            if (pass == 1 && f != 0) break;
            const int s = pass == 0 ? f : 3;
            const int2 lk = a.link[4 * ge + s];
            const int kind = (lk.y >> 2) & 7;
            const int role = (lk.y >> 5) & 1;
            const double2 nvd = a.normal[4 * ge + s];
            const float nx = static_cast<float>(nvd.x), ny = static_cast<float>(nvd.y);
            const int o = (e * 4 + s) * n + m;
            const float op = own_s[o], ou = own_s[FS + o], ov = own_s[2 * FS + o];
            float fp_, fu_, fv_;
            if (kind == kInterior) {
                fp_ = far_s[o];
                fu_ = far_s[FS + o];
                fv_ = far_s[2 * FS + o];
            } else if (kind == kMirror || kind == kCopy) {
                const float gsc = static_cast<float>(a.gscale[4 * ge + s]);
                fp_ = op * gsc;
                const float gu = ou * gsc, gv = ov * gsc;
                if (kind == kMirror) {
                    const float tx = -ny, ty = nx;
                    const float l0 = -(gu * nx + gv * ny);
                    const float l1 = gu * tx + gv * ty;
                    fu_ = nx * l0 + tx * l1;
                    fv_ = ny * l0 + ty * l1;
                } else {
                    fu_ = gu;
                    fv_ = gv;
                }
            } else if (kind == kAnalytic) {
                const double4 gq = a.inflow[4 * ge + s];
                const double rr2 = (static_cast<double>(xn[N - m]) + 1.0) * 0.5;
                double pd, ud, vd;
                plane_wave(gq.z * rr2 + gq.x * (1.0 - rr2), gq.w * rr2 + gq.y * (1.0 - rr2), time + a.rk_b * dt, pd, ud, vd);
                fp_ = static_cast<float>(pd);
                fu_ = static_cast<float>(ud);
                fv_ = static_cast<float>(vd);
            } else {
                fp_ = fu_ = fv_ = 0.0f;
            }
            const float Lp = role ? fp_ : op, Lu = role ? fu_ : ou, Lv = role ? fv_ : ov;
            const float Rp = role ? op : fp_, Ru = role ? ou : fu_, Rv = role ? ov : fv_;
            const float wL = Lp + (Lu * nx + Lv * ny);
            const float wR = Rp - (Ru * nx + Rv * ny);
            const float sum = wL + wR;
            const float sf = ss[e * 4 + s] * 0.5f;
            far_s[o] = (role ? -(wL - wR) : (wL - wR)) * sf;
            far_s[FS + o] = (role ? -nx : nx) * sum * sf;
            far_s[2 * FS + o] = (role ? -ny : ny) * sum * sf;
        }
    }
    __syncthreads();

    const float* Dh = cf.dhat;
    const float* iw = cf.iw;
    const float* F = far_s + f * FS + e * 4 * n;
    if (active) {
        const int j = m;
        float col[n];
#pragma unroll
        for (int i = 0; i < n; ++i) col[i] = y_eta(xn[i]) * Xe[i * n + j] - x_eta(xn[i]) * Ye[i * n + j];
        const float fr = F[1 * n + j], fl3 = F[3 * n + (N - j)];
        float* G = gs + (f * EPB + e) * NN + j;
#pragma unroll
        for (int i = 0; i < n; ++i) {
            float acc = 0.0f;
#pragma unroll
            for (int mm = 0; mm < n; ++mm) acc = fmaf(Dh[i * n + mm], col[mm], acc);
            G[i * n] = -(acc + (fr * lp[i] + fl3 * lm[i]) * iw[i]);
        }
    }
    __syncthreads();

    if (active) {
        const int i = m;
        float line[n];
#pragma unroll
        for (int j = 0; j < n; ++j) line[j] = -y_xi(xn[j]) * Xe[i * n + j] + x_xi(xn[j]) * Ye[i * n + j];
        const float ft = F[2 * n + (N - i)], fb = F[0 * n + i];
        float* G = gs + (f * EPB + e) * NN + i * n;
        const float* jrow = js + e * NN + i * n;
#pragma unroll
        for (int j = 0; j < n; ++j) {
            float acc = 0.0f;
#pragma unroll
            for (int mm = 0; mm < n; ++mm) acc = fmaf(Dh[j * n + mm], line[mm], acc);
            G[j] = (G[j] - (acc + (ft * lp[j] + fb * lm[j]) * iw[j])) * jrow[j];
        }
    }
    __syncthreads();

    // RK3 update in FP64 (Solver2D_t.cpp:138-172); the new q also refreshes
    // the FP32 tile for the traces.
    const double gdt = a.rk_g * dt;
    double kold[T::kNodeIters];
#pragma unroll
    for (int c = 0; c < T::kNodeIters; ++c) {
        const int idx = tid + c * T::kThreads;
        const int ff = idx / (EPB * NN), r = idx - ff * (EPB * NN);
        kold[c] = (!a.first && ff < 3 && r < ne * NN) ? k[(ff * Kp + e0) * NN + r] : 0.0;
    }
#pragma unroll
    for (int c = 0; c < T::kNodeIters; ++c) {
        const int idx = tid + c * T::kThreads;
        const int ff = idx / (EPB * NN), r = idx - ff * (EPB * NN);
        if (ff < 3 && r < ne * NN) {
            const double G = static_cast<double>(gs[ff * EPB * NN + r]);
            const double kn = a.first ? G : fma(a.rk_a, kold[c], G);
            const double qn = fma(gdt, kn, qs[ff * EPB * NN + r]);
            const int64_t gi = (ff * Kp + e0) * NN + r;
            k[gi] = kn;
            q[gi] = qn;
            qf[ff * EPB * NN + r] = static_cast<float>(qn);
            if (a.G_out) a.G_out[inst * 3 * Kp * NN + gi] = G;
        }
    }
    __syncthreads();

    if (active) {
        const float* row = qf + (f * EPB + e) * NN + m * n;
        const float* cl = qf + (f * EPB + e) * NN + m;
        float b = 0.0f, t = 0.0f, r = 0.0f, l = 0.0f;
#pragma unroll
        for (int j = 0; j < n; ++j) {
            b = fmaf(lm[j], row[j], b);
            t = fmaf(lp[j], row[j], t);
            r = fmaf(lp[j], cl[j * n], r);
            l = fmaf(lm[j], cl[j * n], l);
        }
        float* to = tr_out + (f * Kp + ge) * 4 * n;
        to[0 * n + m] = b;
        to[2 * n + (N - m)] = t;
        to[1 * n + m] = r;
        to[3 * n + (N - m)] = l;
    }
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
        a.trace_out_f[((fi * Kp + e) * 4 + s) * n + m] = acc;
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
        a.trace_out[((fi * Kp + e) * 4 + s) * n + m] = side_trace<N, S>(qf, s, m);
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

// ---------------------------------------------------------------------------
// Host launchers.

template <int N, bool S>
static cudaError_t launch_stage_t(const StageArgs& a, cudaStream_t stream) {
    using T = Tile<N>;
    const dim3 grid(static_cast<unsigned>((a.n_elements + T::EPB - 1) / T::EPB), static_cast<unsigned>(a.n_instances));
    stage_kernel<N, S><<<grid, T::kThreads, T::kBytes, stream>>>(a, make_coeffs<N>());
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
    return cudaFuncSetAttribute(stage_kernel<N, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(Tile<N>::kBytes));
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
    return c;
}

template <int N, bool Unused>
static cudaError_t prepare_f32_t() {
    return cudaFuncSetAttribute(stage_kernel_f32<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(TileF<N>::kBytes));
}

template <int N, bool Unused>
static cudaError_t launch_stage_f32_t(const StageArgs& a, cudaStream_t stream) {
    using T = TileF<N>;
    const dim3 grid(static_cast<unsigned>((a.n_elements + T::EPB - 1) / T::EPB), static_cast<unsigned>(a.n_instances));
    stage_kernel_f32<N><<<grid, T::kThreads, T::kBytes, stream>>>(a, make_coeffs_f<N>());
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
