// Variable-speed forward stage and its discrete adjoint for sm_100a.
//
// speed_stage_kernel  one low-storage RK3 stage of L(c) (the operator of
//                     adjoint.cuh), fused like the uniform-order stage kernel:
//                     cp.async copy of the q tile into a padded shared
//                     layout free of bank conflicts, own traces, upwind flux with
//                     the face speed, volume term times c_e, RK update,
//                     traces of the new q; optionally it keeps the stage
//                     input (for the adjoint's c-gradient) and samples the
//                     receivers' pressure of the new q.
// adjoint_stage_kernel  the exact transpose of one stage, run backwards:
//                     every forward pass (trace extraction, ghost traces,
//                     upwind flux, lift, volume derivative, RK update) is
//                     replaced by its transpose, in reverse order, within
//                     one CTA per tile of elements. The neighbour coupling
//                     runs through "adjoint far traces": the transpose of
//                     the flux with respect to the far-side trace, which the
//                     neighbour published at the end of the previous adjoint
//                     stage, exactly as the forward reads the neighbour's
//                     traces of the previous stage.
//
// The c-gradient uses that L(c) is linear in c: the volume term scales with
// c_e and the face flux with (c_e + c_nb) / 2. Per element and stage the
// kernel accumulates mu . (volume term at c = 1) and, per side, the flux
// part U_s = own trace . (adjoint of the own trace) / c_face; for a shared
// face U_s + U_nb,s' is the face flux's derivative with respect to c_face
// (both sides' flux transposes meet in it), so the gradient gathers
// (U_s + U_nb,s') / 2 from both elements (launch_speed_gradient).
//
// Both kernels are templates over R, the type of the operator's arithmetic:
// double (the FP64 form, FMA contraction) or float (the FP32 form: traces,
// fluxes, metrics, contractions and their transposes in FP32, traces stored
// in FP32). The states copied into shared memory, the RK updates, the
// misfit and the gradient accumulators are FP64 in both.
#include "adjoint.cuh"
#include "stage_common.cuh"
#include "stage_kernels.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <type_traits>

namespace ndg {
namespace dev {

template <typename R>
__device__ __forceinline__ R rcp(R x) {
    if constexpr (std::is_same_v<R, double>)
        return __drcp_rn(x);
    else
        return __frcp_rn(x);
}

// ((1 - t) d0 + (1 + t) d1) / 4 of quad_metrics as fma(t, (d1 - d0)/4, (d0 + d1)/4).
template <typename R>
struct LineR {
    R d0, d1, a, b;
    __device__ __forceinline__ LineR(R d0_, R d1_) : d0(d0_), d1(d1_), a(R(0.25) * (d0_ + d1_)), b(R(0.25) * (d1_ - d0_)) {}
    __device__ __forceinline__ R operator()(R t) const { return fma(t, b, a); }
};

// The edge metric term of a side at t = +-1, in the reference's expression.
template <typename R>
__device__ __forceinline__ R edge_term(R t, R d0, R d1) {
    return ((R(1) - t) * d0 + (R(1) + t) * d1) * R(0.25);
}

// The form's trace buffer.
template <typename R>
__device__ __forceinline__ const R* pick(const double* d, const float* f) {
    if constexpr (std::is_same_v<R, double>)
        return d;
    else
        return f;
}
template <typename R>
__device__ __forceinline__ R* pick(double* d, float* f) {
    if constexpr (std::is_same_v<R, double>)
        return d;
    else
        return f;
}

template <int N, typename R>
struct SpeedCoeffs {
    R dhat[(N + 1) * (N + 1)];
    R xn[N + 1], lm[N + 1], lp[N + 1], iw[N + 1];
};

// Coefficients of the adjoint: Dhat, nodes, Lagrange end values, 1/w and
// the lift weights l(-1)/w, l(+1)/w.
template <int N, typename R>
struct AdjCoeffs {
    R dhat[(N + 1) * (N + 1)];
    R xn[N + 1], lm[N + 1], lp[N + 1], iw[N + 1], lmw[N + 1], lpw[N + 1];
};

template <int N, typename R>
static SpeedCoeffs<N, R> make_speed_coeffs() {
    constexpr int n = N + 1;
    double dh[n * n], xn[n], lm[n], lp[n], w[n], iw[n];
    host_coefficients(N, dh, xn, lm, lp, w, iw);
    SpeedCoeffs<N, R> c;
    for (int i = 0; i < n * n; ++i) c.dhat[i] = static_cast<R>(dh[i]);
    for (int i = 0; i < n; ++i) {
        c.xn[i] = static_cast<R>(xn[i]);
        c.lm[i] = static_cast<R>(lm[i]);
        c.lp[i] = static_cast<R>(lp[i]);
        c.iw[i] = static_cast<R>(iw[i]);
    }
    return c;
}

template <int N, typename R>
static AdjCoeffs<N, R> make_adj_coeffs() {
    constexpr int n = N + 1;
    double dh[n * n], xn[n], lm[n], lp[n], w[n], iw[n];
    host_coefficients(N, dh, xn, lm, lp, w, iw);
    AdjCoeffs<N, R> c;
    for (int i = 0; i < n * n; ++i) c.dhat[i] = static_cast<R>(dh[i]);
    for (int i = 0; i < n; ++i) {
        c.xn[i] = static_cast<R>(xn[i]);
        c.lm[i] = static_cast<R>(lm[i]);
        c.lp[i] = static_cast<R>(lp[i]);
        c.iw[i] = static_cast<R>(iw[i]);
        c.lmw[i] = static_cast<R>(lm[i] * iw[i]);
        c.lpw[i] = static_cast<R>(lp[i] * iw[i]);
    }
    return c;
}

// Pressure at the receivers of a tile, one warp: sum of w_r . p over the
// element's nodes, lanes striding the nodes, then a shuffle reduction in a
// fixed order (the same result wherever it is evaluated). FP64 in both forms.
// Receiver sample sum_i w_i p_i over an element's nodes, with the element's
// tile block p laid out in rows of pitch P (node i of n per row).
template <int n, int P>
__device__ __forceinline__ double receiver_value(const double* __restrict__ w, const double* p, int lane) {
    double s = 0.0;
    for (int i = lane; i < n * n; i += 32) s = fma(w[i], p[(i / n) * P + i % n], s);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    return s;
}

// ---------------------------------------------------------------------------
// Forward stage with a wave speed per element, one thread per (field,
// element, line), the line fastest: the FP64 q tile, then R arrays
// (offsets in R values past it). Node arrays have rows of pitch P and
// element strides chosen by bank::search for this thread order (for even n,
// e.g. N = 7: pitch 9, element stride 72, both sweeps conflict-free); the q
// tile arrives by 8-byte cp.async copies into that layout.
template <int N, typename R>
struct SpeedTile {
    static constexpr int n = N + 1, NN = n * n;
    // as many elements as fit ~60 KB of shared memory and 256 threads, rounded down to a power of two
    static constexpr int per_element_doubles = 2 * 3 * NN + 2 * 3 * 4 * n + NN + 4;
    static constexpr int by_smem = (60 * 1024 / 8) / per_element_doubles;
    static constexpr int by_threads = 256 / (3 * n);
    static constexpr int raw = by_smem < by_threads ? by_smem : by_threads;
    static constexpr int EPB = bank::pow2_floor(raw >= 2 ? (raw < 16 ? raw : 16) : 2);
    static constexpr int kThreads = (3 * EPB * n + 31) / 32 * 32;
    static constexpr int kWarps = kThreads / 32;
    static constexpr int kBlockIters = (3 * EPB + kWarps - 1) / kWarps;
    static constexpr int kLaneIters = (NN + 31) / 32;
    static constexpr bank::Strides Ld = bank::search(N, EPB, 16, false);                              // FP64 tile
    static constexpr bank::Strides Lr = bank::search(N, EPB, static_cast<int>(128 / sizeof(R)), false);  // R arrays
    static constexpr int P = Ld.P, ESd = Ld.ES, QSd = Ld.QS, ESr = Lr.ES, QSr = Lr.QS, SE = Lr.SE, FS = Lr.FS;
    static constexpr int kQd = 3 * QSd;              // doubles: the q tile
    static constexpr int kG = 0;                     // [3][QSr] time derivative G
    static constexpr int kOwn = kG + 3 * QSr;        // [3][FS] own side traces
    static constexpr int kFar = kOwn + 3 * FS;       // [3][FS] far traces, then element side fluxes
    static constexpr int kJ = kFar + 3 * FS;         // [EPB][ESr] 1/J
    static constexpr int kS = kJ + EPB * ESr;        // [EPB][4] edge metric per side
    static constexpr int kRs = kS + EPB * 4;
    static constexpr size_t kBytes = sizeof(double) * kQd + sizeof(R) * kRs;
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

template <int N, typename R>
__global__ void __launch_bounds__(SpeedTile<N, R>::kThreads) speed_stage_kernel(SpeedStageArgs a, const __grid_constant__ SpeedCoeffs<N, R> cf) {
    using T = SpeedTile<N, R>;
    constexpr int n = T::n, NN = T::NN, EPB = T::EPB;
    constexpr int P = T::P, ESd = T::ESd, QSd = T::QSd, ESr = T::ESr, QSr = T::QSr, SE = T::SE, FS = T::FS;
    extern __shared__ __align__(128) double smem[];
    double* qs = smem;
    R* rs = reinterpret_cast<R*>(smem + T::kQd);
    R* gs = rs + T::kG;
    R* own_s = rs + T::kOwn;
    R* far_s = rs + T::kFar;
    R* js = rs + T::kJ;
    R* ss = rs + T::kS;

    const int tid = threadIdx.x;
    const int64_t K = a.n_elements;
    const int64_t Kp = a.field_stride;
    const int64_t e0 = static_cast<int64_t>(blockIdx.x) * EPB;
    const int ne = static_cast<int>((K - e0) < EPB ? (K - e0) : EPB);
    double* q = a.q;
    double* k = a.k;
    const R* tr_in = pick<R>(a.trace_in, a.trace_in_f);
    R* tr_out = pick<R>(a.trace_out, a.trace_out_f);
    const R* xn = cf.xn;
    const R* lm = cf.lm;
    const R* lp = cf.lp;

    const int f = tid / (EPB * n);
    const int rr = tid - f * (EPB * n);
    const int e = rr / n;
    const int m = rr - e * n;
    const bool active = f < 3 && e < ne;
    const int64_t ge = e0 + e;

    // q tile: warps take (field, element) blocks, lanes their nodes.
    const int warp = tid >> 5, lane = tid & 31;
    int lane_node[T::kLaneIters];
#pragma unroll
    for (int it = 0; it < T::kLaneIters; ++it) lane_node[it] = T::node(lane + 32 * it);
#pragma unroll
    for (int bi = 0; bi < T::kBlockIters; ++bi) {
        const int b = warp + bi * T::kWarps, ff = b / EPB, el = b - ff * EPB;
        if (b < 3 * EPB && el < ne) {
            const double* src = q + (ff * Kp + e0 + el) * NN;
            double* dst = qs + ff * QSd + el * ESd;
#pragma unroll
            for (int it = 0; it < T::kLaneIters; ++it)
                if (lane + 32 * it < NN) cp_async8(dst + lane_node[it], src + lane + 32 * it);
        }
    }
    // Corners in FP64: their differences are formed before rounding to R.
    double x0 = 0, y0 = 0, x1 = 0, y1 = 0, x2 = 0, y2 = 0, x3 = 0, y3 = 0;
    R ce = 1;
    if (active) {
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            const int2 lk = a.link[4 * ge + s];
            const R v = (((lk.y >> 2) & 7) == kInterior) ? tr_in[((f * Kp + lk.x) * 4 + (lk.y & 3)) * n + (N - m)] : R(0);
            far_s[f * FS + e * SE + s * n + m] = v;
        }
        const double* c = a.corners + 8 * ge;
        x0 = c[0]; y0 = c[1]; x1 = c[2]; y1 = c[3]; x2 = c[4]; y2 = c[5]; x3 = c[6]; y3 = c[7];
        ce = R(a.c[ge]);
    }
    const LineR<R> x_xi(R(x1 - x0), R(x2 - x3)), y_xi(R(y1 - y0), R(y2 - y3));
    const LineR<R> x_eta(R(x3 - x0), R(x2 - x1)), y_eta(R(y3 - y0), R(y2 - y1));
    if (active) {
        const R tm = xn[m];
        if (f == 2) {
            for (int sd = m; sd < 4; sd += n) {
                const R at = (sd == 0 || sd == 3) ? R(-1) : R(1);
                const R dx = (sd == 0 || sd == 2) ? edge_term<R>(at, x_xi.d0, x_xi.d1) : edge_term<R>(at, x_eta.d0, x_eta.d1);
                const R dy = (sd == 0 || sd == 2) ? edge_term<R>(at, y_xi.d0, y_xi.d1) : edge_term<R>(at, y_eta.d0, y_eta.d1);
                ss[e * 4 + sd] = sqrt(dx * dx + dy * dy);
            }
        }
        const R xe = x_eta(tm), ye = y_eta(tm);
        for (int j = f; j < n; j += 3) {
            const R tj = xn[j];
            js[e * ESr + m * P + j] = rcp<R>(x_xi(tj) * ye - xe * y_xi(tj));
        }
    }
    cp_async_wait_all();
    __syncthreads();

    // Flux lines (X, Y) = (u, v), (p, 0), (0, p) for the fields p, u, v: the
    // absent component is scaled by zero.
    const double* Qe = qs + e * ESd;
    const double* Xe = f == 0 ? Qe + 1 * QSd : Qe;
    const double* Ye = f == 0 ? Qe + 2 * QSd : Qe;
    const R sx = f == 2 ? R(0) : R(1), sy = f == 1 ? R(0) : R(1);
    if (active) {
        const double* Qf = Qe + f * QSd;
        R b = 0, t = 0, r = 0, l = 0;
#pragma unroll
        for (int j = 0; j < n; ++j) {
            const R qr = R(Qf[m * P + j]), qc = R(Qf[j * P + m]);
            b = fma(lm[j], qr, b);
            t = fma(lp[j], qr, t);
            r = fma(lp[j], qc, r);
            l = fma(lm[j], qc, l);
        }
        R* o = own_s + f * FS + e * SE;
        o[0 * n + m] = b;
        o[2 * n + (N - m)] = t;
        o[1 * n + m] = r;
        o[3 * n + (N - m)] = l;
    }
    __syncthreads();

    // Flux pass: the unit-speed upwind flux of the face, times the face
    // speed, the edge metric and the element's orientation sign.
    if (active) {
        for (int pass = 0; pass < 2; ++pass) {
            if (pass == 1 && f != 0) break;
            const int s = pass == 0 ? f : 3;
            const int2 lk = a.link[4 * ge + s];
            const int kind = (lk.y >> 2) & 7;
            const int role = (lk.y >> 5) & 1;
            const double2 nd = a.normal[4 * ge + s];
            const R nx = R(nd.x), ny = R(nd.y);
            const int o = e * SE + s * n + m;
            const R op = own_s[o], ou = own_s[FS + o], ov = own_s[2 * FS + o];
            R fp_, fu_, fv_, cface = ce;
            if (kind == kInterior) {
                fp_ = far_s[o];
                fu_ = far_s[FS + o];
                fv_ = far_s[2 * FS + o];
                cface = R(0.5) * (ce + R(a.c[lk.x]));
            } else if (kind == kMirror || kind == kCopy) {
                const R gsc = R(a.gscale[4 * ge + s]);
                fp_ = op * gsc;
                const R gu = ou * gsc, gv = ov * gsc;
                if (kind == kMirror) {
                    const R tx = -ny, ty = nx;
                    const R l0 = -(gu * nx + gv * ny);
                    const R l1 = gu * tx + gv * ty;
                    fu_ = nx * l0 + tx * l1;
                    fv_ = ny * l0 + ty * l1;
                } else {
                    fu_ = gu;
                    fv_ = gv;
                }
            } else {
                fp_ = fu_ = fv_ = R(0);
            }
            const R Lp = role ? fp_ : op, Lu = role ? fu_ : ou, Lv = role ? fv_ : ov;
            const R Rp = role ? op : fp_, Ru = role ? ou : fu_, Rv = role ? ov : fv_;
            const R wL = Lp + (Lu * nx + Lv * ny);
            const R wR = Rp - (Ru * nx + Rv * ny);
            const R sc = (role ? -ss[e * 4 + s] : ss[e * 4 + s]) * cface;
            const R sum = wL + wR;
            far_s[o] = sc * ((wL - wR) * R(0.5));
            far_s[FS + o] = sc * (nx * sum * R(0.5));
            far_s[2 * FS + o] = sc * (ny * sum * R(0.5));
        }
    }
    __syncthreads();

    const R* Dh = cf.dhat;
    const R* iw = cf.iw;
    const R* F = far_s + f * FS + e * SE;

    if (active) {
        const int j = m;
        R col[n];
#pragma unroll
        for (int i = 0; i < n; ++i) col[i] = y_eta(xn[i]) * (sx * R(Xe[i * P + j])) - x_eta(xn[i]) * (sy * R(Ye[i * P + j]));
        const R fr = F[1 * n + j], fl3 = F[3 * n + (N - j)];
        R* G = gs + f * QSr + e * ESr + j;
#pragma unroll
        for (int i = 0; i < n; ++i) {
            R acc = 0;
#pragma unroll
            for (int mm = 0; mm < n; ++mm) acc = fma(Dh[i * n + mm], col[mm], acc);
            G[i * P] = -fma(acc, ce, (fr * lp[i] + fl3 * lm[i]) * iw[i]);
        }
    }
    __syncthreads();

    if (active) {
        const int i = m;
        R line[n];
#pragma unroll
        for (int j = 0; j < n; ++j) line[j] = -y_xi(xn[j]) * (sx * R(Xe[i * P + j])) + x_xi(xn[j]) * (sy * R(Ye[i * P + j]));
        const R ft = F[2 * n + (N - i)], fb = F[0 * n + i];
        R* G = gs + f * QSr + e * ESr + i * P;
        const R* jrow = js + e * ESr + i * P;
#pragma unroll
        for (int j = 0; j < n; ++j) {
            R acc = 0;
#pragma unroll
            for (int mm = 0; mm < n; ++mm) acc = fma(Dh[j * n + mm], line[mm], acc);
            G[j] = (G[j] - fma(acc, ce, (ft * lp[j] + fb * lm[j]) * iw[j])) * jrow[j];
        }
    }
    __syncthreads();

    // RK update in FP64: warps take (field, element) blocks, lanes their nodes.
    double kold[T::kBlockIters][T::kLaneIters];
#pragma unroll
    for (int bi = 0; bi < T::kBlockIters; ++bi) {
        const int b = warp + bi * T::kWarps, ff = b / EPB, el = b - ff * EPB;
        const bool live = !a.first && b < 3 * EPB && el < ne;
        const double* kb = k + (ff * Kp + e0 + el) * NN;
#pragma unroll
        for (int it = 0; it < T::kLaneIters; ++it) kold[bi][it] = (live && lane + 32 * it < NN) ? kb[lane + 32 * it] : 0.0;
    }
#pragma unroll
    for (int bi = 0; bi < T::kBlockIters; ++bi) {
        const int b = warp + bi * T::kWarps, ff = b / EPB, el = b - ff * EPB;
        if (b < 3 * EPB && el < ne) {
            const int64_t gb = (ff * Kp + e0 + el) * NN;
#pragma unroll
            for (int it = 0; it < T::kLaneIters; ++it) {
                const int nd = lane + 32 * it;
                if (nd < NN) {
                    const int sd = ff * QSd + el * ESd + lane_node[it];
                    const double G = static_cast<double>(gs[ff * QSr + el * ESr + lane_node[it]]);
                    const double kn = a.first ? G : fma(a.rk_a, kold[bi][it], G);
                    const double qo = qs[sd];
                    const double qn = fma(a.gdt, kn, qo);
                    if (a.q_save) a.q_save[gb + nd] = qo;
                    k[gb + nd] = kn;
                    q[gb + nd] = qn;
                    qs[sd] = qn;
                    if (a.G_out) a.G_out[gb + nd] = G;
                }
            }
        }
    }
    __syncthreads();

    if (active) {
        const double* row = qs + f * QSd + e * ESd + m * P;
        const double* cl = qs + f * QSd + e * ESd + m;
        R b = 0, t = 0, r = 0, l = 0;
#pragma unroll
        for (int j = 0; j < n; ++j) {
            const R qr = R(row[j]), qc = R(cl[j * P]);
            b = fma(lm[j], qr, b);
            t = fma(lp[j], qr, t);
            r = fma(lp[j], qc, r);
            l = fma(lm[j], qc, l);
        }
        R* to = tr_out + (f * Kp + ge) * 4 * n;
        to[0 * n + m] = b;
        to[2 * n + (N - m)] = t;
        to[1 * n + m] = r;
        to[3 * n + (N - m)] = l;
    }
    if (a.samples && tid < 32) {
        for (int r = 0; r < a.rec.n; ++r) {
            const int64_t el = a.rec.elem[r] - e0;
            if (el < 0 || el >= ne) continue;
            const double v = receiver_value<n, P>(a.rec.w + static_cast<int64_t>(r) * NN, qs + el * ESd, tid);
            if (tid == 0) a.samples[r] = v;
        }
    }
}

// ---------------------------------------------------------------------------
// Adjoint stage. Tile of EPB elements, one thread per (field, element, line)
// as the forward. Shared memory: FP64 arrays first (the lq and qs tiles,
// copied by 8-byte cp.async into rows of pitch P, the receiver residuals
// and masks), then R arrays; node and side arrays use the strides
// bank::search finds for this thread order.
template <int N, typename R>
struct AdjTile {
    static constexpr int n = N + 1;
    static constexpr int NN = n * n;
    static constexpr int per_element_bytes = 8 * (6 * NN + 1) + static_cast<int>(sizeof(R)) * (5 * NN + 43 * n + 8);
    static constexpr int fixed_bytes = 8 * kMaxReceivers + 64;
    static constexpr int by_smem = (60 * 1024 - fixed_bytes) / per_element_bytes;
    static constexpr int by_threads = 256 / (3 * n);
    static constexpr int raw = by_smem < by_threads ? by_smem : by_threads;
    // FP64: 2 elements per CTA (half the shared memory of 4, so more CTAs
    // and warps per SM: 37.6 against 41.2 µs per launch at N = 7 on the
    // 96 x 96 adjoint workload); the FP32 form keeps 4 (31.2 against 35.3 µs).
    static constexpr int EPB = sizeof(R) == 8 ? 2 : (raw >= 4 ? 4 : (raw >= 2 ? (raw & ~1) : 2));
    static constexpr int kThreads = (3 * EPB * n + 31) / 32 * 32;
    static constexpr int kWarps = kThreads / 32;
    static constexpr int kBlockIters = (3 * EPB + kWarps - 1) / kWarps;
    static constexpr int kLaneIters = (NN + 31) / 32;
    static constexpr bank::Strides Ld = bank::search(N, EPB, 16, false);                              // FP64 tiles
    static constexpr bank::Strides Lr = bank::search(N, EPB, static_cast<int>(128 / sizeof(R)), false);  // R arrays
    static constexpr int P = Ld.P, ESd = Ld.ES, QSd = Ld.QS, ESr = Lr.ES, QSr = Lr.QS, SE = Lr.SE, FS = Lr.FS;
    // doubles
    static constexpr int kL = 0;                    // [3][QSd] lq, then lq + volume transpose
    static constexpr int kQ = kL + 3 * QSd;         // [3][QSd] forward stage input qs
    static constexpr int kRes = kQ + 3 * QSd;       // [kMaxReceivers] weighted misfit residuals
    static constexpr int kMask = kRes + kMaxReceivers;  // [EPB] receivers of each element (bit mask)
    static constexpr int kDoubles = kMask + EPB;
    // R values past the doubles
    static constexpr int kNu = 0;                   // [3][QSr] nu = -mu / J, later nu'
    static constexpr int kTp = kNu + 3 * QSr;       // [EPB][ESr] second accumulator of the pressure's transpose
    static constexpr int kJ = kTp + EPB * ESr;      // [EPB][ESr] 1/J
    static constexpr int kOwn = kJ + EPB * ESr;     // [3][FS] side traces of qs
    static constexpr int kEll = kOwn + 3 * FS;      // [3][FS] lift transpose, then own-trace adjoint, then next lift transpose
    static constexpr int kFar = kEll + 3 * FS;      // [3][FS] neighbours' adjoint far traces
    static constexpr int kUp = kFar + 3 * FS;       // [EPB][SE] flux part of the c-derivative per side node
    static constexpr int kVd = kUp + EPB * SE;      // [3][EPB][n] volume part of the c-derivative per line
    static constexpr int kS = kVd + 3 * EPB * n;    // [EPB][4] edge metric
    static constexpr int kCf = kS + 4 * EPB;        // [EPB][4] face speed
    static constexpr int kRs = kCf + 4 * EPB;
    static constexpr size_t kBytes = sizeof(double) * kDoubles + sizeof(R) * kRs;
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

// t += c v with the form's rounding: one FMA in FP64; in the FP32 form the
// FP32 product accumulated in the target's type.
template <typename T, typename R>
__device__ __forceinline__ void add_scaled(T* t, R c, R v) {
    *t = fma(static_cast<T>(c), static_cast<T>(v), *t);
}

template <int N, typename R>
__global__ void __launch_bounds__(AdjTile<N, R>::kThreads) adjoint_stage_kernel(AdjointStageArgs a, const __grid_constant__ AdjCoeffs<N, R> cf) {
    using T = AdjTile<N, R>;
    constexpr int n = T::n, NN = T::NN, EPB = T::EPB, FS = T::FS;
    constexpr int P = T::P, ESd = T::ESd, QSd = T::QSd, ESr = T::ESr, QSr = T::QSr, SE = T::SE;
    extern __shared__ __align__(128) double smem[];
    double* ls = smem + T::kL;
    double* qs = smem + T::kQ;
    double* res = smem + T::kRes;
    unsigned long long* rmask = reinterpret_cast<unsigned long long*>(smem + T::kMask);
    R* rs = reinterpret_cast<R*>(smem + T::kDoubles);
    R* nu = rs + T::kNu;
    R* tp = rs + T::kTp;
    R* js = rs + T::kJ;
    R* own_s = rs + T::kOwn;
    R* ell = rs + T::kEll;
    R* far_s = rs + T::kFar;
    R* up = rs + T::kUp;
    R* vd = rs + T::kVd;
    R* ss = rs + T::kS;
    R* cfs = rs + T::kCf;
    const R* atr_in = pick<R>(a.atr_in, a.atr_in_f);
    R* atr_out = pick<R>(a.atr_out, a.atr_out_f);

    const int tid = threadIdx.x;
    const int64_t K = a.n_elements;
    const int64_t Kp = a.field_stride;
    const int64_t e0 = static_cast<int64_t>(blockIdx.x) * EPB;
    const int ne = static_cast<int>((K - e0) < EPB ? (K - e0) : EPB);
    const R* xn = cf.xn;
    const R* lm = cf.lm;
    const R* lp = cf.lp;
    const R* lmw = cf.lmw;
    const R* lpw = cf.lpw;
    const R* Dh = cf.dhat;

    const int f = tid / (EPB * n);
    const int rr = tid - f * (EPB * n);
    const int e = rr / n;
    const int m = rr - e * n;
    const bool active = f < 3 && e < ne;
    const int64_t ge = e0 + e;

    // Prologue: asynchronous copies of the lq and qs tiles (warps take
    // (field, element) blocks, lanes their nodes); adjoint far traces of the
    // neighbours, metrics, J, edge metrics and face speeds.
    const int warp = tid >> 5, lane = tid & 31;
    int lane_node[T::kLaneIters];
#pragma unroll
    for (int it = 0; it < T::kLaneIters; ++it) lane_node[it] = T::node(lane + 32 * it);
#pragma unroll
    for (int bi = 0; bi < T::kBlockIters; ++bi) {
        const int b = warp + bi * T::kWarps, ff = b / EPB, el = b - ff * EPB;
        if (b < 3 * EPB && el < ne) {
            const int64_t gb = (ff * Kp + e0 + el) * NN;
            const int sb = ff * QSd + el * ESd;
#pragma unroll
            for (int it = 0; it < T::kLaneIters; ++it)
                if (lane + 32 * it < NN) {
                    cp_async8(ls + sb + lane_node[it], a.lq + gb + lane + 32 * it);
                    cp_async8(qs + sb + lane_node[it], a.qs + gb + lane + 32 * it);
                }
        }
    }
    for (int i = tid; i < EPB * ESr; i += T::kThreads) tp[i] = R(0);
    if (tid < EPB) rmask[tid] = 0ull;
    // Corners in FP64: their differences are formed before rounding to R.
    double x0 = 0, y0 = 0, x1 = 0, y1 = 0, x2 = 0, y2 = 0, x3 = 0, y3 = 0;
    R ce = 1;
    if (active) {
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            const int2 lk = a.link[4 * ge + s];
            const R v = (((lk.y >> 2) & 7) == kInterior) ? atr_in[((f * Kp + lk.x) * 4 + (lk.y & 3)) * n + (N - m)] : R(0);
            far_s[f * FS + e * SE + s * n + m] = v;
        }
        const double* c = a.corners + 8 * ge;
        x0 = c[0]; y0 = c[1]; x1 = c[2]; y1 = c[3]; x2 = c[4]; y2 = c[5]; x3 = c[6]; y3 = c[7];
        ce = R(a.c[ge]);
    }
    const LineR<R> x_xi(R(x1 - x0), R(x2 - x3)), y_xi(R(y1 - y0), R(y2 - y3));
    const LineR<R> x_eta(R(x3 - x0), R(x2 - x1)), y_eta(R(y3 - y0), R(y2 - y1));
    if (active) {
        const R tm = xn[m];
        if (f == 2) {
            for (int sd = m; sd < 4; sd += n) {
                const R at = (sd == 0 || sd == 3) ? R(-1) : R(1);
                const R dx = (sd == 0 || sd == 2) ? edge_term<R>(at, x_xi.d0, x_xi.d1) : edge_term<R>(at, x_eta.d0, x_eta.d1);
                const R dy = (sd == 0 || sd == 2) ? edge_term<R>(at, y_xi.d0, y_xi.d1) : edge_term<R>(at, y_eta.d0, y_eta.d1);
                ss[e * 4 + sd] = sqrt(dx * dx + dy * dy);
                const int2 lk = a.link[4 * ge + sd];
                cfs[e * 4 + sd] = (((lk.y >> 2) & 7) == kInterior) ? R(0.5) * (ce + R(a.c[lk.x])) : ce;
            }
        }
        const R xe = x_eta(tm), ye = y_eta(tm);
        for (int j = f; j < n; j += 3) {
            const R tj = xn[j];
            js[e * ESr + m * P + j] = rcp<R>(x_xi(tj) * ye - xe * y_xi(tj));
        }
    }
    cp_async_wait_all();
    __syncthreads();

    // Node pass: mu = lk + gdt lq; lk = a mu (kept in registers for mu');
    // nu = -mu / J. One warp evaluates the misfit residuals of the
    // receivers in the tile at the state qs.
    double kn[T::kBlockIters][T::kLaneIters];
#pragma unroll
    for (int bi = 0; bi < T::kBlockIters; ++bi) {
        const int b = warp + bi * T::kWarps, ff = b / EPB, el = b - ff * EPB;
        const bool live = b < 3 * EPB && el < ne;
        const int64_t gb = (ff * Kp + e0 + el) * NN;
#pragma unroll
        for (int it = 0; it < T::kLaneIters; ++it) {
            const int nd = lane + 32 * it;
            kn[bi][it] = 0.0;
            if (live && nd < NN) {
                const int64_t gi = gb + nd;
                const double mu = fma(a.gdt, ls[ff * QSd + el * ESd + lane_node[it]], a.lk[gi]);
                kn[bi][it] = a.rk_a * mu;
                a.lk[gi] = kn[bi][it];
                nu[ff * QSr + el * ESr + lane_node[it]] = R(-mu) * js[el * ESr + lane_node[it]];
            }
        }
    }
    if (a.inject && tid < 32) {
        for (int r = 0; r < a.rec.n; ++r) {
            const int64_t el = a.rec.elem[r] - e0;
            if (el < 0 || el >= ne) continue;
            const double v = receiver_value<n, P>(a.rec.w + static_cast<int64_t>(r) * NN, qs + el * ESd, tid);
            if (tid == 0) {
                res[r] = a.wdt * (v - a.target[r]);
                rmask[el] |= 1ull << r;
            }
        }
    }
    __syncthreads();

    // Transposed volume term. The forward's flux lines take (X, Y) = (u, v),
    // (p, 0), (0, p) for the fields p, u, v; the transpose sends field f's
    // line adjoints A (of X) and B (of Y) back to those fields:
    //   f = p: A -> lu, B -> lv;  f = u: A -> lp;  f = v: B -> lp (via tp).
    // vdot accumulates X A + Y B (the volume term's derivative in c_e).
    const double* Qe = qs + e * ESd;
    const double* Xe = f == 0 ? Qe + 1 * QSd : Qe;
    const double* Ye = f == 0 ? Qe + 2 * QSd : Qe;
    const R sx = f == 2 ? R(0) : R(1), sy = f == 1 ? R(0) : R(1);
    double* O1 = f == 0 ? ls + 1 * QSd + e * ESd : ls + e * ESd;  // f = p, u
    R* O1v = tp + e * ESr;                                          // f = v
    double* O2 = ls + 2 * QSd + e * ESd;                            // f = p only
    const R* Nf = nu + f * QSr + e * ESr;
    R vdot = 0;
    // xi columns (eta index j = m): alpha = Dhat^T nu(:, j); lift transpose
    // of sides 1 and 3; the side traces of qs.
    if (active) {
        const int j = m;
        R col[n];
#pragma unroll
        for (int i = 0; i < n; ++i) col[i] = Nf[i * P + j];
        R l1 = 0, l3 = 0;
#pragma unroll
        for (int i = 0; i < n; ++i) {
            l1 = fma(col[i], lpw[i], l1);
            l3 = fma(col[i], lmw[i], l3);
        }
        R* L = ell + f * FS + e * SE;
        L[1 * n + j] = l1;
        L[3 * n + (N - j)] = l3;
#pragma unroll
        for (int mm = 0; mm < n; ++mm) {
            R al = 0;
#pragma unroll
            for (int i = 0; i < n; ++i) al = fma(Dh[i * n + mm], col[i], al);
            const R A = y_eta(xn[mm]) * al, B = -x_eta(xn[mm]) * al;
            const int node = mm * P + j;
            vdot = fma(sx * R(Xe[node]), A, fma(sy * R(Ye[node]), B, vdot));
            if (f == 2)
                add_scaled(O1v + node, ce, B);
            else
                add_scaled(O1 + node, ce, A);
            if (f == 0) add_scaled(O2 + node, ce, B);
        }
        const double* Qf = Qe + f * QSd;
        R b = 0, t = 0, r = 0, l = 0;
#pragma unroll
        for (int jj = 0; jj < n; ++jj) {
            const R qr = R(Qf[m * P + jj]), qc = R(Qf[jj * P + m]);
            b = fma(lm[jj], qr, b);
            t = fma(lp[jj], qr, t);
            r = fma(lp[jj], qc, r);
            l = fma(lm[jj], qc, l);
        }
        R* o = own_s + f * FS + e * SE;
        o[0 * n + m] = b;
        o[2 * n + (N - m)] = t;
        o[1 * n + m] = r;
        o[3 * n + (N - m)] = l;
    }
    __syncthreads();

    // eta rows (xi index i = m): beta = Dhat^T nu(i, :); lift transpose of
    // sides 2 and 0.
    if (active) {
        const int i = m;
        R row[n];
#pragma unroll
        for (int j = 0; j < n; ++j) row[j] = Nf[i * P + j];
        R l2 = 0, l0 = 0;
#pragma unroll
        for (int j = 0; j < n; ++j) {
            l2 = fma(row[j], lpw[j], l2);
            l0 = fma(row[j], lmw[j], l0);
        }
        R* L = ell + f * FS + e * SE;
        L[2 * n + (N - i)] = l2;
        L[0 * n + i] = l0;
#pragma unroll
        for (int mm = 0; mm < n; ++mm) {
            R be = 0;
#pragma unroll
            for (int j = 0; j < n; ++j) be = fma(Dh[j * n + mm], row[j], be);
            const R A = -y_xi(xn[mm]) * be, B = x_xi(xn[mm]) * be;
            const int node = i * P + mm;
            vdot = fma(sx * R(Xe[node]), A, fma(sy * R(Ye[node]), B, vdot));
            if (f == 2)
                add_scaled(O1v + node, ce, B);
            else
                add_scaled(O1 + node, ce, A);
            if (f == 0) add_scaled(O2 + node, ce, B);
        }
        vd[(f * EPB + e) * n + m] = vdot;
    }
    __syncthreads();

    // Transposed flux (side s = f, and s = 3 for f = 0): psi = sign sf c_face
    // ell is the adjoint of the unit-speed flux phi(L, R); its transpose
    // gives the adjoints of the left and right traces. The own side keeps
    // its part; the far part goes to the ghost's source (the own trace,
    // mirrored and scaled) or was published by the neighbour for this side.
    // up = own trace . own-trace adjoint / c_face.
    if (active) {
        for (int pass = 0; pass < 2; ++pass) {
            if (pass == 1 && f != 0) break;
            const int s = pass == 0 ? f : 3;
            const int2 lk = a.link[4 * ge + s];
            const int kind = (lk.y >> 2) & 7;
            const int role = (lk.y >> 5) & 1;
            const double2 nd = a.normal[4 * ge + s];
            const R nx = R(nd.x), ny = R(nd.y);
            const int o = e * SE + s * n + m;
            const R cface = cfs[e * 4 + s];
            const R sc = (role ? -ss[e * 4 + s] : ss[e * 4 + s]) * cface;
            const R pp = sc * ell[o], pu = sc * ell[FS + o], pv = sc * ell[2 * FS + o];
            const R dn = R(0.5) * (nx * pu + ny * pv);
            const R wl = fma(R(0.5), pp, dn), wr = fma(R(-0.5), pp, dn);
            // adjoints of L = (wl, wl nx, wl ny) and R = (wr, -wr nx, -wr ny)
            const R sl = role ? -wr : wl;  // own trace: R for the right element
            const R sf_ = role ? wl : -wr;
            R tp_ = role ? wr : wl, tu = sl * nx, tv = sl * ny;
            const R fp_ = role ? wl : wr, fu_ = sf_ * nx, fv_ = sf_ * ny;
            if (kind == kInterior) {
                tp_ += far_s[o];
                tu += far_s[FS + o];
                tv += far_s[2 * FS + o];
            } else if (kind == kMirror || kind == kCopy) {
                const R gsc = R(a.gscale[4 * ge + s]);
                R gu = fu_, gv = fv_;
                if (kind == kMirror) {
                    const R tx = -ny, ty = nx;
                    const R l0 = -(fu_ * nx + fv_ * ny);
                    const R l1 = fu_ * tx + fv_ * ty;
                    gu = nx * l0 + tx * l1;
                    gv = ny * l0 + ty * l1;
                }
                tp_ = fma(gsc, fp_, tp_);
                tu = fma(gsc, gu, tu);
                tv = fma(gsc, gv, tv);
            }
            ell[o] = tp_;
            ell[FS + o] = tu;
            ell[2 * FS + o] = tv;
            up[o] = (own_s[o] * tp_ + own_s[FS + o] * tu + own_s[2 * FS + o] * tv) / cface;
        }
    }
    __syncthreads();

    // Node pass: lq' = lq + volume transpose + trace transpose (the four
    // side-trace adjoints back to the nodes), the misfit injection, then
    // nu' = -(lk' + gdt_next lq') / J for the next stage.
#pragma unroll
    for (int bi = 0; bi < T::kBlockIters; ++bi) {
        const int b = warp + bi * T::kWarps, ff = b / EPB, el = b - ff * EPB;
        if (!(b < 3 * EPB && el < ne)) continue;
        const int64_t gb = (ff * Kp + e0 + el) * NN;
#pragma unroll
        for (int it = 0; it < T::kLaneIters; ++it) {
            const int node = lane + 32 * it;
            if (node >= NN) continue;
            const int i = node / n, j = node - i * n;
            const R* Lo = ell + ff * FS + el * SE;
            double v = ls[ff * QSd + el * ESd + lane_node[it]];
            if (ff == 0) v += static_cast<double>(tp[el * ESr + lane_node[it]]);
            if constexpr (std::is_same_v<R, double>) {
                v = fma(lm[j], Lo[0 * n + i], v);
                v = fma(lp[j], Lo[2 * n + (N - i)], v);
                v = fma(lp[i], Lo[1 * n + j], v);
                v = fma(lm[i], Lo[3 * n + (N - j)], v);
            } else {
                R t4 = lm[j] * Lo[0 * n + i];
                t4 = fma(lp[j], Lo[2 * n + (N - i)], t4);
                t4 = fma(lp[i], Lo[1 * n + j], t4);
                t4 = fma(lm[i], Lo[3 * n + (N - j)], t4);
                v += static_cast<double>(t4);
            }
            if (ff == 0) {
                unsigned long long mask = rmask[el];
                while (mask) {
                    const int rc = __ffsll(static_cast<long long>(mask)) - 1;
                    mask &= mask - 1;
                    v = fma(res[rc], a.rec.w[static_cast<int64_t>(rc) * NN + node], v);
                }
            }
            a.lq[gb + node] = v;
            nu[ff * QSr + el * ESr + lane_node[it]] = R(-fma(a.gdt_next, v, kn[bi][it])) * js[el * ESr + lane_node[it]];
        }
    }
    __syncthreads();

    // Lift transpose of nu' on the four sides (column m: sides 1, 3; row m:
    // sides 2, 0); per element, the c-derivative accumulators (FP64).
    if (active) {
        const R* Nn = nu + f * QSr + e * ESr;
        R l1 = 0, l3 = 0, l2 = 0, l0 = 0;
#pragma unroll
        for (int i = 0; i < n; ++i) {
            const R cv = Nn[i * P + m], rv = Nn[m * P + i];
            l1 = fma(cv, lpw[i], l1);
            l3 = fma(cv, lmw[i], l3);
            l2 = fma(rv, lpw[i], l2);
            l0 = fma(rv, lmw[i], l0);
        }
        R* L = ell + f * FS + e * SE;
        L[1 * n + m] = l1;
        L[3 * n + (N - m)] = l3;
        L[2 * n + (N - m)] = l2;
        L[0 * n + m] = l0;
    }
    if (tid < ne) {
        double vsum = 0.0;
        for (int ff = 0; ff < 3; ++ff)
            for (int i = 0; i < n; ++i) vsum += static_cast<double>(vd[(ff * EPB + tid) * n + i]);
        double* A = a.acc + (e0 + tid) * 5;
        A[0] += vsum;
        for (int s = 0; s < 4; ++s) {
            double us = 0.0;
            for (int i = 0; i < n; ++i) us += static_cast<double>(up[tid * SE + s * n + i]);
            A[1 + s] += us;
        }
    }
    __syncthreads();

    // Adjoint far traces of mu' for the neighbours (interior sides): the
    // transpose of the flux with respect to the far-side trace.
    if (active) {
        for (int pass = 0; pass < 2; ++pass) {
            if (pass == 1 && f != 0) break;
            const int s = pass == 0 ? f : 3;
            const int2 lk = a.link[4 * ge + s];
            if (((lk.y >> 2) & 7) != kInterior) continue;
            const int role = (lk.y >> 5) & 1;
            const double2 nd = a.normal[4 * ge + s];
            const R nx = R(nd.x), ny = R(nd.y);
            const int o = e * SE + s * n + m;
            const R sc = (role ? -ss[e * 4 + s] : ss[e * 4 + s]) * cfs[e * 4 + s];
            const R pp = sc * ell[o], pu = sc * ell[FS + o], pv = sc * ell[2 * FS + o];
            const R dn = R(0.5) * (nx * pu + ny * pv);
            const R wl = fma(R(0.5), pp, dn), wr = fma(R(-0.5), pp, dn);
            const R sf_ = role ? wl : -wr;
            R* to = atr_out + (ge * 4 + s) * n + m;
            to[0] = role ? wl : wr;
            to[Kp * 4 * n] = sf_ * nx;
            to[2 * Kp * 4 * n] = sf_ * ny;
        }
    }
}

// ---------------------------------------------------------------------------
__global__ void speed_gradient_kernel(const double* __restrict__ acc, const int2* __restrict__ link, int64_t K, double* __restrict__ grad) {
    for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < K; e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        double g = acc[5 * e];
        for (int s = 0; s < 4; ++s) {
            const int2 lk = link[4 * e + s];
            const double own = acc[5 * e + 1 + s];
            g += (((lk.y >> 2) & 7) == kInterior) ? 0.5 * (own + acc[5 * static_cast<int64_t>(lk.x) + 1 + (lk.y & 3)]) : own;
        }
        grad[e] = g;
    }
}

// ---------------------------------------------------------------------------
// Host launchers.
template <int N, typename R>
static cudaError_t prepare_speed_t() {
    cudaError_t err =
        cudaFuncSetAttribute(speed_stage_kernel<N, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(SpeedTile<N, R>::kBytes));
    if (err != cudaSuccess) return err;
    return cudaFuncSetAttribute(adjoint_stage_kernel<N, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(AdjTile<N, R>::kBytes));
}

template <int N, typename R>
static cudaError_t launch_speed_stage_t(const SpeedStageArgs& a, cudaStream_t stream) {
    using T = SpeedTile<N, R>;
    speed_stage_kernel<N, R><<<static_cast<unsigned>((a.n_elements + T::EPB - 1) / T::EPB), T::kThreads, T::kBytes, stream>>>(a, make_speed_coeffs<N, R>());
    return cudaGetLastError();
}

template <int N, typename R>
static cudaError_t launch_adjoint_stage_t(const AdjointStageArgs& a, cudaStream_t stream) {
    using T = AdjTile<N, R>;
    adjoint_stage_kernel<N, R><<<static_cast<unsigned>((a.n_elements + T::EPB - 1) / T::EPB), T::kThreads, T::kBytes, stream>>>(a, make_adj_coeffs<N, R>());
    return cudaGetLastError();
}

template <int N, typename R>
static int adjoint_epb_t() {
    return AdjTile<N, R>::EPB;
}

#define NDG_SPEED_DISPATCH(FN, N_, F32_, ...)                                                   \
    switch (N_) {                                                                               \
        case 1: return F32_ ? FN<1, float>(__VA_ARGS__) : FN<1, double>(__VA_ARGS__);           \
        case 2: return F32_ ? FN<2, float>(__VA_ARGS__) : FN<2, double>(__VA_ARGS__);           \
        case 3: return F32_ ? FN<3, float>(__VA_ARGS__) : FN<3, double>(__VA_ARGS__);           \
        case 4: return F32_ ? FN<4, float>(__VA_ARGS__) : FN<4, double>(__VA_ARGS__);           \
        case 5: return F32_ ? FN<5, float>(__VA_ARGS__) : FN<5, double>(__VA_ARGS__);           \
        case 6: return F32_ ? FN<6, float>(__VA_ARGS__) : FN<6, double>(__VA_ARGS__);           \
        case 7: return F32_ ? FN<7, float>(__VA_ARGS__) : FN<7, double>(__VA_ARGS__);           \
        case 8: return F32_ ? FN<8, float>(__VA_ARGS__) : FN<8, double>(__VA_ARGS__);           \
        case 9: return F32_ ? FN<9, float>(__VA_ARGS__) : FN<9, double>(__VA_ARGS__);           \
        case 10: return F32_ ? FN<10, float>(__VA_ARGS__) : FN<10, double>(__VA_ARGS__);        \
        case 11: return F32_ ? FN<11, float>(__VA_ARGS__) : FN<11, double>(__VA_ARGS__);        \
        case 12: return F32_ ? FN<12, float>(__VA_ARGS__) : FN<12, double>(__VA_ARGS__);        \
        default: break;                                                                         \
    }

cudaError_t prepare_speed_kernels(int N, bool fp32) {
    NDG_SPEED_DISPATCH(prepare_speed_t, N, fp32)
    return cudaErrorInvalidValue;
}

cudaError_t launch_speed_stage(int N, bool fp32, const SpeedStageArgs& a, cudaStream_t stream) {
    NDG_SPEED_DISPATCH(launch_speed_stage_t, N, fp32, a, stream)
    return cudaErrorInvalidValue;
}

cudaError_t launch_adjoint_stage(int N, bool fp32, const AdjointStageArgs& a, cudaStream_t stream) {
    NDG_SPEED_DISPATCH(launch_adjoint_stage_t, N, fp32, a, stream)
    return cudaErrorInvalidValue;
}

int adjoint_elements_per_block(int N, bool fp32) {
    NDG_SPEED_DISPATCH(adjoint_epb_t, N, fp32)
    return 0;
}

cudaError_t launch_speed_gradient(const double* acc, const int2* link, int64_t K, double* grad_c, cudaStream_t stream) {
    const int blocks = static_cast<int>(std::min<int64_t>((K + 255) / 256, 148 * 8));
    speed_gradient_kernel<<<blocks, 256, 0, stream>>>(acc, link, K, grad_c);
    return cudaGetLastError();
}

}  // namespace dev
}  // namespace ndg
