// Variable-speed forward stage and its discrete adjoint for sm_100a.
//
// speed_stage_kernel  one low-storage RK3 stage of L(c) (the operator of
//                     adjoint.cuh), fused like the uniform-order stage kernel:
//                     bulk copy of the q tile, own traces, upwind flux with
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
// FP64 with FMA contraction; the RK register and the solution stay FP64.
#include "adjoint.cuh"
#include "stage_common.cuh"
#include "stage_kernels.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

namespace ndg {
namespace dev {

// Coefficients of the adjoint: Dhat, nodes, Lagrange end values and the
// lift weights l(-1)/w, l(+1)/w.
template <int N>
struct AdjCoeffs {
    double dhat[(N + 1) * (N + 1)];
    double xn[N + 1], lm[N + 1], lp[N + 1], iw[N + 1], lmw[N + 1], lpw[N + 1];
};

template <int N>
static AdjCoeffs<N> make_adj_coeffs() {
    constexpr int n = N + 1;
    double w[n];
    AdjCoeffs<N> c;
    host_coefficients(N, c.dhat, c.xn, c.lm, c.lp, w, c.iw);
    for (int i = 0; i < n; ++i) {
        c.lmw[i] = c.lm[i] * c.iw[i];
        c.lpw[i] = c.lp[i] * c.iw[i];
    }
    return c;
}

template <int N>
static Coeffs<N> make_speed_coeffs() {
    Coeffs<N> c;
    host_coefficients(N, c.dhat, c.xn, c.lm, c.lp, c.w, c.iw);
    return c;
}

// Pressure at the receivers of a tile, one warp: sum of w_r . p over the
// element's nodes, lanes striding the nodes, then a shuffle reduction in a
// fixed order (the same result wherever it is evaluated).
template <int NN>
__device__ __forceinline__ double receiver_value(const double* __restrict__ w, const double* p, int lane) {
    double s = 0.0;
    for (int i = lane; i < NN; i += 32) s = fma(w[i], p[i], s);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    return s;
}

// ---------------------------------------------------------------------------
// Forward stage with a wave speed per element. Same tile, thread layout and
// passes as stage_kernel<N, false> (stage_kernels.cu).
template <int N>
__global__ void __launch_bounds__(Tile<N>::kThreads) speed_stage_kernel(SpeedStageArgs a, const __grid_constant__ Coeffs<N> cf) {
    using T = Tile<N>;
    constexpr int n = T::n, NN = T::NN, EPB = T::EPB;
    extern __shared__ __align__(128) double smem[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + T::kBar);
    double* qs = smem + T::kQ;
    double* gs = smem + T::kG;
    double* own_s = smem + T::kOwn;
    double* far_s = smem + T::kFar;
    double* js = smem + T::kJ;
    double* ss = smem + T::kS;
    double* zs = smem + T::kZ;
    constexpr int FS = EPB * 4 * n;

    const int tid = threadIdx.x;
    const int64_t K = a.n_elements;
    const int64_t Kp = a.field_stride;
    const int64_t e0 = static_cast<int64_t>(blockIdx.x) * EPB;
    const int ne = static_cast<int>((K - e0) < EPB ? (K - e0) : EPB);
    const int ne_copy = (ne + 1) & ~1;
    double* q = a.q;
    double* k = a.k;
    const double* xn = cf.xn;
    const double* lm = cf.lm;
    const double* lp = cf.lp;

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
    for (int i = tid; i < NN; i += T::kThreads) zs[i] = 0.0;
    double x0 = 0, y0 = 0, x1 = 0, y1 = 0, x2 = 0, y2 = 0, x3 = 0, y3 = 0, ce = 1.0;
    if (active) {
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            const int2 lk = a.link[4 * ge + s];
            const double v = (((lk.y >> 2) & 7) == kInterior) ? a.trace_in[((f * Kp + lk.x) * 4 + (lk.y & 3)) * n + (N - m)] : 0.0;
            far_s[f * FS + (e * 4 + s) * n + m] = v;
        }
        const double* c = a.corners + 8 * ge;
        x0 = c[0]; y0 = c[1]; x1 = c[2]; y1 = c[3]; x2 = c[4]; y2 = c[5]; x3 = c[6]; y3 = c[7];
        ce = a.c[ge];
    }
    const MetricLine<false> x_xi(x1 - x0, x2 - x3), y_xi(y1 - y0, y2 - y3);
    const MetricLine<false> x_eta(x3 - x0, x2 - x1), y_eta(y3 - y0, y2 - y1);
    if (active) {
        const double tm = xn[m];
        if (f == 2) {
            for (int sd = m; sd < 4; sd += n) {
                const double at = (sd == 0 || sd == 3) ? -1.0 : 1.0;
                const double dx = (sd == 0 || sd == 2) ? metric<false>(at, x_xi.d0, x_xi.d1) : metric<false>(at, x_eta.d0, x_eta.d1);
                const double dy = (sd == 0 || sd == 2) ? metric<false>(at, y_xi.d0, y_xi.d1) : metric<false>(at, y_eta.d0, y_eta.d1);
                ss[e * 4 + sd] = sqrt(dx * dx + dy * dy);
            }
        }
        const double xe = x_eta(tm), ye = y_eta(tm);
        for (int j = f; j < n; j += 3) {
            const double tj = xn[j];
            js[e * NN + m * n + j] = __drcp_rn(x_xi(tj) * ye - xe * y_xi(tj));
        }
    }
    __syncthreads();
    if (!mbar_wait(bar, a.error, kWaitLimitNs)) return;

    const double* Qe = qs + e * NN;
    const double* Xe = f == 0 ? Qe + 1 * EPB * NN : (f == 1 ? Qe : zs);
    const double* Ye = f == 0 ? Qe + 2 * EPB * NN : (f == 1 ? zs : Qe);
    if (active) {
        const double* Qf = Qe + f * EPB * NN;
        double b = 0.0, t = 0.0, r = 0.0, l = 0.0;
#pragma unroll
        for (int j = 0; j < n; ++j) {
            const double qr = Qf[m * n + j], qc = Qf[j * n + m];
            b = fma(lm[j], qr, b);
            t = fma(lp[j], qr, t);
            r = fma(lp[j], qc, r);
            l = fma(lm[j], qc, l);
        }
        double* o = own_s + f * FS + e * 4 * n;
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
            const double2 nv = a.normal[4 * ge + s];
            const int o = (e * 4 + s) * n + m;
            const double op = own_s[o], ou = own_s[FS + o], ov = own_s[2 * FS + o];
            double fp_, fu_, fv_, cface = ce;
            if (kind == kInterior) {
                fp_ = far_s[o];
                fu_ = far_s[FS + o];
                fv_ = far_s[2 * FS + o];
                cface = 0.5 * (ce + a.c[lk.x]);
            } else if (kind == kMirror || kind == kCopy) {
                const double gsc = a.gscale[4 * ge + s];
                fp_ = op * gsc;
                const double gu = ou * gsc, gv = ov * gsc;
                if (kind == kMirror) {
                    const double tx = -nv.y, ty = nv.x;
                    const double l0 = -(gu * nv.x + gv * nv.y);
                    const double l1 = gu * tx + gv * ty;
                    fu_ = nv.x * l0 + tx * l1;
                    fv_ = nv.y * l0 + ty * l1;
                } else {
                    fu_ = gu;
                    fv_ = gv;
                }
            } else {
                fp_ = fu_ = fv_ = 0.0;
            }
            const double Lp = role ? fp_ : op, Lu = role ? fu_ : ou, Lv = role ? fv_ : ov;
            const double Rp = role ? op : fp_, Ru = role ? ou : fu_, Rv = role ? ov : fv_;
            const double wL = Lp + (Lu * nv.x + Lv * nv.y);
            const double wR = Rp - (Ru * nv.x + Rv * nv.y);
            const double sc = (role ? -ss[e * 4 + s] : ss[e * 4 + s]) * cface;
            const double sum = wL + wR;
            far_s[o] = sc * ((wL - wR) * 0.5);
            far_s[FS + o] = sc * (nv.x * sum * 0.5);
            far_s[2 * FS + o] = sc * (nv.y * sum * 0.5);
        }
    }
    __syncthreads();

    const double* Dh = cf.dhat;
    const double* iw = cf.iw;
    const double* F = far_s + f * FS + e * 4 * n;

    if (active) {
        const int j = m;
        double col[n];
#pragma unroll
        for (int i = 0; i < n; ++i) col[i] = y_eta(xn[i]) * Xe[i * n + j] - x_eta(xn[i]) * Ye[i * n + j];
        const double fr = F[1 * n + j], fl3 = F[3 * n + (N - j)];
        double* G = gs + (f * EPB + e) * NN + j;
#pragma unroll
        for (int i = 0; i < n; ++i) {
            double acc = 0.0;
#pragma unroll
            for (int mm = 0; mm < n; ++mm) acc = fma(Dh[i * n + mm], col[mm], acc);
            G[i * n] = -fma(acc, ce, (fr * lp[i] + fl3 * lm[i]) * iw[i]);
        }
    }
    __syncthreads();

    if (active) {
        const int i = m;
        double line[n];
#pragma unroll
        for (int j = 0; j < n; ++j) line[j] = -y_xi(xn[j]) * Xe[i * n + j] + x_xi(xn[j]) * Ye[i * n + j];
        const double ft = F[2 * n + (N - i)], fb = F[0 * n + i];
        double* G = gs + (f * EPB + e) * NN + i * n;
        const double* jrow = js + e * NN + i * n;
#pragma unroll
        for (int j = 0; j < n; ++j) {
            double acc = 0.0;
#pragma unroll
            for (int mm = 0; mm < n; ++mm) acc = fma(Dh[j * n + mm], line[mm], acc);
            G[j] = (G[j] - fma(acc, ce, (ft * lp[j] + fb * lm[j]) * iw[j])) * jrow[j];
        }
    }
    __syncthreads();

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
            const double kn = a.first ? G : fma(a.rk_a, kold[c], G);
            const double qo = qs[ff * EPB * NN + r];
            const double qn = fma(a.gdt, kn, qo);
            const int64_t gi = (ff * Kp + e0) * NN + r;
            if (a.q_save) a.q_save[gi] = qo;
            k[gi] = kn;
            q[gi] = qn;
            qs[ff * EPB * NN + r] = qn;
            if (a.G_out) a.G_out[gi] = G;
        }
    }
    __syncthreads();

    if (active) {
        const double* row = qs + (f * EPB + e) * NN + m * n;
        const double* cl = qs + (f * EPB + e) * NN + m;
        double b = 0.0, t = 0.0, r = 0.0, l = 0.0;
#pragma unroll
        for (int j = 0; j < n; ++j) {
            b = fma(lm[j], row[j], b);
            t = fma(lp[j], row[j], t);
            r = fma(lp[j], cl[j * n], r);
            l = fma(lm[j], cl[j * n], l);
        }
        double* to = a.trace_out + (f * Kp + ge) * 4 * n;
        to[0 * n + m] = b;
        to[2 * n + (N - m)] = t;
        to[1 * n + m] = r;
        to[3 * n + (N - m)] = l;
    }
    if (a.samples && tid < 32) {
        for (int r = 0; r < a.rec.n; ++r) {
            const int64_t el = a.rec.elem[r] - e0;
            if (el < 0 || el >= ne) continue;
            const double v = receiver_value<NN>(a.rec.w + static_cast<int64_t>(r) * NN, qs + el * NN, tid);
            if (tid == 0) a.samples[r] = v;
        }
    }
}

// ---------------------------------------------------------------------------
// Adjoint stage. Tile of EPB elements, one thread per (field, element, line)
// as the forward. Shared memory (doubles):
template <int N>
struct AdjTile {
    static constexpr int n = N + 1;
    static constexpr int NN = n * n;
    static constexpr int per_element_doubles = 11 * NN + 43 * n + 9;
    static constexpr int fixed_doubles = NN + kMaxReceivers + 2;
    static constexpr int by_smem = (60 * 1024 / 8 - fixed_doubles) / per_element_doubles;
    static constexpr int by_threads = 256 / (3 * n);
    static constexpr int raw = by_smem < by_threads ? by_smem : by_threads;
    static constexpr int EPB = raw >= 2 ? (raw & ~1) : 2;
    static constexpr int kThreads = (3 * EPB * n + 31) / 32 * 32;
    static constexpr int kNodeIters = (3 * EPB * NN + kThreads - 1) / kThreads;
    static constexpr int FS = EPB * 4 * n;
    static constexpr int kL = 0;                   // [3][EPB][NN] lq (bulk copy), then lq + volume transpose
    static constexpr int kQ = kL + 3 * EPB * NN;   // [3][EPB][NN] forward stage input qs (bulk copy)
    static constexpr int kNu = kQ + 3 * EPB * NN;  // [3][EPB][NN] nu = -mu / J, later nu'
    static constexpr int kTp = kNu + 3 * EPB * NN; // [EPB][NN] second accumulator of the pressure's transpose
    static constexpr int kJ = kTp + EPB * NN;      // [EPB][NN] 1/J
    static constexpr int kOwn = kJ + EPB * NN;     // [3][EPB][4][n] side traces of qs
    static constexpr int kEll = kOwn + 3 * FS;     // [3][EPB][4][n] lift transpose, then own-trace adjoint, then next lift transpose
    static constexpr int kFar = kEll + 3 * FS;     // [3][EPB][4][n] neighbours' adjoint far traces
    static constexpr int kUp = kFar + 3 * FS;      // [EPB][4][n] flux part of the c-derivative per side node
    static constexpr int kVd = kUp + FS;           // [3][EPB][n] volume part of the c-derivative per line
    static constexpr int kS = kVd + 3 * EPB * n;   // [EPB][4] edge metric
    static constexpr int kCf = kS + 4 * EPB;       // [EPB][4] face speed
    static constexpr int kMask = kCf + 4 * EPB;    // [EPB] receivers of each element (bit mask)
    static constexpr int kZ = kMask + EPB;         // [NN] zeros
    static constexpr int kRes = kZ + NN;           // [kMaxReceivers] weighted residuals
    static constexpr int kBar = kRes + kMaxReceivers;
    static constexpr int kDoubles = kBar + 2;
    static constexpr size_t kBytes = sizeof(double) * kDoubles;
    static_assert(kDoubles <= EPB * per_element_doubles + fixed_doubles, "layout exceeds its budget");
};

template <int N>
__global__ void __launch_bounds__(AdjTile<N>::kThreads) adjoint_stage_kernel(AdjointStageArgs a, const __grid_constant__ AdjCoeffs<N> cf) {
    using T = AdjTile<N>;
    constexpr int n = T::n, NN = T::NN, EPB = T::EPB, FS = T::FS;
    extern __shared__ __align__(128) double smem[];
    double* ls = smem + T::kL;
    double* qs = smem + T::kQ;
    double* nu = smem + T::kNu;
    double* tp = smem + T::kTp;
    double* js = smem + T::kJ;
    double* own_s = smem + T::kOwn;
    double* ell = smem + T::kEll;
    double* far_s = smem + T::kFar;
    double* up = smem + T::kUp;
    double* vd = smem + T::kVd;
    double* ss = smem + T::kS;
    double* cfs = smem + T::kCf;
    unsigned long long* rmask = reinterpret_cast<unsigned long long*>(smem + T::kMask);
    double* zs = smem + T::kZ;
    double* res = smem + T::kRes;
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + T::kBar);

    const int tid = threadIdx.x;
    const int64_t K = a.n_elements;
    const int64_t Kp = a.field_stride;
    const int64_t e0 = static_cast<int64_t>(blockIdx.x) * EPB;
    const int ne = static_cast<int>((K - e0) < EPB ? (K - e0) : EPB);
    const int ne_copy = (ne + 1) & ~1;
    const double* xn = cf.xn;
    const double* lm = cf.lm;
    const double* lp = cf.lp;
    const double* lmw = cf.lmw;
    const double* lpw = cf.lpw;
    const double* Dh = cf.dhat;

    const int f = tid / (EPB * n);
    const int rr = tid - f * (EPB * n);
    const int e = rr / n;
    const int m = rr - e * n;
    const bool active = f < 3 && e < ne;
    const int64_t ge = e0 + e;

    // Prologue: bulk copies of the lq and qs tiles; adjoint far traces of
    // the neighbours, metrics, J, edge metrics and face speeds.
    if (tid == 0) {
        mbar_init(bar, 1);
        mbar_fence_init();
        const uint32_t bytes = static_cast<uint32_t>(ne_copy * NN * sizeof(double));
        mbar_expect_tx(bar, 6 * bytes);
        for (int ff = 0; ff < 3; ++ff) {
            bulk_load(ls + ff * EPB * NN, a.lq + (ff * Kp + e0) * NN, bytes, bar);
            bulk_load(qs + ff * EPB * NN, a.qs + (ff * Kp + e0) * NN, bytes, bar);
        }
    }
    for (int i = tid; i < NN; i += T::kThreads) zs[i] = 0.0;
    for (int i = tid; i < EPB * NN; i += T::kThreads) tp[i] = 0.0;
    if (tid < EPB) rmask[tid] = 0ull;
    double x0 = 0, y0 = 0, x1 = 0, y1 = 0, x2 = 0, y2 = 0, x3 = 0, y3 = 0, ce = 1.0;
    if (active) {
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            const int2 lk = a.link[4 * ge + s];
            const double v = (((lk.y >> 2) & 7) == kInterior) ? a.atr_in[((f * Kp + lk.x) * 4 + (lk.y & 3)) * n + (N - m)] : 0.0;
            far_s[f * FS + (e * 4 + s) * n + m] = v;
        }
        const double* c = a.corners + 8 * ge;
        x0 = c[0]; y0 = c[1]; x1 = c[2]; y1 = c[3]; x2 = c[4]; y2 = c[5]; x3 = c[6]; y3 = c[7];
        ce = a.c[ge];
    }
    const MetricLine<false> x_xi(x1 - x0, x2 - x3), y_xi(y1 - y0, y2 - y3);
    const MetricLine<false> x_eta(x3 - x0, x2 - x1), y_eta(y3 - y0, y2 - y1);
    if (active) {
        const double tm = xn[m];
        if (f == 2) {
            for (int sd = m; sd < 4; sd += n) {
                const double at = (sd == 0 || sd == 3) ? -1.0 : 1.0;
                const double dx = (sd == 0 || sd == 2) ? metric<false>(at, x_xi.d0, x_xi.d1) : metric<false>(at, x_eta.d0, x_eta.d1);
                const double dy = (sd == 0 || sd == 2) ? metric<false>(at, y_xi.d0, y_xi.d1) : metric<false>(at, y_eta.d0, y_eta.d1);
                ss[e * 4 + sd] = sqrt(dx * dx + dy * dy);
                const int2 lk = a.link[4 * ge + sd];
                cfs[e * 4 + sd] = (((lk.y >> 2) & 7) == kInterior) ? 0.5 * (ce + a.c[lk.x]) : ce;
            }
        }
        const double xe = x_eta(tm), ye = y_eta(tm);
        for (int j = f; j < n; j += 3) {
            const double tj = xn[j];
            js[e * NN + m * n + j] = __drcp_rn(x_xi(tj) * ye - xe * y_xi(tj));
        }
    }
    __syncthreads();
    if (!mbar_wait(bar, a.error, kWaitLimitNs)) return;

    // Node pass: mu = lk + gdt lq; lk = a mu (kept in registers for mu');
    // nu = -mu / J. One warp evaluates the misfit residuals of the
    // receivers in the tile at the state qs.
    double kn[T::kNodeIters];
#pragma unroll
    for (int c = 0; c < T::kNodeIters; ++c) {
        const int idx = tid + c * T::kThreads;
        const int ff = idx / (EPB * NN), r = idx - ff * (EPB * NN);
        kn[c] = 0.0;
        if (ff < 3 && r < ne * NN) {
            const int64_t gi = (ff * Kp + e0) * NN + r;
            const double mu = fma(a.gdt, ls[ff * EPB * NN + r], a.lk[gi]);
            kn[c] = a.rk_a * mu;
            a.lk[gi] = kn[c];
            nu[ff * EPB * NN + r] = -mu * js[r];
        }
    }
    if (a.inject && tid < 32) {
        for (int r = 0; r < a.rec.n; ++r) {
            const int64_t el = a.rec.elem[r] - e0;
            if (el < 0 || el >= ne) continue;
            const double v = receiver_value<NN>(a.rec.w + static_cast<int64_t>(r) * NN, qs + el * NN, tid);
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
    const double* Qe = qs + e * NN;
    const double* Xe = f == 0 ? Qe + 1 * EPB * NN : (f == 1 ? Qe : zs);
    const double* Ye = f == 0 ? Qe + 2 * EPB * NN : (f == 1 ? zs : Qe);
    double* O1 = f == 0 ? ls + (1 * EPB + e) * NN : (f == 1 ? ls + e * NN : tp + e * NN);
    double* O2 = ls + (2 * EPB + e) * NN;  // f = p only
    const double* Nf = nu + (f * EPB + e) * NN;
    double vdot = 0.0;
    // xi columns (eta index j = m): alpha = Dhat^T nu(:, j); lift transpose
    // of sides 1 and 3; the side traces of qs.
    if (active) {
        const int j = m;
        double col[n];
#pragma unroll
        for (int i = 0; i < n; ++i) col[i] = Nf[i * n + j];
        double l1 = 0.0, l3 = 0.0;
#pragma unroll
        for (int i = 0; i < n; ++i) {
            l1 = fma(col[i], lpw[i], l1);
            l3 = fma(col[i], lmw[i], l3);
        }
        double* L = ell + f * FS + e * 4 * n;
        L[1 * n + j] = l1;
        L[3 * n + (N - j)] = l3;
#pragma unroll
        for (int mm = 0; mm < n; ++mm) {
            double al = 0.0;
#pragma unroll
            for (int i = 0; i < n; ++i) al = fma(Dh[i * n + mm], col[i], al);
            const double A = y_eta(xn[mm]) * al, B = -x_eta(xn[mm]) * al;
            const int node = mm * n + j;
            vdot = fma(Xe[node], A, fma(Ye[node], B, vdot));
            O1[node] = fma(ce, f == 2 ? B : A, O1[node]);
            if (f == 0) O2[node] = fma(ce, B, O2[node]);
        }
        const double* Qf = Qe + f * EPB * NN;
        double b = 0.0, t = 0.0, r = 0.0, l = 0.0;
#pragma unroll
        for (int jj = 0; jj < n; ++jj) {
            const double qr = Qf[m * n + jj], qc = Qf[jj * n + m];
            b = fma(lm[jj], qr, b);
            t = fma(lp[jj], qr, t);
            r = fma(lp[jj], qc, r);
            l = fma(lm[jj], qc, l);
        }
        double* o = own_s + f * FS + e * 4 * n;
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
        double row[n];
#pragma unroll
        for (int j = 0; j < n; ++j) row[j] = Nf[i * n + j];
        double l2 = 0.0, l0 = 0.0;
#pragma unroll
        for (int j = 0; j < n; ++j) {
            l2 = fma(row[j], lpw[j], l2);
            l0 = fma(row[j], lmw[j], l0);
        }
        double* L = ell + f * FS + e * 4 * n;
        L[2 * n + (N - i)] = l2;
        L[0 * n + i] = l0;
#pragma unroll
        for (int mm = 0; mm < n; ++mm) {
            double be = 0.0;
#pragma unroll
            for (int j = 0; j < n; ++j) be = fma(Dh[j * n + mm], row[j], be);
            const double A = -y_xi(xn[mm]) * be, B = x_xi(xn[mm]) * be;
            const int node = i * n + mm;
            vdot = fma(Xe[node], A, fma(Ye[node], B, vdot));
            O1[node] = fma(ce, f == 2 ? B : A, O1[node]);
            if (f == 0) O2[node] = fma(ce, B, O2[node]);
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
            const double2 nv = a.normal[4 * ge + s];
            const int o = (e * 4 + s) * n + m;
            const double cface = cfs[e * 4 + s];
            const double sc = (role ? -ss[e * 4 + s] : ss[e * 4 + s]) * cface;
            const double pp = sc * ell[o], pu = sc * ell[FS + o], pv = sc * ell[2 * FS + o];
            const double dn = 0.5 * (nv.x * pu + nv.y * pv);
            const double wl = fma(0.5, pp, dn), wr = fma(-0.5, pp, dn);
            // adjoints of L = (wl, wl nx, wl ny) and R = (wr, -wr nx, -wr ny)
            const double sl = role ? -wr : wl;  // own trace: R for the right element
            const double sf_ = role ? wl : -wr;
            double tp_ = role ? wr : wl, tu = sl * nv.x, tv = sl * nv.y;
            const double fp_ = role ? wl : wr, fu_ = sf_ * nv.x, fv_ = sf_ * nv.y;
            if (kind == kInterior) {
                tp_ += far_s[o];
                tu += far_s[FS + o];
                tv += far_s[2 * FS + o];
            } else if (kind == kMirror || kind == kCopy) {
                const double gsc = a.gscale[4 * ge + s];
                double gu = fu_, gv = fv_;
                if (kind == kMirror) {
                    const double tx = -nv.y, ty = nv.x;
                    const double l0 = -(fu_ * nv.x + fv_ * nv.y);
                    const double l1 = fu_ * tx + fv_ * ty;
                    gu = nv.x * l0 + tx * l1;
                    gv = nv.y * l0 + ty * l1;
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
    for (int c = 0; c < T::kNodeIters; ++c) {
        const int idx = tid + c * T::kThreads;
        const int ff = idx / (EPB * NN), r = idx - ff * (EPB * NN);
        if (ff < 3 && r < ne * NN) {
            const int el = r / NN, node = r - el * NN;
            const int i = node / n, j = node - i * n;
            const double* Lo = ell + ff * FS + el * 4 * n;
            double v = ls[ff * EPB * NN + r];
            if (ff == 0) v += tp[r];
            v = fma(lm[j], Lo[0 * n + i], v);
            v = fma(lp[j], Lo[2 * n + (N - i)], v);
            v = fma(lp[i], Lo[1 * n + j], v);
            v = fma(lm[i], Lo[3 * n + (N - j)], v);
            if (ff == 0) {
                unsigned long long mask = rmask[el];
                while (mask) {
                    const int rc = __ffsll(static_cast<long long>(mask)) - 1;
                    mask &= mask - 1;
                    v = fma(res[rc], a.rec.w[static_cast<int64_t>(rc) * NN + node], v);
                }
            }
            a.lq[(ff * Kp + e0) * NN + r] = v;
            nu[ff * EPB * NN + r] = -fma(a.gdt_next, v, kn[c]) * js[r];
        }
    }
    __syncthreads();

    // Lift transpose of nu' on the four sides (column m: sides 1, 3; row m:
    // sides 2, 0); per element, the c-derivative accumulators.
    if (active) {
        const double* Nn = nu + (f * EPB + e) * NN;
        double l1 = 0.0, l3 = 0.0, l2 = 0.0, l0 = 0.0;
#pragma unroll
        for (int i = 0; i < n; ++i) {
            const double cv = Nn[i * n + m], rv = Nn[m * n + i];
            l1 = fma(cv, lpw[i], l1);
            l3 = fma(cv, lmw[i], l3);
            l2 = fma(rv, lpw[i], l2);
            l0 = fma(rv, lmw[i], l0);
        }
        double* L = ell + f * FS + e * 4 * n;
        L[1 * n + m] = l1;
        L[3 * n + (N - m)] = l3;
        L[2 * n + (N - m)] = l2;
        L[0 * n + m] = l0;
    }
    if (tid < ne) {
        double vsum = 0.0;
        for (int ff = 0; ff < 3; ++ff)
            for (int i = 0; i < n; ++i) vsum += vd[(ff * EPB + tid) * n + i];
        double* A = a.acc + (e0 + tid) * 5;
        A[0] += vsum;
        for (int s = 0; s < 4; ++s) {
            double us = 0.0;
            for (int i = 0; i < n; ++i) us += up[(tid * 4 + s) * n + i];
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
            const double2 nv = a.normal[4 * ge + s];
            const int o = (e * 4 + s) * n + m;
            const double sc = (role ? -ss[e * 4 + s] : ss[e * 4 + s]) * cfs[e * 4 + s];
            const double pp = sc * ell[o], pu = sc * ell[FS + o], pv = sc * ell[2 * FS + o];
            const double dn = 0.5 * (nv.x * pu + nv.y * pv);
            const double wl = fma(0.5, pp, dn), wr = fma(-0.5, pp, dn);
            const double sf_ = role ? wl : -wr;
            double* to = a.atr_out + (ge * 4 + s) * n + m;
            to[0] = role ? wl : wr;
            to[Kp * 4 * n] = sf_ * nv.x;
            to[2 * Kp * 4 * n] = sf_ * nv.y;
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
template <int N>
static cudaError_t prepare_speed_t() {
    cudaError_t err = cudaFuncSetAttribute(speed_stage_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(Tile<N>::kBytes));
    if (err != cudaSuccess) return err;
    return cudaFuncSetAttribute(adjoint_stage_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(AdjTile<N>::kBytes));
}

template <int N>
static cudaError_t launch_speed_stage_t(const SpeedStageArgs& a, cudaStream_t stream) {
    using T = Tile<N>;
    speed_stage_kernel<N><<<static_cast<unsigned>((a.n_elements + T::EPB - 1) / T::EPB), T::kThreads, T::kBytes, stream>>>(a, make_speed_coeffs<N>());
    return cudaGetLastError();
}

template <int N>
static cudaError_t launch_adjoint_stage_t(const AdjointStageArgs& a, cudaStream_t stream) {
    using T = AdjTile<N>;
    adjoint_stage_kernel<N><<<static_cast<unsigned>((a.n_elements + T::EPB - 1) / T::EPB), T::kThreads, T::kBytes, stream>>>(a, make_adj_coeffs<N>());
    return cudaGetLastError();
}

template <int N>
static int adjoint_epb_t() {
    return AdjTile<N>::EPB;
}

#define NDG_SPEED_DISPATCH(FN, N_, ...)        \
    switch (N_) {                              \
        case 1: return FN<1>(__VA_ARGS__);     \
        case 2: return FN<2>(__VA_ARGS__);     \
        case 3: return FN<3>(__VA_ARGS__);     \
        case 4: return FN<4>(__VA_ARGS__);     \
        case 5: return FN<5>(__VA_ARGS__);     \
        case 6: return FN<6>(__VA_ARGS__);     \
        case 7: return FN<7>(__VA_ARGS__);     \
        case 8: return FN<8>(__VA_ARGS__);     \
        case 9: return FN<9>(__VA_ARGS__);     \
        case 10: return FN<10>(__VA_ARGS__);   \
        case 11: return FN<11>(__VA_ARGS__);   \
        case 12: return FN<12>(__VA_ARGS__);   \
        default: break;                        \
    }

cudaError_t prepare_speed_kernels(int N) {
    NDG_SPEED_DISPATCH(prepare_speed_t, N)
    return cudaErrorInvalidValue;
}

cudaError_t launch_speed_stage(int N, const SpeedStageArgs& a, cudaStream_t stream) {
    NDG_SPEED_DISPATCH(launch_speed_stage_t, N, a, stream)
    return cudaErrorInvalidValue;
}

cudaError_t launch_adjoint_stage(int N, const AdjointStageArgs& a, cudaStream_t stream) {
    NDG_SPEED_DISPATCH(launch_adjoint_stage_t, N, a, stream)
    return cudaErrorInvalidValue;
}

int adjoint_elements_per_block(int N) {
    NDG_SPEED_DISPATCH(adjoint_epb_t, N)
    return 0;
}

cudaError_t launch_speed_gradient(const double* acc, const int2* link, int64_t K, double* grad_c, cudaStream_t stream) {
    const int blocks = static_cast<int>(std::min<int64_t>((K + 255) / 256, 148 * 8));
    speed_gradient_kernel<<<blocks, 256, 0, stream>>>(acc, link, K, grad_c);
    return cudaGetLastError();
}

}  // namespace dev
}  // namespace ndg
