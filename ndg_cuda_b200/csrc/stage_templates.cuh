// The fused uniform-order stage kernels (FP64 and the FP32 form), as
// templates over the order N, the rounding mode and the tile size E
// (elements per CTA; 0 = the default of Tile). Instantiated by
// stage_kernels.cu (default tiles) and stage_variants.cu (the autotuner's
// candidate tiles). The design notes are at the top of stage_kernels.cu.
#pragma once

#include "ndg_internal.hpp"
#include "stage_common.cuh"
#include "stage_kernels.cuh"

#include <cuda_runtime.h>

#include <cstdint>

namespace ndg {
namespace dev {

// Tensor-core form of the two contraction passes (TC = true; FP64 with DMMA
// m16n8k4, the FP32 form with 3xTF32 m16n8k8). The tile's 3 EPB (N+1) flux
// lines, in the threads' (field, line, element) order with the element
// fastest, are the M rows of 16-row MMA tiles; the node index along the line
// is K and the output node is N, both padded with zeros:
// out[line][i] = sum_k line[k] Dhat[i][k], so B holds Dhat transposed and
// stays in registers for both passes. With EPB dividing 8, rows g and g + 8
// of lane 4g + t belong to element g mod EPB in every MMA tile, so a lane
// evaluates the metric terms of its lines' element once. Warps take the MMA
// tiles round robin. The line values are formed in registers from the
// shared q tile as in the SIMT passes, and the lift, the sign, 1/J and the
// stores to G follow from the accumulator fragments.
template <int N, int EPB>
struct TcLines {
    static_assert(EPB == 2 || EPB == 4 || EPB == 8, "the tensor-core passes need EPB dividing 8");
    static constexpr int kTiles = (3 * EPB * (N + 1) + 15) / 16;
};

template <int N, bool S, int E, bool TC = false>
__global__ void __launch_bounds__(Tile<N, E>::kThreads, TC ? 0 : Tile<N, E>::kMinBlocks) stage_kernel(StageArgs a, const __grid_constant__ Coeffs<N> cf) {
    static_assert(!(TC && S), "the strict form rounds every operation in the reference's order: no tensor cores");
    using T = Tile<N, E>;
    constexpr int n = T::n, NN = T::NN, EPB = T::EPB;
    // padded strides of the tile (Tile): row pitch, element and field strides
    // of node arrays, element and field strides of side arrays
    constexpr int P = T::P, ES = T::ES, QS = T::QS, SE = T::SE, FS = T::FS;
    extern __shared__ __align__(128) double smem[];
    double* qs = smem + T::kQ;
    double* gs = smem + T::kG;
    double* own_s = smem + T::kOwn;
    double* far_s = smem + T::kFar;  // far traces, then element side fluxes in place
    double* js = smem + T::kJ;
    double* ss = smem + T::kS;
    double* zs = smem + T::kZ;

    const int tid = threadIdx.x;
    const int64_t K = a.n_elements;
    const int64_t Kp = a.field_stride;  // elements per field block (K rounded up to even)
    const int64_t e0 = static_cast<int64_t>(blockIdx.x) * EPB;
    const int ne = static_cast<int>((K - e0) < EPB ? (K - e0) : EPB);
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

    // Line threads: (field f, line or node index m, element e of the tile),
    // e fastest (the order the bank-conflict-free strides assume).
    const int f = tid / (EPB * n);
    const int rr = tid - f * (EPB * n);
    const int m = rr / EPB;
    const int e = rr - m * EPB;
    const bool active = f < 3 && e < ne;
    const int64_t ge = e0 + e;

    // Prologue: 8-byte asynchronous copies place the q tile in the padded
    // layout (coalesced reads; a padded tile is not one contiguous range).
    // Warps take (field, element) blocks, lanes their nodes.
    const int warp = tid >> 5, lane = tid & 31;
    int lane_node[T::kLaneIters];  // padded offsets of this lane's nodes within an element
#pragma unroll
    for (int it = 0; it < T::kLaneIters; ++it) lane_node[it] = T::node(lane + 32 * it);
#pragma unroll
    for (int bi = 0; bi < T::kBlockIters; ++bi) {
        const int b = warp + bi * T::kWarps, ff = b / EPB, el = b - ff * EPB;
        if (b < 3 * EPB && el < ne) {
            const double* src = q + (ff * Kp + e0 + el) * NN;
            double* dst = qs + ff * QS + el * ES;
#pragma unroll
            for (int it = 0; it < T::kLaneIters; ++it)
                if (lane + 32 * it < NN) cp_async8(dst + lane_node[it], src + lane + 32 * it);
        }
    }
    // Far traces: the previous stage wrote each neighbour's trace into this
    // element's far slots ([field][element][side][node], 4 (N+1) contiguous
    // values per field and element), so they arrive like the q tile, with
    // no link to follow.
#pragma unroll
    for (int bi = 0; bi < T::kBlockIters; ++bi) {
        const int b = warp + bi * T::kWarps, ff = b / EPB, el = b - ff * EPB;
        if (b < 3 * EPB && el < ne) {
            const double* src = tr_in + (ff * Kp + e0 + el) * 4 * n;
            double* dst = far_s + ff * FS + el * SE;
#pragma unroll
            for (int it = 0; it < (4 * n + 31) / 32; ++it)
                if (lane + 32 * it < 4 * n) cp_async8(dst + lane + 32 * it, src + lane + 32 * it);
        }
    }
    for (int i = tid; i < n * P; i += T::kThreads) zs[i] = 0.0;
    // Element metrics, edge metrics and J.
    double x0 = 0, y0 = 0, x1 = 0, y1 = 0, x2 = 0, y2 = 0, x3 = 0, y3 = 0;
    if (active) {
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
            js[e * ES + m * P + j] = S ? jac : __drcp_rn(jac);
        }
    }
    cp_async_wait_all();
    __syncthreads();  // q tile, far traces, zeros, edge metrics, J

    // Own side traces of this thread's field (Element2D_t.cpp:86-125):
    // bottom and top from row m, right and left from column m.
    // The flux lines take (X, Y) = (u, v), (p, 0), (0, p) for f = 0, 1, 2:
    // x_flux = (c u, p, 0), y_flux = (c v, 0, p) (Solver2D_t.cpp:31-37).
    const double* Qe = qs + e * ES;
    const double* Xe = f == 0 ? Qe + 1 * QS : (f == 1 ? Qe : zs);
    const double* Ye = f == 0 ? Qe + 2 * QS : (f == 1 ? zs : Qe);
    if (active) {
        const double* Qf = Qe + f * QS;
        double b = 0.0, t = 0.0, r = 0.0, l = 0.0;
#pragma unroll
        for (int j = 0; j < n; ++j) {
            const double qr = Qf[m * P + j], qc = Qf[j * P + m];
            b = madd<S>(b, lm[j], qr);
            t = madd<S>(t, lp[j], qr);
            r = madd<S>(r, lp[j], qc);
            l = madd<S>(l, lm[j], qc);
        }
        double* o = own_s + f * FS + e * SE;
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
            const int o = e * SE + s * n + m;
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
    const double* F = far_s + f * FS + e * SE;  // this thread's field, element side fluxes

    // Tensor-core passes: the lane's fragments of Dhat transposed, its lift
    // weights and the metric terms of its rows' element.
    using TT = TcTable64<N>;
    [[maybe_unused]] double tb[TT::KS][TT::NT], tlpw[TT::NT][2], tlmw[TT::NT][2], tcx[8];
    [[maybe_unused]] const int tg = lane >> 2, tt = lane & 3, tel = tg % (EPB < 8 ? EPB : 8);
    [[maybe_unused]] const bool tlive = tel < ne;
    if constexpr (TC) {
        const double* tab = a.tc64;
#pragma unroll
        for (int s = 0; s < TT::KS; ++s)
#pragma unroll
            for (int u = 0; u < TT::NT; ++u) tb[s][u] = tab[TT::kB + (s * TT::NT + u) * 32 + lane];
#pragma unroll
        for (int u = 0; u < TT::NT; ++u)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                tlpw[u][h] = tab[TT::kLPW + (u * 2 + h) * 32 + lane];
                tlmw[u][h] = tab[TT::kLMW + (u * 2 + h) * 32 + lane];
            }
        const double* cc = a.corners + 8 * (e0 + tel);
#pragma unroll
        for (int k = 0; k < 8; ++k) tcx[k] = tlive ? cc[k] : 0.0;
    }

    // xi pass (eta index j = m): contravariant flux line eta_y X - eta_x Y
    // (Solver2D_t.cpp:72-80), Dhat . line + lift, G = -(...) (:82-101); G column j.
    if constexpr (TC) {
        const MetricLine<false> mx_eta(tcx[6] - tcx[0], tcx[4] - tcx[2]), my_eta(tcx[7] - tcx[1], tcx[5] - tcx[3]);
        double ka[TT::KS], kb[TT::KS];  // eta_y, eta_x at the lane's nodes k = 4s + t (0 beyond N)
#pragma unroll
        for (int s = 0; s < TT::KS; ++s) {
            const double xv = a.tc64[TT::kXK + s * 32 + lane];
            const bool kv = 4 * s + tt < n;
            ka[s] = kv ? my_eta(xv) : 0.0;
            kb[s] = kv ? mx_eta(xv) : 0.0;
        }
        for (int mt = warp; mt < TcLines<N, EPB>::kTiles; mt += T::kWarps) {
            int rf[2], rj[2];
            bool rv[2];
            double av[2][TT::KS];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int qq = (16 * mt + tg + 8 * h) / EPB;
                rf[h] = qq / n;
                rj[h] = qq - rf[h] * n;
                rv[h] = tlive && rf[h] < 3;
                const double* Xr = rf[h] == 0 ? qs + QS + tel * ES : (rf[h] == 1 ? qs + tel * ES : zs);
                const double* Yr = rf[h] == 0 ? qs + 2 * QS + tel * ES : (rf[h] == 1 ? zs : qs + tel * ES);
#pragma unroll
                for (int s = 0; s < TT::KS; ++s) {
                    const int k = 4 * s + tt;
                    av[h][s] = (rv[h] && k < n) ? ka[s] * Xr[k * P + rj[h]] - kb[s] * Yr[k * P + rj[h]] : 0.0;
                }
            }
            double acc[TT::NT][4];
#pragma unroll
            for (int u = 0; u < TT::NT; ++u) {
                acc[u][0] = acc[u][1] = acc[u][2] = acc[u][3] = 0.0;
#pragma unroll
                for (int s = 0; s < TT::KS; ++s) dmma_16x8x4(acc[u], av[0][s], av[1][s], tb[s][u]);
            }
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                if (!rv[h]) continue;
                const double* Fr = far_s + rf[h] * FS + tel * SE;
                const double fr = Fr[1 * n + rj[h]], fl3 = Fr[3 * n + (N - rj[h])];
                double* G = gs + rf[h] * QS + tel * ES + rj[h];
#pragma unroll
                for (int u = 0; u < TT::NT; ++u)
#pragma unroll
                    for (int c = 0; c < 2; ++c) {
                        const int i = 8 * u + 2 * tt + c;
                        if (i < n) G[i * P] = -(acc[u][2 * h + c] + fr * tlpw[u][c] + fl3 * tlmw[u][c]);
                    }
            }
        }
    } else if (active) {
        const int j = m;
        double col[n];
#pragma unroll
        for (int i = 0; i < n; ++i) col[i] = sub<S>(mul<S>(y_eta(xn[i]), Xe[i * P + j]), mul<S>(x_eta(xn[i]), Ye[i * P + j]));
        const double fr = F[1 * n + j], fl3 = F[3 * n + (N - j)];
        double* G = gs + f * QS + e * ES + j;
        constexpr bool EO = !S && N >= kEvenOddMinOrder64;
        if constexpr (EO) {
            dhat_even_odd<n>(cf.ea, cf.so, col, [&](int i, double y) { G[i * P] = -(y + (fr * lp[i] + fl3 * lm[i]) * iw[i]); });
        }
        // Otherwise the plain product (in the reference's order in the strict
        // form), up to 9 outputs accumulating side by side (independent FMA
        // chains).
        constexpr int GR = n < 9 ? n : 9;
#pragma unroll
        for (int i0 = 0; i0 < (EO ? 0 : n); i0 += GR) {
            double acc[GR];
#pragma unroll
            for (int g = 0; g < GR; ++g) acc[g] = 0.0;
#pragma unroll
            for (int mm = 0; mm < n; ++mm)
#pragma unroll
                for (int g = 0; g < GR; ++g)
                    if (i0 + g < n) acc[g] = madd<S>(acc[g], Dh[(i0 + g) * n + mm], col[mm]);
#pragma unroll
            for (int g = 0; g < GR; ++g) {
                const int i = i0 + g;
                if (i >= n) break;
                const double lift = S ? __ddiv_rn(add<S>(mul<S>(fr, lp[i]), mul<S>(fl3, lm[i])), w[i]) : (fr * lp[i] + fl3 * lm[i]) * iw[i];
                G[i * P] = -add<S>(acc[g], lift);
            }
        }
    }
    __syncthreads();

    // eta pass (xi index i = m): line -xi_y X + xi_x Y (Solver2D_t.cpp:103-113),
    // G = (G - (Dhat . line + lift)) / J (:114-133); G row i.
    if constexpr (TC) {
        const MetricLine<false> mx_xi(tcx[2] - tcx[0], tcx[4] - tcx[6]), my_xi(tcx[3] - tcx[1], tcx[5] - tcx[7]);
        double ka[TT::KS], kb[TT::KS];  // -xi_y, xi_x at the lane's nodes k = 4s + t (0 beyond N)
#pragma unroll
        for (int s = 0; s < TT::KS; ++s) {
            const double xv = a.tc64[TT::kXK + s * 32 + lane];
            const bool kv = 4 * s + tt < n;
            ka[s] = kv ? -my_xi(xv) : 0.0;
            kb[s] = kv ? mx_xi(xv) : 0.0;
        }
        for (int mt = warp; mt < TcLines<N, EPB>::kTiles; mt += T::kWarps) {
            int rf[2], ri[2];
            bool rv[2];
            double av[2][TT::KS];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int qq = (16 * mt + tg + 8 * h) / EPB;
                rf[h] = qq / n;
                ri[h] = qq - rf[h] * n;
                rv[h] = tlive && rf[h] < 3;
                const double* Xr = rf[h] == 0 ? qs + QS + tel * ES : (rf[h] == 1 ? qs + tel * ES : zs);
                const double* Yr = rf[h] == 0 ? qs + 2 * QS + tel * ES : (rf[h] == 1 ? zs : qs + tel * ES);
#pragma unroll
                for (int s = 0; s < TT::KS; ++s) {
                    const int k = 4 * s + tt;
                    av[h][s] = (rv[h] && k < n) ? ka[s] * Xr[ri[h] * P + k] + kb[s] * Yr[ri[h] * P + k] : 0.0;
                }
            }
            double acc[TT::NT][4];
#pragma unroll
            for (int u = 0; u < TT::NT; ++u) {
                acc[u][0] = acc[u][1] = acc[u][2] = acc[u][3] = 0.0;
#pragma unroll
                for (int s = 0; s < TT::KS; ++s) dmma_16x8x4(acc[u], av[0][s], av[1][s], tb[s][u]);
            }
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                if (!rv[h]) continue;
                const double* Fr = far_s + rf[h] * FS + tel * SE;
                const double ft = Fr[2 * n + (N - ri[h])], fb = Fr[0 * n + ri[h]];
                double* G = gs + rf[h] * QS + tel * ES + ri[h] * P;
                const double* jrow = js + tel * ES + ri[h] * P;
#pragma unroll
                for (int u = 0; u < TT::NT; ++u)
#pragma unroll
                    for (int c = 0; c < 2; ++c) {
                        const int j = 8 * u + 2 * tt + c;
                        if (j < n) G[j] = (G[j] - (acc[u][2 * h + c] + ft * tlpw[u][c] + fb * tlmw[u][c])) * jrow[j];
                    }
            }
        }
    } else if (active) {
        const int i = m;
        double line[n];
#pragma unroll
        for (int j = 0; j < n; ++j) line[j] = add<S>(mul<S>(-y_xi(xn[j]), Xe[i * P + j]), mul<S>(x_xi(xn[j]), Ye[i * P + j]));
        const double ft = F[2 * n + (N - i)], fb = F[0 * n + i];
        double* G = gs + f * QS + e * ES + i * P;
        const double* jrow = js + e * ES + i * P;
        constexpr bool EO = !S && N >= kEvenOddMinOrder64;
        if constexpr (EO) {
            dhat_even_odd<n>(cf.ea, cf.so, line, [&](int j, double y) { G[j] = (G[j] - (y + (ft * lp[j] + fb * lm[j]) * iw[j])) * jrow[j]; });
        }
        constexpr int GR = n < 9 ? n : 9;  // otherwise as in the xi pass
#pragma unroll
        for (int j0 = 0; j0 < (EO ? 0 : n); j0 += GR) {
            double acc[GR];
#pragma unroll
            for (int g = 0; g < GR; ++g) acc[g] = 0.0;
#pragma unroll
            for (int mm = 0; mm < n; ++mm)
#pragma unroll
                for (int g = 0; g < GR; ++g)
                    if (j0 + g < n) acc[g] = madd<S>(acc[g], Dh[(j0 + g) * n + mm], line[mm]);
#pragma unroll
            for (int g = 0; g < GR; ++g) {
                const int j = j0 + g;
                if (j >= n) break;
                const double lift = S ? __ddiv_rn(add<S>(mul<S>(ft, lp[j]), mul<S>(fb, lm[j])), w[j]) : (ft * lp[j] + fb * lm[j]) * iw[j];
                const double num = sub<S>(G[j], add<S>(acc[g], lift));
                G[j] = S ? __ddiv_rn(num, jrow[j]) : num * jrow[j];
            }
        }
    }
    __syncthreads();

    // Low-storage RK3 update (Solver2D_t.cpp:138-172), node by node:
    // coalesced reads of k (all prefetched) and writes of k and q.
    const double gdt = mul<S>(a.rk_g, dt);
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
            const int sb = ff * QS + el * ES;
#pragma unroll
            for (int it = 0; it < T::kLaneIters; ++it) {
                const int nd = lane + 32 * it;
                if (nd < NN) {
                    const int sn = sb + lane_node[it];
                    const double G = gs[sn];
                    const double kn = a.first ? G : add<S>(mul<S>(a.rk_a, kold[bi][it]), G);
                    const double qn = add<S>(qs[sn], mul<S>(gdt, kn));
                    k[gb + nd] = kn;
                    q[gb + nd] = qn;
                    qs[sn] = qn;
                    if (a.G_out) a.G_out[inst * 3 * Kp * NN + gb + nd] = G;
                }
            }
        }
    }
    __syncthreads();

    // Side traces of the new solution for the next stage: bottom/top from
    // row m, right/left from column m (Element2D_t.cpp:86-125), written into
    // the far slots of the neighbour across each interior side (its side
    // lk.y & 3, node N - k for this side's node k; links are reciprocal).
    if (active) {
        const double* row = qs + f * QS + e * ES + m * P;
        const double* cl = qs + f * QS + e * ES + m;
        double b = 0.0, t = 0.0, r = 0.0, l = 0.0;
#pragma unroll
        for (int j = 0; j < n; ++j) {
            b = madd<S>(b, lm[j], row[j]);
            t = madd<S>(t, lp[j], row[j]);
            r = madd<S>(r, lp[j], cl[j * P]);
            l = madd<S>(l, lm[j], cl[j * P]);
        }
        const double v[4] = {b, r, t, l};
        const int at[4] = {N - m, N - m, m, m};  // N - (own node of side s)
#pragma unroll
        for (int sd = 0; sd < 4; ++sd) {
            const int2 lk = a.link[4 * ge + sd];
            if (((lk.y >> 2) & 7) == kInterior) tr_out[((f * Kp + lk.x) * 4 + (lk.y & 3)) * n + at[sd]] = v[sd];
        }
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
    float ea[Coeffs<N>::H * Coeffs<N>::HO], so[Coeffs<N>::HO * Coeffs<N>::H];  // as Coeffs
};

template <int N, int E>
struct TileF {
    static constexpr int n = N + 1;
    static constexpr int NN = n * n;
    static constexpr int EPB = Tile<N, E>::EPB;
    static constexpr int kThreads = Tile<N, E>::kThreads;
    // bank-conflict-free strides of the FP32 arrays (32 four-byte values per wavefront)
    static constexpr bank::Strides L = bank::search(N, EPB, 32);
    static constexpr int P = L.P, ES = L.ES, QS = L.QS, SE = L.SE, FS = L.FS;
    // the bulk-copied FP64 q tile, then FP32 arrays (offsets in floats past it)
    static constexpr int kQd = 3 * EPB * NN;             // doubles
    static constexpr int kQf = 0;                        // [3][QS] q in FP32
    static constexpr int kG = kQf + 3 * QS;              // [3][QS]
    static constexpr int kOwn = kG + 3 * QS;             // [3][FS]
    static constexpr int kFar = kOwn + 3 * FS;           // [3][FS] far traces, then side fluxes
    static constexpr int kJ = kFar + 3 * FS;             // [EPB][ES] 1/J
    static constexpr int kS = kJ + EPB * ES;             // [EPB][4]
    static constexpr int kZ = bank::place(kS + EPB * 4, L.Z, 32);  // [n P] zeros
    static constexpr int kFloats = (kZ + n * P + 3) / 4 * 4;  // keeps the mbarrier 16-byte aligned
    static constexpr size_t kBytes = sizeof(double) * kQd + sizeof(float) * kFloats + 16;
    // CTAs per SM of the launch bound (occupancy_target at 56 registers; 0: none)
    static constexpr int kMinBlocks = bound_blocks(kBytes, kThreads, 56);
    // Offset within a field of node r = e NN + i n + j of the tile's elements.
    __device__ static __forceinline__ int node(int r) {
        const int el = r / NN, nd = r - el * NN;
        if constexpr (P == n) {
            return el * ES + nd;
        } else {
            const int i = nd / n;
            return el * ES + i * P + (nd - i * n);
        }
    }
};

// ((1 - t) d0 + (1 + t) d1) / 4 as fma(t, (d1 - d0) / 4, (d0 + d1) / 4) in FP32.
struct MetricLineF {
    float a, b;
    __device__ __forceinline__ MetricLineF(float d0, float d1) : a(0.25f * (d0 + d1)), b(0.25f * (d1 - d0)) {}
    __device__ __forceinline__ float operator()(float t) const { return fmaf(t, b, a); }
};

// One 3xTF32 product accumulation: c += a b with a = a_hi + a_lo split in
// TF32 and b's parts (b_hi, b_lo) from the lane table, the small terms first:
// c += a_lo b_hi, c += a_hi b_lo, c += a_hi b_hi.
__device__ __forceinline__ void tf32x3_mma(float (&c)[4], const float (&a)[4], const float (&b)[4]) {
    uint32_t hi[4], lo[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        hi[r] = to_tf32(a[r]);
        lo[r] = to_tf32(a[r] - __uint_as_float(hi[r]));
    }
    tf32mma_16x8x8(c, lo, __float_as_uint(b[0]), __float_as_uint(b[1]));
    tf32mma_16x8x8(c, hi, __float_as_uint(b[2]), __float_as_uint(b[3]));
    tf32mma_16x8x8(c, hi, __float_as_uint(b[0]), __float_as_uint(b[1]));
}

template <int N, int E, bool TC = false>
__global__ void __launch_bounds__(TileF<N, E>::kThreads, TC ? 0 : TileF<N, E>::kMinBlocks) stage_kernel_f32(StageArgs a, const __grid_constant__ CoeffsF<N> cf) {
    using T = TileF<N, E>;
    constexpr int n = T::n, NN = T::NN, EPB = T::EPB;
    constexpr int P = T::P, ES = T::ES, QS = T::QS, SE = T::SE, FS = T::FS;
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
    const int m = rr / EPB;
    const int e = rr - m * EPB;
    const bool active = f < 3 && e < ne;
    const int64_t ge = e0 + e;

    if (tid == 0) {
        mbar_init(bar, 1);
        mbar_fence_init();
        const uint32_t bytes = static_cast<uint32_t>(ne_copy * NN * sizeof(double));
        mbar_expect_tx(bar, 3 * bytes);
        for (int ff = 0; ff < 3; ++ff) bulk_load(qs + ff * EPB * NN, q + (ff * Kp + e0) * NN, bytes, bar);
    }
    // Far traces (written into this element's far slots by its neighbours
    // in the previous stage): 4-byte asynchronous copies of the contiguous
    // [field][element] blocks.
    {
        const int warp0 = tid >> 5, lane0 = tid & 31;
#pragma unroll
        for (int bi = 0; bi < Tile<N, E>::kBlockIters; ++bi) {
            const int b = warp0 + bi * Tile<N, E>::kWarps, ff = b / EPB, el = b - ff * EPB;
            if (b < 3 * EPB && el < ne) {
                const float* src = tr_in + (ff * Kp + e0 + el) * 4 * n;
                float* dst = far_s + ff * FS + el * SE;
#pragma unroll
                for (int it = 0; it < (4 * n + 31) / 32; ++it)
                    if (lane0 + 32 * it < 4 * n) cp_async4(dst + lane0 + 32 * it, src + lane0 + 32 * it);
            }
        }
    }
    for (int i = tid; i < n * P; i += T::kThreads) zs[i] = 0.0f;
    // Corners in FP64: their differences are formed before rounding to FP32
    // (on a fine mesh a difference is far smaller than the coordinates).
    double x0 = 0, y0 = 0, x1 = 0, y1 = 0, x2 = 0, y2 = 0, x3 = 0, y3 = 0;
    if (active) {
        const double* c = a.corners + 8 * ge;
        x0 = c[0]; y0 = c[1]; x1 = c[2]; y1 = c[3]; x2 = c[4]; y2 = c[5]; x3 = c[6]; y3 = c[7];
    }
    const MetricLineF x_xi(static_cast<float>(x1 - x0), static_cast<float>(x2 - x3)), y_xi(static_cast<float>(y1 - y0), static_cast<float>(y2 - y3));
    const MetricLineF x_eta(static_cast<float>(x3 - x0), static_cast<float>(x2 - x1)), y_eta(static_cast<float>(y3 - y0), static_cast<float>(y2 - y1));
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
            js[e * ES + m * P + j] = __frcp_rn(x_xi(tj) * ye - xe * y_xi(tj));
        }
    }
    cp_async_wait_all();
    // Every thread waits on the mbarrier only after thread 0 initialised it
    // (polling an uninitialised mbarrier is undefined).
    __syncthreads();
    if (!mbar_wait(bar, a.error, kWaitLimitNs)) return;  // also the barrier for zeros, far traces, edge metrics and J
    // FP32 copy of the tile in the padded layout: warps take (field,
    // element) blocks, lanes their nodes.
    const int warp = tid >> 5, lane = tid & 31;
    int lane_node[Tile<N, E>::kLaneIters];  // padded offsets of this lane's nodes within an element
#pragma unroll
    for (int it = 0; it < Tile<N, E>::kLaneIters; ++it) lane_node[it] = T::node(lane + 32 * it);
#pragma unroll
    for (int bi = 0; bi < Tile<N, E>::kBlockIters; ++bi) {
        const int b = warp + bi * Tile<N, E>::kWarps, ff = b / EPB, el = b - ff * EPB;
        if (b < 3 * EPB && el < ne) {
#pragma unroll
            for (int it = 0; it < Tile<N, E>::kLaneIters; ++it)
                if (lane + 32 * it < NN) qf[ff * QS + el * ES + lane_node[it]] = static_cast<float>(qs[(ff * EPB + el) * NN + lane + 32 * it]);
        }
    }
    __syncthreads();

    const float* Qe = qf + e * ES;
    const float* Xe = f == 0 ? Qe + 1 * QS : (f == 1 ? Qe : zs);
    const float* Ye = f == 0 ? Qe + 2 * QS : (f == 1 ? zs : Qe);
    if (active) {
        const float* Qf = Qe + f * QS;
        float b = 0.0f, t = 0.0f, r = 0.0f, l = 0.0f;
#pragma unroll
        for (int j = 0; j < n; ++j) {
            const float qr = Qf[m * P + j], qc = Qf[j * P + m];
            b = fmaf(lm[j], qr, b);
            t = fmaf(lp[j], qr, t);
            r = fmaf(lp[j], qc, r);
            l = fmaf(lm[j], qc, l);
        }
        float* o = own_s + f * FS + e * SE;
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
            const int o = e * SE + s * n + m;
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
    const float* F = far_s + f * FS + e * SE;
    // Tensor-core passes (3xTF32): the lane's fragments of Dhat transposed
    // (high and low TF32 parts), its lift weights and the corners of its
    // rows' element.
    using TT = TcTable32<N>;
    constexpr int EPBc = Tile<N, E>::EPB;
    [[maybe_unused]] float tb[TT::KS][TT::NT][4], tlpw[TT::NT][2], tlmw[TT::NT][2];
    [[maybe_unused]] double tcx[8];
    [[maybe_unused]] const int tg = lane >> 2, tt = lane & 3, tel = tg % (EPBc < 8 ? EPBc : 8);
    [[maybe_unused]] const bool tlive = tel < ne;
    if constexpr (TC) {
        const float* tab = a.tc32;
#pragma unroll
        for (int s = 0; s < TT::KS; ++s)
#pragma unroll
            for (int u = 0; u < TT::NT; ++u)
#pragma unroll
                for (int r = 0; r < 4; ++r) tb[s][u][r] = tab[TT::kB + ((s * TT::NT + u) * 32 + lane) * 4 + r];
#pragma unroll
        for (int u = 0; u < TT::NT; ++u)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                tlpw[u][h] = tab[TT::kLPW + (u * 2 + h) * 32 + lane];
                tlmw[u][h] = tab[TT::kLMW + (u * 2 + h) * 32 + lane];
            }
        const double* cc = a.corners + 8 * (e0 + tel);
#pragma unroll
        for (int k = 0; k < 8; ++k) tcx[k] = tlive ? cc[k] : 0.0;
    }
    if constexpr (TC) {
        // xi pass: rows (field, eta line j, element), K along xi.
        const MetricLineF mx_eta(static_cast<float>(tcx[6] - tcx[0]), static_cast<float>(tcx[4] - tcx[2]));
        const MetricLineF my_eta(static_cast<float>(tcx[7] - tcx[1]), static_cast<float>(tcx[5] - tcx[3]));
        float ka[TT::KS][2], kb[TT::KS][2];
#pragma unroll
        for (int s = 0; s < TT::KS; ++s)
#pragma unroll
            for (int r = 0; r < 2; ++r) {
                const float xv = a.tc32[TT::kXK + (s * 32 + lane) * 2 + r];
                const bool kv = 8 * s + tt + 4 * r < n;
                ka[s][r] = kv ? my_eta(xv) : 0.0f;
                kb[s][r] = kv ? mx_eta(xv) : 0.0f;
            }
        for (int mt = warp; mt < TcLines<N, EPBc>::kTiles; mt += Tile<N, E>::kWarps) {
            int rf[2], rj[2];
            bool rv[2];
            const float* Xr[2];
            const float* Yr[2];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int qq = (16 * mt + tg + 8 * h) / EPBc;
                rf[h] = qq / n;
                rj[h] = qq - rf[h] * n;
                rv[h] = tlive && rf[h] < 3;
                Xr[h] = rf[h] == 0 ? qf + QS + tel * ES : (rf[h] == 1 ? qf + tel * ES : zs);
                Yr[h] = rf[h] == 0 ? qf + 2 * QS + tel * ES : (rf[h] == 1 ? zs : qf + tel * ES);
            }
            float acc[TT::NT][4];
#pragma unroll
            for (int u = 0; u < TT::NT; ++u) acc[u][0] = acc[u][1] = acc[u][2] = acc[u][3] = 0.0f;
#pragma unroll
            for (int s = 0; s < TT::KS; ++s) {
                float av[4];  // (row h, column r) at fragment register h + 2r
#pragma unroll
                for (int r = 0; r < 2; ++r)
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const int k = 8 * s + tt + 4 * r;
                        av[h + 2 * r] = (rv[h] && k < n) ? ka[s][r] * Xr[h][k * P + rj[h]] - kb[s][r] * Yr[h][k * P + rj[h]] : 0.0f;
                    }
#pragma unroll
                for (int u = 0; u < TT::NT; ++u) tf32x3_mma(acc[u], av, tb[s][u]);
            }
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                if (!rv[h]) continue;
                const float* Fr = far_s + rf[h] * FS + tel * SE;
                const float fr = Fr[1 * n + rj[h]], fl3 = Fr[3 * n + (N - rj[h])];
                float* G = gs + rf[h] * QS + tel * ES + rj[h];
#pragma unroll
                for (int u = 0; u < TT::NT; ++u)
#pragma unroll
                    for (int c = 0; c < 2; ++c) {
                        const int i = 8 * u + 2 * tt + c;
                        if (i < n) G[i * P] = -(acc[u][2 * h + c] + fr * tlpw[u][c] + fl3 * tlmw[u][c]);
                    }
            }
        }
    } else if (active) {
        const int j = m;
        float col[n];
#pragma unroll
        for (int i = 0; i < n; ++i) col[i] = y_eta(xn[i]) * Xe[i * P + j] - x_eta(xn[i]) * Ye[i * P + j];
        const float fr = F[1 * n + j], fl3 = F[3 * n + (N - j)];
        float* G = gs + f * QS + e * ES + j;
        if constexpr (N >= kEvenOddMinOrder32) {
            dhat_even_odd<n>(cf.ea, cf.so, col, [&](int i, float y) { G[i * P] = -(y + (fr * lp[i] + fl3 * lm[i]) * iw[i]); });
        } else {
#pragma unroll
            for (int i = 0; i < n; ++i) {
                float acc = 0.0f;
#pragma unroll
                for (int mm = 0; mm < n; ++mm) acc = fmaf(Dh[i * n + mm], col[mm], acc);
                G[i * P] = -(acc + (fr * lp[i] + fl3 * lm[i]) * iw[i]);
            }
        }
    }
    __syncthreads();

    if constexpr (TC) {
        // eta pass: rows (field, xi line i, element), K along eta.
        const MetricLineF mx_xi(static_cast<float>(tcx[2] - tcx[0]), static_cast<float>(tcx[4] - tcx[6]));
        const MetricLineF my_xi(static_cast<float>(tcx[3] - tcx[1]), static_cast<float>(tcx[5] - tcx[7]));
        float ka[TT::KS][2], kb[TT::KS][2];
#pragma unroll
        for (int s = 0; s < TT::KS; ++s)
#pragma unroll
            for (int r = 0; r < 2; ++r) {
                const float xv = a.tc32[TT::kXK + (s * 32 + lane) * 2 + r];
                const bool kv = 8 * s + tt + 4 * r < n;
                ka[s][r] = kv ? -my_xi(xv) : 0.0f;
                kb[s][r] = kv ? mx_xi(xv) : 0.0f;
            }
        for (int mt = warp; mt < TcLines<N, EPBc>::kTiles; mt += Tile<N, E>::kWarps) {
            int rf[2], ri[2];
            bool rv[2];
            const float* Xr[2];
            const float* Yr[2];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int qq = (16 * mt + tg + 8 * h) / EPBc;
                rf[h] = qq / n;
                ri[h] = qq - rf[h] * n;
                rv[h] = tlive && rf[h] < 3;
                Xr[h] = rf[h] == 0 ? qf + QS + tel * ES : (rf[h] == 1 ? qf + tel * ES : zs);
                Yr[h] = rf[h] == 0 ? qf + 2 * QS + tel * ES : (rf[h] == 1 ? zs : qf + tel * ES);
            }
            float acc[TT::NT][4];
#pragma unroll
            for (int u = 0; u < TT::NT; ++u) acc[u][0] = acc[u][1] = acc[u][2] = acc[u][3] = 0.0f;
#pragma unroll
            for (int s = 0; s < TT::KS; ++s) {
                float av[4];
#pragma unroll
                for (int r = 0; r < 2; ++r)
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const int k = 8 * s + tt + 4 * r;
                        av[h + 2 * r] = (rv[h] && k < n) ? ka[s][r] * Xr[h][ri[h] * P + k] + kb[s][r] * Yr[h][ri[h] * P + k] : 0.0f;
                    }
#pragma unroll
                for (int u = 0; u < TT::NT; ++u) tf32x3_mma(acc[u], av, tb[s][u]);
            }
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                if (!rv[h]) continue;
                const float* Fr = far_s + rf[h] * FS + tel * SE;
                const float ft = Fr[2 * n + (N - ri[h])], fb = Fr[0 * n + ri[h]];
                float* G = gs + rf[h] * QS + tel * ES + ri[h] * P;
                const float* jrow = js + tel * ES + ri[h] * P;
#pragma unroll
                for (int u = 0; u < TT::NT; ++u)
#pragma unroll
                    for (int c = 0; c < 2; ++c) {
                        const int j = 8 * u + 2 * tt + c;
                        if (j < n) G[j] = (G[j] - (acc[u][2 * h + c] + ft * tlpw[u][c] + fb * tlmw[u][c])) * jrow[j];
                    }
            }
        }
    } else if (active) {
        const int i = m;
        float line[n];
#pragma unroll
        for (int j = 0; j < n; ++j) line[j] = -y_xi(xn[j]) * Xe[i * P + j] + x_xi(xn[j]) * Ye[i * P + j];
        const float ft = F[2 * n + (N - i)], fb = F[0 * n + i];
        float* G = gs + f * QS + e * ES + i * P;
        const float* jrow = js + e * ES + i * P;
        if constexpr (N >= kEvenOddMinOrder32) {
            dhat_even_odd<n>(cf.ea, cf.so, line, [&](int j, float y) { G[j] = (G[j] - (y + (ft * lp[j] + fb * lm[j]) * iw[j])) * jrow[j]; });
        } else {
#pragma unroll
            for (int j = 0; j < n; ++j) {
                float acc = 0.0f;
#pragma unroll
                for (int mm = 0; mm < n; ++mm) acc = fmaf(Dh[j * n + mm], line[mm], acc);
                G[j] = (G[j] - (acc + (ft * lp[j] + fb * lm[j]) * iw[j])) * jrow[j];
            }
        }
    }
    __syncthreads();

    // RK3 update in FP64 (Solver2D_t.cpp:138-172); the new q also refreshes
    // the FP32 tile for the traces.
    using U = Tile<N, E>;
    const double gdt = a.rk_g * dt;
    double kold[U::kBlockIters][U::kLaneIters];
#pragma unroll
    for (int bi = 0; bi < U::kBlockIters; ++bi) {
        const int b = warp + bi * U::kWarps, ff = b / EPB, el = b - ff * EPB;
        const bool live = !a.first && b < 3 * EPB && el < ne;
        const double* kb = k + (ff * Kp + e0 + el) * NN;
#pragma unroll
        for (int it = 0; it < U::kLaneIters; ++it) kold[bi][it] = (live && lane + 32 * it < NN) ? kb[lane + 32 * it] : 0.0;
    }
#pragma unroll
    for (int bi = 0; bi < U::kBlockIters; ++bi) {
        const int b = warp + bi * U::kWarps, ff = b / EPB, el = b - ff * EPB;
        if (b < 3 * EPB && el < ne) {
            const int64_t gb = (ff * Kp + e0 + el) * NN;
            const int sb = ff * QS + el * ES, db = (ff * EPB + el) * NN;
#pragma unroll
            for (int it = 0; it < U::kLaneIters; ++it) {
                const int nd = lane + 32 * it;
                if (nd < NN) {
                    const int sn = sb + lane_node[it];
                    const double G = static_cast<double>(gs[sn]);
                    const double kn = a.first ? G : fma(a.rk_a, kold[bi][it], G);
                    const double qn = fma(gdt, kn, qs[db + nd]);
                    k[gb + nd] = kn;
                    q[gb + nd] = qn;
                    qf[sn] = static_cast<float>(qn);
                    if (a.G_out) a.G_out[inst * 3 * Kp * NN + gb + nd] = G;
                }
            }
        }
    }
    __syncthreads();

    if (active) {
        const float* row = qf + f * QS + e * ES + m * P;
        const float* cl = qf + f * QS + e * ES + m;
        float b = 0.0f, t = 0.0f, r = 0.0f, l = 0.0f;
#pragma unroll
        for (int j = 0; j < n; ++j) {
            b = fmaf(lm[j], row[j], b);
            t = fmaf(lp[j], row[j], t);
            r = fmaf(lp[j], cl[j * P], r);
            l = fmaf(lm[j], cl[j * P], l);
        }
        // into the neighbours' far slots (as the FP64 kernel)
        const float v[4] = {b, r, t, l};
        const int at[4] = {N - m, N - m, m, m};
#pragma unroll
        for (int sd = 0; sd < 4; ++sd) {
            const int2 lk = a.link[4 * ge + sd];
            if (((lk.y >> 2) & 7) == kInterior) tr_out[((f * Kp + lk.x) * 4 + (lk.y & 3)) * n + at[sd]] = v[sd];
        }
    }
}

}  // namespace dev
}  // namespace ndg
