// Stage kernel of the conforming elements of a mixed-order mesh (sm_100a).
//
// After adaptation most elements still have, on each of their four sides,
// one face of their own order shared with a neighbour (or ghost) of the same
// order whose nodes match theirs. For those elements the face flux needs no
// interpolation and the element side flux no mortar projection
// (Mesh2D_t.cpp:3803-3929: the copy and reversed-copy branches), so their
// stage is the uniform-order stage: the padded, bank-conflict-free tile of
// the uniform kernels (Tile, stage_common.cuh), the neighbour traces
// gathered into it (each side's trace base comes from the plan), the upwind
// flux, both contraction passes, the RK update and the new side traces into
// the element's own trace slots, which the general kernels and the ghost
// kernel read. Where they are at least half of an order group the plan
// lists them last in it and they run here as a group of their own; the rest
// of the group runs general_fused_kernel.
//
// Every value is computed with the operations, in the order, of the general
// kernel's conforming branches, so STRICT instantiations reproduce the
// reference's CPU results bit for bit; the default form contracts by the
// even-odd decomposition where the uniform kernels do (kEvenOddMinOrder64).
// The FP32 form (conforming_stage_kernel_f32) follows the uniform FP32
// kernel: traces, fluxes and the volume term in FP32 over FP32 trace
// buffers, q, k and the RK update in FP64.
//
// PRE forms: the element side fluxes arrive precomputed (side_flux_kernel,
// general_kernels.cu, in the trace layout of sflux), so that any element,
// conforming or not, runs the tile: it copies them where the neighbour
// traces go and skips its own traces, the edge metrics and the flux pass.
#include "general_kernels.cuh"
#include "stage_common.cuh"
#include "stage_kernels.cuh"
#include "stage_templates.cuh"

#include <cuda_runtime.h>

#include <cstdint>

namespace ndg {
namespace dev {

namespace {

template <int N, bool S, bool PRE>
__global__ void __launch_bounds__(Tile<N>::kThreads, Tile<N>::kMinBlocks)
    conforming_stage_kernel(GeneralStage a, OrderGroup grp, const __grid_constant__ Coeffs<N> cf) {
    using T = Tile<N>;
    constexpr int n = T::n, NN = T::NN, EPB = T::EPB;
    constexpr int P = T::P, ES = T::ES, QS = T::QS, SE = T::SE, FS = T::FS;
    extern __shared__ __align__(128) double smem[];
    double* qs = smem + T::kQ;
    double* gs = smem + T::kG;
    double* own_s = smem + T::kOwn;
    double* far_s = smem + T::kFar;  // neighbour traces, then element side fluxes in place
    double* js = smem + T::kJ;
    double* ss = smem + T::kS;
    double* zs = smem + T::kZ;

    const GeneralMesh& M = a.m;
    const int tid = threadIdx.x;
    const int64_t base = static_cast<int64_t>(blockIdx.x) * EPB;
    const int64_t p0 = grp.first + base;  // list position of the tile's first element
    const int ne = static_cast<int>((grp.count - base) < EPB ? (grp.count - base) : EPB);
    const int64_t inst = blockIdx.y;
    const int64_t fb = M.block, ft = M.trace_total;
    double* q = a.q + inst * 3 * fb;
    double* k = a.k + inst * 3 * fb;
    const double* tr_in = a.etr + inst * 3 * ft;
    double* tr_out = a.etr_out + inst * 3 * ft;
    const double* sf_in = PRE ? a.sflux + inst * 3 * ft : nullptr;  // element side fluxes (PRE)
    const double* xn = cf.xn;
    const double* lm = cf.lm;
    const double* lp = cf.lp;
    const double dt = a.step[1];

    // Line threads (field f, line m, element e), e fastest, as in the uniform
    // stage kernel.
    const int f = tid / (EPB * n);
    const int rr = tid - f * (EPB * n);
    const int m = rr / EPB;
    const int e = rr - m * EPB;
    const bool active = f < 3 && e < ne;
    const int64_t pe = p0 + e;

    // Prologue: the q tile by 8-byte asynchronous copies into the padded
    // layout, warps over (field, element) blocks; the neighbour traces
    // likewise, node N - k of the neighbour's side for node k of this side
    // (two elements traverse a shared side in opposite directions).
    const int warp = tid >> 5, lane = tid & 31;
    const uint64_t stream_policy = evict_first_policy();  // q and k: read and rewritten once per stage
    int lane_node[T::kLaneIters];
#pragma unroll
    for (int it = 0; it < T::kLaneIters; ++it) lane_node[it] = T::node(lane + 32 * it);
#pragma unroll
    for (int bi = 0; bi < T::kBlockIters; ++bi) {
        const int b = warp + bi * T::kWarps, ff = b / EPB, el = b - ff * EPB;
        if (b < 3 * EPB && el < ne) {
            const double* src = q + ff * fb + M.poff2[p0 + el];
            double* dst = qs + ff * QS + el * ES;
#pragma unroll
            for (int it = 0; it < T::kLaneIters; ++it)
                if (lane + 32 * it < NN) cp_async8_stream(dst + lane_node[it], src + lane + 32 * it, stream_policy);
        }
    }
#pragma unroll
    for (int bi = 0; bi < T::kBlockIters; ++bi) {
        const int b = warp + bi * T::kWarps, ff = b / EPB, el = b - ff * EPB;
        if (b < 3 * EPB && el < ne) {
            double* dst = far_s + ff * FS + el * SE;
#pragma unroll
            for (int it = 0; it < (4 * n + 31) / 32; ++it) {
                const int idx = lane + 32 * it;
                if (idx < 4 * n) {
                    if constexpr (PRE) {
                        cp_async8(dst + idx, sf_in + ff * ft + M.poff1[p0 + el] + idx);
                    } else {
                        const int sd = idx / n, kk = idx - sd * n;
                        cp_async8(dst + idx, tr_in + ff * ft + M.cnb[4 * (p0 + el) + sd] + (N - kk));
                    }
                }
            }
        }
    }
    for (int i = tid; i < n * P; i += T::kThreads) zs[i] = 0.0;
    double x0 = 0, y0 = 0, x1 = 0, y1 = 0, x2 = 0, y2 = 0, x3 = 0, y3 = 0;
    if (active) {
        const double* c = M.pcorners + 8 * pe;
        x0 = c[0]; y0 = c[1]; x1 = c[2]; y1 = c[3]; x2 = c[4]; y2 = c[5]; x3 = c[6]; y3 = c[7];
    }
    const MetricLine<S> x_xi(sub<S>(x1, x0), sub<S>(x2, x3)), y_xi(sub<S>(y1, y0), sub<S>(y2, y3));
    const MetricLine<S> x_eta(sub<S>(x3, x0), sub<S>(x2, x1)), y_eta(sub<S>(y3, y0), sub<S>(y2, y1));
    if (active) {
        const double tm = xn[m];
        if (!PRE && f == 2) {
            // Edge metric of each side (Element2D_t.cpp:756-769).
            for (int sd = m; sd < 4; sd += n) {
                const double at = (sd == 0 || sd == 3) ? -1.0 : 1.0;
                const double dx = (sd == 0 || sd == 2) ? metric<S>(at, x_xi.d0, x_xi.d1) : metric<S>(at, x_eta.d0, x_eta.d1);
                const double dy = (sd == 0 || sd == 2) ? metric<S>(at, y_xi.d0, y_xi.d1) : metric<S>(at, y_eta.d0, y_eta.d1);
                ss[e * 4 + sd] = sqrt(add<S>(mul<S>(dx, dx), mul<S>(dy, dy)));
            }
        }
        // J (1/J outside the strict form) at nodes (m, j), j = f, f + 3, ...
        // (Element2D_t.cpp:752).
        const double xe = x_eta(tm), ye = y_eta(tm);
        for (int j = f; j < n; j += 3) {
            const double tj = xn[j];
            const double jac = sub<S>(mul<S>(x_xi(tj), ye), mul<S>(xe, y_xi(tj)));
            js[e * ES + m * P + j] = S ? jac : __drcp_rn(jac);
        }
    }
    cp_async_wait_all();
    __syncthreads();  // q tile, neighbour traces, zeros, edge metrics, J

    // Own side traces of this thread's field (Element2D_t.cpp:86-125): bottom
    // and top from row m, right and left from column m. Flux lines (X, Y) =
    // (u, v), (p, 0), (0, p) for f = 0, 1, 2 (Solver2D_t.cpp:31-37).
    const double* Qe = qs + e * ES;
    const double* Xe = f == 0 ? Qe + 1 * QS : (f == 1 ? Qe : zs);
    const double* Ye = f == 0 ? Qe + 2 * QS : (f == 1 ? zs : Qe);
    if constexpr (!PRE) {
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

        // Flux pass: side nodes m of side f, and of side 3 for f = 0. The upwind
        // flux in the face's own left/right order (Solver2D_t.cpp:48-63), then
        // the element's view of it: times the edge metric, negated for the
        // face's right element, whose side runs against the face's nodes
        // (Mesh2D_t.cpp:3895-3929).
        if (active) {
            for (int pass = 0; pass < 2; ++pass) {
                if (pass == 1 && f != 0) break;
                const int s = pass == 0 ? f : 3;
                const int role = M.crole[4 * pe + s];
                const double nx = M.cnormal[2 * (4 * pe + s)], ny = M.cnormal[2 * (4 * pe + s) + 1];
                const int o = e * SE + s * n + m;
                const double op = own_s[o], ou = own_s[FS + o], ov = own_s[2 * FS + o];
                const double fp_ = far_s[o], fu_ = far_s[FS + o], fv_ = far_s[2 * FS + o];
                const double Lp = role ? fp_ : op, Lu = role ? fu_ : ou, Lv = role ? fv_ : ov;
                const double Rp = role ? op : fp_, Ru = role ? ou : fu_, Rv = role ? ov : fv_;
                const double wL = add<S>(Lp, add<S>(mul<S>(Lu, nx), mul<S>(Lv, ny)));
                const double wR = sub<S>(Rp, add<S>(mul<S>(Ru, nx), mul<S>(Rv, ny)));
                const double flp = mul<S>(sub<S>(wL, wR), 0.5);
                const double sum = add<S>(wL, wR);
                const double flu = mul<S>(mul<S>(nx, sum), 0.5);
                const double flv = mul<S>(mul<S>(ny, sum), 0.5);
                const double sf = ss[e * 4 + s];
                far_s[o] = mul<S>(role ? -flp : flp, sf);
                far_s[FS + o] = mul<S>(role ? -flu : flu, sf);
                far_s[2 * FS + o] = mul<S>(role ? -flv : flv, sf);
            }
        }
        __syncthreads();
    }

    const double* Dh = cf.dhat;
    const double* w = cf.w;
    const double* iw = cf.iw;
    const double* F = far_s + f * FS + e * SE;
    constexpr bool EO = !S && N >= kEvenOddMinOrder64;
    constexpr int GR = n < 9 ? n : 9;

    // xi pass (eta index j = m): Dhat . line + lift, G = -(...) (Solver2D_t.cpp:72-101).
    if (active) {
        const int j = m;
        double col[n];
#pragma unroll
        for (int i = 0; i < n; ++i) col[i] = sub<S>(mul<S>(y_eta(xn[i]), Xe[i * P + j]), mul<S>(x_eta(xn[i]), Ye[i * P + j]));
        const double fr = F[1 * n + j], fl3 = F[3 * n + (N - j)];
        double* G = gs + f * QS + e * ES + j;
        if constexpr (EO) {
            dhat_even_odd<n>(cf.ea, cf.so, col, [&](int i, double y) { G[i * P] = -(y + (fr * lp[i] + fl3 * lm[i]) * iw[i]); });
        }
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

    // eta pass (xi index i = m): G = (G - (Dhat . line + lift)) / J (Solver2D_t.cpp:103-133).
    if (active) {
        const int i = m;
        double line[n];
#pragma unroll
        for (int j = 0; j < n; ++j) line[j] = add<S>(mul<S>(-y_xi(xn[j]), Xe[i * P + j]), mul<S>(x_xi(xn[j]), Ye[i * P + j]));
        const double ftp = F[2 * n + (N - i)], fbm = F[0 * n + i];
        double* G = gs + f * QS + e * ES + i * P;
        const double* jrow = js + e * ES + i * P;
        if constexpr (EO) {
            dhat_even_odd<n>(cf.ea, cf.so, line, [&](int j, double y) { G[j] = (G[j] - (y + (ftp * lp[j] + fbm * lm[j]) * iw[j])) * jrow[j]; });
        }
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
                const double lift = S ? __ddiv_rn(add<S>(mul<S>(ftp, lp[j]), mul<S>(fbm, lm[j])), w[j]) : (ftp * lp[j] + fbm * lm[j]) * iw[j];
                const double num = sub<S>(G[j], add<S>(acc[g], lift));
                G[j] = S ? __ddiv_rn(num, jrow[j]) : num * jrow[j];
            }
        }
    }
    __syncthreads();

    // Low-storage RK3 update (Solver2D_t.cpp:138-172), node by node over
    // (field, element) blocks; each block's k values are loaded together.
    const double gdt = mul<S>(a.rk_g, dt);
#pragma unroll
    for (int bi = 0; bi < T::kBlockIters; ++bi) {
        const int b = warp + bi * T::kWarps, ff = b / EPB, el = b - ff * EPB;
        if (b < 3 * EPB && el < ne) {
            const int64_t gb = ff * fb + M.poff2[p0 + el];
            const int sb = ff * QS + el * ES;
            double kold[T::kLaneIters];
#pragma unroll
            for (int it = 0; it < T::kLaneIters; ++it) kold[it] = (!a.first && lane + 32 * it < NN) ? __ldcs(k + gb + lane + 32 * it) : 0.0;
#pragma unroll
            for (int it = 0; it < T::kLaneIters; ++it) {
                const int nd = lane + 32 * it;
                if (nd < NN) {
                    const int sn = sb + lane_node[it];
                    const double G = gs[sn];
                    const double kn = a.first ? G : add<S>(mul<S>(a.rk_a, kold[it]), G);
                    const double qn = add<S>(qs[sn], mul<S>(gdt, kn));
                    __stcs(k + gb + nd, kn);
                    __stcs(q + gb + nd, qn);
                    qs[sn] = qn;
                    if (a.G_out) a.G_out[inst * 3 * fb + gb + nd] = G;
                }
            }
        }
    }
    __syncthreads();

    // Side traces of the new state into the element's own trace slots
    // (Element2D_t.cpp:86-125; top and left run reversed).
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
        double* o = tr_out + f * ft + M.poff1[pe];
        o[0 * n + m] = b;
        o[1 * n + m] = r;
        o[2 * n + (N - m)] = t;
        o[3 * n + (N - m)] = l;
    }
}

// FP32 form. The FP64 q tile arrives unpadded by 8-byte copies (warps over
// (field, element) blocks, as above) and each thread converts the values it
// copied into the padded FP32 tile once its own copies have landed.
template <int N, bool PRE>
__global__ void __launch_bounds__(TileF<N, 0>::kThreads, TileF<N, 0>::kMinBlocks)
    conforming_stage_kernel_f32(GeneralStage a, OrderGroup grp, const __grid_constant__ CoeffsF<N> cf) {
    using T = TileF<N, 0>;
    using U = Tile<N, 0>;
    constexpr int n = T::n, NN = T::NN, EPB = T::EPB;
    constexpr int P = T::P, ES = T::ES, QS = T::QS, SE = T::SE, FS = T::FS;
    extern __shared__ __align__(128) double smem[];
    double* qs = smem;  // [3][EPB][NN] FP64 q, unpadded
    float* fsm = reinterpret_cast<float*>(smem + T::kQd);
    float* qf = fsm + T::kQf;
    float* gs = fsm + T::kG;
    float* own_s = fsm + T::kOwn;
    float* far_s = fsm + T::kFar;
    float* js = fsm + T::kJ;
    float* ss = fsm + T::kS;
    float* zs = fsm + T::kZ;

    const GeneralMesh& M = a.m;
    const int tid = threadIdx.x;
    const int64_t base = static_cast<int64_t>(blockIdx.x) * EPB;
    const int64_t p0 = grp.first + base;
    const int ne = static_cast<int>((grp.count - base) < EPB ? (grp.count - base) : EPB);
    const int64_t inst = blockIdx.y;
    const int64_t fb = M.block, ft = M.trace_total;
    double* q = a.q + inst * 3 * fb;
    double* k = a.k + inst * 3 * fb;
    const float* tr_in = a.etr_f + inst * 3 * ft;
    float* tr_out = a.etr_out_f + inst * 3 * ft;
    const float* sf_in = PRE ? a.sflux_f + inst * 3 * ft : nullptr;  // element side fluxes (PRE)
    const float* xn = cf.xn;
    const float* lm = cf.lm;
    const float* lp = cf.lp;
    const double dt = a.step[1];

    const int f = tid / (EPB * n);
    const int rr = tid - f * (EPB * n);
    const int m = rr / EPB;
    const int e = rr - m * EPB;
    const bool active = f < 3 && e < ne;
    const int64_t pe = p0 + e;

    const int warp = tid >> 5, lane = tid & 31;
    const uint64_t stream_policy = evict_first_policy();  // q and k: read and rewritten once per stage
    int lane_node[U::kLaneIters];
#pragma unroll
    for (int it = 0; it < U::kLaneIters; ++it) lane_node[it] = T::node(lane + 32 * it);
#pragma unroll
    for (int bi = 0; bi < U::kBlockIters; ++bi) {
        const int b = warp + bi * U::kWarps, ff = b / EPB, el = b - ff * EPB;
        if (b < 3 * EPB && el < ne) {
            const double* src = q + ff * fb + M.poff2[p0 + el];
#pragma unroll
            for (int it = 0; it < U::kLaneIters; ++it)
                if (lane + 32 * it < NN) cp_async8_stream(qs + b * NN + lane + 32 * it, src + lane + 32 * it, stream_policy);
        }
    }
#pragma unroll
    for (int bi = 0; bi < U::kBlockIters; ++bi) {
        const int b = warp + bi * U::kWarps, ff = b / EPB, el = b - ff * EPB;
        if (b < 3 * EPB && el < ne) {
            float* dst = far_s + ff * FS + el * SE;
#pragma unroll
            for (int it = 0; it < (4 * n + 31) / 32; ++it) {
                const int idx = lane + 32 * it;
                if (idx < 4 * n) {
                    if constexpr (PRE) {
                        cp_async4(dst + idx, sf_in + ff * ft + M.poff1[p0 + el] + idx);
                    } else {
                        const int sd = idx / n, kk = idx - sd * n;
                        cp_async4(dst + idx, tr_in + ff * ft + M.cnb[4 * (p0 + el) + sd] + (N - kk));
                    }
                }
            }
        }
    }
    for (int i = tid; i < n * P; i += T::kThreads) zs[i] = 0.0f;
    double x0 = 0, y0 = 0, x1 = 0, y1 = 0, x2 = 0, y2 = 0, x3 = 0, y3 = 0;
    if (active) {
        const double* c = M.pcorners + 8 * pe;
        x0 = c[0]; y0 = c[1]; x1 = c[2]; y1 = c[3]; x2 = c[4]; y2 = c[5]; x3 = c[6]; y3 = c[7];
    }
    const MetricLineF x_xi(static_cast<float>(x1 - x0), static_cast<float>(x2 - x3)), y_xi(static_cast<float>(y1 - y0), static_cast<float>(y2 - y3));
    const MetricLineF x_eta(static_cast<float>(x3 - x0), static_cast<float>(x2 - x1)), y_eta(static_cast<float>(y3 - y0), static_cast<float>(y2 - y1));
    if (active) {
        const float tm = xn[m];
        if (!PRE && f == 2) {
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
#pragma unroll
    for (int bi = 0; bi < U::kBlockIters; ++bi) {
        const int b = warp + bi * U::kWarps, ff = b / EPB, el = b - ff * EPB;
        if (b < 3 * EPB && el < ne) {
#pragma unroll
            for (int it = 0; it < U::kLaneIters; ++it)
                if (lane + 32 * it < NN) qf[ff * QS + el * ES + lane_node[it]] = static_cast<float>(qs[b * NN + lane + 32 * it]);
        }
    }
    __syncthreads();  // FP32 q tile, neighbour traces, zeros, edge metrics, J

    const float* Qe = qf + e * ES;
    const float* Xe = f == 0 ? Qe + 1 * QS : (f == 1 ? Qe : zs);
    const float* Ye = f == 0 ? Qe + 2 * QS : (f == 1 ? zs : Qe);
    if constexpr (!PRE) {
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
                const int role = M.crole[4 * pe + s];
                const float nx = static_cast<float>(M.cnormal[2 * (4 * pe + s)]), ny = static_cast<float>(M.cnormal[2 * (4 * pe + s) + 1]);
                const int o = e * SE + s * n + m;
                const float op = own_s[o], ou = own_s[FS + o], ov = own_s[2 * FS + o];
                const float fp_ = far_s[o], fu_ = far_s[FS + o], fv_ = far_s[2 * FS + o];
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
    }

    const float* Dh = cf.dhat;
    const float* iw = cf.iw;
    const float* F = far_s + f * FS + e * SE;
    if (active) {
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
    if (active) {
        const int i = m;
        float line[n];
#pragma unroll
        for (int j = 0; j < n; ++j) line[j] = -y_xi(xn[j]) * Xe[i * P + j] + x_xi(xn[j]) * Ye[i * P + j];
        const float ftp = F[2 * n + (N - i)], fbm = F[0 * n + i];
        float* G = gs + f * QS + e * ES + i * P;
        const float* jrow = js + e * ES + i * P;
        if constexpr (N >= kEvenOddMinOrder32) {
            dhat_even_odd<n>(cf.ea, cf.so, line, [&](int j, float y) { G[j] = (G[j] - (y + (ftp * lp[j] + fbm * lm[j]) * iw[j])) * jrow[j]; });
        } else {
#pragma unroll
            for (int j = 0; j < n; ++j) {
                float acc = 0.0f;
#pragma unroll
                for (int mm = 0; mm < n; ++mm) acc = fmaf(Dh[j * n + mm], line[mm], acc);
                G[j] = (G[j] - (acc + (ftp * lp[j] + fbm * lm[j]) * iw[j])) * jrow[j];
            }
        }
    }
    __syncthreads();

    // RK update in FP64; the new state also into the FP32 tile for the traces.
    const double gdt = a.rk_g * dt;
#pragma unroll
    for (int bi = 0; bi < U::kBlockIters; ++bi) {
        const int b = warp + bi * U::kWarps, ff = b / EPB, el = b - ff * EPB;
        if (b < 3 * EPB && el < ne) {
            const int64_t gb = ff * fb + M.poff2[p0 + el];
            const int sb = ff * QS + el * ES, db = b * NN;
            double kold[U::kLaneIters];
#pragma unroll
            for (int it = 0; it < U::kLaneIters; ++it) kold[it] = (!a.first && lane + 32 * it < NN) ? __ldcs(k + gb + lane + 32 * it) : 0.0;
#pragma unroll
            for (int it = 0; it < U::kLaneIters; ++it) {
                const int nd = lane + 32 * it;
                if (nd < NN) {
                    const int sn = sb + lane_node[it];
                    const double G = static_cast<double>(gs[sn]);
                    const double kn = a.first ? G : fma(a.rk_a, kold[it], G);
                    const double qn = fma(gdt, kn, qs[db + nd]);
                    __stcs(k + gb + nd, kn);
                    __stcs(q + gb + nd, qn);
                    qf[sn] = static_cast<float>(qn);
                    if (a.G_out) a.G_out[inst * 3 * fb + gb + nd] = G;
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
        float* o = tr_out + f * ft + M.poff1[pe];
        o[0 * n + m] = b;
        o[1 * n + m] = r;
        o[2 * n + (N - m)] = t;
        o[3 * n + (N - m)] = l;
    }
}

template <int N>
Coeffs<N> conforming_coeffs() {
    Coeffs<N> c;
    host_coefficients(N, c.dhat, c.xn, c.lm, c.lp, c.w, c.iw);
    c.fill_even_odd();
    return c;
}

template <int N, bool S, bool PRE>
cudaError_t launch_t(const GeneralStage& a, const OrderGroup& g, cudaStream_t stream) {
    using T = Tile<N>;
    const dim3 grid(static_cast<unsigned>((g.count + T::EPB - 1) / T::EPB), static_cast<unsigned>(a.n_instances));
    conforming_stage_kernel<N, S, PRE><<<grid, T::kThreads, T::kBytes, stream>>>(a, g, conforming_coeffs<N>());
    return cudaGetLastError();
}

template <int N>
CoeffsF<N> conforming_coeffs_f() {
    const Coeffs<N> d = conforming_coeffs<N>();
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

template <int N, bool PRE>
cudaError_t launch_f32_t(const GeneralStage& a, const OrderGroup& g, cudaStream_t stream) {
    using T = TileF<N, 0>;
    const dim3 grid(static_cast<unsigned>((g.count + T::EPB - 1) / T::EPB), static_cast<unsigned>(a.n_instances));
    conforming_stage_kernel_f32<N, PRE><<<grid, T::kThreads, T::kBytes, stream>>>(a, g, conforming_coeffs_f<N>());
    return cudaGetLastError();
}

template <int N, bool PRE>
cudaError_t prepare_form() {
    cudaError_t err = cudaFuncSetAttribute(conforming_stage_kernel<N, false, PRE>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(Tile<N>::kBytes));
    if (err == cudaSuccess)
        err = cudaFuncSetAttribute(conforming_stage_kernel<N, true, PRE>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(Tile<N>::kBytes));
    if (err == cudaSuccess)
        err = cudaFuncSetAttribute(conforming_stage_kernel_f32<N, PRE>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(TileF<N, 0>::kBytes));
    return err;
}
template <int N>
cudaError_t prepare_t() {
    const cudaError_t err = prepare_form<N, false>();
    return err == cudaSuccess ? prepare_form<N, true>() : err;
}

#define NDG_CONFORMING_ORDERS(X) X(1) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14) X(15) X(16)

}  // namespace

cudaError_t prepare_conforming_kernels(int N) {
    switch (N) {
#define NDG_CASE(n_) \
    case n_: return prepare_t<n_>();
        NDG_CONFORMING_ORDERS(NDG_CASE)
#undef NDG_CASE
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_conforming_group(const GeneralStage& a, const OrderGroup& g, bool strict, bool fp32, cudaStream_t stream, bool pre) {
    if (g.count <= 0) return cudaSuccess;
    switch (g.N) {
#define NDG_CASE(n_)                                                                                                          \
    case n_:                                                                                                                  \
        if (pre) return fp32 ? launch_f32_t<n_, true>(a, g, stream) : (strict ? launch_t<n_, true, true>(a, g, stream) : launch_t<n_, false, true>(a, g, stream)); \
        return fp32 ? launch_f32_t<n_, false>(a, g, stream) : (strict ? launch_t<n_, true, false>(a, g, stream) : launch_t<n_, false, false>(a, g, stream));
        NDG_CONFORMING_ORDERS(NDG_CASE)
#undef NDG_CASE
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace dev
}  // namespace ndg
