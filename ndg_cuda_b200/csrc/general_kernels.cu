// Stage kernels for mixed-order meshes with nonconforming faces (sm_100a).
//
// After adaptation elements differ in order and faces carry mortar offsets
// and scales. A stage (include/solvers/Solver2D_t.tcu:46-70) is two kinds of
// launch over device arrays, with the element side traces double-buffered
// between stages:
//
//   ghost traces   walls, symmetry planes, outflow: the neighbours' traces
//                  projected onto the ghost; inflow: the plane wave; periodic
//                  interfaces: the origin's side trace
//                  (Mesh2D_t.cpp:4298-4730)
//   fused stage    per order group, one CTA per tile of elements: the face
//                  fluxes of the elements' sides (both traces brought to the
//                  face order, copy when conforming, interpolation otherwise;
//                  upwind flux; Mesh2D_t.cpp:3803-3893, Solver2D_t.cpp:48-63),
//                  the element side fluxes (mortar projection,
//                  Mesh2D_t.cpp:3895-4006), the derivative
//                  (Solver2D_t.cpp:66-136), the RK3 update
//                  (Solver2D_t.cpp:138-172) and the side traces of the new
//                  state for the next stage (Element2D_t.cpp:86-125)
//
// Where at least half of an order group's elements are conforming (one
// same-order face per side, shared with a same-order neighbour), they come
// last in the plan's list and run conforming_stage_kernel
// (conforming_kernels.cu) instead of the fused stage; the two parts are
// separate groups and concurrent branches. A large group whose order has no
// conforming part runs split instead of fused: side_flux_kernel (the fused
// stage's face and element-side fluxes, into a trace-layout buffer), then
// conforming_stage_kernel's PRE form over those side fluxes.
//
// The mortar weights of the plan are computed once (side_weights_kernel,
// face_weights_kernel). A face's flux is evaluated by each of its two
// elements, with the same operations, so both see the same value.
//
// STRICT instantiations round every operation in the reference's order and
// reproduce its CPU results bit for bit; node matching (almost_equal) is
// always evaluated exactly as the reference does, since it is a decision.
#include "general_kernels.cuh"
#include "stage_common.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <vector>

namespace ndg {
namespace dev {

namespace {

constexpr int kGVecTotal = (kMaxOrder + 1) * (kMaxOrder + 2) / 2;
constexpr int kGMatTotal = (kMaxOrder + 1) * (kMaxOrder + 2) * (2 * kMaxOrder + 3) / 6;
__host__ __device__ constexpr int gvec(int N) { return N * (N + 1) / 2; }
__host__ __device__ constexpr int gmat(int N) { return N * (N + 1) * (2 * N + 1) / 6; }

__constant__ double g_nodes[kGVecTotal];
__constant__ double g_weights[kGVecTotal];
__constant__ double g_inv_weights[kGVecTotal];
__constant__ double g_bary[kGVecTotal];
__constant__ double g_lagrange_left[kGVecTotal];
__constant__ double g_lagrange_right[kGVecTotal];
__constant__ double g_dhat[kGMatTotal];
// FP32 copies for the FP32 form
__constant__ float gf_nodes[kGVecTotal];
__constant__ float gf_weights[kGVecTotal];
__constant__ float gf_inv_weights[kGVecTotal];
__constant__ float gf_lagrange_left[kGVecTotal];
__constant__ float gf_lagrange_right[kGVecTotal];
__constant__ float gf_dhat[kGMatTotal];

// The table (or trace buffer) of the arithmetic type R.
template <typename R>
__device__ __forceinline__ const R* tab(const double* d, const float* f) {
    if constexpr (sizeof(R) == 8)
        return d;
    else
        return f;
}
template <typename R>
__device__ __forceinline__ const R* pick(const double* d, const float* f) {
    return tab<R>(d, f);
}
template <typename R>
__device__ __forceinline__ R* pick(double* d, float* f) {
    if constexpr (sizeof(R) == 8)
        return d;
    else
        return f;
}

// Mesh2D_t::almost_equal (src/meshes/Mesh2D_t.cpp:3785-3792): 2 ulp relative,
// or an absolute difference below DBL_MIN.
__device__ __forceinline__ bool almost_equal(double x, double y) {
    const double d = fabs(__dsub_rn(x, y));
    return d <= __dmul_rn(__dmul_rn(DBL_EPSILON, fabs(__dadd_rn(x, y))), 2.0) || d < DBL_MIN;
}

// Reference coordinate on an element side of face node coordinate xf:
// (xf + 1) scale + 2 offset - 1 (Mesh2D_t.cpp:3847, 3954).
__device__ __forceinline__ double mortar_coord(double xf, double scale, double offset) {
    return __dsub_rn(__dadd_rn(__dmul_rn(__dadd_rn(xf, 1.0), scale), __dmul_rn(2.0, offset)), 1.0);
}

// ---------------------------------------------------------------------------
// Side traces of the domain elements of one order group: thread per
// (element, side, node), three fields each.
template <int N, bool S, typename R>
__global__ void __launch_bounds__(256) general_traces_kernel(GeneralStage a, const int64_t* __restrict__ ids, int64_t count) {
    constexpr int n = N + 1;
    const R* lm = tab<R>(g_lagrange_left, gf_lagrange_left) + gvec(N);
    const R* lp = tab<R>(g_lagrange_right, gf_lagrange_right) + gvec(N);
    const int64_t total = count * 4 * n;
    const int64_t fb = a.m.block, ft = a.m.trace_total;
    R* etr = pick<R>(a.etr, a.etr_f);
    for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < total * a.n_instances;
         idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t inst = idx / total;
        const int64_t r = idx - inst * total;
        const int64_t le = r / (4 * n);
        const int sm = static_cast<int>(r - le * 4 * n);
        const int s = sm / n, m = sm - s * n;
        const int64_t e = ids[le];
        const R* l = (s == 0 || s == 3) ? lm : lp;
        const int line = (s < 2) ? m : N - m;
        const int base = (s == 0 || s == 2) ? line * n : line;
        const int stride = (s == 0 || s == 2) ? 1 : n;
        const double* q = a.q + inst * 3 * fb + a.m.off2[e] + base;
        R* out = etr + inst * 3 * ft + a.m.off1[e] + s * n + m;
#pragma unroll
        for (int f = 0; f < 3; ++f) {
            R acc = 0;
#pragma unroll
            for (int j = 0; j < n; ++j) acc = madd<S>(acc, l[j], R(q[f * fb + j * stride]));
            out[f * ft] = acc;
        }
    }
}

// Ghost traces: thread per (instance, ghost element, node); each node
// gathers the contributions the reference's loops add to it, in their order.
template <bool S, typename R>
__global__ void __launch_bounds__(128) general_ghosts_kernel(GeneralStage a, int max_n) {
    const GeneralMesh& M = a.m;
    const int64_t n_ghosts = M.n_total - M.n_domain;
    const int64_t ft = M.trace_total;
    const double t = add<S>(a.step[0], mul<S>(a.rk_b, a.step[1]));
    const int64_t per_inst = n_ghosts * max_n;
    for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < per_inst * a.n_instances;
         idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t inst = idx / per_inst;
        const int64_t r = idx - inst * per_inst;
        const int64_t gi = r / max_n;
        const int i = static_cast<int>(r - gi * max_n);
        const int64_t ge = M.n_domain + gi;
        const int N = M.eN[ge];
        if (i > N) continue;
        const double* xe = g_nodes + gvec(N);
        R* tr = pick<R>(a.etr, a.etr_f) + inst * 3 * ft;
        R* gp = tr + M.off1[ge];
        R* gu = gp + ft;
        R* gv = gu + ft;
        const int kind = M.gkind[gi];
        if (kind == kGhostMirror || kind == kGhostCopy) {
            // Mesh2D_t.cpp:4366-4434 (multi-face branch) and 4601-4710, with
            // the plan's weights (ghost_weights_kernel).
            const R sf = R(M.gscale[gi]);
            R vp = 0, vu = 0, vv = 0;
            const int64_t e0 = M.gq_start[gi], e1 = M.gq_start[gi + 1];
            const int64_t direct = M.gdirect[gi];
            if (direct >= 0) {
                // The one term of the loop below (neighbour node N - i, weight
                // exactly 1), without its chain of plan loads.
                const R* np_ = tr + direct + (N - i);
                vp = add<S>(vp, mul<S>(mul<S>(R(1), np_[0]), sf));
                vu = add<S>(vu, mul<S>(mul<S>(R(1), np_[ft]), sf));
                vv = add<S>(vv, mul<S>(mul<S>(R(1), np_[2 * ft]), sf));
            }
            for (int64_t qe = (direct >= 0 ? e1 : e0); qe < e1; ++qe) {
                const int Nn = M.gq_N[qe];
                const R* np_ = tr + M.gq_base[qe];
                const R* nu_ = np_ + ft;
                const R* nv_ = nu_ + ft;
                const double* W = M.sw + M.gq_woff[qe] + i * (Nn + 1);
                const int* match = M.smatch + M.gq_moff[qe];
                // Every node's loads are issued before its match decides
                // whether it adds (the sums keep their order), so that
                // unrolled iterations overlap their loads.
#pragma unroll 4
                for (int j = 0; j <= Nn; ++j) {
                    const int mt = match[j];
                    const R w = R(W[j]), xp = np_[j], xu = nu_[j], xv = nv_[j];
                    if (mt >= 0 && mt != i) continue;
                    vp = add<S>(vp, mul<S>(mul<S>(w, xp), sf));
                    vu = add<S>(vu, mul<S>(mul<S>(w, xu), sf));
                    vv = add<S>(vv, mul<S>(mul<S>(w, xv), sf));
                }
            }
            if (kind == kGhostMirror && e1 > e0) {
                const R nx = R(M.gframe[4 * gi]), ny = R(M.gframe[4 * gi + 1]);
                const R tx = R(M.gframe[4 * gi + 2]), ty = R(M.gframe[4 * gi + 3]);
                const R l0 = -add<S>(mul<S>(vu, nx), mul<S>(vv, ny));
                const R l1 = add<S>(mul<S>(vu, tx), mul<S>(vv, ty));
                vu = add<S>(mul<S>(nx, l0), mul<S>(tx, l1));
                vv = add<S>(mul<S>(ny, l0), mul<S>(ty, l1));
            }
            gp[i] = vp;
            gu[i] = vu;
            gv[i] = vv;
        } else if (kind == kGhostAnalytic) {
            // Mesh2D_t.cpp:4575-4599.
            const int64_t n0 = M.enodes[4 * ge], n1 = M.enodes[4 * ge + 1];
            const double p0x = M.node_xy[2 * n0], p0y = M.node_xy[2 * n0 + 1];
            const double p1x = M.node_xy[2 * n1], p1y = M.node_xy[2 * n1 + 1];
            const double rr = __dmul_rn(__dadd_rn(xe[i], 1.0), 0.5);
            const double gx = __dadd_rn(__dmul_rn(p1x, rr), __dmul_rn(p0x, __dsub_rn(1.0, rr)));
            const double gy = __dadd_rn(__dmul_rn(p1y, rr), __dmul_rn(p0y, __dsub_rn(1.0, rr)));
            double pw, uw, vw;
            plane_wave(gx, gy, t, pw, uw, vw);
            gp[i] = R(pw);
            gu[i] = R(uw);
            gv[i] = R(vw);
        } else if (kind == kGhostInterface) {
            // Mesh2D_t.cpp:4712-4730: the origin's side trace, up to its order.
            const int64_t src = M.gsrc[gi];
            const int Ns = M.eN[src];
            if (i <= Ns) {
                const R* sp = tr + M.off1[src] + M.gsrc_side[gi] * (Ns + 1);
                gp[i] = sp[i];
                gu[i] = sp[i + ft];
                gv[i] = sp[i + 2 * ft];
            }
        } else {
            gp[i] = gu[i] = gv[i] = R(0);
        }
    }
}

// Mortar weights of the element sides (Mesh2D_t.cpp:3895-4006, the
// multi-face branch): per face node j the element node it matches
// (almost_equal) or -1, and the weight of every element node i,
// sign w_f[j] / w_e[i] at the match or sign T_i w_f[j] / w_e[i] with the
// barycentric T_i, in the reference's rounding. Thread per domain element
// side.
__global__ void __launch_bounds__(128) side_weights_kernel(GeneralMesh M, double* __restrict__ sw, int* __restrict__ smatch) {
    for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < 4 * M.n_domain;
         idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t e = idx / 4;
        const int s = static_cast<int>(idx - 4 * e);
        const int N = M.eN[e];
        const double* xe = g_nodes + gvec(N);
        const double* we = g_weights + gvec(N);
        const double* bwe = g_bary + gvec(N);
        for (int64_t q = M.sface_start[4 * e + s]; q < M.sface_start[4 * e + s + 1]; ++q) {
            if (M.sw_off[q] < 0) continue;
            const int64_t f = M.sface[q];
            const int Nf = M.fN[f];
            const double* xf = g_nodes + gvec(Nf);
            const double* wf = g_weights + gvec(Nf);
            const bool fwd = e == M.felem[2 * f];
            const int fs = fwd ? 0 : 1;
            const double sgn = fwd ? 1.0 : -1.0;
            const double scale = M.fscale[2 * f + fs], offset = M.foffset[2 * f + fs];
            double* W = sw + M.sw_off[q];
            int* match = smatch + M.sm_off[q];
            for (int j = 0; j <= Nf; ++j) {
                const double coord = mortar_coord(xf[fwd ? j : Nf - j], scale, offset);
                int found = -1;
                for (int ii = 0; ii <= N; ++ii)
                    if (almost_equal(coord, xe[ii])) {
                        found = ii;
                        break;
                    }
                match[j] = found;
                if (found >= 0) {
                    for (int i = 0; i <= N; ++i) W[i * (Nf + 1) + j] = (i == found) ? __ddiv_rn(__dmul_rn(sgn, wf[j]), we[i]) : 0.0;
                } else {
                    double sb = 0.0;
                    for (int ii = 0; ii <= N; ++ii) sb = __dadd_rn(sb, __ddiv_rn(bwe[ii], __dsub_rn(coord, xe[ii])));
                    for (int i = 0; i <= N; ++i) {
                        const double T = __ddiv_rn(bwe[i], __dmul_rn(__dsub_rn(coord, xe[i]), sb));
                        W[i * (Nf + 1) + j] = __ddiv_rn(__dmul_rn(__dmul_rn(sgn, T), wf[j]), we[i]);
                    }
                }
            }
        }
    }
}

// Interpolation weights of the non-conforming face sides
// (Mesh2D_t.cpp:3803-3893): per face node i the element node it matches or
// -1, the barycentric terms t_j = w_j / (x - x_j) and their sum, in the
// reference's rounding. Thread per face side.
__global__ void __launch_bounds__(128) face_weights_kernel(GeneralMesh M, double* __restrict__ fw, int* __restrict__ fmatch) {
    for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < 2 * M.n_faces;
         idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        if (M.fw_off[idx] < 0) continue;
        const int64_t f = idx / 2;
        const int side = static_cast<int>(idx - 2 * f);
        const int Nf = M.fN[f];
        const int64_t e = M.felem[2 * f + side];
        const int Ne = M.eN[e];
        const double* xf = g_nodes + gvec(Nf);
        const double* xe = g_nodes + gvec(Ne);
        const double* bwe = g_bary + gvec(Ne);
        double* tw = fw + M.fw_off[idx];
        int* match = fmatch + M.fm_off[idx];
        for (int i = 0; i <= Nf; ++i) {
            const double coord = mortar_coord(xf[side == 0 ? i : Nf - i], M.fscale[2 * f + side], M.foffset[2 * f + side]);
            int found = -1;
            double den = 0.0;
            for (int j = 0; j <= Ne; ++j) {
                if (almost_equal(coord, xe[j])) {
                    found = j;
                    break;
                }
                const double tj = __ddiv_rn(bwe[j], __dsub_rn(coord, xe[j]));
                tw[i * (Ne + 1) + j] = tj;
                den = __dadd_rn(den, tj);
            }
            match[i] = found;
            tw[(Nf + 1) * (Ne + 1) + i] = den;
        }
    }
}

// Weights of the ghost side-0 gathers (Mesh2D_t.cpp:4366-4434, 4601-4710):
// per neighbour node j the ghost node it matches (almost_equal) or -1, and
// the weight of every ghost node i, w_n[j] / w_g[i] at the match or
// T_i w_n[j] / w_g[i] with the barycentric T_i, in the reference's rounding.
// Thread per ghost.
__global__ void __launch_bounds__(128) ghost_weights_kernel(GeneralMesh M, double* __restrict__ sw, int* __restrict__ smatch) {
    const int64_t n_ghosts = M.n_total - M.n_domain;
    for (int64_t gi = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; gi < n_ghosts;
         gi += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int N = M.eN[M.n_domain + gi];
        const double* xe = g_nodes + gvec(N);
        const double* we = g_weights + gvec(N);
        const double* bwe = g_bary + gvec(N);
        for (int64_t qe = M.gq_start[gi]; qe < M.gq_start[gi + 1]; ++qe) {
            const int64_t f = M.gq_face[qe];
            const int fs = M.gq_fs[qe];
            const int Nn = M.gq_N[qe];
            const double* xnb = g_nodes + gvec(Nn);
            const double* wnb = g_weights + gvec(Nn);
            const double scale = M.fscale[2 * f + fs], offset = M.foffset[2 * f + fs];
            double* W = sw + M.gq_woff[qe];
            int* match = smatch + M.gq_moff[qe];
            for (int j = 0; j <= Nn; ++j) {
                const double coord = mortar_coord(xnb[Nn - j], scale, offset);
                int found = -1;
                for (int ii = 0; ii <= N; ++ii)
                    if (almost_equal(coord, xe[ii])) {
                        found = ii;
                        break;
                    }
                match[j] = found;
                if (found >= 0) {
                    for (int i = 0; i <= N; ++i) W[i * (Nn + 1) + j] = (i == found) ? __ddiv_rn(wnb[j], we[i]) : 0.0;
                } else {
                    double sb = 0.0;
                    for (int ii = 0; ii <= N; ++ii) sb = __dadd_rn(sb, __ddiv_rn(bwe[ii], __dsub_rn(coord, xe[ii])));
                    for (int i = 0; i <= N; ++i) {
                        const double T = __ddiv_rn(bwe[i], __dmul_rn(__dsub_rn(coord, xe[i]), sb));
                        W[i * (Nn + 1) + j] = __ddiv_rn(__dmul_rn(T, wnb[j]), we[i]);
                    }
                }
            }
        }
    }
}

// Trace value each face-node slot reads on each face side
// (Mesh2D_t::project_to_faces, Mesh2D_t.cpp:3803-3893): the element side's
// node (side 0) or its mirror (side 1) where the face side is conforming, the
// matched node where the face node coincides with an element node, otherwise
// -1 - (32 (2 f + side) + j): the face side and node to interpolate at.
__global__ void __launch_bounds__(128) slot_sources_kernel(GeneralMesh M, int64_t* __restrict__ src) {
    for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < 2 * M.n_slots;
         idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t slot = idx / 2;
        const int side = static_cast<int>(idx - 2 * slot);
        const int64_t d = M.slot_desc[slot];
        const int64_t f = d / 32;
        const int j = static_cast<int>(d - 32 * f);
        const int64_t b = M.fbase[2 * f + side];
        int64_t v;
        if (M.fw_off[2 * f + side] < 0) {
            v = b + (side == 0 ? j : M.fN[f] - j);
        } else {
            const int match = M.fmatch[M.fm_off[2 * f + side] + j];
            v = match >= 0 ? b + match : -1 - (32 * (2 * f + side) + j);
        }
        src[idx] = v;
    }
}

}  // namespace

cudaError_t launch_general_weights(const GeneralMesh& m, double* sw, int* smatch, double* fw, int* fmatch, int64_t* slot_src, cudaStream_t stream) {
    if (m.n_domain > 0) {
        const int blocks = static_cast<int>(std::min<int64_t>((4 * m.n_domain + 127) / 128, 148 * 8));
        side_weights_kernel<<<blocks, 128, 0, stream>>>(m, sw, smatch);
    }
    if (m.n_faces > 0) {
        const int blocks = static_cast<int>(std::min<int64_t>((2 * m.n_faces + 127) / 128, 148 * 8));
        face_weights_kernel<<<blocks, 128, 0, stream>>>(m, fw, fmatch);
    }
    if (m.n_total > m.n_domain) {
        const int blocks = static_cast<int>(std::min<int64_t>((m.n_total - m.n_domain + 127) / 128, 148 * 8));
        ghost_weights_kernel<<<blocks, 128, 0, stream>>>(m, sw, smatch);
    }
    if (m.n_slots > 0) {
        const int blocks = static_cast<int>(std::min<int64_t>((2 * m.n_slots + 127) / 128, 148 * 8));
        slot_sources_kernel<<<blocks, 128, 0, stream>>>(m, slot_src);
    }
    return cudaGetLastError();
}

namespace {

// ---------------------------------------------------------------------------
// Fused stage of one order group: the face fluxes of the elements' sides,
// the derivative, the RK3 update and the new side traces, one CTA per tile
// of EPB elements of the group, one thread per (field, element, line) in the
// derivative as in the uniform kernel. Face values come from the side traces
// of the stage's input (etr: the previous stage's output, and the ghost
// traces of general_ghosts_kernel); the new traces go to etr_out. Every value
// is computed with the operations, in the order, of the reference's separate
// steps, so strict instantiations stay bit-identical to its CPU path.

// Values of the three fields at node j of face side fs2 = 2 f + side whose
// element side is interpolated to the face (Mesh2D_t::project_to_faces,
// Mesh2D_t.cpp:3803-3893): the barycentric sum with the plan's weights over
// its denominator. code = 32 fs2 + j.
template <bool S, typename R>
__device__ __forceinline__ void slot_interp(const GeneralMesh& M, const R* __restrict__ tr, int64_t ft, int64_t code, R v[3]) {
    const int64_t fs2 = code / 32;
    const int j = static_cast<int>(code - 32 * fs2);
    const int Ne = M.fsN[fs2], Nf = M.fN[fs2 / 2];
    const R* ep = tr + M.fbase[fs2];
    const double* tw = M.fw + M.fw_off[fs2];
    const double* tj = tw + j * (Ne + 1);
    const R den = R(tw[(Nf + 1) * (Ne + 1) + j]);
    R pn = 0, un = 0, vn = 0;
    for (int i = 0; i <= Ne; ++i) {
        const R t = R(tj[i]);
        pn = madd<S>(pn, t, ep[i]);
        un = madd<S>(un, t, ep[i + ft]);
        vn = madd<S>(vn, t, ep[i + 2 * ft]);
    }
    v[0] = div<S>(pn, den);
    v[1] = div<S>(un, den);
    v[2] = div<S>(vn, den);
}

// Tile of the fused stage: FP64 arrays (the q tile, element numbers
// and offsets, the sides' slot ranges and flux modes) then arrays of the
// arithmetic type R. About 128 threads per CTA: the stage's time on a small
// order group is one CTA's dependent chain, so tiles are kept short.
template <int N, typename R>
struct FusedTile {
    static constexpr int n = N + 1;
    static constexpr int NN = n * n;
    static constexpr int raw = 128 / (3 * n);
    static constexpr int EPB = raw >= 1 ? raw : 1;
    static constexpr int kThreads = (3 * EPB * n + 31) / 32 * 32;
    static constexpr int kVals = 3 * EPB * NN;     // values of a [3][EPB][NN] field tile
    static_assert(4 * EPB < kThreads, "one thread per tile side and one more");
    // doubles (the RK register k is read from global memory in the update:
    // a k tile here measured 3.4% slower per step, its shared memory costing
    // a CTA per SM)
    static constexpr int kQ = 0;                   // [3][EPB][NN] q, then the new q
    static constexpr int kOff = kQ + kVals;        // [EPB] field offset, [EPB] trace offset,
                                                   // [4 EPB + 1] first slot of each side, then the end,
                                                   // [4 EPB + 1] first mortar entry of each side, then the end (int64)
    static constexpr int kMode = kOff + 10 * EPB + 2;  // [4 EPB] side flux modes (ints)
    static constexpr int kDoubles = kMode + 2 * EPB;
    // R values past the doubles
    static constexpr int kF = 0;                   // [3][EPB][4][n] element side fluxes
    static constexpr int kJ = kF + 3 * EPB * 4 * n;  // [EPB][NN] J (1/J in the default mode)
    static constexpr int kS = kJ + EPB * NN;       // [EPB][4] edge metric per side
    static constexpr bool kCopy = sizeof(R) != sizeof(double);  // the FP32 form keeps an FP32 copy of the q tile
    static constexpr int kQr = kS + EPB * 4;       // [3][EPB][NN] q in R (FP32 form only)
    // [3][EPB][NN] G and [3][EPB][4][slots] face fluxes at the sides' face
    // nodes. In the FP32 form G takes the face fluxes' place once they are
    // dead (after the element side fluxes), which fits more CTAs per SM; in
    // FP64 that measured slower, so there G has a place of its own.
    static constexpr int kG = kQr + (kCopy ? kVals : 0);
    static constexpr int kFF = kCopy ? kG : kG + kVals;
    static constexpr size_t bytes(int slots) {
        const size_t ff = static_cast<size_t>(3 * EPB * 4) * static_cast<size_t>(slots);
        return sizeof(double) * kDoubles + sizeof(R) * (kFF + (kCopy ? (ff > kVals ? ff : static_cast<size_t>(kVals)) : ff));
    }
};

// One tile of EPB elements of an order group: list positions
// first + base .. first + base + EPB - 1 (at most count - base of them), of
// instance inst, by THREADS threads (at least the tile's own kThreads; the
// extra threads take part in the strided loops and the barriers only).
template <int N, bool S, typename R, int THREADS>
__device__ __forceinline__ void fused_tile(const GeneralStage& a, const int64_t first, const int64_t count, const int64_t base,
                                           const int64_t inst, double* smem) {
    using T = FusedTile<N, R>;
    static_assert(T::kThreads <= THREADS, "a tile needs at least its own threads");
    constexpr int n = T::n, NN = T::NN, EPB = T::EPB;
    double* qs = smem + T::kQ;
    int64_t* eo2 = reinterpret_cast<int64_t*>(smem + T::kOff);  // first value of the tile's elements in a field block
    int64_t* eo1 = eo2 + EPB;                                    // their first side-trace value
    int64_t* sst = eo1 + EPB;                                    // first slot of each tile side, then the end
    int64_t* sqs = sst + 4 * EPB + 1;                            // first mortar entry of each tile side, then the end
    int* smode = reinterpret_cast<int*>(smem + T::kMode);
    R* rs = reinterpret_cast<R*>(smem + T::kDoubles);
    R* gs = rs + T::kG;
    R* fs = rs + T::kF;
    R* js = rs + T::kJ;
    R* ss = rs + T::kS;
    R* ffs = rs + T::kFF;
    // q in the arithmetic type: a converted copy in the FP32 form, the tile itself in FP64
    const R* qv;
    R* qw;
    if constexpr (T::kCopy) {
        qw = rs + T::kQr;
        qv = qw;
    } else {
        qw = nullptr;
        qv = qs;
    }
    constexpr int FS = EPB * 4 * n;
    const int SL = a.side_slots;
    const int FFS = EPB * 4 * SL;
    const GeneralMesh& M = a.m;
    const int tid = threadIdx.x;
    const int ne = static_cast<int>((count - base) < EPB ? (count - base) : EPB);
    const int64_t fb = M.block, ft = M.trace_total;
    double* q = a.q + inst * 3 * fb;
    double* k = a.k + inst * 3 * fb;
    const R* tr = pick<R>(a.etr, a.etr_f) + inst * 3 * ft;
    R* tr_out = pick<R>(a.etr_out, a.etr_out_f) + inst * 3 * ft;
    const R* xn = tab<R>(g_nodes, gf_nodes) + gvec(N);
    const R* lm = tab<R>(g_lagrange_left, gf_lagrange_left) + gvec(N);
    const R* lp = tab<R>(g_lagrange_right, gf_lagrange_right) + gvec(N);
    const double dt = a.step[1];

    // The tile's sides: slot ranges, mortar entries and flux modes, and per
    // element its offsets (plan arrays in list order).
    if (tid <= 4 * ne) {
        const int64_t ps = 4 * (first + base) + tid;
        sst[tid] = M.pslot_start[ps];
        sqs[tid] = M.pq_start[ps];
        if (tid < 4 * ne) smode[tid] = M.pside_mode[ps];
        if (tid < ne) {
            eo2[tid] = M.poff2[first + base + tid];
            eo1[tid] = M.poff1[first + base + tid];
        }
    }
    __syncthreads();
    // q tile: asynchronous copies, waited for before the volume terms. The
    // state is read and rewritten once per stage, evict-first in L2.
    const uint64_t stream_policy = evict_first_policy();
    for (int idx = tid; idx < T::kVals; idx += THREADS) {
        const int f = idx / (EPB * NN), r = idx - f * (EPB * NN);
        const int e = r / NN, node = r - e * NN;
        if (e < ne) {
            const int64_t gi = f * fb + eo2[e] + node;
            cp_async8_stream(qs + idx, q + gi, stream_policy);
        }
    }
    // The RK register of the tile into L2 while the stage runs (the update
    // reads it last, after the CTA's longest chains of dependent loads).
    if (!a.first) {
        constexpr int kLines = (NN + 15) / 16 + 1;  // 128-byte lines an element's NN values can touch
        for (int idx = tid; idx < 3 * ne * kLines; idx += THREADS) {
            const int f = idx / (ne * kLines), r = idx - f * (ne * kLines);
            const int e = r / kLines, l = r - e * kLines;
            prefetch_l2(k + f * fb + eo2[e] + (16 * l < NN ? 16 * l : NN - 1));
        }
    }
    // Face fluxes at every face node of every side (Mesh2D_t.cpp:3803-3893,
    // Solver2D_t.cpp:48-63): one item per slot of the tile's contiguous slot
    // range; the plan names each slot's position side (slot_side).
    const int64_t g0 = sst[0];
    const int n_items = static_cast<int>(sst[4 * ne] - g0);
    const int64_t side0 = 4 * (first + base);
    for (int idx = tid; idx < n_items; idx += THREADS) {
        const int64_t g = g0 + idx;
        const int lo = static_cast<int>(M.slot_side[g] - side0);
        const int slot = static_cast<int>(g - sst[lo]);
        const int64_t src0 = M.slot_src[2 * g], src1 = M.slot_src[2 * g + 1];
        const R nx = R(M.slot_normal[2 * g]), ny = R(M.slot_normal[2 * g + 1]);
        R L[3], Rv[3];
        if (src0 >= 0) {
            L[0] = tr[src0];
            L[1] = tr[src0 + ft];
            L[2] = tr[src0 + 2 * ft];
        } else {
            slot_interp<S, R>(M, tr, ft, -1 - src0, L);
        }
        if (src1 >= 0) {
            Rv[0] = tr[src1];
            Rv[1] = tr[src1 + ft];
            Rv[2] = tr[src1 + 2 * ft];
        } else {
            slot_interp<S, R>(M, tr, ft, -1 - src1, Rv);
        }
        const R wL = add<S>(L[0], add<S>(mul<S>(L[1], nx), mul<S>(L[2], ny)));
        const R wR = sub<S>(Rv[0], add<S>(mul<S>(Rv[1], nx), mul<S>(Rv[2], ny)));
        const R sum = add<S>(wL, wR);
        R* o = ffs + lo * SL + slot;
        o[0] = mul<S>(sub<S>(wL, wR), R(0.5));
        o[FFS] = mul<S>(mul<S>(nx, sum), R(0.5));
        o[2 * FFS] = mul<S>(mul<S>(ny, sum), R(0.5));
    }

    const int f = tid / (EPB * n);
    const int rr = tid - f * (EPB * n);
    const int e = rr / n;
    const int m = rr - e * n;
    const bool active = f < 3 && e < ne;
    const int64_t pe = active ? first + base + e : 0;
    // Corners in FP64: their differences are formed before rounding to R.
    double x0 = 0, y0 = 0, x1 = 0, y1 = 0, x2 = 0, y2 = 0, x3 = 0, y3 = 0;
    if (active) {
        const double* c = M.pcorners + 8 * pe;
        x0 = c[0]; y0 = c[1]; x1 = c[2]; y1 = c[3]; x2 = c[4]; y2 = c[5]; x3 = c[6]; y3 = c[7];
    }
    const MetricLine<S, R> x_xi(R(sub<S>(x1, x0)), R(sub<S>(x2, x3))), y_xi(R(sub<S>(y1, y0)), R(sub<S>(y2, y3)));
    const MetricLine<S, R> x_eta(R(sub<S>(x3, x0)), R(sub<S>(x2, x1))), y_eta(R(sub<S>(y3, y0)), R(sub<S>(y2, y1)));
    if (active) {
        const R tm = xn[m];
        if (f == 2) {
            for (int sd = m; sd < 4; sd += n) {
                const R at = (sd == 0 || sd == 3) ? R(-1) : R(1);
                const R dx = (sd == 0 || sd == 2) ? metric<S, R>(at, x_xi.d0, x_xi.d1) : metric<S, R>(at, x_eta.d0, x_eta.d1);
                const R dy = (sd == 0 || sd == 2) ? metric<S, R>(at, y_xi.d0, y_xi.d1) : metric<S, R>(at, y_eta.d0, y_eta.d1);
                ss[e * 4 + sd] = sqrt(add<S>(mul<S>(dx, dx), mul<S>(dy, dy)));
            }
        }
        const R xe = x_eta(tm), ye = y_eta(tm);
        for (int j = f; j < n; j += 3) {
            const R tj = xn[j];
            const R jac = sub<S>(mul<S>(x_xi(tj), ye), mul<S>(xe, y_xi(tj)));
            js[e * NN + m * n + j] = S ? jac : R(1) / jac;
        }
    }
    // Each thread converts the q values it copied (FP32 form).
    cp_async_wait_all();
    if constexpr (T::kCopy) {
        for (int idx = tid; idx < T::kVals; idx += THREADS) qw[idx] = R(qs[idx]);
    }
    __syncthreads();  // q tile, face fluxes, J, edge metrics

    // Element side fluxes (Mesh2D_t::project_to_elements, Mesh2D_t.cpp:3895-4006):
    // the face flux times the edge metric where one face of the element's
    // order covers the side (reversed and negated for the face's right
    // element), otherwise the mortar projection with the plan's weights.
    for (int idx = tid; idx < ne * 4 * n; idx += THREADS) {
        const int ee = idx / (4 * n), sm = idx - ee * 4 * n;
        const int s = sm / n, i = sm - s * n;
        const int mode = smode[ee * 4 + s];
        const R sfv = ss[ee * 4 + s];
        const R* fl = ffs + (ee * 4 + s) * SL;
        R out[3] = {0, 0, 0};
        if (mode == 1) {
            for (int c = 0; c < 3; ++c) out[c] = mul<S>(fl[c * FFS + i], sfv);
        } else if (mode == 2) {
            for (int c = 0; c < 3; ++c) out[c] = mul<S>(-fl[c * FFS + (N - i)], sfv);
        } else if (mode == 3) {
            const int64_t q0 = sqs[ee * 4 + s], q1 = sqs[ee * 4 + s + 1];
            int slot0 = 0;
            for (int64_t qq = q0; qq < q1; ++qq) {
                const int Nf = M.pq_N[qq];
                const R scale = R(M.pq_scale[qq]);
                const double* W = M.sw + M.pq_woff[qq] + i * (Nf + 1);
                const int* match = M.smatch + M.pq_moff[qq];
                for (int j = 0; j <= Nf; ++j) {
                    const int mt = match[j];
                    const R w = R(W[j]);  // loaded with the match (the sums keep their order)
                    if (mt >= 0 && mt != i) continue;
#pragma unroll
                    for (int c = 0; c < 3; ++c) out[c] = add<S>(out[c], mul<S>(mul<S>(mul<S>(w, fl[c * FFS + slot0 + j]), sfv), scale));
                }
                slot0 += Nf + 1;
            }
        }
        fs[0 * FS + idx] = out[0];
        fs[1 * FS + idx] = out[1];
        fs[2 * FS + idx] = out[2];
    }
    __syncthreads();

    const R* Dh = tab<R>(g_dhat, gf_dhat) + gmat(N);
    const R* w = tab<R>(g_weights, gf_weights) + gvec(N);
    const R* iw = tab<R>(g_inv_weights, gf_inv_weights) + gvec(N);
    const R* F = fs + f * FS + e * 4 * n;

    // xi pass (eta index j = m): Dhat . line + lift, G = -(...) (Solver2D_t.cpp:82-101).
    if (active) {
        const int j = m;
        R col[n];
        const R* P = qv + (0 * EPB + e) * NN + j;
        const R* U = qv + (1 * EPB + e) * NN + j;
        const R* V = qv + (2 * EPB + e) * NN + j;
#pragma unroll
        for (int i = 0; i < n; ++i) {
            if (f == 0) col[i] = sub<S>(mul<S>(y_eta(xn[i]), U[i * n]), mul<S>(x_eta(xn[i]), V[i * n]));
            else if (f == 1) col[i] = mul<S>(y_eta(xn[i]), P[i * n]);
            else col[i] = -mul<S>(x_eta(xn[i]), P[i * n]);
        }
        const R fr = F[1 * n + j], fl3 = F[3 * n + (N - j)];
        R* G = gs + (f * EPB + e) * NN + j;
#pragma unroll
        for (int i = 0; i < n; ++i) {
            R acc = 0;
#pragma unroll
            for (int mm = 0; mm < n; ++mm) acc = madd<S>(acc, Dh[i * n + mm], col[mm]);
            const R lift = S ? div<S>(add<S>(mul<S>(fr, lp[i]), mul<S>(fl3, lm[i])), w[i]) : (fr * lp[i] + fl3 * lm[i]) * iw[i];
            G[i * n] = -add<S>(acc, lift);
        }
    }
    __syncthreads();

    // eta pass (xi index i = m): G = (G - (Dhat . line + lift)) / J (Solver2D_t.cpp:103-133).
    if (active) {
        const int i = m;
        R line[n];
        const R* P = qv + (0 * EPB + e) * NN + i * n;
        const R* U = qv + (1 * EPB + e) * NN + i * n;
        const R* V = qv + (2 * EPB + e) * NN + i * n;
#pragma unroll
        for (int j = 0; j < n; ++j) {
            if (f == 0) line[j] = add<S>(mul<S>(-y_xi(xn[j]), U[j]), mul<S>(x_xi(xn[j]), V[j]));
            else if (f == 1) line[j] = mul<S>(-y_xi(xn[j]), P[j]);
            else line[j] = mul<S>(x_xi(xn[j]), P[j]);
        }
        const R ftp = F[2 * n + (N - i)], fbm = F[0 * n + i];
        R* G = gs + (f * EPB + e) * NN + i * n;
        const R* jrow = js + e * NN + i * n;
#pragma unroll
        for (int j = 0; j < n; ++j) {
            R acc = 0;
#pragma unroll
            for (int mm = 0; mm < n; ++mm) acc = madd<S>(acc, Dh[j * n + mm], line[mm]);
            const R lift = S ? div<S>(add<S>(mul<S>(ftp, lp[j]), mul<S>(fbm, lm[j])), w[j]) : (ftp * lp[j] + fbm * lm[j]) * iw[j];
            const R num = sub<S>(G[j], add<S>(acc, lift));
            G[j] = S ? div<S>(num, jrow[j]) : num * jrow[j];
        }
    }
    __syncthreads();

    // Low-storage RK3 update (Solver2D_t.cpp:138-172), node by node, in FP64.
    const double gdt = mul<S>(a.rk_g, dt);
    for (int idx = tid; idx < T::kVals; idx += THREADS) {
        const int ff = idx / (EPB * NN), r = idx - ff * (EPB * NN);
        const int ee = r / NN, node = r - ee * NN;
        if (ee >= ne) continue;
        const int64_t gi = ff * fb + eo2[ee] + node;
        const double G = static_cast<double>(gs[idx]);
        const double kn = a.first ? G : add<S>(mul<S>(a.rk_a, __ldcs(k + gi)), G);
        const double qn = add<S>(qs[idx], mul<S>(gdt, kn));
        __stcs(k + gi, kn);
        __stcs(q + gi, qn);
        qs[idx] = qn;
        if constexpr (T::kCopy) qw[idx] = R(qn);
        if (a.G_out) a.G_out[inst * 3 * fb + gi] = G;
    }
    __syncthreads();

    // Side traces of the new q for the next stage (Element2D_t.cpp:86-125):
    // item (element, side, node), three fields each.
    for (int idx = tid; idx < ne * 4 * n; idx += THREADS) {
        const int ee = idx / (4 * n), sm = idx - ee * 4 * n;
        const int s = sm / n, mm = sm - s * n;
        const R* l = (s == 0 || s == 3) ? lm : lp;
        const int line = (s < 2) ? mm : N - mm;
        const int b0 = (s == 0 || s == 2) ? line * n : line;
        const int stride = (s == 0 || s == 2) ? 1 : n;
        R* out = tr_out + eo1[ee] + s * n + mm;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const R* qe = qv + (c * EPB + ee) * NN + b0;
            R acc = 0;
#pragma unroll
            for (int j = 0; j < n; ++j) acc = madd<S>(acc, l[j], qe[j * stride]);
            out[c * ft] = acc;
        }
    }
}

// Fused stage of one order group: one CTA per tile.
template <int N, bool S, typename R>
__global__ void __launch_bounds__(FusedTile<N, R>::kThreads) general_fused_kernel(GeneralStage a, OrderGroup grp) {
    extern __shared__ __align__(128) double smem[];
    fused_tile<N, S, R, FusedTile<N, R>::kThreads>(a, grp.first, grp.count, static_cast<int64_t>(blockIdx.x) * FusedTile<N, R>::EPB,
                                                   blockIdx.y, smem);
}

// Element side fluxes of one order group for its split form: the fused
// tile's face-flux and element-side-flux phases, with the same operations
// in the same order, written to sflux in the trace layout (field, then the
// element's four sides of N + 1 values) for conforming_stage_kernel's PRE
// form, which runs the rest of the stage on the uniform kernels' tile. Tiles
// of about 32 side nodes a field (128 threads), with no q tile, so that many
// short tiles share an SM and hide the gathers' latency.
template <int N, typename R>
struct FluxTile {
    static constexpr int n = N + 1;
    static constexpr int EPB = 32 / n >= 1 ? 32 / n : 1;
    static constexpr int kThreads = 128;
    // FP64: 8 CTAs per SM (64 registers, 24 bytes of spills) rather than the
    // free allocation's 7 at 66: mixed 128² step 0.2545 → 0.2507 ms, the hp
    // refining run unchanged. Bounds of 10 and 12 CTAs spill 80-108 bytes and
    // cost the hp run 2-3%; the FP32 form fits 10 at its free 48 registers.
    static constexpr int kMinBlocks = sizeof(R) == 8 ? 8 : 0;
    // doubles: [EPB] trace offsets, [4 EPB + 1] first slot of each side and
    // the end, the same for mortar entries (int64), [4 EPB] flux modes (ints)
    static constexpr int kDoubles = EPB + 2 * (4 * EPB + 1) + 2 * EPB;
    // then R: [EPB][4] edge metrics, [3][EPB][4][slots] face fluxes
    static constexpr size_t bytes(int slots) {
        return sizeof(double) * kDoubles + sizeof(R) * (4 * EPB + static_cast<size_t>(3 * EPB * 4) * static_cast<size_t>(slots));
    }
};

template <int N, bool S, typename R>
__global__ void __launch_bounds__(FluxTile<N, R>::kThreads, FluxTile<N, R>::kMinBlocks) side_flux_kernel(GeneralStage a, OrderGroup grp) {
    using T = FluxTile<N, R>;
    constexpr int n = T::n, EPB = T::EPB, THREADS = T::kThreads;
    extern __shared__ __align__(128) double smem[];
    int64_t* eo1 = reinterpret_cast<int64_t*>(smem);
    int64_t* sst = eo1 + EPB;
    int64_t* sqs = sst + 4 * EPB + 1;
    int* smode = reinterpret_cast<int*>(sqs + 4 * EPB + 1);
    R* ss = reinterpret_cast<R*>(smem + T::kDoubles);
    R* ffs = ss + 4 * EPB;
    const GeneralMesh& M = a.m;
    const int tid = threadIdx.x;
    const int64_t first = grp.first;
    const int64_t base = static_cast<int64_t>(blockIdx.x) * EPB;
    const int ne = static_cast<int>((grp.count - base) < EPB ? (grp.count - base) : EPB);
    const int64_t inst = blockIdx.y;
    const int64_t ft = M.trace_total;
    const R* tr = pick<R>(a.etr, a.etr_f) + inst * 3 * ft;
    R* out_flux = pick<R>(a.sflux, a.sflux_f) + inst * 3 * ft;
    const int SL = a.side_slots;
    const int FFS = EPB * 4 * SL;

    if (tid <= 4 * ne) {
        const int64_t ps = 4 * (first + base) + tid;
        sst[tid] = M.pslot_start[ps];
        sqs[tid] = M.pq_start[ps];
        if (tid < 4 * ne) smode[tid] = M.pside_mode[ps];
        if (tid < ne) eo1[tid] = M.poff1[first + base + tid];
    }
    // Edge metric of each side (Element2D_t.cpp:756-769), thread per side.
    if (tid < 4 * ne) {
        const int ee = tid / 4, sd = tid - 4 * ee;
        const double* c = M.pcorners + 8 * (first + base + ee);
        const double x0 = c[0], y0 = c[1], x1 = c[2], y1 = c[3], x2 = c[4], y2 = c[5], x3 = c[6], y3 = c[7];
        const MetricLine<S, R> x_xi(R(sub<S>(x1, x0)), R(sub<S>(x2, x3))), y_xi(R(sub<S>(y1, y0)), R(sub<S>(y2, y3)));
        const MetricLine<S, R> x_eta(R(sub<S>(x3, x0)), R(sub<S>(x2, x1))), y_eta(R(sub<S>(y3, y0)), R(sub<S>(y2, y1)));
        const R at = (sd == 0 || sd == 3) ? R(-1) : R(1);
        const R dx = (sd == 0 || sd == 2) ? metric<S, R>(at, x_xi.d0, x_xi.d1) : metric<S, R>(at, x_eta.d0, x_eta.d1);
        const R dy = (sd == 0 || sd == 2) ? metric<S, R>(at, y_xi.d0, y_xi.d1) : metric<S, R>(at, y_eta.d0, y_eta.d1);
        ss[tid] = sqrt(add<S>(mul<S>(dx, dx), mul<S>(dy, dy)));
    }
    __syncthreads();

    // Face fluxes at every face node of the tile's sides (Mesh2D_t.cpp:3803-3893,
    // Solver2D_t.cpp:48-63), as in fused_tile.
    const int64_t g0 = sst[0];
    const int n_items = static_cast<int>(sst[4 * ne] - g0);
    const int64_t side0 = 4 * (first + base);
    for (int idx = tid; idx < n_items; idx += THREADS) {
        const int64_t g = g0 + idx;
        const int lo = static_cast<int>(M.slot_side[g] - side0);
        const int slot = static_cast<int>(g - sst[lo]);
        const int64_t src0 = M.slot_src[2 * g], src1 = M.slot_src[2 * g + 1];
        const R nx = R(M.slot_normal[2 * g]), ny = R(M.slot_normal[2 * g + 1]);
        R L[3], Rv[3];
        if (src0 >= 0) {
            L[0] = tr[src0];
            L[1] = tr[src0 + ft];
            L[2] = tr[src0 + 2 * ft];
        } else {
            slot_interp<S, R>(M, tr, ft, -1 - src0, L);
        }
        if (src1 >= 0) {
            Rv[0] = tr[src1];
            Rv[1] = tr[src1 + ft];
            Rv[2] = tr[src1 + 2 * ft];
        } else {
            slot_interp<S, R>(M, tr, ft, -1 - src1, Rv);
        }
        const R wL = add<S>(L[0], add<S>(mul<S>(L[1], nx), mul<S>(L[2], ny)));
        const R wR = sub<S>(Rv[0], add<S>(mul<S>(Rv[1], nx), mul<S>(Rv[2], ny)));
        const R sum = add<S>(wL, wR);
        R* o = ffs + lo * SL + slot;
        o[0] = mul<S>(sub<S>(wL, wR), R(0.5));
        o[FFS] = mul<S>(mul<S>(nx, sum), R(0.5));
        o[2 * FFS] = mul<S>(mul<S>(ny, sum), R(0.5));
    }
    __syncthreads();

    // Element side fluxes (Mesh2D_t::project_to_elements, Mesh2D_t.cpp:3895-4006),
    // as in fused_tile, into the element's trace-layout slots of sflux.
    for (int idx = tid; idx < ne * 4 * n; idx += THREADS) {
        const int ee = idx / (4 * n), sm = idx - ee * 4 * n;
        const int s = sm / n, i = sm - s * n;
        const int mode = smode[ee * 4 + s];
        const R sfv = ss[ee * 4 + s];
        const R* fl = ffs + (ee * 4 + s) * SL;
        R out[3] = {0, 0, 0};
        if (mode == 1) {
            for (int c = 0; c < 3; ++c) out[c] = mul<S>(fl[c * FFS + i], sfv);
        } else if (mode == 2) {
            for (int c = 0; c < 3; ++c) out[c] = mul<S>(-fl[c * FFS + (N - i)], sfv);
        } else if (mode == 3) {
            const int64_t q0 = sqs[ee * 4 + s], q1 = sqs[ee * 4 + s + 1];
            int slot0 = 0;
            for (int64_t qq = q0; qq < q1; ++qq) {
                const int Nf = M.pq_N[qq];
                const R scale = R(M.pq_scale[qq]);
                const double* W = M.sw + M.pq_woff[qq] + i * (Nf + 1);
                const int* match = M.smatch + M.pq_moff[qq];
                for (int j = 0; j <= Nf; ++j) {
                    const int mt = match[j];
                    const R w = R(W[j]);  // loaded with the match (the sums keep their order)
                    if (mt >= 0 && mt != i) continue;
#pragma unroll
                    for (int c = 0; c < 3; ++c) out[c] = add<S>(out[c], mul<S>(mul<S>(mul<S>(w, fl[c * FFS + slot0 + j]), sfv), scale));
                }
                slot0 += Nf + 1;
            }
        }
        R* o = out_flux + eo1[ee] + sm;
        o[0] = out[0];
        o[ft] = out[1];
        o[2 * ft] = out[2];
    }
}

// Fused stage of every order group in one launch: one CTA of kQueueThreads
// threads per entry of the stage queue (the tiles of every group, largest
// order first, then the next instance), which names the tile's order; the
// CTA runs that order's tile. The block scheduler hands out the entries in
// queue order as CTAs retire, so the long high-order tiles start first.
// One order's tile as a function of its own (not inlined), so that each
// order is register-allocated on its own rather than the sixteen together;
// the stage arguments reach it through a restrict pointer to the kernel's
// parameter, so the mesh arrays' addresses stay in registers across the
// tile's stores.
template <int N, bool S, typename R>
__device__ __noinline__ void queue_tile(const GeneralStage* __restrict__ ap, int64_t first, int64_t count, int64_t base, int64_t inst,
                                        double* smem) {
    fused_tile<N, S, R, kQueueThreads>(*ap, first, count, base, inst, smem);
}

template <bool S, typename R>
__global__ void __launch_bounds__(kQueueThreads, 6) general_stage_kernel(const __grid_constant__ GeneralStage a, StageQueue wq) {
    extern __shared__ __align__(128) double smem[];
    const int64_t it = blockIdx.x;
    const int64_t inst = it / wq.n_tiles;
    const QueueTile w = wq.tiles[it - inst * wq.n_tiles];
    switch (w.N) {
#define NDG_TILE_CASE(n_) \
    case n_: queue_tile<n_, S, R>(&a, w.first, w.count, w.base, inst, smem); break;
        NDG_TILE_CASE(1) NDG_TILE_CASE(2) NDG_TILE_CASE(3) NDG_TILE_CASE(4) NDG_TILE_CASE(5) NDG_TILE_CASE(6)
        NDG_TILE_CASE(7) NDG_TILE_CASE(8) NDG_TILE_CASE(9) NDG_TILE_CASE(10) NDG_TILE_CASE(11) NDG_TILE_CASE(12)
        NDG_TILE_CASE(13) NDG_TILE_CASE(14) NDG_TILE_CASE(15) NDG_TILE_CASE(16)
#undef NDG_TILE_CASE
        default: break;
    }
}

// Plane-wave initial condition at every node of a group (Mesh2D_t.cpp:1192-1216).
template <int N>
__global__ void __launch_bounds__(256) general_ic_kernel(GeneralStage a, const int64_t* __restrict__ ids, int64_t count) {
    constexpr int n = N + 1, NN = n * n;
    const double* xn = g_nodes + gvec(N);
    const int64_t fb = a.m.block;
    const int64_t total = count * NN;
    for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < total * a.n_instances;
         idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t inst = idx / total;
        const int64_t r = idx - inst * total;
        const int64_t le = r / NN;
        const int node = static_cast<int>(r - le * NN);
        const int i = node / n, j = node - i * n;
        const int64_t e = ids[le];
        const double* c = a.m.corners + 8 * e;
        // quad_map (include/functions/quad_map.tpp): bilinear map of (xi_i, eta_j).
        const double xi = xn[i], eta = xn[j];
        const double am = __dsub_rn(1.0, xi), bp = __dadd_rn(xi, 1.0), cm = __dsub_rn(1.0, eta), dp = __dadd_rn(eta, 1.0);
        const double x = __dmul_rn(__dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(__dmul_rn(c[0], am), cm), __dmul_rn(__dmul_rn(c[2], bp), cm)), __dmul_rn(__dmul_rn(c[4], bp), dp)),
                                             __dmul_rn(__dmul_rn(c[6], am), dp)),
                                   0.25);
        const double y = __dmul_rn(__dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(__dmul_rn(c[1], am), cm), __dmul_rn(__dmul_rn(c[3], bp), cm)), __dmul_rn(__dmul_rn(c[5], bp), dp)),
                                             __dmul_rn(__dmul_rn(c[7], am), dp)),
                                   0.25);
        double p, u, v;
        plane_wave(x, y, 0.0, p, u, v);
        const int64_t gi = inst * 3 * fb + a.m.off2[e] + node;
        a.q[gi] = p;
        a.q[gi + fb] = u;
        a.q[gi + 2 * fb] = v;
        a.k[gi] = 0.0;
        a.k[gi + fb] = 0.0;
        a.k[gi + 2 * fb] = 0.0;
    }
}

// Field transfer, one thread per (instance, field, new element, node)
// (Element2D_t::interpolate_from, same points; Element2D_t.cpp:464-579),
// always rounded as the reference rounds.
__global__ void __launch_bounds__(256) transfer_kernel(Transfer t, int max_nn) {
    const int64_t per_field = t.n_elements * max_nn;
    const int64_t total = per_field * t.n_fields * t.n_instances;
    for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < total; idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t fi = idx / per_field;  // instance * n_fields + field
        const int64_t r = idx - fi * per_field;
        const int64_t e = r / max_nn;
        const int node = static_cast<int>(r - e * max_nn);
        const int Nn = t.new_N[e], No = t.old_N[e];
        const int nn = Nn + 1, no = No + 1;
        if (node >= nn * nn) continue;
        const double* src = t.src + fi * t.old_block + t.old_off2[e];
        double* dst = t.dst + fi * t.new_block + t.new_off2[e] + node;
        const int mode = t.mode ? t.mode[e] : (Nn == No ? 0 : 1);
        if (mode == 0) {
            *dst = src[node];
            continue;
        }
        if (t.zero_changed) {
            *dst = 0.0;
            continue;
        }
        const int i = node / nn, j = node - i * nn;
        const double x = mode == 2 ? t.coords[t.coord_off[e] + 2 * node] : g_nodes[gvec(Nn) + i];
        const double y = mode == 2 ? t.coords[t.coord_off[e] + 2 * node + 1] : g_nodes[gvec(Nn) + j];
        const double* xo = g_nodes + gvec(No);
        const double* bo = g_bary + gvec(No);
        int row = -1, col = -1;
        for (int mm = 0; mm <= No; ++mm) {
            if (almost_equal(x, xo[mm])) col = mm;
            if (almost_equal(y, xo[mm])) row = mm;
        }
        double v;
        if (row != -1 && col != -1) {
            v = src[col * no + row];
        } else if (row != -1) {
            double num = 0.0, den = 0.0;
            for (int mm = 0; mm <= No; ++mm) {
                const double tt = __ddiv_rn(bo[mm], __dsub_rn(x, xo[mm]));
                num = __dadd_rn(num, __dmul_rn(tt, src[mm * no + row]));
                den = __dadd_rn(den, tt);
            }
            v = __ddiv_rn(num, den);
        } else if (col != -1) {
            double num = 0.0, den = 0.0;
            for (int mm = 0; mm <= No; ++mm) {
                const double tt = __ddiv_rn(bo[mm], __dsub_rn(y, xo[mm]));
                num = __dadd_rn(num, __dmul_rn(tt, src[col * no + mm]));
                den = __dadd_rn(den, tt);
            }
            v = __ddiv_rn(num, den);
        } else {
            double dx = 0.0, dy = 0.0;
            for (int kk = 0; kk <= No; ++kk) {
                dx = __dadd_rn(dx, __ddiv_rn(bo[kk], __dsub_rn(x, xo[kk])));
                dy = __dadd_rn(dy, __ddiv_rn(bo[kk], __dsub_rn(y, xo[kk])));
            }
            v = 0.0;
            for (int mm = 0; mm <= No; ++mm) {
                const double tx = __ddiv_rn(bo[mm], __dmul_rn(__dsub_rn(x, xo[mm]), dx));
                for (int nn2 = 0; nn2 <= No; ++nn2) {
                    const double ty = __ddiv_rn(bo[nn2], __dmul_rn(__dsub_rn(y, xo[nn2]), dy));
                    v = __dadd_rn(v, __dmul_rn(__dmul_rn(src[mm * no + nn2], tx), ty));
                }
            }
        }
        *dst = v;
    }
}

int grid_for(int64_t items, int threads) {
    const int64_t b = (items + threads - 1) / threads;
    return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(b, 148 * 32)));
}

template <int N, bool S, typename R>
cudaError_t launch_group_traces(const GeneralStage& a, const OrderGroup& g, cudaStream_t stream) {
    general_traces_kernel<N, S, R><<<grid_for(g.count * 4 * (N + 1) * a.n_instances, 256), 256, 0, stream>>>(a, g.ids, g.count);
    return cudaGetLastError();
}

template <int N, bool S, typename R>
cudaError_t launch_fused(const GeneralStage& a, const OrderGroup& g, cudaStream_t stream) {
    using T = FusedTile<N, R>;
    const dim3 grid(static_cast<unsigned>((g.count + T::EPB - 1) / T::EPB), static_cast<unsigned>(a.n_instances));
    general_fused_kernel<N, S, R><<<grid, T::kThreads, T::bytes(a.side_slots), stream>>>(a, g);
    return cudaGetLastError();
}

template <bool S, typename R>
cudaError_t launch_queue_t(const GeneralStage& a, const StageQueue& wq, cudaStream_t stream) {
    const int64_t ctas = wq.n_tiles * a.n_instances;
    if (ctas > 0x7fffffff) return cudaErrorInvalidValue;
    general_stage_kernel<S, R><<<static_cast<unsigned>(ctas), kQueueThreads, wq.smem_bytes, stream>>>(a, wq);
    return cudaGetLastError();
}

template <int N>
cudaError_t set_attrs(int side_slots) {
    const int b64 = static_cast<int>(FusedTile<N, double>::bytes(side_slots));
    const int b32 = static_cast<int>(FusedTile<N, float>::bytes(side_slots));
    cudaError_t err = cudaFuncSetAttribute(general_fused_kernel<N, false, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, b64);
    if (err == cudaSuccess) err = cudaFuncSetAttribute(general_fused_kernel<N, true, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, b64);
    if (err == cudaSuccess) err = cudaFuncSetAttribute(general_fused_kernel<N, false, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, b32);
    const int f64 = static_cast<int>(FluxTile<N, double>::bytes(side_slots));
    const int f32 = static_cast<int>(FluxTile<N, float>::bytes(side_slots));
    if (err == cudaSuccess) err = cudaFuncSetAttribute(side_flux_kernel<N, false, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, f64);
    if (err == cudaSuccess) err = cudaFuncSetAttribute(side_flux_kernel<N, true, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, f64);
    if (err == cudaSuccess) err = cudaFuncSetAttribute(side_flux_kernel<N, false, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, f32);
    return err;
}

template <int N, bool S, typename R>
cudaError_t launch_side_fluxes(const GeneralStage& a, const OrderGroup& g, cudaStream_t stream) {
    using T = FluxTile<N, R>;
    const dim3 grid(static_cast<unsigned>((g.count + T::EPB - 1) / T::EPB), static_cast<unsigned>(a.n_instances));
    side_flux_kernel<N, S, R><<<grid, T::kThreads, T::bytes(a.side_slots), stream>>>(a, g);
    return cudaGetLastError();
}

template <int N>
cudaError_t launch_ic(const GeneralStage& a, const OrderGroup& g, cudaStream_t stream) {
    general_ic_kernel<N><<<grid_for(g.count * (N + 1) * (N + 1) * a.n_instances, 256), 256, 0, stream>>>(a, g.ids, g.count);
    return cudaGetLastError();
}

// Calls fn.template operator()<N>() for a runtime order 1..16.
template <typename F>
cudaError_t by_order(int N, F&& fn) {
    switch (N) {
        case 1: return fn(std::integral_constant<int, 1>{});
        case 2: return fn(std::integral_constant<int, 2>{});
        case 3: return fn(std::integral_constant<int, 3>{});
        case 4: return fn(std::integral_constant<int, 4>{});
        case 5: return fn(std::integral_constant<int, 5>{});
        case 6: return fn(std::integral_constant<int, 6>{});
        case 7: return fn(std::integral_constant<int, 7>{});
        case 8: return fn(std::integral_constant<int, 8>{});
        case 9: return fn(std::integral_constant<int, 9>{});
        case 10: return fn(std::integral_constant<int, 10>{});
        case 11: return fn(std::integral_constant<int, 11>{});
        case 12: return fn(std::integral_constant<int, 12>{});
        case 13: return fn(std::integral_constant<int, 13>{});
        case 14: return fn(std::integral_constant<int, 14>{});
        case 15: return fn(std::integral_constant<int, 15>{});
        case 16: return fn(std::integral_constant<int, 16>{});
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace

cudaError_t upload_general_tables(const Tables& t) {
    if (t.N_max < 1) return cudaSuccess;
    std::vector<double> nodes(kGVecTotal, 0.0), weights(kGVecTotal, 0.0), inv_w(kGVecTotal, 0.0), bary(kGVecTotal, 0.0), ll(kGVecTotal, 0.0),
        lr(kGVecTotal, 0.0), dhat(kGMatTotal, 0.0);
    for (int N = 0; N <= std::min(t.N_max, kMaxOrder); ++N) {
        for (int i = 0; i <= N; ++i) {
            const size_t at = static_cast<size_t>(gvec(N) + i);
            nodes[at] = t.get(NDG_TABLE_NODES, N)[static_cast<size_t>(i)];
            weights[at] = t.get(NDG_TABLE_WEIGHTS, N)[static_cast<size_t>(i)];
            inv_w[at] = 1.0 / weights[at];
            bary[at] = t.get(NDG_TABLE_BARYCENTRIC_WEIGHTS, N)[static_cast<size_t>(i)];
            ll[at] = t.get(NDG_TABLE_LAGRANGE_LEFT, N)[static_cast<size_t>(i)];
            lr[at] = t.get(NDG_TABLE_LAGRANGE_RIGHT, N)[static_cast<size_t>(i)];
        }
        const auto& d = t.get(NDG_TABLE_DERIVATIVE_MATRICES_HAT, N);
        std::copy(d.begin(), d.end(), dhat.begin() + gmat(N));
    }
    cudaError_t err;
    if ((err = cudaMemcpyToSymbol(g_nodes, nodes.data(), sizeof(double) * kGVecTotal)) != cudaSuccess) return err;
    if ((err = cudaMemcpyToSymbol(g_weights, weights.data(), sizeof(double) * kGVecTotal)) != cudaSuccess) return err;
    if ((err = cudaMemcpyToSymbol(g_inv_weights, inv_w.data(), sizeof(double) * kGVecTotal)) != cudaSuccess) return err;
    if ((err = cudaMemcpyToSymbol(g_bary, bary.data(), sizeof(double) * kGVecTotal)) != cudaSuccess) return err;
    if ((err = cudaMemcpyToSymbol(g_lagrange_left, ll.data(), sizeof(double) * kGVecTotal)) != cudaSuccess) return err;
    if ((err = cudaMemcpyToSymbol(g_lagrange_right, lr.data(), sizeof(double) * kGVecTotal)) != cudaSuccess) return err;
    if ((err = cudaMemcpyToSymbol(g_dhat, dhat.data(), sizeof(double) * kGMatTotal)) != cudaSuccess) return err;
    auto to_f = [](const std::vector<double>& v) { return std::vector<float>(v.begin(), v.end()); };
    const std::vector<float> fn = to_f(nodes), fw = to_f(weights), fiw = to_f(inv_w), fll = to_f(ll), flr = to_f(lr), fd = to_f(dhat);
    if ((err = cudaMemcpyToSymbol(gf_nodes, fn.data(), sizeof(float) * kGVecTotal)) != cudaSuccess) return err;
    if ((err = cudaMemcpyToSymbol(gf_weights, fw.data(), sizeof(float) * kGVecTotal)) != cudaSuccess) return err;
    if ((err = cudaMemcpyToSymbol(gf_inv_weights, fiw.data(), sizeof(float) * kGVecTotal)) != cudaSuccess) return err;
    if ((err = cudaMemcpyToSymbol(gf_lagrange_left, fll.data(), sizeof(float) * kGVecTotal)) != cudaSuccess) return err;
    if ((err = cudaMemcpyToSymbol(gf_lagrange_right, flr.data(), sizeof(float) * kGVecTotal)) != cudaSuccess) return err;
    return cudaMemcpyToSymbol(gf_dhat, fd.data(), sizeof(float) * kGMatTotal);
}

cudaError_t prepare_general_kernels(int N, int side_slots) {
    const cudaError_t err = prepare_conforming_kernels(N);
    if (err != cudaSuccess) return err;
    return by_order(N, [&](auto c) { return set_attrs<decltype(c)::value>(side_slots); });
}

cudaError_t launch_general_traces(const GeneralStage& a, const OrderGroup* groups, int n_groups, bool strict, bool fp32, cudaStream_t stream) {
    cudaError_t err = cudaSuccess;
    for (int g = 0; g < n_groups && err == cudaSuccess; ++g) {
        if (groups[g].count == 0) continue;
        err = by_order(groups[g].N, [&](auto c) {
            constexpr int N = decltype(c)::value;
            if (fp32) return launch_group_traces<N, false, float>(a, groups[g], stream);
            return strict ? launch_group_traces<N, true, double>(a, groups[g], stream) : launch_group_traces<N, false, double>(a, groups[g], stream);
        });
    }
    return err;
}

cudaError_t launch_general_ghosts(const GeneralStage& a, bool strict, bool fp32, cudaStream_t stream) {
    const int64_t n_ghosts = a.m.n_total - a.m.n_domain;
    if (n_ghosts == 0) return cudaSuccess;
    const int max_n = a.m.max_n;
    const int blocks = grid_for(n_ghosts * max_n * a.n_instances, 128);
    if (fp32) general_ghosts_kernel<false, float><<<blocks, 128, 0, stream>>>(a, max_n);
    else if (strict) general_ghosts_kernel<true, double><<<blocks, 128, 0, stream>>>(a, max_n);
    else general_ghosts_kernel<false, double><<<blocks, 128, 0, stream>>>(a, max_n);
    return cudaGetLastError();
}

cudaError_t launch_general_group(const GeneralStage& a, const OrderGroup& g, bool strict, bool fp32, cudaStream_t stream) {
    if (g.count == 0) return cudaSuccess;
    if (g.conforming) return launch_conforming_group(a, g, strict, fp32, stream);
    if (g.split) {
        const cudaError_t err = by_order(g.N, [&](auto c) {
            constexpr int N = decltype(c)::value;
            if (fp32) return launch_side_fluxes<N, false, float>(a, g, stream);
            return strict ? launch_side_fluxes<N, true, double>(a, g, stream) : launch_side_fluxes<N, false, double>(a, g, stream);
        });
        return err == cudaSuccess ? launch_conforming_group(a, g, strict, fp32, stream, true) : err;
    }
    return by_order(g.N, [&](auto c) {
        constexpr int N = decltype(c)::value;
        if (fp32) return launch_fused<N, false, float>(a, g, stream);
        return strict ? launch_fused<N, true, double>(a, g, stream) : launch_fused<N, false, double>(a, g, stream);
    });
}

size_t general_tile_bytes(int N, int side_slots, bool fp32) {
    size_t b = 0;
    by_order(N, [&](auto c) {
        constexpr int n_ = decltype(c)::value;
        b = fp32 ? FusedTile<n_, float>::bytes(side_slots) : FusedTile<n_, double>::bytes(side_slots);
        return cudaSuccess;
    });
    return b;
}

int general_tile_elements(int N) {
    int e = 0;
    by_order(N, [&](auto c) {
        e = FusedTile<decltype(c)::value, double>::EPB;
        return cudaSuccess;
    });
    return e;
}

cudaError_t prepare_general_queue(size_t smem_bytes) {
    const int b = static_cast<int>(smem_bytes);
    cudaError_t err = cudaFuncSetAttribute(general_stage_kernel<false, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    if (err == cudaSuccess) err = cudaFuncSetAttribute(general_stage_kernel<true, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    if (err == cudaSuccess) err = cudaFuncSetAttribute(general_stage_kernel<false, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    return err;
}

cudaError_t launch_general_queue(const GeneralStage& a, const StageQueue& wq, bool strict, bool fp32, cudaStream_t stream) {
    if (wq.n_tiles == 0) return cudaSuccess;
    if (fp32) return launch_queue_t<false, float>(a, wq, stream);
    return strict ? launch_queue_t<true, double>(a, wq, stream) : launch_queue_t<false, double>(a, wq, stream);
}

cudaError_t launch_general_initial_conditions(const GeneralStage& a, const OrderGroup* groups, int n_groups, cudaStream_t stream) {
    cudaError_t err = cudaSuccess;
    for (int g = 0; g < n_groups && err == cudaSuccess; ++g) {
        if (groups[g].count == 0) continue;
        err = by_order(groups[g].N, [&](auto c) { return launch_ic<decltype(c)::value>(a, groups[g], stream); });
    }
    return err;
}

cudaError_t launch_transfer(const Transfer& t, cudaStream_t stream) {
    if (t.n_elements == 0) return cudaSuccess;
    constexpr int max_nn = (kMaxOrder + 1) * (kMaxOrder + 1);
    transfer_kernel<<<grid_for(t.n_elements * max_nn * t.n_fields * t.n_instances, 256), 256, 0, stream>>>(t, max_nn);
    return cudaGetLastError();
}

}  // namespace dev
}  // namespace ndg
