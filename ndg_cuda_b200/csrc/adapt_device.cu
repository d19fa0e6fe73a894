// The decisions and renumbering counts of an adaptation, on the device
// (Mesh2D_t::adapt, src/meshes/Mesh2D_t.cpp:1644-2268; the reference's device
// version counts per block, include/meshes/Mesh2D_t.tcu:94-707).
//
// From the device-resident error estimate (refine flags and decay rates,
// estimator.cu) and a device copy of the topology (AdaptView), one pass of
// kernels computes what the host's rebuild of the topology needs:
//
//   decisions     per domain element: refine and sigma >= 1 as bits
//                 (Element2D_t::would_p_refine / would_h_refine,
//                 src/entities/Element2D_t.cpp:802-812, follow from them and
//                 the element's order and split level)
//   find_nodes    per side of a splitting element: whether it needs a new
//                 node (no face of the side ends at its midpoint;
//                 Mesh2D_t.cpp:5987-6014)
//   ghosts        copy_interfaces_error and copy_boundaries_error
//                 (Mesh2D_t.cpp:6025-6077): a ghost takes its source's flags
//                 and the new-node flag of the source's side
//   face splits   per face: a new node on one of its elements' sides and
//                 both halves of that side covering part of the face
//                 (Mesh2D_t.cpp:1917-2090)
//   scans         exclusive prefix counts of the splitting elements and of
//                 the split faces, which number the new elements
//                 (i + 3 * splits before i), interior faces, nodes and
//                 second halves of split faces
//
// The host downloads one byte per element side and face plus the two count
// arrays, and rebuilds the element, face, boundary and interface lists with
// them (adapt_h.cpp). Every value a decision depends on is rounded as the
// host's rounds it (explicit IEEE operations, no contraction), so the
// decisions are the reference's.
#include "ndg_internal.hpp"

#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cstdint>

namespace ndg {
namespace dev {

namespace {

constexpr int kScanThreads = 1024;

// Mesh2D_t::almost_equal (Mesh2D_t.cpp:3785-3792).
__device__ __forceinline__ bool same_value(double x, double y) {
    const double d = fabs(__dsub_rn(x, y));
    return d <= __dmul_rn(__dmul_rn(DBL_EPSILON, fabs(__dadd_rn(x, y))), 2.0) || d < DBL_MIN;
}

struct P2 {
    double x, y;
};
__device__ __forceinline__ P2 node_at(const AdaptView& v, int64_t i) { return {v.node_xy[2 * i], v.node_xy[2 * i + 1]}; }
__device__ __forceinline__ P2 midpoint(P2 a, P2 b) { return {__ddiv_rn(__dadd_rn(a.x, b.x), 2.0), __ddiv_rn(__dadd_rn(a.y, b.y), 2.0)}; }
__device__ __forceinline__ P2 minus(P2 a, P2 b) { return {__dsub_rn(a.x, b.x), __dsub_rn(a.y, b.y)}; }
__device__ __forceinline__ double dotp(P2 a, P2 b) { return __dadd_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)); }
__device__ __forceinline__ bool same_point(P2 a, P2 b) { return same_value(a.x, b.x) && same_value(a.y, b.y); }

__device__ __forceinline__ bool wants_h(uint8_t code) { return (code & 1u) && !(code & 2u); }  // refine and sigma < 1

// Per domain element: bit 0 refine, bit 1 sigma >= 1 (from instance 0's
// estimate); new-node flags cleared for every element.
__global__ void decisions_kernel(AdaptView v, const int32_t* __restrict__ refine, const double* __restrict__ sigma, uint8_t* __restrict__ code,
                                 uint8_t* __restrict__ add) {
    for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < v.n_total; e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        code[e] = e < v.n_domain ? static_cast<uint8_t>((refine[e] != 0 ? 1u : 0u) | (sigma[e] >= 1.0 ? 2u : 0u)) : 0;
        reinterpret_cast<uint32_t*>(add)[e] = 0u;
    }
}

// find_nodes (Mesh2D_t.cpp:5987-6014) for the splitting domain elements.
__global__ void find_nodes_kernel(AdaptView v, const uint8_t* __restrict__ code, uint8_t* __restrict__ add) {
    for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < v.n_domain; e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        if (!(wants_h(code[e]) && v.split[e] < v.max_split)) continue;
        for (int s = 0; s < 4; ++s) {
            const P2 mid = midpoint(node_at(v, v.enodes[4 * e + s]), node_at(v, v.enodes[4 * e + (s + 1) % 4]));
            uint8_t a = 1;
            for (int64_t q = v.sface_start[4 * e + s]; q < v.sface_start[4 * e + s + 1]; ++q) {
                const int64_t f = v.sface[q];
                if (same_point(node_at(v, v.fnodes[2 * f]), mid) || same_point(node_at(v, v.fnodes[2 * f + 1]), mid)) {
                    a = 0;
                    break;
                }
            }
            add[4 * e + s] = a;
        }
    }
}

// copy_interfaces_error (Mesh2D_t.cpp:6054-6077): the destination ghost takes
// the origin's flags and the new-node flag of the origin's side.
__global__ void interface_ghosts_kernel(AdaptView v, uint8_t* __restrict__ code_all, uint8_t* __restrict__ add) {
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < v.n_interfaces; i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t src = v.if_origin[i], dst = v.if_destination[i];
        add[4 * dst] = add[4 * src + v.if_origin_side[i]];
        code_all[dst] = code_all[src];
    }
}

// copy_boundaries_error (Mesh2D_t.cpp:6025-6053): a ghost with one face takes
// its neighbour's flags and the new-node flag of the neighbour's side.
__global__ void boundary_ghosts_kernel(AdaptView v, uint8_t* __restrict__ code_all, uint8_t* __restrict__ add) {
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < v.n_boundary; i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int64_t g = v.boundary[i];
        if (v.sface_start[4 * g + 1] - v.sface_start[4 * g] != 1) continue;
        const int64_t f = v.sface[v.sface_start[4 * g]];
        const int fs = v.felem[2 * f] == g ? 1 : 0;
        const int64_t src = v.felem[2 * f + fs];
        add[4 * g] = add[4 * src + v.fside[2 * f + fs]];
        code_all[g] = code_all[src];
    }
}

// "The face lies within this half" (adapt, Mesh2D_t.cpp:2025-2034).
__device__ __forceinline__ bool in_half(double c, double d) {
    return (__dadd_rn(c, DBL_EPSILON) <= 1.0 && d >= __dadd_rn(0.0, DBL_EPSILON)) || (__dadd_rn(d, DBL_EPSILON) <= 1.0 && c >= __dadd_rn(0.0, DBL_EPSILON));
}

// Face split decisions (Mesh2D_t.cpp:1917-2090): the left element's side if it
// gets a new node, else the right one's; the face splits when both halves of
// that side cover part of it.
__global__ void face_split_kernel(AdaptView v, const uint8_t* __restrict__ add, uint8_t* __restrict__ frefine) {
    for (int64_t f = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; f < v.n_faces; f += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        uint8_t r = 0;
        for (int side = 0; side < 2; ++side) {
            const int64_t x = v.felem[2 * f + side];
            const int s = static_cast<int>(v.fside[2 * f + side]);
            if (!add[4 * x + s]) continue;
            const P2 a = node_at(v, v.enodes[4 * x + s]), b = node_at(v, v.enodes[4 * x + (s + 1) % 4]);
            const P2 mid = midpoint(a, b);
            const P2 AB[2] = {minus(mid, a), minus(b, mid)};
            const double inv[2] = {__ddiv_rn(1.0, dotp(AB[0], AB[0])), __ddiv_rn(1.0, dotp(AB[1], AB[1]))};
            const P2 C = node_at(v, v.fnodes[2 * f]), D = node_at(v, v.fnodes[2 * f + 1]);
            const P2 AC[2] = {minus(C, a), minus(C, mid)}, AD[2] = {minus(D, a), minus(D, mid)};
            bool in[2];
            for (int h = 0; h < 2; ++h) in[h] = in_half(__dmul_rn(dotp(AC[h], AB[h]), inv[h]), __dmul_rn(dotp(AD[h], AB[h]), inv[h]));
            r = (in[0] && in[1]) ? 1 : 0;
            break;
        }
        frefine[f] = r;
    }
}

// Splitting domain elements as 0/1 (would_h_refine), for the scan.
__global__ void split_flags_kernel(AdaptView v, const uint8_t* __restrict__ code, uint8_t* __restrict__ out) {
    for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < v.n_domain; e += static_cast<int64_t>(gridDim.x) * blockDim.x)
        out[e] = (wants_h(code[e]) && v.split[e] < v.max_split) ? 1 : 0;
}

// Exclusive scan of 0/1 flags into int64 counts, n + 1 values (the last is
// the total): block sums, a scan of the block sums by one block, then each
// block's scan plus its offset.
__device__ __forceinline__ int64_t block_exclusive_scan(int64_t v, int64_t* red, int64_t* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int64_t x = v;
    for (int o = 1; o < 32; o <<= 1) {
        const int64_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) red[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int64_t w = lane < (kScanThreads / 32) ? red[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            const int64_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        red[lane] = w;  // inclusive over warps
    }
    __syncthreads();
    const int64_t before = (warp > 0 ? red[warp - 1] : 0) + x - v;
    if (total) *total = red[kScanThreads / 32 - 1];
    __syncthreads();
    return before;
}

__global__ void __launch_bounds__(kScanThreads) scan_sums_kernel(const uint8_t* __restrict__ flags, int64_t n, int64_t* __restrict__ sums) {
    __shared__ int64_t red[kScanThreads / 32];
    const int64_t i = blockIdx.x * static_cast<int64_t>(kScanThreads) + threadIdx.x;
    int64_t total = 0;
    block_exclusive_scan(i < n ? flags[i] : 0, red, &total);
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanThreads) scan_offsets_kernel(int64_t* __restrict__ sums, int64_t n_blocks) {
    __shared__ int64_t red[kScanThreads / 32];
    int64_t carry = 0;
    for (int64_t b0 = 0; b0 < n_blocks; b0 += kScanThreads) {
        const int64_t b = b0 + threadIdx.x;
        const int64_t v = b < n_blocks ? sums[b] : 0;
        int64_t total = 0;
        const int64_t ex = block_exclusive_scan(v, red, &total);
        if (b < n_blocks) sums[b] = carry + ex;
        carry += total;
    }
    if (threadIdx.x == 0) sums[n_blocks] = carry;
}

__global__ void __launch_bounds__(kScanThreads) scan_apply_kernel(const uint8_t* __restrict__ flags, int64_t n, const int64_t* __restrict__ sums,
                                                                  int64_t n_blocks, int64_t* __restrict__ out) {
    __shared__ int64_t red[kScanThreads / 32];
    const int64_t i = blockIdx.x * static_cast<int64_t>(kScanThreads) + threadIdx.x;
    const int64_t ex = block_exclusive_scan(i < n ? flags[i] : 0, red, nullptr);
    if (i < n) out[i] = sums[blockIdx.x] + ex;
    if (blockIdx.x == 0 && threadIdx.x == 0) out[n] = sums[n_blocks];
}

cudaError_t exclusive_count(const uint8_t* flags, int64_t n, int64_t* out, int64_t* sums, cudaStream_t stream) {
    const int64_t blocks = std::max<int64_t>(1, (n + kScanThreads - 1) / kScanThreads);
    scan_sums_kernel<<<static_cast<unsigned>(blocks), kScanThreads, 0, stream>>>(flags, n, sums);
    scan_offsets_kernel<<<1, kScanThreads, 0, stream>>>(sums, blocks);
    scan_apply_kernel<<<static_cast<unsigned>(blocks), kScanThreads, 0, stream>>>(flags, n, sums, blocks, out);
    return cudaGetLastError();
}

int grid_of(int64_t n) { return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 16))); }

}  // namespace

int64_t adapt_scan_scratch(int64_t n) { return (std::max<int64_t>(1, (n + kScanThreads - 1) / kScanThreads)) + 1; }

cudaError_t launch_adapt_decisions(const AdaptView& v, const int32_t* refine, const double* sigma, const AdaptOutputs& o, cudaStream_t stream) {
    decisions_kernel<<<grid_of(v.n_total), 256, 0, stream>>>(v, refine, sigma, o.code, o.add);
    find_nodes_kernel<<<grid_of(v.n_domain), 256, 0, stream>>>(v, o.code, o.add);
    if (v.n_interfaces > 0) interface_ghosts_kernel<<<grid_of(v.n_interfaces), 256, 0, stream>>>(v, o.code, o.add);
    if (v.n_boundary > 0) boundary_ghosts_kernel<<<grid_of(v.n_boundary), 256, 0, stream>>>(v, o.code, o.add);
    if (v.n_faces > 0) face_split_kernel<<<grid_of(v.n_faces), 256, 0, stream>>>(v, o.add, o.frefine);
    split_flags_kernel<<<grid_of(v.n_domain), 256, 0, stream>>>(v, o.code, o.split_flags);
    cudaError_t err = cudaGetLastError();
    if (err == cudaSuccess) err = exclusive_count(o.split_flags, v.n_domain, o.split_prefix, o.scan_sums, stream);
    if (err == cudaSuccess) err = exclusive_count(o.frefine, v.n_faces, o.refined_prefix, o.scan_sums, stream);
    return err;
}

}  // namespace dev
}  // namespace ndg
