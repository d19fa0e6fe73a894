// Stage kernels for meshes of mixed order and nonconforming faces
// (general_kernels.cu): the state after p- or h-adaptation.
#pragma once

#include "ndg_internal.hpp"

#include <cuda_runtime.h>

#include <cstdint>

namespace ndg {
namespace dev {

// What a ghost element's side-0 trace is made of at each stage
// (Mesh2D_t::boundary_conditions, src/meshes/Mesh2D_t.cpp:3731-3782).
enum GhostKind : int {
    kGhostMirror = 0,     // wall and symmetry: projected neighbour trace, normal velocity mirrored
    kGhostAnalytic = 1,   // inflow: the plane wave on the ghost's edge
    kGhostCopy = 2,       // outflow: projected neighbour trace
    kGhostInterface = 3,  // periodic destination: the origin element's side trace
    kGhostNone = 4
};

// Device view of a mixed-order mesh, in the reference's numbering:
// elements 0 .. n_domain-1 are the domain, the rest ghosts.
struct GeneralMesh {
    int64_t n_domain = 0, n_total = 0, n_faces = 0;
    int64_t trace_total = 0;  // values per field of the element side-trace array
    int64_t face_total = 0;   // values per field of the face flux array
    int64_t block = 0;        // values per field block of q, k and G
    int max_n = 1;            // largest order + 1 over elements and faces
    const int* eN = nullptr;            // [n_total] order
    const int64_t* off2 = nullptr;      // [n_domain] first value of the element in a field block
    const int64_t* off1 = nullptr;      // [n_total] first side-trace value (4 (N+1) domain, N+1 ghost)
    const int64_t* enodes = nullptr;    // [4 n_total]
    const int64_t* sface_start = nullptr;  // [4 n_total + 1] faces of side s of element e:
    const int64_t* sface = nullptr;        //   sface[sface_start[4e+s] .. sface_start[4e+s+1])
    const double* corners = nullptr;    // [8 n_domain]
    const double* node_xy = nullptr;    // [2 n_nodes]
    const int* fN = nullptr;            // [n_faces]
    const int64_t* foff = nullptr;      // [n_faces] first flux value of the face
    const int64_t* fnodes = nullptr;    // [2 n_faces]
    const int64_t* felem = nullptr;     // [2 n_faces]
    const int64_t* fside = nullptr;     // [2 n_faces]
    const double* fnormal = nullptr;    // [2 n_faces]
    const double* ftangent = nullptr;   // [2 n_faces]
    const double* foffset = nullptr;    // [2 n_faces]
    const double* fscale = nullptr;     // [2 n_faces]
    const int* gkind = nullptr;         // [n_total - n_domain] GhostKind
    const double* gscale = nullptr;     // [n_total - n_domain] side-0 scaling factor
    const int64_t* gsrc = nullptr;      // [n_total - n_domain] interface origin element
    const int* gsrc_side = nullptr;     // [n_total - n_domain] interface origin side
    // Precomputed mortar weights (launch_general_weights): element side
    // projections per sface entry (weights [N_e+1][N_f+1], node match per
    // face node, -1 = barycentric) and face-side interpolations per
    // (face, side) (weights [N_f+1][N_e+1] then N_f+1 denominators, node
    // match per face node); offsets -1 where the fast conforming path runs.
    const int64_t* fbase = nullptr;     // [2 n_faces] first trace value of each face side's element side
    const int* fsN = nullptr;           // [2 n_faces] order of each face side's element
    const int64_t* sw_off = nullptr;
    const int64_t* sm_off = nullptr;
    const int64_t* fw_off = nullptr;
    const int64_t* fm_off = nullptr;
    const double* sw = nullptr;
    const int* smatch = nullptr;
    const double* fw = nullptr;
    const int* fmatch = nullptr;
    // Face-node slots of the domain element sides in group-list order (side
    // s of list position p owns [pslot_start[4 p + s], pslot_start[4 p + s + 1])):
    // per slot the face and node (32 f + j), the face normal, and per face
    // side the trace value the slot reads (first of the three fields), or,
    // where the face side interpolates, -1 - (32 (2 f + side) + j); per
    // position side its flux mode (0 no face, 1 one conforming face, 2 the
    // same reversed, 3 mortar).
    int64_t n_slots = 0;
    const int64_t* pslot_start = nullptr;  // [4 n_domain + 1]
    const int64_t* slot_desc = nullptr;    // [n_slots]
    const double* slot_normal = nullptr;   // [2 n_slots]
    const int64_t* slot_src = nullptr;     // [2 n_slots], filled by launch_general_weights
    const int* pside_mode = nullptr;       // [4 n_domain]
    const int* slot_side = nullptr;        // [n_slots] the position side 4 p + s owning each slot
    // Conforming position sides (conforming_stage_kernel): the first trace
    // value of the neighbour's side, 1 when the element is the face's right
    // element, and the face normal.
    const int64_t* cnb = nullptr;          // [4 n_domain]
    const int* crole = nullptr;            // [4 n_domain]
    const double* cnormal = nullptr;       // [8 n_domain]
    // Mortar sides (mode 3) in list order: side s of list position p owns
    // entries [pq_start[4 p + s], pq_start[4 p + s + 1]), one per face, with
    // the face order, the element's scaling factor on the face and the
    // offsets of its weights and node matches in sw / smatch.
    const int64_t* pq_start = nullptr;     // [4 n_domain + 1]
    const int* pq_N = nullptr;
    const double* pq_scale = nullptr;
    const int64_t* pq_woff = nullptr;
    const int64_t* pq_moff = nullptr;
    const int64_t* poff2 = nullptr;        // [n_domain] off2 in list order
    const int64_t* poff1 = nullptr;        // [n_domain] off1 in list order
    const double* pcorners = nullptr;      // [8 n_domain] corners in list order
    // Ghost side-0 gathers of the mirror and copy ghosts (ghost g - n_domain
    // owns entries [gq_start[.], gq_start[. + 1])): per entry the face and the
    // neighbour's face side, the neighbour side's trace base and order, and
    // the offsets of its weights and node matches in sw / smatch; gframe is
    // the normal and tangent of each ghost's first face.
    const int64_t* gq_start = nullptr;     // [n_total - n_domain + 1]
    const int64_t* gq_face = nullptr;
    const int* gq_fs = nullptr;
    const int64_t* gq_base = nullptr;
    const int* gq_N = nullptr;
    const int64_t* gq_woff = nullptr;
    const int64_t* gq_moff = nullptr;
    const double* gframe = nullptr;        // [4 (n_total - n_domain)]
    const int64_t* gdirect = nullptr;      // [n_total - n_domain] trace base of a direct one-face gather, or -1
};

// One RK3 stage on a mixed-order mesh.
struct GeneralStage {
    GeneralMesh m;
    double* q = nullptr;      // [instance][field][block]
    double* k = nullptr;
    double* G_out = nullptr;  // optional copy of the stage's time derivative
    double* etr = nullptr;      // [instance][field][trace_total] element side traces of q (ghosts filled by the stage)
    double* etr_out = nullptr;  // the same for the stage's output
    float* etr_f = nullptr;     // the two trace buffers of the FP32 form
    float* etr_out_f = nullptr;
    double* sflux = nullptr;    // [instance][field][trace_total] element side fluxes of a split group
    float* sflux_f = nullptr;   // the same in the FP32 form
    int side_slots = 1;         // largest sum of (face order + 1) over the faces of one element side
    const double* step = nullptr;  // {time, dt, dt_mesh, t_end}
    double rk_a = 0, rk_b = 0, rk_g = 0;
    int first = 0;
    int n_instances = 1;
};

// Elements of one order, processed by one launch of the order's kernels.
struct OrderGroup {
    int N = 0;
    int64_t count = 0;
    const int64_t* ids = nullptr;  // device, element numbers
    int64_t first = 0;             // list position of the group's first element
    int conforming = 0;            // 1: every side one same-order face with a same-order neighbour (conforming_stage_kernel)
    int split = 0;                 // 1: side_flux_kernel, then conforming_stage_kernel over its side fluxes
};

// The stage queue of a mixed-order mesh: every tile of every order group
// (largest order first), one CTA each in one launch per stage
// (launch_general_queue).
constexpr int kQueueThreads = 128;
struct QueueTile {
    int N = 0;
    int64_t first = 0;  // list position of the group's first element
    int64_t count = 0;  // elements of the group
    int64_t base = 0;   // the tile's first element within the group
};
struct StageQueue {
    const QueueTile* tiles = nullptr;
    int64_t n_tiles = 0;    // per instance
    size_t smem_bytes = 0;  // the largest tile of the orders present
};

cudaError_t upload_general_tables(const Tables& t);
// Fills the mortar weights of a plan (once per plan): the same arithmetic,
// in the reference's rounding, as the per-node computation they replace.
// Then the ghost gathers' weights (into sw, smatch) and the trace sources of
// the face-node slots (slot_src).
cudaError_t launch_general_weights(const GeneralMesh& m, double* sw, int* smatch, double* fw, int* fmatch, int64_t* slot_src, cudaStream_t stream);
cudaError_t prepare_general_kernels(int N, int side_slots);
// Side traces of q into etr (before the first stage, or after q changed).
cudaError_t launch_general_traces(const GeneralStage& a, const OrderGroup* groups, int n_groups, bool strict, bool fp32, cudaStream_t stream);
// One stage is the ghost traces into etr, then for every order group the
// fused face fluxes, volume term, RK update and traces of the new state
// into etr_out. The groups read only etr and write disjoint elements, so
// they may run concurrently after the ghost launch.
// fp32: the FP32 form (traces, fluxes and the volume term in FP32 over the
// FP32 trace buffers; q, k and the RK update in FP64).
cudaError_t launch_general_ghosts(const GeneralStage& a, bool strict, bool fp32, cudaStream_t stream);
cudaError_t launch_general_group(const GeneralStage& a, const OrderGroup& g, bool strict, bool fp32, cudaStream_t stream);
// Shared memory and elements of the fused tile of order N.
size_t general_tile_bytes(int N, int side_slots, bool fp32);
int general_tile_elements(int N);
// Opts the queue kernels into smem_bytes of dynamic shared memory.
cudaError_t prepare_general_queue(size_t smem_bytes);
// The fused stage of every order group in one launch (after the ghosts).
cudaError_t launch_general_queue(const GeneralStage& a, const StageQueue& wq, bool strict, bool fp32, cudaStream_t stream);
// Stage kernel of a group of conforming elements (conforming_kernels.cu):
// the uniform-order stage with the neighbour traces gathered by the plan, in
// FP64 (strict or not) or in the FP32 form.
cudaError_t prepare_conforming_kernels(int N);
// pre: the group's element side fluxes are in sflux (sflux_f) already.
cudaError_t launch_conforming_group(const GeneralStage& a, const OrderGroup& g, bool strict, bool fp32, cudaStream_t stream, bool pre = false);
// The plane-wave initial condition at every node of a mixed-order mesh.
cudaError_t launch_general_initial_conditions(const GeneralStage& a, const OrderGroup* groups, int n_groups, cudaStream_t stream);

// Field transfer to a re-ordered mesh (Element2D_t::interpolate_from, same
// element points; src/entities/Element2D_t.cpp:464-579): for new element e,
// old order old_N[e] at old offset old_off2[e]; equal orders copy, others
// interpolate, or write zeros when zero_changed is set (the RK register of a
// re-ordered element starts at zero). Fields: n_fields blocks of old_block /
// new_block values per instance.
struct Transfer {
    const double* src = nullptr;
    double* dst = nullptr;
    int64_t old_block = 0, new_block = 0;
    int n_fields = 3;
    int n_instances = 1;
    int64_t n_elements = 0;
    const int* old_N = nullptr;
    const int64_t* old_off2 = nullptr;
    const int* new_N = nullptr;
    const int64_t* new_off2 = nullptr;
    int zero_changed = 0;  // 1: write zeros where the order changed (RK register)
    // Optional, after h-adaptation: per new element 0 copy, 1 new order at the
    // same points, 2 a child at the node coordinates coords[coord_off[e] ..]
    // (2 per node, in the parent's reference square). Zeros replace every
    // non-copied element when zero_changed is set.
    const int* mode = nullptr;
    const double* coords = nullptr;
    const int64_t* coord_off = nullptr;
};
cudaError_t launch_transfer(const Transfer& t, cudaStream_t stream);

}  // namespace dev
}  // namespace ndg
