// Internal types shared by the host (C++) and device (CUDA) parts of the
// library. Not installed; the public surface is include/ndg_b200.h.
#pragma once

#include "../../include/ndg_b200.h"

#include <cuda_runtime_api.h>

#include <array>
#include <cstdint>
#include <string>
#include <vector>

namespace ndg {

constexpr int kMaxOrder = 16;  // highest polynomial order with a compiled kernel

// ---------------------------------------------------------------------------
// Errors: every C entry point converts an ndg::Error into a status and a
// thread-local message.
struct Error {
    ndg_status status;
    std::string message;
};
[[noreturn]] void fail(ndg_status status, const std::string& message);
void set_last_error(const std::string& message);

// ---------------------------------------------------------------------------
// Polynomial tables of NDG_t<LegendrePolynomial_t>, one vector per order.
struct Tables {
    int N_max = -1;
    int64_t n_interp = 0;
    // [table][N] with table in ndg_table order.
    std::array<std::vector<std::vector<double>>, 12> t;
    const std::vector<double>& get(ndg_table table, int N) const { return t[table][static_cast<size_t>(N)]; }
};
Tables build_tables(int N_max, int64_t n_interp);
bool almost_equal(double x, double y);

// ---------------------------------------------------------------------------
// Mesh topology with the reference's numbering.
enum BoundaryKind : int { kWall = 0, kSymmetry = 1, kInflow = 2, kOutflow = 3 };

struct Topology {
    std::vector<double> node_x, node_y;
    int64_t n_domain = 0;                 // domain elements come first
    std::vector<int> elem_N;              // all elements
    std::vector<std::array<int64_t, 4>> elem_nodes;
    std::vector<std::array<int64_t, 4>> elem_face;  // face of each side, -1 when none
    // faces
    std::vector<int> face_N;
    std::vector<std::array<int64_t, 2>> face_nodes, face_elems, face_sides;
    std::vector<std::array<double, 2>> face_normal, face_tangent, face_offset, face_scale;
    std::vector<double> face_length;
    // boundaries and self interfaces
    std::array<std::vector<int64_t>, 4> boundary;
    std::vector<int64_t> if_origin, if_origin_side, if_destination;
    // geometry
    std::vector<double> delta_xy_min;
    std::vector<std::array<double, 2>> center;
    std::vector<std::array<double, 4>> ghost_scale;  // scaling_factor_[s] (constant along a straight side)
    // adaptivity state: Element2D_t::split_level_, status_ (Hilbert H, A, R,
    // B = 0..3), rotation_, the faces of every side (faces_; ghosts use side
    // 0), and ghosts whose boundary storage was resized without new geometry
    // (their scaling factor stays zero, as in the reference)
    std::vector<int> elem_split, elem_status, elem_rotation;
    std::vector<std::array<std::vector<int64_t>, 4>> elem_faces;
    std::vector<uint8_t> ghost_sf_zero;
};

Topology build_topology(const ndg_zone& zone, int initial_N);
Topology read_su2(const std::string& path, int initial_N);
void compute_geometry(Topology& topo, const Tables& tables);
// Fills the adaptivity state of a freshly read mesh: face lists from the
// single faces, split level 0, Hilbert status and rotation of the domain
// elements (Mesh2D_t.cpp:4055-4178), status A and rotation 0 for ghosts.
void init_adaptivity_state(Topology& topo);

// ---------------------------------------------------------------------------
// Device plan of one mesh for the fused stage kernels (uniform order N,
// conforming faces). Per domain element side:
//   link.x = neighbour element whose side trace feeds the face (-1: none),
//   link.y = neighbour side | kind << 2 | role << 5,
// where kind is a SideKind and role is 1 when the element is the face's
// right (second) element.
enum SideKind : int { kInterior = 0, kMirror = 1, kCopy = 2, kAnalytic = 3, kZero = 4 };

struct SidePlan {
    std::vector<int32_t> link;      // 2 per side, 8 per element
    std::vector<double> normal;     // 2 per side, 8 per element
    std::vector<double> gscale;     // ghost scaling factor per side (kMirror/kCopy), 4 per element
    std::vector<double> inflow_xy;  // 4 per side (ghost end points, kAnalytic), 16 per element
    std::vector<double> corners;    // 8 per element: x0, y0, x1, y1, x2, y2, x3, y3
};
SidePlan build_side_plan(const Topology& topo, const Tables& tables);

// True when every element and face has one order and every face is
// conforming, so the fused uniform-order kernels apply.
bool fused_path_applies(const Topology& t);

// Host arrays of the general (mixed-order, mortar) stage path; the field
// names match dev::GeneralMesh.
struct GeneralPlan {
    int64_t n_domain = 0, n_total = 0, n_faces = 0, trace_total = 0, face_total = 0, block = 0;
    std::vector<int32_t> eN;
    std::vector<int64_t> off2, off1, enodes, sface_start, sface;
    std::vector<double> corners, node_xy;
    std::vector<int32_t> fN;
    std::vector<int64_t> foff, fnodes, felem, fside;
    std::vector<double> fnormal, ftangent, foffset, fscale;
    std::vector<int32_t> gkind;
    std::vector<double> gscale;
    std::vector<int64_t> gsrc;
    std::vector<int32_t> gsrc_side;
    std::vector<std::pair<int, std::vector<int64_t>>> groups;  // order, its domain elements
    // Per group, how many of its last elements are conforming and run the
    // conforming stage kernel (0 where they are fewer than half the group,
    // which then keeps its order): on each side one face of the element's
    // order whose nodes are the side's, shared with a neighbour (or ghost) of
    // the same order. Per position side: the first
    // trace value of the neighbour's side, 1 when the element is the face's
    // right element, the face normal (2 values); meaningful for conforming
    // positions only.
    std::vector<int64_t> group_conforming;
    std::vector<int64_t> cnb;
    std::vector<int32_t> crole;
    std::vector<double> cnormal;
    // Mortar weights, filled on the device once per plan. Per entry of
    // sface on a domain element side that is not one conforming face of the
    // element's order: offsets of its (N_e+1) x (N_f+1) projection weights
    // and of its N_f+1 node matches (-1 elsewhere). Per face side that is not
    // conforming: offsets of its (N_f+1) x (N_e+1) interpolation weights
    // followed by N_f+1 denominators, and of its N_f+1 node matches.
    std::vector<int64_t> sw_off, sm_off, fw_off, fm_off;
    int64_t sw_total = 0, sm_total = 0, fw_total = 0, fm_total = 0;
    int64_t side_slots = 1;  // largest sum of (face order + 1) over the faces of one domain element side
    // per face side (2 per face): first value of the element side's trace
    // (off1 + side (N_e + 1)) and the element's order
    std::vector<int64_t> fbase;
    std::vector<int32_t> fsN;
    // Face-node slots of the domain element sides, numbered in the order of
    // the group lists (position p = index of the element in the
    // concatenated lists): side s of position p owns slots
    // [pslot_start[4 p + s], pslot_start[4 p + s + 1]), running over the
    // side's faces in list order and each face's nodes; per slot the face and
    // node as 32 f + j, the face normal (2 values) and the position side
    // 4 p + s that owns the slot (slot_side). pside_mode per position
    // side: 0 no face, 1 one face of the element's order from the side's
    // first to its second node, 2 the same face reversed, 3 mortar.
    std::vector<int64_t> pslot_start, slot_desc;
    std::vector<double> slot_normal;
    std::vector<int32_t> pside_mode, slot_side;
    int64_t n_slots = 0;
    // Mortar sides (mode 3) in list order: side s of position p owns face
    // entries [pq_start[4 p + s], pq_start[4 p + s + 1]), one per face in list
    // order, each with the face order, the element's scaling factor on the
    // face, and the offsets of its weights and node matches (sw_off, sm_off).
    std::vector<int64_t> pq_start, pq_woff, pq_moff;
    std::vector<int32_t> pq_N;
    std::vector<double> pq_scale;
    // off2, off1 and corners of the domain elements in list order.
    std::vector<int64_t> poff2, poff1;
    std::vector<double> pcorners;
    // Ghost side-0 gathers (wall, symmetry and outflow ghosts): ghost g (from
    // n_domain) owns entries [gq_start[g - n_domain], gq_start[g - n_domain + 1]),
    // one per face of its side 0 in list order, each with the face and the
    // neighbour's face side, the neighbour side's trace base and order, and
    // the offsets of its weights [(N_g+1) x (N_n+1)] and node matches [N_n+1]
    // in the side-weight arrays (filled on the device). gframe: normal and
    // tangent of the ghost's first face (4 per ghost). gdirect: where the
    // ghost's gather is one face of its own order whose every node matches
    // the reversed neighbour node with weight exactly 1 (checked with the
    // gather's arithmetic), the neighbour side's trace base; -1 elsewhere.
    std::vector<int64_t> gq_start, gq_face, gq_base, gq_woff, gq_moff, gdirect;
    std::vector<int32_t> gq_fs, gq_N;
    std::vector<double> gframe;
};
// tab: the host tables of the context (node matching of the direct ghost
// gathers; without them no gather is direct).
GeneralPlan build_general_plan(const Topology& t, const Tables* tab = nullptr);

// p-adaptation of the topology (orders of elements, ghosts and faces) from
// per-element refine flags and decay rates. Returns whether an order changed.
bool p_adapt(Topology& t, const int32_t* refine, const double* p_sigma, int N_max, int max_split_level);

// Where a domain element of an adapted mesh takes its solution from.
struct ElementSource {
    int64_t old = -1;  // element of the mesh before adaptation
    int kind = 0;      // 0: same order, copied; 1: new order, same points; 2: child of a split element
    std::array<double, 8> child{}, parent{};  // kind 2: corners x0, y0, ..., x3, y3 of the child and its parent
};
// Decisions of one adaptation computed on the device (adapt_device.cu):
// per element (domain and ghosts) bit 0 refine and bit 1 sigma >= 1, ghosts
// holding their source's (copy_interfaces_error, copy_boundaries_error); per
// element side whether it gets a new node (find_nodes); per face whether it
// splits; the exclusive counts of splitting domain elements (n_domain + 1
// values) and of split faces (n_faces + 1 values).
struct AdaptDecisions {
    std::vector<uint8_t> code, add, face_split;
    std::vector<int64_t> split_prefix, split_face_prefix;
};
// h-adaptation (with the p-refinement of the same pass) of the topology.
// Returns false, leaving t untouched, when no element splits; otherwise
// rebuilds t, recomputes its geometry and fills sources for the new domain
// elements. With `dec` the new-node flags, face splits and counts are the
// device's (refine and p_sigma then carry dec's bits); without, the host
// computes them.
bool h_adapt(Topology& t, const Tables& tables, const int32_t* refine, const double* p_sigma, int N_max, int max_split_level,
             std::vector<ElementSource>& sources, const AdaptDecisions* dec = nullptr);

namespace dev {
// Device copy of the topology that the decisions read (adapt_device.cu).
struct AdaptView {
    int64_t n_domain = 0, n_total = 0, n_faces = 0, n_interfaces = 0, n_boundary = 0;
    int max_split = 0;
    const int* split = nullptr;               // [n_domain] split levels
    const int64_t* enodes = nullptr;          // [4 n_total]
    const int64_t* sface_start = nullptr;     // [4 n_total + 1]
    const int64_t* sface = nullptr;
    const int64_t* fnodes = nullptr;          // [2 n_faces]
    const int64_t* felem = nullptr;
    const int64_t* fside = nullptr;
    const int64_t* if_origin = nullptr;       // [n_interfaces]
    const int64_t* if_origin_side = nullptr;
    const int64_t* if_destination = nullptr;
    const int64_t* boundary = nullptr;        // [n_boundary] the ghosts of the four boundary lists
    const double* node_xy = nullptr;          // [2 n_nodes]
};
struct AdaptOutputs {
    uint8_t* code = nullptr;         // [n_total]
    uint8_t* add = nullptr;          // [4 n_total]
    uint8_t* frefine = nullptr;      // [n_faces]
    uint8_t* split_flags = nullptr;  // [n_domain]
    int64_t* split_prefix = nullptr;      // [n_domain + 1]
    int64_t* refined_prefix = nullptr;    // [n_faces + 1]
    int64_t* scan_sums = nullptr;         // [adapt_scan_scratch(max(n_domain, n_faces))]
};
int64_t adapt_scan_scratch(int64_t n);
cudaError_t launch_adapt_decisions(const AdaptView& v, const int32_t* refine, const double* sigma, const AdaptOutputs& o, cudaStream_t stream);
}  // namespace dev
// Coordinates, in the parent's reference square, of the nodes of order N of
// a child (Element2D_t::interpolate_from with quad_map and inverse_quad_map):
// 2 (N+1)^2 values, node i*(N+1)+j.
void child_coordinates(const ElementSource& src, const std::vector<double>& nodes_N, std::vector<double>& out);

}  // namespace ndg
