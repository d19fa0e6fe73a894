// Host construction of the mesh topology with the reference's numbering, and
// the per-element-side plan that the fused stage kernels read.
//
// The numbering must be bit-for-bit the reference's (faces, element order,
// ghost order, boundary and interface lists), because connectivity, flags
// and solution arrays are compared against it element by element:
//  - elements: QUAD_4 sections in section order, then BAR_2 ghost sections
//    (src/meshes/Mesh2D_t.cpp:658-713);
//  - faces: created in the order domain elements traverse their sides, a side
//    whose reversed node pair already has a face becomes that face's second
//    element; ghosts attach as second elements, flipping their node order
//    when they run the same way as the face (src/meshes/Mesh2D_t.cpp:1110-1190);
//  - boundary lists per CGNS boundary in file order, periodic self interfaces
//    per connectivity (src/meshes/Mesh2D_t.cpp:725-875).
// Faces are looked up by directed node pair in a hash map instead of the
// reference's per-node face lists; for any mesh in which a directed edge
// belongs to at most one domain element (every valid conforming mesh) both
// lookups find the same face, so the numbering is identical.
#include "ndg_internal.hpp"

#include <algorithm>
#include <cmath>
#include <fstream>
#include <sstream>
#include <unordered_map>

namespace ndg {
namespace {

struct EdgeKey {
    int64_t a, b;
    bool operator==(const EdgeKey& o) const { return a == o.a && b == o.b; }
};
struct EdgeHash {
    size_t operator()(const EdgeKey& k) const {
        const uint64_t h = static_cast<uint64_t>(k.a) * 0x9E3779B97F4A7C15ull ^ (static_cast<uint64_t>(k.b) + 0x632BE59BD9B4E019ull);
        return static_cast<size_t>(h ^ (h >> 29));
    }
};

double magnitude(double x, double y) { return std::sqrt(x * x + y * y); }

// quad_metrics (include/functions/quad_metrics.tpp:2-7): returns
// {dx/dxi, dx/deta, dy/dxi, dy/deta} at (xi, eta).
std::array<double, 4> quad_metrics(double xi, double eta, const double* px, const double* py) {
    return {((1 - eta) * (px[1] - px[0]) + (1 + eta) * (px[2] - px[3])) / 4,
            ((1 - xi) * (px[3] - px[0]) + (1 + xi) * (px[2] - px[1])) / 4,
            ((1 - eta) * (py[1] - py[0]) + (1 + eta) * (py[2] - py[3])) / 4,
            ((1 - xi) * (py[3] - py[0]) + (1 + xi) * (py[2] - py[1])) / 4};
}

// Faces from element sides and ghosts (see the file comment).
void build_faces(Topology& t) {
    const int64_t n_all = static_cast<int64_t>(t.elem_nodes.size());
    std::unordered_map<EdgeKey, int64_t, EdgeHash> by_edge;
    by_edge.reserve(static_cast<size_t>(4 * t.n_domain));
    t.elem_face.assign(static_cast<size_t>(n_all), {-1, -1, -1, -1});
    for (int64_t e = 0; e < t.n_domain; ++e) {
        const auto& nd = t.elem_nodes[static_cast<size_t>(e)];
        for (int s = 0; s < 4; ++s) {
            const int64_t a = nd[static_cast<size_t>(s)], b = nd[static_cast<size_t>((s + 1) % 4)];
            auto it = by_edge.find({b, a});
            if (it != by_edge.end()) {
                const size_t f = static_cast<size_t>(it->second);
                t.face_elems[f][1] = e;
                t.face_sides[f][1] = s;
                t.elem_face[static_cast<size_t>(e)][static_cast<size_t>(s)] = it->second;
                continue;
            }
            const int64_t f = static_cast<int64_t>(t.face_nodes.size());
            by_edge.emplace(EdgeKey{a, b}, f);
            t.face_nodes.push_back({a, b});
            t.face_elems.push_back({e, -1});
            t.face_sides.push_back({s, -1});
            t.elem_face[static_cast<size_t>(e)][static_cast<size_t>(s)] = f;
        }
    }
    for (int64_t g = t.n_domain; g < n_all; ++g) {
        auto& nd = t.elem_nodes[static_cast<size_t>(g)];
        const int64_t a = nd[0], b = nd[1];
        int64_t f = -1;
        bool flip = false;
        auto rev = by_edge.find({b, a});
        if (rev != by_edge.end()) {
            f = rev->second;
        } else {
            auto same = by_edge.find({a, b});
            if (same != by_edge.end()) {
                f = same->second;
                flip = true;
            }
        }
        if (f < 0) continue;  // a ghost on no domain edge stays unattached, as in the reference
        t.face_elems[static_cast<size_t>(f)][1] = g;
        t.face_sides[static_cast<size_t>(f)][1] = 0;
        t.elem_face[static_cast<size_t>(g)][0] = f;
        if (flip) {
            // The reference swaps only the first two nodes of the ghost.
            std::swap(nd[0], nd[1]);
        }
    }
    for (size_t f = 0; f < t.face_elems.size(); ++f)
        if (t.face_elems[f][1] < 0)
            fail(NDG_ERR_MESH, "face " + std::to_string(f) + " has a single element and no boundary element");
    t.face_N.assign(t.face_nodes.size(), t.elem_N.empty() ? 0 : t.elem_N[0]);
}

}  // namespace

Topology build_topology(const ndg_zone& z, int initial_N) {
    if (z.n_nodes <= 0 || !z.x || !z.y) fail(NDG_ERR_INVALID_ARG, "zone has no nodes");
    if (z.n_sections <= 0 || !z.section_type || !z.section_start || !z.section_end || !z.section_connectivity)
        fail(NDG_ERR_INVALID_ARG, "zone has no sections");
    Topology t;
    t.node_x.assign(z.x, z.x + z.n_nodes);
    t.node_y.assign(z.y, z.y + z.n_nodes);

    // Element numbering: QUAD_4 sections first, then BAR_2 (Mesh2D_t.cpp:658-713).
    int64_t n_quad = 0, n_bar = 0;
    for (int32_t s = 0; s < z.n_sections; ++s) {
        const int64_t cnt = z.section_end[s] - z.section_start[s] + 1;
        if (cnt < 0) fail(NDG_ERR_MESH, "section with a negative element range");
        if (z.section_type[s] == 0) n_quad += cnt;
        else if (z.section_type[s] == 1) n_bar += cnt;
        else fail(NDG_ERR_MESH, "only QUAD_4 and BAR_2 sections are supported");
    }
    t.n_domain = n_quad;
    t.elem_N.assign(static_cast<size_t>(n_quad + n_bar), initial_N);
    t.elem_nodes.resize(static_cast<size_t>(n_quad + n_bar));
    std::vector<int64_t> first_index(static_cast<size_t>(z.n_sections));
    int64_t next_quad = 0, next_bar = n_quad, conn = 0;
    auto node_at = [&](int64_t one_based) {
        if (one_based < 1 || one_based > z.n_nodes) fail(NDG_ERR_MESH, "element references node " + std::to_string(one_based) + " out of range");
        return one_based - 1;
    };
    for (int32_t s = 0; s < z.n_sections; ++s) {
        const int64_t cnt = z.section_end[s] - z.section_start[s] + 1;
        if (z.section_type[s] == 0) {
            first_index[static_cast<size_t>(s)] = next_quad;
            for (int64_t j = 0; j < cnt; ++j) {
                auto& nd = t.elem_nodes[static_cast<size_t>(next_quad + j)];
                for (int k = 0; k < 4; ++k) nd[static_cast<size_t>(k)] = node_at(z.section_connectivity[conn + 4 * j + k]);
            }
            next_quad += cnt;
            conn += 4 * cnt;
        } else {
            first_index[static_cast<size_t>(s)] = next_bar;
            for (int64_t j = 0; j < cnt; ++j) {
                const int64_t a = node_at(z.section_connectivity[conn + 2 * j]);
                const int64_t b = node_at(z.section_connectivity[conn + 2 * j + 1]);
                t.elem_nodes[static_cast<size_t>(next_bar + j)] = {a, b, b, a};
            }
            next_bar += cnt;
            conn += 2 * cnt;
        }
    }
    auto element_of = [&](int64_t one_based) -> int64_t {
        for (int32_t s = 0; s < z.n_sections; ++s)
            if (one_based >= z.section_start[s] && one_based <= z.section_end[s])
                return first_index[static_cast<size_t>(s)] + one_based - z.section_start[s];
        fail(NDG_ERR_MESH, "element " + std::to_string(one_based) + " is in no section");
    };

    build_faces(t);

    // Boundary lists (Mesh2D_t.cpp:725-816); NULL boundaries are not listed.
    int64_t off = 0;
    for (int32_t b = 0; b < z.n_bocos; ++b) {
        const int32_t type = z.boco_type[b];
        for (int64_t j = 0; j < z.boco_count[b]; ++j) {
            const int64_t e = element_of(z.boco_points[off + j]);
            if (type >= 0 && type < 4) t.boundary[static_cast<size_t>(type)].push_back(e);
            else if (type != NDG_BC_NULL) fail(NDG_ERR_MESH, "unknown boundary type");
        }
        off += z.boco_count[b];
    }
    // Periodic self interfaces (Mesh2D_t.cpp:818-875): the receiving ghost
    // copies the side trace of the domain element next to the donor ghost.
    off = 0;
    for (int32_t c = 0; c < z.n_conns; ++c) {
        for (int64_t j = 0; j < z.conn_count[c]; ++j) {
            const int64_t dest = element_of(z.conn_points[off + j]);
            const int64_t donor_ghost = element_of(z.conn_donors[off + j]);
            const int64_t f = t.elem_face[static_cast<size_t>(donor_ghost)][0];
            if (f < 0) fail(NDG_ERR_MESH, "periodic donor element is not attached to a face");
            const size_t side = t.face_elems[static_cast<size_t>(f)][0] == donor_ghost ? 1 : 0;
            t.if_origin.push_back(t.face_elems[static_cast<size_t>(f)][side]);
            t.if_origin_side.push_back(t.face_sides[static_cast<size_t>(f)][side]);
            t.if_destination.push_back(dest);
        }
        off += z.conn_count[c];
    }
    return t;
}

// Element and face geometry (Element2D_t.cpp:743-790, Face2D_t.cpp:56-81,
// Mesh2D_t.cpp:4026-4053, 4208-4235).
void compute_geometry(Topology& t, const Tables& tables) {
    const size_t n_all = t.elem_nodes.size();
    t.delta_xy_min.assign(n_all, 0.0);
    t.center.assign(n_all, {0.0, 0.0});
    t.ghost_scale.assign(n_all, {0.0, 0.0, 0.0, 0.0});
    for (size_t e = 0; e < n_all; ++e) {
        double px[4], py[4];
        for (int k = 0; k < 4; ++k) {
            px[k] = t.node_x[static_cast<size_t>(t.elem_nodes[e][static_cast<size_t>(k)])];
            py[k] = t.node_y[static_cast<size_t>(t.elem_nodes[e][static_cast<size_t>(k)])];
        }
        const double x0 = tables.get(NDG_TABLE_NODES, t.elem_N[e])[0];
        if (static_cast<int64_t>(e) < t.n_domain) {
            const double d[6] = {magnitude(px[1] - px[0], py[1] - py[0]), magnitude(px[2] - px[3], py[2] - py[3]),
                                 magnitude(px[1] - px[2], py[1] - py[2]), magnitude(px[0] - px[3], py[0] - py[3]),
                                 magnitude(px[1] - px[3], py[1] - py[3]), magnitude(px[2] - px[0], py[2] - py[0])};
            t.delta_xy_min[e] = std::min(std::min(std::min(d[0], d[1]), std::min(d[2], d[3])), std::min(d[4], d[5]));
            t.center[e] = {(px[0] + px[1] + px[2] + px[3]) / 4, (py[0] + py[1] + py[2] + py[3]) / 4};
            const auto mb = quad_metrics(x0, -1.0, px, py);
            const auto mr = quad_metrics(1.0, x0, px, py);
            const auto mt = quad_metrics(x0, 1.0, px, py);
            const auto ml = quad_metrics(-1.0, x0, px, py);
            t.ghost_scale[e] = {std::sqrt(mb[0] * mb[0] + mb[2] * mb[2]), std::sqrt(mr[1] * mr[1] + mr[3] * mr[3]),
                                std::sqrt(mt[0] * mt[0] + mt[2] * mt[2]), std::sqrt(ml[1] * ml[1] + ml[3] * ml[3])};
        } else {
            t.delta_xy_min[e] = magnitude(px[1] - px[0], py[1] - py[0]);
            t.center[e] = {(px[0] + px[1]) / 2, (py[0] + py[1]) / 2};
            const auto mb = quad_metrics(x0, -1.0, px, py);
            t.ghost_scale[e] = {std::sqrt(mb[0] * mb[0] + mb[2] * mb[2]), 0.0, 0.0, 0.0};
            if (e < t.ghost_sf_zero.size() && t.ghost_sf_zero[e]) t.ghost_scale[e][0] = 0.0;
        }
    }
    const size_t nf = t.face_nodes.size();
    t.face_normal.resize(nf);
    t.face_tangent.resize(nf);
    t.face_offset.resize(nf);
    t.face_scale.resize(nf);
    t.face_length.resize(nf);
    for (size_t f = 0; f < nf; ++f) {
        const auto nx = [&](int64_t i) { return t.node_x[static_cast<size_t>(i)]; };
        const auto ny = [&](int64_t i) { return t.node_y[static_cast<size_t>(i)]; };
        const int64_t a = t.face_nodes[f][0], b = t.face_nodes[f][1];
        std::array<std::array<int64_t, 2>, 2> en;
        for (size_t side = 0; side < 2; ++side) {
            const auto& el = t.elem_nodes[static_cast<size_t>(t.face_elems[f][side])];
            const int64_t s = t.face_sides[f][side];
            en[side] = {el[static_cast<size_t>(s)], el[static_cast<size_t>((s + 1) % 4)]};
        }
        double tx = nx(b) - nx(a), ty = ny(b) - ny(a);
        const double len = magnitude(tx, ty);
        tx /= len;
        ty /= len;
        const double sign = std::copysign(1.0, tx * (nx(en[0][1]) - nx(en[0][0])) + ty * (ny(en[0][1]) - ny(en[0][0])));
        t.face_length[f] = len;
        t.face_normal[f] = {ty * sign, -tx * sign};
        t.face_tangent[f] = {tx * sign, ty * sign};
        const double span = magnitude(nx(b) - nx(a), ny(b) - ny(a));
        for (size_t side = 0; side < 2; ++side) {
            const double edge = magnitude(nx(en[side][1]) - nx(en[side][0]), ny(en[side][1]) - ny(en[side][0]));
            const int64_t start = side == 0 ? a : b;
            t.face_offset[f][side] = magnitude(nx(start) - nx(en[side][0]), ny(start) - ny(en[side][0])) / edge;
            t.face_scale[f][side] = span / edge;
        }
    }
}

// Per-side plan of the stage kernels: which trace feeds the far side of each
// element side, and how (see SidePlan in ndg_internal.hpp). Ghost boundary
// traces follow Mesh2D_t::boundary_conditions (src/meshes/Mesh2D_t.cpp:3731-3782):
// walls and symmetry planes mirror the velocity of the scaled neighbour
// trace, outflow copies it scaled, inflow evaluates the analytic wave,
// periodic ghosts copy the donor's trace, and a later list in that order
// overrides an earlier one for the same ghost.
SidePlan build_side_plan(const Topology& t, const Tables& tables) {
    const int64_t K = t.n_domain;
    if (K <= 0) fail(NDG_ERR_MESH, "mesh has no domain elements");
    const int N = t.elem_N[0];
    for (int64_t e = 0; e < static_cast<int64_t>(t.elem_N.size()); ++e)
        if (t.elem_N[static_cast<size_t>(e)] != N) fail(NDG_ERR_UNSUPPORTED, "elements of different orders need the mortar path");
    for (int Nf : t.face_N)
        if (Nf != N) fail(NDG_ERR_UNSUPPORTED, "faces of a different order than their elements need the mortar path");
    (void)tables;

    // What fills each ghost's side-0 trace: last writer wins.
    const size_t n_all = t.elem_nodes.size();
    std::vector<int> ghost_kind(n_all, kZero);
    std::vector<int64_t> ghost_src(n_all, -1), ghost_src_side(n_all, 0);
    for (int64_t g : t.boundary[kWall]) ghost_kind[static_cast<size_t>(g)] = kMirror;
    for (int64_t g : t.boundary[kSymmetry]) ghost_kind[static_cast<size_t>(g)] = kMirror;
    for (int64_t g : t.boundary[kInflow]) ghost_kind[static_cast<size_t>(g)] = kAnalytic;
    for (int64_t g : t.boundary[kOutflow]) ghost_kind[static_cast<size_t>(g)] = kCopy;
    for (size_t i = 0; i < t.if_destination.size(); ++i) {
        const size_t g = static_cast<size_t>(t.if_destination[i]);
        ghost_kind[g] = kInterior;
        ghost_src[g] = t.if_origin[i];
        ghost_src_side[g] = t.if_origin_side[i];
    }

    SidePlan p;
    p.link.assign(static_cast<size_t>(8 * K), 0);
    p.normal.assign(static_cast<size_t>(8 * K), 0.0);
    p.gscale.assign(static_cast<size_t>(4 * K), 0.0);
    p.inflow_xy.assign(static_cast<size_t>(16 * K), 0.0);
    p.corners.assign(static_cast<size_t>(8 * K), 0.0);
    for (int64_t e = 0; e < K; ++e) {
        const auto& nd = t.elem_nodes[static_cast<size_t>(e)];
        for (int k = 0; k < 4; ++k) {
            p.corners[static_cast<size_t>(8 * e + 2 * k)] = t.node_x[static_cast<size_t>(nd[static_cast<size_t>(k)])];
            p.corners[static_cast<size_t>(8 * e + 2 * k + 1)] = t.node_y[static_cast<size_t>(nd[static_cast<size_t>(k)])];
        }
        for (int s = 0; s < 4; ++s) {
            const size_t ps = static_cast<size_t>(4 * e + s);
            const int64_t f = t.elem_face[static_cast<size_t>(e)][static_cast<size_t>(s)];
            if (f < 0) fail(NDG_ERR_MESH, "domain element side without a face");
            const auto& fe = t.face_elems[static_cast<size_t>(f)];
            const auto& fs = t.face_sides[static_cast<size_t>(f)];
            const auto& fn = t.face_nodes[static_cast<size_t>(f)];
            const int role = fe[0] == e ? 0 : 1;
            const int64_t a = nd[static_cast<size_t>(s)], b = nd[static_cast<size_t>((s + 1) % 4)];
            const bool conforming = role == 0 ? (fn[0] == a && fn[1] == b) : (fn[0] == b && fn[1] == a);
            if (!conforming) fail(NDG_ERR_UNSUPPORTED, "non-conforming face needs the mortar path");
            const int64_t other = fe[static_cast<size_t>(1 - role)];
            const int64_t other_side = fs[static_cast<size_t>(1 - role)];
            int kind = kInterior;
            int64_t src = other, src_side = other_side;
            if (other >= K) {
                const size_t g = static_cast<size_t>(other);
                kind = ghost_kind[g];
                src = kind == kInterior ? ghost_src[g] : -1;
                src_side = kind == kInterior ? ghost_src_side[g] : 0;
                if (kind == kMirror || kind == kCopy) {
                    // Conforming ghosts project by an exact reversed copy scaled
                    // by the ghost's edge metric (Mesh2D_t.cpp:4366-4424 with
                    // scale 1 and offset 0).
                    if (t.face_scale[static_cast<size_t>(f)][1] != 1.0 || t.face_offset[static_cast<size_t>(f)][1] != 0.0)
                        fail(NDG_ERR_UNSUPPORTED, "boundary element that does not match its face");
                    p.gscale[ps] = t.ghost_scale[g][0];
                }
                if (kind == kAnalytic) {
                    const auto& gn = t.elem_nodes[g];
                    p.inflow_xy[4 * ps + 0] = t.node_x[static_cast<size_t>(gn[0])];
                    p.inflow_xy[4 * ps + 1] = t.node_y[static_cast<size_t>(gn[0])];
                    p.inflow_xy[4 * ps + 2] = t.node_x[static_cast<size_t>(gn[1])];
                    p.inflow_xy[4 * ps + 3] = t.node_y[static_cast<size_t>(gn[1])];
                }
            }
            p.link[2 * ps] = static_cast<int32_t>(src);
            p.link[2 * ps + 1] = static_cast<int32_t>(src_side | (kind << 2) | (role << 5));
            p.normal[2 * ps] = t.face_normal[static_cast<size_t>(f)][0];
            p.normal[2 * ps + 1] = t.face_normal[static_cast<size_t>(f)][1];
        }
    }
    return p;
}

// SU2 reader with the semantics of Mesh2D_t::read_su2
// (src/meshes/Mesh2D_t.cpp:78-421): NDIME=2, 0-based node numbers,
// quadrilateral (9) elements, line (3) markers "wall"/"airfoil" (wall),
// "symmetry", "inlet" (inflow) and "farfield" (outflow). Ghost elements are
// numbered by kind: all wall bars in file order, then symmetry, inflow and
// outflow (:312-361). Builds the equivalent zone (one BAR_2 section per kind)
// and delegates to the zone path, which yields the same numbering.
Topology read_su2(const std::string& path, int initial_N) {
    std::ifstream in(path);
    if (!in) fail(NDG_ERR_INVALID_ARG, "cannot open '" + path + "'");
    std::vector<double> xs, ys;
    std::vector<int64_t> quads;
    std::array<std::vector<int64_t>, 4> bars_by_kind;  // wall, symmetry, inflow, outflow
    std::string line;
    auto value_after = [](const std::string& l) { return l.substr(l.find('=') + 1); };
    while (std::getline(in, line)) {
        if (line.rfind("NDIME", 0) == 0) {
            if (std::stoi(value_after(line)) != 2) fail(NDG_ERR_MESH, "only 2D SU2 meshes are supported");
        } else if (line.rfind("NPOIN", 0) == 0) {
            const int64_t n = std::stoll(value_after(line));
            for (int64_t i = 0; i < n && std::getline(in, line); ++i) {
                std::istringstream ss(line);
                double x, y;
                ss >> x >> y;
                xs.push_back(x);
                ys.push_back(y);
            }
        } else if (line.rfind("NELEM", 0) == 0) {
            const int64_t n = std::stoll(value_after(line));
            for (int64_t i = 0; i < n && std::getline(in, line); ++i) {
                std::istringstream ss(line);
                int type;
                ss >> type;
                if (type != 9) fail(NDG_ERR_MESH, "only quadrilateral SU2 elements are supported");
                for (int k = 0; k < 4; ++k) {
                    int64_t v;
                    ss >> v;
                    quads.push_back(v + 1);
                }
            }
        } else if (line.rfind("MARKER_TAG", 0) == 0) {
            std::string tag = value_after(line);
            tag.erase(std::remove_if(tag.begin(), tag.end(), [](unsigned char c) { return std::isspace(c); }), tag.end());
            std::transform(tag.begin(), tag.end(), tag.begin(), [](unsigned char c) { return static_cast<char>(std::tolower(c)); });
            int bc;
            if (tag == "farfield") bc = NDG_BC_OUTFLOW;
            else if (tag == "inlet") bc = NDG_BC_INFLOW;
            else if (tag == "wall" || tag == "airfoil") bc = NDG_BC_WALL;
            else if (tag == "symmetry") bc = NDG_BC_SYMMETRY;
            else fail(NDG_ERR_MESH, "unknown SU2 marker '" + tag + "'");
            if (!std::getline(in, line) || line.rfind("MARKER_ELEMS", 0) != 0) fail(NDG_ERR_MESH, "MARKER_TAG without MARKER_ELEMS");
            const int64_t n = std::stoll(value_after(line));
            auto& bars = bars_by_kind[static_cast<size_t>(bc)];
            for (int64_t i = 0; i < n && std::getline(in, line); ++i) {
                std::istringstream ss(line);
                int type;
                int64_t a, b;
                ss >> type >> a >> b;
                if (type != 3) fail(NDG_ERR_MESH, "only line SU2 markers are supported");
                bars.push_back(a + 1);
                bars.push_back(b + 1);
            }
        }
    }
    const int64_t n_quad = static_cast<int64_t>(quads.size() / 4);
    std::vector<int32_t> sec_type{0};
    std::vector<int64_t> sec_start{1}, sec_end{n_quad}, conn(quads);
    std::vector<int32_t> boco_type;
    std::vector<int64_t> boco_count, boco_points;
    int64_t next = n_quad + 1;
    for (int bc = 0; bc < 4; ++bc) {
        const auto& bars = bars_by_kind[static_cast<size_t>(bc)];
        const int64_t cnt = static_cast<int64_t>(bars.size() / 2);
        if (cnt == 0) continue;
        sec_type.push_back(1);
        sec_start.push_back(next);
        sec_end.push_back(next + cnt - 1);
        conn.insert(conn.end(), bars.begin(), bars.end());
        boco_type.push_back(bc);
        boco_count.push_back(cnt);
        for (int64_t i = 0; i < cnt; ++i) boco_points.push_back(next + i);
        next += cnt;
    }
    ndg_zone z{};
    z.n_nodes = static_cast<int64_t>(xs.size());
    z.x = xs.data();
    z.y = ys.data();
    z.n_sections = static_cast<int32_t>(sec_type.size());
    z.section_type = sec_type.data();
    z.section_start = sec_start.data();
    z.section_end = sec_end.data();
    z.section_connectivity = conn.data();
    z.n_bocos = static_cast<int32_t>(boco_type.size());
    z.boco_type = boco_type.data();
    z.boco_count = boco_count.data();
    z.boco_points = boco_points.data();
    z.n_conns = 0;
    return build_topology(z, initial_N);
}

}  // namespace ndg
