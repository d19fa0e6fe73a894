// h-adaptation (element splitting) of the host topology with the reference's
// rules and numbering: Mesh2D_t::adapt when at least one element splits
// (src/meshes/Mesh2D_t.cpp:1877-2268) for one process, i.e. find_nodes,
// copy_interfaces_error, copy_boundaries_error, the face refine decisions,
// hp_adapt (:5186-5659), split_boundaries (:6232-6342), split_interfaces
// (:6343-6757) and split_faces (:5661-5985).
//
// The rules decide new element, face and node numbers by prefix counts
// (element i moves to i + 3 * splitting elements before it, a split face to
// n_faces + 4 * splitting elements + refined faces before it, and so on) and
// decide which half of a split side a face belongs to by projecting its end
// points on the side. Those projections and midpoints are evaluated in the
// reference's operation order so that every decision is the reference's.
// Face and element geometry (normals, offsets, scales, centres, minimum
// lengths, ghost scaling factors) is recomputed afterwards from the final
// topology; every midpoint it reads was formed from the same operands as the
// reference's, so the values are the same.
#include "ndg_internal.hpp"

#include <algorithm>
#include <array>
#include <cmath>
#include <limits>
#include <vector>

namespace ndg {

namespace {

struct V2 {
    double x = 0.0, y = 0.0;
};
V2 operator+(V2 a, V2 b) { return {a.x + b.x, a.y + b.y}; }
V2 operator-(V2 a, V2 b) { return {a.x - b.x, a.y - b.y}; }
V2 operator/(V2 a, double s) { return {a.x / s, a.y / s}; }
double dot(V2 a, V2 b) { return a.x * b.x + a.y * b.y; }
bool same_point(V2 a, V2 b) { return almost_equal(a.x, b.x) && almost_equal(a.y, b.y); }

constexpr double kEps = std::numeric_limits<double>::epsilon();

// "Both projections lie on the side" (hp_adapt, split_faces, split_interfaces).
bool on_side(double c, double d) { return c + kEps >= 0.0 && c <= 1.0 + kEps && d + kEps >= 0.0 && d <= 1.0 + kEps; }
// "The face lies within this half" of the face refine decisions (adapt, :2025-2034).
bool in_half(double c, double d) { return (c + kEps <= 1.0 && d >= 0.0 + kEps) || (d + kEps <= 1.0 && c >= 0.0 + kEps); }

// Hilbert::child_order and child_statuses (src/functions/Hilbert_splitting.cpp:24-81),
// indexed [rotation][parent status]; statuses H, A, R, B = 0..3. These tables
// define the children's numbering and are the reference's.
constexpr int kChildOrder[4][4][4] = {{{0, 3, 2, 1}, {0, 1, 2, 3}, {2, 1, 0, 3}, {2, 3, 0, 1}},
                                      {{3, 2, 1, 0}, {1, 2, 3, 0}, {1, 0, 3, 2}, {3, 0, 1, 2}},
                                      {{2, 1, 0, 3}, {2, 3, 0, 1}, {0, 3, 2, 1}, {0, 1, 2, 3}},
                                      {{1, 0, 3, 2}, {3, 0, 1, 2}, {3, 2, 1, 0}, {1, 2, 3, 0}}};
constexpr int kChildStatus[4][4][4] = {{{1, 3, 0, 0}, {0, 1, 1, 2}, {2, 2, 3, 1}, {3, 0, 2, 3}},
                                       {{3, 0, 0, 1}, {1, 1, 2, 0}, {2, 3, 1, 2}, {0, 2, 3, 3}},
                                       {{0, 0, 1, 3}, {1, 2, 0, 1}, {3, 1, 2, 2}, {2, 3, 3, 0}},
                                       {{0, 1, 3, 0}, {2, 0, 1, 1}, {1, 2, 2, 3}, {3, 3, 0, 2}}};

// Working copy of an element and a face, with the fields the rules read.
struct Elem {
    int N = 0, split = 0, status = 1, rotation = 0;
    std::array<int64_t, 4> nodes{};
    std::array<std::vector<int64_t>, 4> faces;
    bool refine = false;
    double sigma = 0.0;
    std::array<bool, 4> add{};
    bool sf_zero = false;
};
struct Face {
    int N = 0;
    std::array<int64_t, 2> nodes{}, elems{}, sides{};
    bool refine = false;
};

struct Work {
    int64_t K = 0;  // domain elements
    std::vector<Elem> el;
    std::vector<Face> fa;
    std::vector<V2> nd;
    std::array<std::vector<int64_t>, 4> boundary;
    std::vector<int64_t> if_origin, if_origin_side, if_destination;
    int max_split = 0, N_max = 0;

    bool would_h(const Elem& e) const { return e.refine && e.sigma < 1.0 && e.split < max_split; }
    bool would_p(const Elem& e) const { return e.refine && e.sigma >= 1.0 && e.N + 2 <= N_max; }
    V2 node(int64_t i) const { return nd[static_cast<size_t>(i)]; }
};

}  // namespace

namespace {

// Exclusive prefix count of a flag: out[i] = number of set flags before i
// (out has one more entry, the total). The reference numbers new faces,
// nodes and elements by these counts (its serial loops over j < i,
// src/meshes/Mesh2D_t.cpp:5204-5209 and the split_* functions); one scan
// gives every count at once.
template <typename Flag>
std::vector<int64_t> exclusive_count(size_t n, Flag flag) {
    std::vector<int64_t> out(n + 1, 0);
    for (size_t i = 0; i < n; ++i) out[i + 1] = out[i] + (flag(i) ? 1 : 0);
    return out;
}

// A side's face list with every refined face followed by its second half
// (the move and p-refine branches of hp_adapt, :5576-5605 and :5617-5646);
// refined_before[f] is the number of refined faces before face f.
std::vector<int64_t> expand_side(const std::vector<Face>& fa, const std::vector<int64_t>& refined_before,
                                 const std::vector<int64_t>& side, int64_t second_half_base) {
    std::vector<int64_t> out;
    for (int64_t f : side) {
        out.push_back(f);
        if (fa[static_cast<size_t>(f)].refine) out.push_back(second_half_base + refined_before[static_cast<size_t>(f)]);
    }
    return out;
}

}  // namespace

bool h_adapt(Topology& t, const Tables& tables, const int32_t* refine, const double* p_sigma, int N_max, int max_split_level,
             std::vector<ElementSource>& sources, const AdaptDecisions* dec) {
    // Splitting elements first: without one, t stays untouched.
    int64_t n_split = 0;
    if (dec) {
        n_split = dec->split_prefix[static_cast<size_t>(t.n_domain)];
    } else {
        for (int64_t e = 0; e < t.n_domain; ++e)
            n_split += (refine[e] != 0 && p_sigma[e] < 1.0 && t.elem_split[static_cast<size_t>(e)] < max_split_level) ? 1 : 0;
    }
    if (n_split == 0) return false;

    // The working copy takes t's face lists (t is rebuilt at the end).
    Work w;
    w.K = t.n_domain;
    w.max_split = max_split_level;
    w.N_max = N_max;
    const int64_t total = static_cast<int64_t>(t.elem_N.size());
    const int64_t F = static_cast<int64_t>(t.face_N.size());
    const int64_t n_nodes = static_cast<int64_t>(t.node_x.size());
    w.el.resize(static_cast<size_t>(total));
    for (int64_t e = 0; e < total; ++e) {
        Elem& x = w.el[static_cast<size_t>(e)];
        const size_t ei = static_cast<size_t>(e);
        x.N = t.elem_N[ei];
        x.split = t.elem_split[ei];
        x.status = t.elem_status[ei];
        x.rotation = t.elem_rotation[ei];
        x.nodes = t.elem_nodes[ei];
        x.faces = std::move(t.elem_faces[ei]);
        x.sf_zero = t.ghost_sf_zero[ei] != 0;
        if (e < w.K) {
            x.refine = refine[e] != 0;
            x.sigma = p_sigma[e];
        }
    }
    w.fa.resize(static_cast<size_t>(F));
    for (int64_t f = 0; f < F; ++f) {
        Face& x = w.fa[static_cast<size_t>(f)];
        x.N = t.face_N[static_cast<size_t>(f)];
        x.nodes = t.face_nodes[static_cast<size_t>(f)];
        x.elems = t.face_elems[static_cast<size_t>(f)];
        x.sides = t.face_sides[static_cast<size_t>(f)];
    }
    w.nd.resize(static_cast<size_t>(n_nodes));
    for (int64_t i = 0; i < n_nodes; ++i) w.nd[static_cast<size_t>(i)] = {t.node_x[static_cast<size_t>(i)], t.node_y[static_cast<size_t>(i)]};
    w.boundary = t.boundary;
    w.if_origin = t.if_origin;
    w.if_origin_side = t.if_origin_side;
    w.if_destination = t.if_destination;

    if (dec) {
        // The device's decisions: every element's flags (ghosts holding
        // their source's), new-node flags, face splits and counts.
        for (int64_t e = 0; e < total; ++e) {
            Elem& x = w.el[static_cast<size_t>(e)];
            const uint8_t c = dec->code[static_cast<size_t>(e)];
            x.refine = (c & 1u) != 0;
            x.sigma = (c & 2u) ? 1.0 : 0.0;
            for (size_t s = 0; s < 4; ++s) x.add[s] = dec->add[static_cast<size_t>(4 * e) + s] != 0;
        }
        for (int64_t f = 0; f < F; ++f) w.fa[static_cast<size_t>(f)].refine = dec->face_split[static_cast<size_t>(f)] != 0;
    }

    // find_nodes (:5987-6014): a splitting element needs a new node on a side
    // unless a face of that side already ends at the side's midpoint.
    for (int64_t e = 0; !dec && e < w.K; ++e) {
        Elem& x = w.el[static_cast<size_t>(e)];
        x.add = {false, false, false, false};
        if (!w.would_h(x)) continue;
        x.add = {true, true, true, true};
        for (int s = 0; s < 4; ++s) {
            const V2 mid = (w.node(x.nodes[static_cast<size_t>(s)]) + w.node(x.nodes[static_cast<size_t>((s + 1) % 4)])) / 2;
            for (int64_t f : x.faces[static_cast<size_t>(s)]) {
                const Face& fc = w.fa[static_cast<size_t>(f)];
                if (same_point(w.node(fc.nodes[0]), mid) || same_point(w.node(fc.nodes[1]), mid)) {
                    x.add[static_cast<size_t>(s)] = false;
                    break;
                }
            }
        }
    }
    // copy_interfaces_error (:6054-6077), then copy_boundaries_error (:6025-6053).
    for (size_t i = 0; !dec && i < w.if_origin.size(); ++i) {
        const Elem& src = w.el[static_cast<size_t>(w.if_origin[i])];
        Elem& dst = w.el[static_cast<size_t>(w.if_destination[i])];
        dst.add[0] = src.add[static_cast<size_t>(w.if_origin_side[i])];
        dst.refine = src.refine;
        dst.sigma = src.sigma;
    }
    for (int b = 0; !dec && b < 4; ++b)
        for (int64_t g : w.boundary[static_cast<size_t>(b)]) {
            Elem& dst = w.el[static_cast<size_t>(g)];
            if (dst.faces[0].size() != 1) continue;
            const Face& fc = w.fa[static_cast<size_t>(dst.faces[0][0])];
            const size_t fs = fc.elems[0] == g ? 1 : 0;
            const Elem& src = w.el[static_cast<size_t>(fc.elems[fs])];
            dst.add[0] = src.add[static_cast<size_t>(fc.sides[fs])];
            dst.refine = src.refine;
            dst.sigma = src.sigma;
        }
    // Faces that split: a new node on the side of one of their elements and
    // both halves of the side cover part of the face (:1917-2090).
    int64_t n_split_faces = dec ? dec->split_face_prefix[static_cast<size_t>(F)] : 0;
    for (Face& fc : w.fa) {
        if (dec) break;
        fc.refine = false;
        for (int side = 0; side < 2; ++side) {
            if (side == 1 && fc.refine) break;
            const Elem& x = w.el[static_cast<size_t>(fc.elems[static_cast<size_t>(side)])];
            const int s = static_cast<int>(fc.sides[static_cast<size_t>(side)]);
            if (!x.add[static_cast<size_t>(s)]) continue;
            const V2 a = w.node(x.nodes[static_cast<size_t>(s)]), b = w.node(x.nodes[static_cast<size_t>((s + 1) % 4)]);
            const V2 mid = (a + b) / 2;
            const V2 AB[2] = {mid - a, b - mid};
            const double inv[2] = {1 / dot(AB[0], AB[0]), 1 / dot(AB[1], AB[1])};
            const V2 C = w.node(fc.nodes[0]), D = w.node(fc.nodes[1]);
            const V2 AC[2] = {C - a, C - mid}, AD[2] = {D - a, D - mid};
            bool in[2];
            for (int h = 0; h < 2; ++h) in[h] = in_half(dot(AC[h], AB[h]) * inv[h], dot(AD[h], AB[h]) * inv[h]);
            if (in[0] && in[1]) {
                fc.refine = true;
                ++n_split_faces;
            }
            break;  // the reference checks the right element only when the left one adds no node
        }
    }

    // Index of a refined face's new node, or of the second half of a refined
    // face: base + number of refined faces before it.
    const std::vector<int64_t> refined_prefix =
        dec ? dec->split_face_prefix : exclusive_count(w.fa.size(), [&](size_t f) { return w.fa[f].refine; });
    auto refined_before = [&](int64_t f) { return refined_prefix[static_cast<size_t>(f)]; };
    // Splitting domain elements before element j: element j moves to j + 3 * that.
    const std::vector<int64_t> split_prefix =
        dec ? dec->split_prefix : exclusive_count(static_cast<size_t>(w.K), [&](size_t e) { return w.would_h(w.el[e]); });

    // Sizes of the new arrays (:2091-2151).
    std::array<int64_t, 4> n_split_b{};
    for (int b = 0; b < 4; ++b)
        for (int64_t g : w.boundary[static_cast<size_t>(b)]) {
            const Elem& x = w.el[static_cast<size_t>(g)];
            if (x.faces[0].size() == 1) n_split_b[static_cast<size_t>(b)] += w.fa[static_cast<size_t>(x.faces[0][0])].refine ? 1 : 0;
        }
    int64_t n_split_if = 0;
    for (int64_t o : w.if_origin) n_split_if += w.would_h(w.el[static_cast<size_t>(o)]) ? 1 : 0;
    int64_t new_total = total + 3 * n_split + n_split_if;
    for (int b = 0; b < 4; ++b) new_total += n_split_b[static_cast<size_t>(b)];
    std::vector<Elem> ne(static_cast<size_t>(new_total));
    std::vector<Face> nf(static_cast<size_t>(F + 4 * n_split + n_split_faces));
    w.nd.resize(static_cast<size_t>(n_nodes + n_split + n_split_faces));
    std::vector<int64_t> new_index(static_cast<size_t>(total), -1);
    const int64_t split_face_base = F + 4 * n_split;  // second halves of refined faces
    const int64_t split_node_base = n_nodes + n_split;  // midpoints of refined faces
    sources.assign(static_cast<size_t>(w.K + 3 * n_split), ElementSource{});

    // hp_adapt (:5186-5659) over the domain elements.
    int64_t before = 0;  // splitting elements before element i
    for (int64_t i = 0; i < w.K; ++i) {
        Elem& x = w.el[static_cast<size_t>(i)];
        const int64_t at = i + 3 * before;
        new_index[static_cast<size_t>(i)] = at;
        if (w.would_h(x)) {
            const int64_t centre = n_nodes + before;
            std::array<int64_t, 4> side_node{-1, -1, -1, -1};
            std::array<V2, 4> side_xy{};
            V2 c{};
            for (int s = 0; s < 4; ++s) {
                c = c + w.node(x.nodes[static_cast<size_t>(s)]);
                if (x.add[static_cast<size_t>(s)]) {
                    const int64_t f = x.faces[static_cast<size_t>(s)][0];
                    const Face& fc = w.fa[static_cast<size_t>(f)];
                    side_xy[static_cast<size_t>(s)] = (w.node(fc.nodes[0]) + w.node(fc.nodes[1])) / 2;
                    side_node[static_cast<size_t>(s)] = split_node_base + refined_before(f);
                } else {
                    const V2 mid = (w.node(x.nodes[static_cast<size_t>(s)]) + w.node(x.nodes[static_cast<size_t>((s + 1) % 4)])) / 2;
                    for (int64_t f : x.faces[static_cast<size_t>(s)]) {
                        const Face& fc = w.fa[static_cast<size_t>(f)];
                        if (same_point(w.node(fc.nodes[0]), mid)) {
                            side_node[static_cast<size_t>(s)] = fc.nodes[0];
                            side_xy[static_cast<size_t>(s)] = w.node(fc.nodes[0]);
                            break;
                        } else if (same_point(w.node(fc.nodes[1]), mid)) {
                            side_node[static_cast<size_t>(s)] = fc.nodes[1];
                            side_xy[static_cast<size_t>(s)] = w.node(fc.nodes[1]);
                            break;
                        }
                    }
                }
            }
            w.nd[static_cast<size_t>(centre)] = c / 4.0;
            const V2 cxy = w.nd[static_cast<size_t>(centre)];
            const int* order = kChildOrder[x.rotation][x.status];
            const int* status = kChildStatus[x.rotation][x.status];
            const int64_t interior = F + 4 * before;
            for (int s = 0; s < 4; ++s) {
                const int prev = (s + 3) % 4, next = (s + 1) % 4, opp = (s + 2) % 4;
                Face& inner = nf[static_cast<size_t>(interior + s)];
                inner.N = x.N;
                inner.nodes = {side_node[static_cast<size_t>(s)], centre};
                inner.elems = {at + order[s], at + order[next]};
                inner.sides = {next, prev};
                std::array<std::vector<int64_t>, 4> faces;
                faces[static_cast<size_t>(next)] = {interior + s};
                faces[static_cast<size_t>(opp)] = {interior + prev};
                // The child's part of the parent's side s (first half) and of
                // side prev (second half).
                for (int half = 0; half < 2; ++half) {
                    const int ps = half == 0 ? s : prev;
                    auto& out = faces[static_cast<size_t>(ps)];
                    if (x.add[static_cast<size_t>(ps)]) {
                        const int64_t f = x.faces[static_cast<size_t>(ps)][0];
                        const bool forward = i == w.fa[static_cast<size_t>(f)].elems[0];
                        const int64_t second = split_face_base + refined_before(f);
                        out = {(half == 0) == forward ? f : second};
                        continue;
                    }
                    const V2 a = w.node(x.nodes[static_cast<size_t>(ps)]), b = w.node(x.nodes[static_cast<size_t>((ps + 1) % 4)]);
                    const V2 mid = (a + b) / 2;
                    const V2 A = half == 0 ? a : mid;  // start of this child's half
                    const V2 AB = half == 0 ? mid - a : b - mid;
                    const double inv = 1 / dot(AB, AB);
                    out.clear();
                    for (int64_t f : x.faces[static_cast<size_t>(ps)]) {
                        const Face& fc = w.fa[static_cast<size_t>(f)];
                        if (fc.refine) {
                            const V2 fm = (w.node(fc.nodes[0]) + w.node(fc.nodes[1])) / 2;
                            const double C = dot(w.node(fc.nodes[0]) - A, AB) * inv, D = dot(fm - A, AB) * inv,
                                         E = dot(w.node(fc.nodes[1]) - A, AB) * inv;
                            if (on_side(C, D)) out.push_back(f);
                            if (on_side(D, E)) out.push_back(split_face_base + refined_before(f));
                        } else {
                            const double C = dot(w.node(fc.nodes[0]) - A, AB) * inv, D = dot(w.node(fc.nodes[1]) - A, AB) * inv;
                            if (on_side(C, D)) out.push_back(f);
                        }
                    }
                }
                Elem& child = ne[static_cast<size_t>(at + order[s])];
                child.N = x.N;
                child.split = x.split + 1;
                child.status = status[s];
                child.rotation = x.rotation;
                child.faces = std::move(faces);
                child.nodes[static_cast<size_t>(s)] = x.nodes[static_cast<size_t>(s)];
                child.nodes[static_cast<size_t>(next)] = side_node[static_cast<size_t>(s)];
                child.nodes[static_cast<size_t>(opp)] = centre;
                child.nodes[static_cast<size_t>(prev)] = side_node[static_cast<size_t>(prev)];
                ElementSource& src = sources[static_cast<size_t>(at + order[s])];
                src.old = i;
                src.kind = 2;
                std::array<V2, 4> cp;
                cp[static_cast<size_t>(s)] = w.node(x.nodes[static_cast<size_t>(s)]);
                cp[static_cast<size_t>(next)] = side_xy[static_cast<size_t>(s)];
                cp[static_cast<size_t>(opp)] = cxy;
                cp[static_cast<size_t>(prev)] = side_xy[static_cast<size_t>(prev)];
                for (int k = 0; k < 4; ++k) {
                    src.child[static_cast<size_t>(2 * k)] = cp[static_cast<size_t>(k)].x;
                    src.child[static_cast<size_t>(2 * k + 1)] = cp[static_cast<size_t>(k)].y;
                    src.parent[static_cast<size_t>(2 * k)] = w.node(x.nodes[static_cast<size_t>(k)]).x;
                    src.parent[static_cast<size_t>(2 * k + 1)] = w.node(x.nodes[static_cast<size_t>(k)]).y;
                }
            }
            ++before;
        } else {
            // The element moves (its face lists are rebuilt below; the
            // old lists are read no more).
            Elem y;
            y.N = x.N;
            y.split = x.split;
            y.status = x.status;
            y.rotation = x.rotation;
            y.nodes = x.nodes;
            y.refine = x.refine;
            y.sigma = x.sigma;
            y.add = x.add;
            y.sf_zero = x.sf_zero;
            ElementSource& src = sources[static_cast<size_t>(at)];
            src.old = i;
            src.kind = 0;
            if (w.would_p(x)) {
                y.N = x.N + 2;
                y.refine = false;
                src.kind = 1;
            }
            for (int s = 0; s < 4; ++s) {
                auto& list = x.faces[static_cast<size_t>(s)];
                const bool any_split = std::any_of(list.begin(), list.end(), [&](int64_t f) { return w.fa[static_cast<size_t>(f)].refine; });
                // A side without a split face keeps its list (moved: x is read no more).
                y.faces[static_cast<size_t>(s)] = any_split ? expand_side(w.fa, refined_prefix, list, split_face_base) : std::move(list);
            }
            ne[static_cast<size_t>(at)] = std::move(y);
        }
    }

    // split_boundaries (:6232-6342), walls, symmetry, inflow, outflow in turn.
    std::array<std::vector<int64_t>, 4> new_boundary;
    int64_t offset = w.K + 3 * n_split;
    for (int b = 0; b < 4; ++b) {
        const auto& list = w.boundary[static_cast<size_t>(b)];
        auto& out = new_boundary[static_cast<size_t>(b)];
        out.assign(list.size() + static_cast<size_t>(n_split_b[static_cast<size_t>(b)]), 0);
        int64_t shift = 0;  // split boundaries before this one
        for (size_t bi = 0; bi < list.size(); ++bi) {
            const int64_t g = list[bi];
            Elem& dst = w.el[static_cast<size_t>(g)];
            const int64_t nb = static_cast<int64_t>(bi) + shift;
            const int64_t at = offset + nb;
            new_index[static_cast<size_t>(g)] = at;
            const bool splits = dst.faces[0].size() == 1 && w.fa[static_cast<size_t>(dst.faces[0][0])].refine;
            if (splits) {
                const int64_t f = dst.faces[0][0];
                const int64_t mid_node = split_node_base + refined_before(f);
                const int64_t second = split_face_base + refined_before(f);
                out[static_cast<size_t>(nb)] = at;
                out[static_cast<size_t>(nb + 1)] = at + 1;
                for (int h = 0; h < 2; ++h) {
                    Elem& y = ne[static_cast<size_t>(at + h)];
                    y.N = dst.N;
                    y.nodes = h == 0 ? std::array<int64_t, 4>{dst.nodes[0], mid_node, mid_node, dst.nodes[0]}
                                     : std::array<int64_t, 4>{mid_node, dst.nodes[1], dst.nodes[1], mid_node};
                    y.status = dst.status;
                    y.rotation = dst.rotation;
                    y.split = dst.split + 1;
                    y.faces = {};
                    y.faces[0] = {h == 0 ? second : f};
                    y.sf_zero = false;
                }
                ++shift;
            } else {
                out[static_cast<size_t>(nb)] = at;
                int N_el = dst.N;
                for (int64_t f : dst.faces[0]) {
                    const Face& fc = w.fa[static_cast<size_t>(f)];
                    N_el = std::max(N_el, w.el[static_cast<size_t>(fc.elems[fc.elems[0] == g ? 1 : 0])].N);
                }
                // The reference resizes the old ghost in place, so split_faces
                // below sees the new order.
                if (dst.N != N_el) {
                    dst.N = N_el;
                    dst.sf_zero = false;  // resized with its geometry recomputed
                }
                // Moved: split_faces reads only its order, flags and nodes.
                ne[static_cast<size_t>(at)] = std::move(dst);
            }
        }
        offset += static_cast<int64_t>(list.size()) + n_split_b[static_cast<size_t>(b)];
    }

    // split_interfaces (:6343-6757).
    std::vector<int64_t> new_origin, new_origin_side, new_destination;
    const size_t n_if = w.if_origin.size();
    new_origin.assign(n_if + static_cast<size_t>(n_split_if), 0);
    new_origin_side = new_origin;
    new_destination = new_origin;
    {
        int64_t shift = 0;
        for (size_t ii = 0; ii < n_if; ++ii) {
            const int64_t si = w.if_origin[ii], di = w.if_destination[ii];
            const Elem& src = w.el[static_cast<size_t>(si)];
            Elem& dst = w.el[static_cast<size_t>(di)];
            const int side = static_cast<int>(w.if_origin_side[ii]);
            const int64_t src_new = si + 3 * split_prefix[static_cast<size_t>(si)];
            const int64_t nii = static_cast<int64_t>(ii) + shift;
            const int64_t at = offset + nii;
            new_index[static_cast<size_t>(di)] = at;
            if (w.would_h(src)) {
                const int* order = kChildOrder[src.rotation][src.status];
                new_origin[static_cast<size_t>(nii)] = src_new + order[side];
                new_origin[static_cast<size_t>(nii + 1)] = src_new + order[(side + 1) % 4];
                new_origin_side[static_cast<size_t>(nii)] = side;
                new_origin_side[static_cast<size_t>(nii + 1)] = side;
                new_destination[static_cast<size_t>(nii)] = at;
                new_destination[static_cast<size_t>(nii + 1)] = at + 1;
                V2 mid{};
                int64_t mid_node = -1;
                if (dst.add[0]) {
                    const int64_t f = dst.faces[0][0];
                    mid = (w.node(w.fa[static_cast<size_t>(f)].nodes[0]) + w.node(w.fa[static_cast<size_t>(f)].nodes[1])) / 2;
                    mid_node = split_node_base + refined_before(f);
                } else {
                    const V2 m2 = (w.node(dst.nodes[0]) + w.node(dst.nodes[1])) / 2;
                    for (int64_t f : dst.faces[0]) {
                        const Face& fc = w.fa[static_cast<size_t>(f)];
                        if (same_point(w.node(fc.nodes[0]), m2)) {
                            mid_node = fc.nodes[0];
                            mid = w.node(fc.nodes[0]);
                            break;
                        } else if (same_point(w.node(fc.nodes[1]), m2)) {
                            mid_node = fc.nodes[1];
                            mid = w.node(fc.nodes[1]);
                            break;
                        }
                    }
                }
                for (int h = 0; h < 2; ++h) {
                    Elem& y = ne[static_cast<size_t>(at + h)];
                    y.N = src.N;
                    y.nodes = h == 0 ? std::array<int64_t, 4>{dst.nodes[0], mid_node, mid_node, dst.nodes[0]}
                                     : std::array<int64_t, 4>{mid_node, dst.nodes[1], dst.nodes[1], mid_node};
                    y.status = dst.status;
                    y.rotation = dst.rotation;
                    y.split = dst.split + 1;
                    y.faces = {};
                    y.sf_zero = false;
                }
                if (dst.add[0]) {
                    const int64_t f = dst.faces[0][0];
                    ne[static_cast<size_t>(at)].faces[0] = {split_face_base + refined_before(f)};
                    ne[static_cast<size_t>(at + 1)].faces[0] = {f};
                } else {
                    const V2 n0 = w.node(dst.nodes[0]), n1 = w.node(dst.nodes[1]);
                    const V2 AB[2] = {mid - n0, n1 - mid};
                    const double inv[2] = {1 / dot(AB[0], AB[0]), 1 / dot(AB[1], AB[1])};
                    const V2 A[2] = {n0, mid};
                    auto& f0 = ne[static_cast<size_t>(at)].faces[0];
                    auto& f1 = ne[static_cast<size_t>(at + 1)].faces[0];
                    for (int64_t f : dst.faces[0]) {
                        const Face& fc = w.fa[static_cast<size_t>(f)];
                        if (fc.refine) {
                            const int64_t second = split_face_base + refined_before(f);
                            const V2 fm = (w.node(fc.nodes[0]) + w.node(fc.nodes[1])) / 2;
                            double C[2], D[2], E[2];
                            for (int h = 0; h < 2; ++h) {
                                C[h] = dot(w.node(fc.nodes[0]) - A[h], AB[h]) * inv[h];
                                D[h] = dot(fm - A[h], AB[h]) * inv[h];
                                E[h] = dot(w.node(fc.nodes[1]) - A[h], AB[h]) * inv[h];
                            }
                            if (on_side(C[0], D[0])) f0.push_back(f);
                            if (on_side(C[1], D[1])) f1.push_back(f);
                            if (on_side(D[0], E[0])) f0.push_back(second);
                            if (on_side(D[1], E[1])) f1.push_back(second);
                        } else {
                            double C[2], D[2];
                            for (int h = 0; h < 2; ++h) {
                                C[h] = dot(w.node(fc.nodes[0]) - A[h], AB[h]) * inv[h];
                                D[h] = dot(w.node(fc.nodes[1]) - A[h], AB[h]) * inv[h];
                            }
                            if (on_side(C[0], D[0])) f0.push_back(f);
                            if (on_side(C[1], D[1])) f1.push_back(f);
                        }
                    }
                }
                ++shift;
            } else {
                new_origin[static_cast<size_t>(nii)] = src_new;
                new_origin_side[static_cast<size_t>(nii)] = side;
                new_destination[static_cast<size_t>(nii)] = at;
                // Resized in place, as in the reference (split_faces sees it).
                if (w.would_p(src)) {
                    dst.N = src.N + 2;
                    dst.sf_zero = false;
                }
                Elem y = dst;
                y.faces[0] = expand_side(w.fa, refined_prefix, dst.faces[0], split_face_base);
                ne[static_cast<size_t>(at)] = std::move(y);
            }
        }
    }

    // split_faces (:5661-5985): old faces keep their numbers, second halves
    // follow the new interior faces; element numbers move to the children
    // that now carry each face.
    auto child_shift = [&](const Elem& x, int xs, V2 p0, V2 p1, V2 p2, int which) {
        // which = 0: faces (p0, p1) of an unsplit face; 1, 2: the halves
        // (p0, p1), (p1, p2) of a refined face. Returns the child offset to add.
        const int* order = kChildOrder[x.rotation][x.status];
        const V2 e0 = w.node(x.nodes[static_cast<size_t>(xs)]), e1 = w.node(x.nodes[static_cast<size_t>((xs + 1) % 4)]);
        const V2 em = (e0 + e1) / 2;
        const V2 AB[2] = {em - e0, e1 - em};
        const double inv[2] = {1 / dot(AB[0], AB[0]), 1 / dot(AB[1], AB[1])};
        const V2 A[2] = {e0, em};
        int add = 0;
        for (int h = 0; h < 2; ++h) {
            const double C = dot(p0 - A[h], AB[h]) * inv[h], D = dot(p1 - A[h], AB[h]) * inv[h];
            if (which == 0) {
                if (on_side(C, D)) add += order[(xs + h) % 4];
            } else {
                const double E = dot(p2 - A[h], AB[h]) * inv[h];
                if (which == 1 ? on_side(C, D) : on_side(D, E)) add += order[(xs + h) % 4];
            }
        }
        return add;
    };
    for (int64_t fi = 0; fi < F; ++fi) {
        Face fc = w.fa[static_cast<size_t>(fi)];
        const Elem& L = w.el[static_cast<size_t>(fc.elems[0])];
        const Elem& R = w.el[static_cast<size_t>(fc.elems[1])];
        const int Ls = static_cast<int>(fc.sides[0]), Rs = static_cast<int>(fc.sides[1]);
        const int64_t Ln = new_index[static_cast<size_t>(fc.elems[0])], Rn = new_index[static_cast<size_t>(fc.elems[1])];
        const int face_N = std::max(L.N + 2 * (w.would_p(L) ? 1 : 0), R.N + 2 * (w.would_p(R) ? 1 : 0));
        const V2 p0 = w.node(fc.nodes[0]), p2 = w.node(fc.nodes[1]);
        if (fc.refine) {
            const int64_t mid_node = split_node_base + refined_before(fi);
            const int64_t second = split_face_base + refined_before(fi);
            const V2 p1 = (p0 + p2) / 2;
            w.nd[static_cast<size_t>(mid_node)] = p1;
            std::array<int64_t, 2> e1{Ln, Rn}, e2{Ln, Rn};
            if (w.would_h(L)) {
                e1[0] += child_shift(L, Ls, p0, p1, p2, 1);
                e2[0] += child_shift(L, Ls, p0, p1, p2, 2);
            }
            if (w.would_h(R)) {
                e1[1] += child_shift(R, Rs, p0, p1, p2, 1);
                e2[1] += child_shift(R, Rs, p0, p1, p2, 2);
            }
            Face a, b;
            a.N = b.N = face_N;
            a.nodes = {fc.nodes[0], mid_node};
            b.nodes = {mid_node, fc.nodes[1]};
            a.elems = e1;
            b.elems = e2;
            a.sides = b.sides = fc.sides;
            nf[static_cast<size_t>(fi)] = a;
            nf[static_cast<size_t>(second)] = b;
        } else {
            fc.N = face_N;
            std::array<int64_t, 2> e{Ln, Rn};
            if (w.would_h(L)) e[0] += child_shift(L, Ls, p0, p2, p2, 0);
            if (w.would_h(R)) e[1] += child_shift(R, Rs, p0, p2, p2, 0);
            fc.elems = e;
            fc.refine = false;
            nf[static_cast<size_t>(fi)] = fc;
        }
    }

    // Write the new mesh back.
    const int64_t K_new = w.K + 3 * n_split;
    t.n_domain = K_new;
    const size_t E = ne.size();
    t.elem_N.resize(E);
    t.elem_nodes.resize(E);
    t.elem_face.resize(E);
    t.elem_faces.resize(E);
    t.elem_split.resize(E);
    t.elem_status.resize(E);
    t.elem_rotation.resize(E);
    t.ghost_sf_zero.assign(E, 0);
    for (size_t e = 0; e < E; ++e) {
        Elem& x = ne[e];
        t.elem_N[e] = x.N;
        t.elem_nodes[e] = x.nodes;
        t.elem_faces[e] = std::move(x.faces);
        for (size_t s = 0; s < 4; ++s) t.elem_face[e][s] = t.elem_faces[e][s].empty() ? -1 : t.elem_faces[e][s][0];
        t.elem_split[e] = x.split;
        t.elem_status[e] = x.status;
        t.elem_rotation[e] = x.rotation;
        t.ghost_sf_zero[e] = (static_cast<int64_t>(e) >= K_new && x.sf_zero) ? 1 : 0;
    }
    const size_t NF = nf.size();
    t.face_N.resize(NF);
    t.face_nodes.resize(NF);
    t.face_elems.resize(NF);
    t.face_sides.resize(NF);
    for (size_t f = 0; f < NF; ++f) {
        t.face_N[f] = nf[f].N;
        t.face_nodes[f] = nf[f].nodes;
        t.face_elems[f] = nf[f].elems;
        t.face_sides[f] = nf[f].sides;
    }
    t.node_x.resize(w.nd.size());
    t.node_y.resize(w.nd.size());
    for (size_t i = 0; i < w.nd.size(); ++i) {
        t.node_x[i] = w.nd[i].x;
        t.node_y[i] = w.nd[i].y;
    }
    t.boundary = new_boundary;
    t.if_origin = new_origin;
    t.if_origin_side = new_origin_side;
    t.if_destination = new_destination;
    compute_geometry(t, tables);
    return true;
}

}  // namespace ndg

namespace ndg {

namespace {

// quad_map (include/functions/quad_map.tpp): the bilinear map of (x, y).
V2 quad_map(double x, double y, const std::array<double, 8>& p) {
    auto P = [&](int k) { return V2{p[static_cast<size_t>(2 * k)], p[static_cast<size_t>(2 * k + 1)]}; };
    auto scaled = [](V2 v, double a, double b) { return V2{v.x * a * b, v.y * a * b}; };
    const V2 s = scaled(P(0), 1 - x, 1 - y) + scaled(P(1), x + 1, 1 - y) + scaled(P(2), x + 1, y + 1) + scaled(P(3), 1 - x, y + 1);
    return s / 4;
}

double cross(V2 a, V2 b) { return a.x * b.y - a.y * b.x; }

// inverse_quad_map (include/functions/inverse_quad_map.tpp:42-77, the code
// that runs): reference-square coordinates of a point of a quad.
V2 inverse_quad_map(V2 q, const std::array<double, 8>& p) {
    const V2 p0{p[0], p[1]}, p1{p[2], p[3]}, p2{p[4], p[5]}, p3{p[6], p[7]};
    const V2 e = p1 - p0, f = p3 - p0, g = p0 - p1 + p2 - p3, h = q - p0;
    const double k2 = cross(g, f);
    const double k1 = cross(e, f) + cross(h, g);
    const double k0 = cross(h, e);
    if (std::abs(k2) < std::numeric_limits<double>::min()) {
        const double ux = e.x * k1 - g.x * k0, uy = e.y * k1 - g.y * k0;
        const double u = (std::abs(ux) > std::abs(uy)) ? (h.x * k1 + f.x * k0) / ux : (h.y * k1 + f.y * k0) / uy;
        return {u * 2 - 1, -k0 / k1 * 2 - 1};
    }
    double w = k1 * k1 - 4 * k0 * k2;
    if (w < 0.0) return {-1, -1};
    w = std::sqrt(w);
    const double ik2 = 1 / (2 * k2);
    double v = (-k1 - w) * ik2;
    double ux = e.x + g.x * v, uy = e.y + g.y * v;
    double u = (std::abs(ux) > std::abs(uy)) ? (h.x - f.x * v) / ux : (h.y - f.y * v) / uy;
    if (u < 0.0 || u > 1.0 || v < 0.0 || v > 1.0) {
        v = (-k1 + w) * ik2;
        ux = e.x + g.x * v;
        uy = e.y + g.y * v;
        u = (std::abs(ux) > std::abs(uy)) ? (h.x - f.x * v) / ux : (h.y - f.y * v) / uy;
    }
    return {u * 2 - 1, v * 2 - 1};
}

}  // namespace

void child_coordinates(const ElementSource& src, const std::vector<double>& nodes_N, std::vector<double>& out) {
    const size_t n = nodes_N.size();
    out.resize(2 * n * n);
    for (size_t i = 0; i < n; ++i)
        for (size_t j = 0; j < n; ++j) {
            const V2 gxy = quad_map(nodes_N[i], nodes_N[j], src.child);
            const V2 local = inverse_quad_map(gxy, src.parent);
            out[2 * (i * n + j)] = local.x;
            out[2 * (i * n + j) + 1] = local.y;
        }
}

}  // namespace ndg
