// Host side of mixed-order meshes: the device plan of the general stage
// path, and p-adaptation of the topology with the reference's rules.
#include "ndg_internal.hpp"

#include <algorithm>
#include <cmath>
#include <map>

namespace ndg {

namespace {
constexpr double kPi = 3.14159265358979323846;
enum HilbertStatus : int { kH = 0, kA = 1, kR = 2, kB = 3 };

// Hilbert::deduct_*_element_status (src/functions/Hilbert_splitting.cpp:3-22):
// the curve's shape in an element from the sides it enters and leaves by.
int first_status(int outgoing) {
    constexpr int t[4] = {kB, kH, kA, kR};
    return t[outgoing];
}
int last_status(int incoming) {
    constexpr int t[4] = {kA, kR, kB, kH};
    return t[incoming];
}
int middle_status(int incoming, int outgoing) {
    constexpr int t[4][4] = {{kH, kH, kA, kA}, {kB, kB, kR, kR}, {kB, kB, kR, kR}, {kH, kH, kA, kA}};
    return t[incoming][outgoing];
}

// Side of an element through which the neighbouring centre lies.
int side_towards(double dx, double dy) {
    if (std::abs(dy) > std::abs(dx)) return dy < 0 ? 0 : 2;
    return dx < 0 ? 3 : 1;
}
}  // namespace

void init_adaptivity_state(Topology& t) {
    const size_t total = t.elem_N.size();
    const int64_t K = t.n_domain;
    t.elem_split.assign(total, 0);
    t.elem_status.assign(total, kA);
    t.elem_rotation.assign(total, 0);
    t.ghost_sf_zero.assign(total, 0);
    t.elem_faces.assign(total, {});
    for (size_t e = 0; e < total; ++e)
        for (int s = 0; s < 4; ++s) {
            const int64_t f = t.elem_face[e][static_cast<size_t>(s)];
            if (f >= 0 && (static_cast<int64_t>(e) < K || s == 0)) t.elem_faces[e][static_cast<size_t>(s)].push_back(f);
        }
    // Mesh2D_t::compute_element_status (src/meshes/Mesh2D_t.cpp:4055-4178).
    constexpr double targets[4] = {-3 * kPi / 4, -kPi / 4, kPi / 4, 3 * kPi / 4};
    for (int64_t e = 0; e < K; ++e) {
        const size_t ei = static_cast<size_t>(e);
        long rotation = 0;
        for (size_t i = 0; i < 4; ++i) {
            const size_t nd = static_cast<size_t>(t.elem_nodes[ei][i]);
            const double angle = std::atan2(t.node_y[nd] - t.center[ei][1], t.node_x[nd] - t.center[ei][0]);
            const double offset = std::atan2(std::sin(angle - targets[i]), std::cos(angle - targets[i]));
            const long turns = std::lround(offset * 2 / kPi + 4 * (offset < 0));
            rotation += turns * (turns < 4);
        }
        t.elem_rotation[ei] = static_cast<int>(rotation / 4);
        auto toward = [&](int64_t o) {
            const size_t oi = static_cast<size_t>(o);
            return side_towards(t.center[oi][0] - t.center[ei][0], t.center[oi][1] - t.center[ei][1]);
        };
        if (K == 1) t.elem_status[ei] = kH;
        else if (e == 0) t.elem_status[ei] = first_status(toward(e + 1));
        else if (e == K - 1) t.elem_status[ei] = last_status(toward(e - 1));
        else t.elem_status[ei] = middle_status(toward(e - 1), toward(e + 1));
    }
}

bool fused_path_applies(const Topology& t) {
    if (t.n_domain <= 0) return false;
    const int N = t.elem_N[0];
    for (int Ne : t.elem_N)
        if (Ne != N) return false;
    for (int Nf : t.face_N)
        if (Nf != N) return false;
    for (int64_t e = 0; e < t.n_domain; ++e) {
        const auto& nd = t.elem_nodes[static_cast<size_t>(e)];
        for (int s = 0; s < 4; ++s) {
            if (t.elem_faces[static_cast<size_t>(e)][static_cast<size_t>(s)].size() != 1) return false;
            const int64_t f = t.elem_face[static_cast<size_t>(e)][static_cast<size_t>(s)];
            if (f < 0) return false;
            const auto& fe = t.face_elems[static_cast<size_t>(f)];
            const auto& fn = t.face_nodes[static_cast<size_t>(f)];
            const int64_t a = nd[static_cast<size_t>(s)], b = nd[static_cast<size_t>((s + 1) % 4)];
            const bool conforming = fe[0] == e ? (fn[0] == a && fn[1] == b) : (fn[0] == b && fn[1] == a);
            if (!conforming) return false;
            const int64_t other = fe[0] == e ? fe[1] : fe[0];
            if (other >= t.n_domain && (t.face_scale[static_cast<size_t>(f)][1] != 1.0 || t.face_offset[static_cast<size_t>(f)][1] != 0.0))
                return false;
        }
    }
    return true;
}

GeneralPlan build_general_plan(const Topology& t, const Tables* tab) {
    GeneralPlan p;
    const int64_t K = t.n_domain;
    const int64_t total = static_cast<int64_t>(t.elem_N.size());
    const int64_t F = static_cast<int64_t>(t.face_N.size());
    p.n_domain = K;
    p.n_total = total;
    p.n_faces = F;
    p.eN.assign(t.elem_N.begin(), t.elem_N.end());
    p.off2.resize(static_cast<size_t>(K));
    p.off1.resize(static_cast<size_t>(total));
    int64_t o2 = 0, o1 = 0;
    for (int64_t e = 0; e < total; ++e) {
        const int64_t n = t.elem_N[static_cast<size_t>(e)] + 1;
        if (e < K) {
            p.off2[static_cast<size_t>(e)] = o2;
            o2 += n * n;
            p.off1[static_cast<size_t>(e)] = o1;
            o1 += 4 * n;
        } else {
            p.off1[static_cast<size_t>(e)] = o1;
            o1 += n;
        }
    }
    p.block = o2 + (o2 & 1);
    p.trace_total = o1;
    p.enodes.resize(static_cast<size_t>(4 * total));
    p.sface_start.assign(static_cast<size_t>(4 * total + 1), 0);
    {
        size_t n_entries = 0;  // the side face lists' total, so that sface grows once
        for (const auto& sides : t.elem_faces)
            for (const auto& list : sides) n_entries += list.size();
        p.sface.reserve(n_entries);
    }
    for (int64_t e = 0; e < total; ++e) {
        for (int s = 0; s < 4; ++s) {
            p.enodes[static_cast<size_t>(4 * e + s)] = t.elem_nodes[static_cast<size_t>(e)][static_cast<size_t>(s)];
            const auto& list = t.elem_faces[static_cast<size_t>(e)][static_cast<size_t>(s)];
            p.sface_start[static_cast<size_t>(4 * e + s + 1)] = p.sface_start[static_cast<size_t>(4 * e + s)] + static_cast<int64_t>(list.size());
            p.sface.insert(p.sface.end(), list.begin(), list.end());
        }
    }
    p.corners.resize(static_cast<size_t>(8 * K));
    for (int64_t e = 0; e < K; ++e)
        for (int k = 0; k < 4; ++k) {
            const size_t nd = static_cast<size_t>(t.elem_nodes[static_cast<size_t>(e)][static_cast<size_t>(k)]);
            p.corners[static_cast<size_t>(8 * e + 2 * k)] = t.node_x[nd];
            p.corners[static_cast<size_t>(8 * e + 2 * k + 1)] = t.node_y[nd];
        }
    p.node_xy.resize(2 * t.node_x.size());
    for (size_t i = 0; i < t.node_x.size(); ++i) {
        p.node_xy[2 * i] = t.node_x[i];
        p.node_xy[2 * i + 1] = t.node_y[i];
    }
    p.fN.assign(t.face_N.begin(), t.face_N.end());
    p.foff.resize(static_cast<size_t>(F));
    int64_t of = 0;
    for (int64_t f = 0; f < F; ++f) {
        p.foff[static_cast<size_t>(f)] = of;
        of += t.face_N[static_cast<size_t>(f)] + 1;
    }
    p.face_total = of;
    auto put2 = [F](const auto& src, auto& dst) {
        dst.resize(static_cast<size_t>(2 * F));
        for (int64_t f = 0; f < F; ++f) {
            dst[static_cast<size_t>(2 * f)] = src[static_cast<size_t>(f)][0];
            dst[static_cast<size_t>(2 * f + 1)] = src[static_cast<size_t>(f)][1];
        }
    };
    put2(t.face_nodes, p.fnodes);
    put2(t.face_elems, p.felem);
    put2(t.face_sides, p.fside);
    put2(t.face_normal, p.fnormal);
    put2(t.face_tangent, p.ftangent);
    put2(t.face_offset, p.foffset);
    put2(t.face_scale, p.fscale);

    // What fills each ghost's side-0 trace (Mesh2D_t::boundary_conditions
    // runs walls, symmetry, inflow, outflow, then interfaces: last writer wins).
    const int64_t G = total - K;
    p.gkind.assign(static_cast<size_t>(G), 4);
    p.gscale.assign(static_cast<size_t>(G), 0.0);
    p.gsrc.assign(static_cast<size_t>(G), 0);
    p.gsrc_side.assign(static_cast<size_t>(G), 0);
    const int kinds[4] = {0, 0, 1, 2};  // wall, symmetry: mirror; inflow: analytic; outflow: copy
    for (int b = 0; b < 4; ++b)
        for (int64_t g : t.boundary[static_cast<size_t>(b)]) p.gkind[static_cast<size_t>(g - K)] = kinds[b];
    for (size_t i = 0; i < t.if_destination.size(); ++i) {
        const size_t g = static_cast<size_t>(t.if_destination[i] - K);
        p.gkind[g] = 3;
        p.gsrc[g] = t.if_origin[i];
        p.gsrc_side[g] = static_cast<int32_t>(t.if_origin_side[i]);
    }
    for (int64_t g = K; g < total; ++g) p.gscale[static_cast<size_t>(g - K)] = t.ghost_scale[static_cast<size_t>(g)][0];

    std::map<int, std::vector<int64_t>> by_order;
    for (int64_t e = 0; e < K; ++e) by_order[t.elem_N[static_cast<size_t>(e)]].push_back(e);
    for (auto& kv : by_order) p.groups.emplace_back(kv.first, std::move(kv.second));

    // Mortar weight blocks for the sides and face sides that need them.
    auto conforming = [&](int64_t f, int64_t e, int64_t es, bool left) {
        const int64_t a = t.elem_nodes[static_cast<size_t>(e)][static_cast<size_t>(es)];
        const int64_t b = t.elem_nodes[static_cast<size_t>(e)][static_cast<size_t>((es + 1) & 3)];
        const auto& fn = t.face_nodes[static_cast<size_t>(f)];
        return t.face_N[static_cast<size_t>(f)] == t.elem_N[static_cast<size_t>(e)] && (left ? (fn[0] == a && fn[1] == b) : (fn[1] == a && fn[0] == b));
    };
    // Conforming elements (conforming_stage_kernel): on each side one face
    // of the element's order from the side's first to its second node (or
    // reversed, for the face's right element), whose other element (a domain
    // element or a ghost) sees it the same way. Where they are at least half
    // of their order group they go last in it (the rest, whose tiles take
    // longest, first) and form a group of their own at run time; elsewhere
    // the group keeps its order and runs as one.
    auto conforming_side = [&](int64_t e, int s, int64_t& nb, int32_t& role, int64_t& face) {
        const auto& list = t.elem_faces[static_cast<size_t>(e)][static_cast<size_t>(s)];
        if (list.size() != 1) return false;
        const int64_t f = list[0];
        const auto& fe = t.face_elems[static_cast<size_t>(f)];
        const auto& fs = t.face_sides[static_cast<size_t>(f)];
        const bool left = fe[0] == e && fs[0] == s, right = fe[1] == e && fs[1] == s;
        if (left == right) return false;
        const size_t oi = left ? 1 : 0;
        const int64_t o = fe[oi], os = fs[oi];
        if (o >= K && os != 0) return false;  // a ghost's only trace is its side 0
        if (!conforming(f, e, s, left) || !conforming(f, o, os, !left)) return false;
        nb = p.off1[static_cast<size_t>(o)] + os * (t.elem_N[static_cast<size_t>(o)] + 1);
        role = left ? 0 : 1;
        face = f;
        return true;
    };
    std::vector<char> conf(static_cast<size_t>(K), 0);
    for (int64_t e = 0; e < K; ++e) {
        bool ok = true;
        for (int s = 0; s < 4 && ok; ++s) {
            int64_t nb, face;
            int32_t role;
            ok = conforming_side(e, s, nb, role, face);
        }
        conf[static_cast<size_t>(e)] = ok ? 1 : 0;
    }
    p.group_conforming.assign(p.groups.size(), 0);
    for (size_t gi = 0; gi < p.groups.size(); ++gi) {
        auto& list = p.groups[gi].second;
        int64_t nconf = 0;
        for (int64_t e : list) nconf += conf[static_cast<size_t>(e)];
        if (2 * nconf < static_cast<int64_t>(list.size())) continue;
        std::stable_partition(list.begin(), list.end(), [&](int64_t e) { return conf[static_cast<size_t>(e)] == 0; });
        p.group_conforming[gi] = nconf;
    }
    for (int64_t e = 0; e < K; ++e)
        for (int s = 0; s < 4; ++s) {
            int64_t slots = 0;
            for (int64_t q = p.sface_start[static_cast<size_t>(4 * e + s)]; q < p.sface_start[static_cast<size_t>(4 * e + s + 1)]; ++q)
                slots += t.face_N[static_cast<size_t>(p.sface[static_cast<size_t>(q)])] + 1;
            p.side_slots = std::max(p.side_slots, slots);
        }
    p.sw_off.assign(p.sface.size(), -1);
    p.sm_off.assign(p.sface.size(), -1);
    for (int64_t e = 0; e < K; ++e)
        for (int s = 0; s < 4; ++s) {
            const int64_t q0 = p.sface_start[static_cast<size_t>(4 * e + s)], q1 = p.sface_start[static_cast<size_t>(4 * e + s + 1)];
            if (q1 == q0) continue;
            const int64_t f0 = p.sface[static_cast<size_t>(q0)];
            if (q1 - q0 == 1 && (conforming(f0, e, s, true) || conforming(f0, e, s, false))) continue;
            const int64_t ne_ = t.elem_N[static_cast<size_t>(e)] + 1;
            for (int64_t q = q0; q < q1; ++q) {
                const int64_t nf = t.face_N[static_cast<size_t>(p.sface[static_cast<size_t>(q)])] + 1;
                p.sw_off[static_cast<size_t>(q)] = p.sw_total;
                p.sw_total += ne_ * nf;
                p.sm_off[static_cast<size_t>(q)] = p.sm_total;
                p.sm_total += nf;
            }
        }
    p.fbase.resize(static_cast<size_t>(2 * F));
    p.fsN.resize(static_cast<size_t>(2 * F));
    for (int64_t f = 0; f < F; ++f)
        for (int side = 0; side < 2; ++side) {
            const int64_t e = t.face_elems[static_cast<size_t>(f)][static_cast<size_t>(side)];
            const int64_t es = t.face_sides[static_cast<size_t>(f)][static_cast<size_t>(side)];
            const int Ne = t.elem_N[static_cast<size_t>(e)];
            p.fbase[static_cast<size_t>(2 * f + side)] = p.off1[static_cast<size_t>(e)] + es * (Ne + 1);
            p.fsN[static_cast<size_t>(2 * f + side)] = Ne;
        }
    p.fw_off.assign(static_cast<size_t>(2 * F), -1);
    p.fm_off.assign(static_cast<size_t>(2 * F), -1);
    for (int64_t f = 0; f < F; ++f)
        for (int side = 0; side < 2; ++side) {
            const int64_t e = t.face_elems[static_cast<size_t>(f)][static_cast<size_t>(side)];
            const int64_t es = t.face_sides[static_cast<size_t>(f)][static_cast<size_t>(side)];
            if (conforming(f, e, es, side == 0)) continue;
            const int64_t nf = t.face_N[static_cast<size_t>(f)] + 1, ne_ = t.elem_N[static_cast<size_t>(e)] + 1;
            p.fw_off[static_cast<size_t>(2 * f + side)] = p.fw_total;
            p.fw_total += nf * ne_ + nf;
            p.fm_off[static_cast<size_t>(2 * f + side)] = p.fm_total;
            p.fm_total += nf;
        }

    // Ghost side-0 gathers, for the ghosts whose trace is projected from
    // their neighbours (mirror and copy kinds).
    p.gq_start.assign(static_cast<size_t>(G + 1), 0);
    p.gframe.assign(static_cast<size_t>(4 * G), 0.0);
    p.gdirect.assign(static_cast<size_t>(G), -1);
    for (auto* v : {&p.gq_face, &p.gq_base, &p.gq_woff, &p.gq_moff}) v->reserve(static_cast<size_t>(G));
    p.gq_fs.reserve(static_cast<size_t>(G));
    p.gq_N.reserve(static_cast<size_t>(G));
    for (int64_t g = K; g < total; ++g) {
        const size_t gi = static_cast<size_t>(g - K);
        p.gq_start[gi] = static_cast<int64_t>(p.gq_face.size());
        if (p.gkind[gi] != 0 && p.gkind[gi] != 2) continue;
        const int Ng = t.elem_N[static_cast<size_t>(g)];
        const int64_t q0 = p.sface_start[static_cast<size_t>(4 * g)], q1 = p.sface_start[static_cast<size_t>(4 * g + 1)];
        for (int64_t q = q0; q < q1; ++q) {
            const int64_t f = p.sface[static_cast<size_t>(q)];
            const int fs = t.face_elems[static_cast<size_t>(f)][0] == g ? 1 : 0;
            const int Nn = p.fsN[static_cast<size_t>(2 * f + fs)];
            p.gq_face.push_back(f);
            p.gq_fs.push_back(fs);
            p.gq_base.push_back(p.fbase[static_cast<size_t>(2 * f + fs)]);
            p.gq_N.push_back(Nn);
            p.gq_woff.push_back(p.sw_total);
            p.sw_total += static_cast<int64_t>(Ng + 1) * (Nn + 1);
            p.gq_moff.push_back(p.sm_total);
            p.sm_total += Nn + 1;
        }
        if (q1 - q0 == 1 && tab != nullptr && Ng <= tab->N_max) {
            // Direct gather: ghost_weights_kernel would match neighbour node j
            // to ghost node N - j with weight w_n[j] / w_g[N - j] == 1.
            const int64_t f = p.sface[static_cast<size_t>(q0)];
            const int fs = p.gq_fs.back(), Nn = p.gq_N.back();
            bool direct = Nn == Ng;
            const auto& x = tab->get(NDG_TABLE_NODES, Ng);
            const auto& w = tab->get(NDG_TABLE_WEIGHTS, Ng);
            const double scale = t.face_scale[static_cast<size_t>(f)][static_cast<size_t>(fs)];
            const double offset = t.face_offset[static_cast<size_t>(f)][static_cast<size_t>(fs)];
            for (int j = 0; j <= Nn && direct; ++j) {
                const double coord = ((x[static_cast<size_t>(Nn - j)] + 1.0) * scale + 2.0 * offset) - 1.0;  // mortar_coord
                int found = -1;
                for (int ii = 0; ii <= Ng && found < 0; ++ii)
                    if (almost_equal(coord, x[static_cast<size_t>(ii)])) found = ii;
                direct = found == Ng - j && w[static_cast<size_t>(j)] == w[static_cast<size_t>(Ng - j)];
            }
            if (direct) p.gdirect[gi] = p.gq_base.back();
        }
        if (q1 > q0) {
            const size_t f0 = static_cast<size_t>(p.sface[static_cast<size_t>(q0)]);
            p.gframe[4 * gi] = t.face_normal[f0][0];
            p.gframe[4 * gi + 1] = t.face_normal[f0][1];
            p.gframe[4 * gi + 2] = t.face_tangent[f0][0];
            p.gframe[4 * gi + 3] = t.face_tangent[f0][1];
        }
    }
    p.gq_start[static_cast<size_t>(G)] = static_cast<int64_t>(p.gq_face.size());

    // Slots and side modes in group-list order, so that the sides of one
    // tile of a group own one contiguous slot range. A slot stores its face
    // node j as 32 f + j, and the kernels decode it with the same base.
    static_assert(kMaxOrder < 32, "face node index of a slot must fit below 32");
    p.pslot_start.assign(static_cast<size_t>(4 * K + 1), 0);
    p.pside_mode.assign(static_cast<size_t>(4 * K), 0);
    p.pq_start.assign(static_cast<size_t>(4 * K + 1), 0);
    {
        // Sizes first, so that the slot and list-order arrays grow once.
        size_t n_slots = 0;
        for (int64_t q = 0; q < p.sface_start[static_cast<size_t>(4 * K)]; ++q)
            n_slots += static_cast<size_t>(t.face_N[static_cast<size_t>(p.sface[static_cast<size_t>(q)])] + 1);
        p.slot_desc.reserve(n_slots);
        p.slot_normal.reserve(2 * n_slots);
        p.slot_side.reserve(n_slots);
        const size_t n_q = static_cast<size_t>(p.sface_start[static_cast<size_t>(4 * K)]);
        p.pq_N.reserve(n_q);
        p.pq_scale.reserve(n_q);
        p.pq_woff.reserve(n_q);
        p.pq_moff.reserve(n_q);
        p.poff2.reserve(static_cast<size_t>(K));
        p.cnb.reserve(static_cast<size_t>(4 * K));
        p.crole.reserve(static_cast<size_t>(4 * K));
        p.cnormal.reserve(static_cast<size_t>(8 * K));
        p.poff1.reserve(static_cast<size_t>(K));
        p.pcorners.reserve(static_cast<size_t>(8 * K));
    }
    int64_t pos = 0, slot = 0;
    for (const auto& grp : p.groups)
        for (int64_t e : grp.second) {
            const int Ne = t.elem_N[static_cast<size_t>(e)];
            p.poff2.push_back(p.off2[static_cast<size_t>(e)]);
            p.poff1.push_back(p.off1[static_cast<size_t>(e)]);
            p.pcorners.insert(p.pcorners.end(), p.corners.begin() + 8 * e, p.corners.begin() + 8 * e + 8);
            for (int s = 0; s < 4; ++s) {
                int64_t nb = 0, face = -1;
                int32_t role = 0;
                if (!conf[static_cast<size_t>(e)] || !conforming_side(e, s, nb, role, face)) nb = 0, role = 0, face = -1;
                p.cnb.push_back(nb);
                p.crole.push_back(role);
                p.cnormal.push_back(face >= 0 ? t.face_normal[static_cast<size_t>(face)][0] : 0.0);
                p.cnormal.push_back(face >= 0 ? t.face_normal[static_cast<size_t>(face)][1] : 0.0);
                const size_t ps = static_cast<size_t>(4 * pos + s);
                p.pslot_start[ps] = slot;
                p.pq_start[ps] = static_cast<int64_t>(p.pq_N.size());
                const int64_t q0 = p.sface_start[static_cast<size_t>(4 * e + s)], q1 = p.sface_start[static_cast<size_t>(4 * e + s + 1)];
                for (int64_t q = q0; q < q1; ++q) {
                    const int64_t f = p.sface[static_cast<size_t>(q)];
                    for (int j = 0; j <= t.face_N[static_cast<size_t>(f)]; ++j) {
                        p.slot_desc.push_back(32 * f + j);
                        p.slot_normal.push_back(t.face_normal[static_cast<size_t>(f)][0]);
                        p.slot_normal.push_back(t.face_normal[static_cast<size_t>(f)][1]);
                        p.slot_side.push_back(static_cast<int32_t>(ps));
                        ++slot;
                    }
                }
                if (q1 == q0) continue;
                const int64_t f0 = p.sface[static_cast<size_t>(q0)];
                const auto& fn = t.face_nodes[static_cast<size_t>(f0)];
                const int64_t en0 = p.enodes[static_cast<size_t>(4 * e + s)], en1 = p.enodes[static_cast<size_t>(4 * e + ((s + 1) & 3))];
                const bool one = q1 - q0 == 1 && t.face_N[static_cast<size_t>(f0)] == Ne;
                p.pside_mode[ps] = one && fn[0] == en0 && fn[1] == en1 ? 1 : one && fn[1] == en0 && fn[0] == en1 ? 2 : 3;
                if (p.pside_mode[ps] != 3) continue;
                for (int64_t q = q0; q < q1; ++q) {
                    const size_t f = static_cast<size_t>(p.sface[static_cast<size_t>(q)]);
                    const int fsd = t.face_elems[f][0] == e ? 0 : 1;
                    p.pq_N.push_back(t.face_N[f]);
                    p.pq_scale.push_back(t.face_scale[f][static_cast<size_t>(fsd)]);
                    p.pq_woff.push_back(p.sw_off[static_cast<size_t>(q)]);
                    p.pq_moff.push_back(p.sm_off[static_cast<size_t>(q)]);
                }
            }
            ++pos;
        }
    p.pslot_start[static_cast<size_t>(4 * K)] = slot;
    p.pq_start[static_cast<size_t>(4 * K)] = static_cast<int64_t>(p.pq_N.size());
    p.n_slots = slot;
    return p;
}

// Mesh2D_t::adapt when no element splits (src/meshes/Mesh2D_t.cpp:1644-1700):
// p_adapt (:5026-5049; Element2D_t::would_p_refine, Element2D_t.cpp:802-806),
// then adjust_boundaries for walls, symmetry, inflow and outflow
// (:7482-7504), adjust_interfaces (:7506-7520) and adjust_faces (:7522-7538).
// A ghost whose order changes gets new, zeroed boundary storage in the
// reference (Element2D_t::resize_boundary_storage, Element2D_t.cpp:735-741),
// scaling factor included; that is kept.
bool p_adapt(Topology& t, const int32_t* refine, const double* p_sigma, int N_max, int max_split_level) {
    const int64_t K = t.n_domain;
    (void)max_split_level;  // element splitting is h_adapt's branch
    bool changed = false;
    for (int64_t e = 0; e < K; ++e) {
        int& N = t.elem_N[static_cast<size_t>(e)];
        if (refine[e] && p_sigma[e] >= 1.0 && N + 2 <= N_max) {
            N += 2;
            changed = true;
        }
    }
    for (int b = 0; b < 4; ++b)
        for (int64_t g : t.boundary[static_cast<size_t>(b)]) {
            int N_el = t.elem_N[static_cast<size_t>(g)];
            for (int64_t f : t.elem_faces[static_cast<size_t>(g)][0]) {
                const auto& fe = t.face_elems[static_cast<size_t>(f)];
                const int64_t src = fe[fe[0] == g ? 1 : 0];
                N_el = std::max(N_el, t.elem_N[static_cast<size_t>(src)]);
            }
            if (t.elem_N[static_cast<size_t>(g)] != N_el) {
                t.elem_N[static_cast<size_t>(g)] = N_el;
                t.ghost_scale[static_cast<size_t>(g)][0] = 0.0;
                t.ghost_sf_zero[static_cast<size_t>(g)] = 1;
                changed = true;
            }
        }
    for (size_t i = 0; i < t.if_origin.size(); ++i) {
        const int Ns = t.elem_N[static_cast<size_t>(t.if_origin[i])];
        int& Nd = t.elem_N[static_cast<size_t>(t.if_destination[i])];
        if (Nd != Ns) {
            Nd = Ns;
            t.ghost_scale[static_cast<size_t>(t.if_destination[i])][0] = 0.0;
            t.ghost_sf_zero[static_cast<size_t>(t.if_destination[i])] = 1;
            changed = true;
        }
    }
    for (size_t f = 0; f < t.face_N.size(); ++f) {
        const int Nf = std::max(t.elem_N[static_cast<size_t>(t.face_elems[f][0])], t.elem_N[static_cast<size_t>(t.face_elems[f][1])]);
        if (t.face_N[f] != Nf) {
            t.face_N[f] = Nf;
            changed = true;
        }
    }
    return changed;
}

}  // namespace ndg
