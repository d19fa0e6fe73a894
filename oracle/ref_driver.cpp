// Test-only C driver over the reference's own CPU path (SEM::Host::*),
// compiled unmodified from the reference sources into oracle/_ref/libndgref.so
// by oracle/Makefile. Tests use it to pin the oracle restatement and the CUDA
// path: it is the checker, never the product.
//
// The stage sequence below is the body of the reference's time loop
// (include/solvers/Solver2D_t.tpp:44-70) without the progress bar and output
// calls; dt is the reference's Solver2D_t::get_delta_t
// (src/solvers/Solver2D_t.cpp:19-29).
#include "cgnslib.h"
#include "entities/NDG_t.h"
#include "polynomials/LegendrePolynomial_t.h"
#include "meshes/Mesh2D_t.h"
#include "solvers/Solver2D_t.h"
#include <array>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

NdgMemZone ndg_mem_cgns;

namespace {
using NDG = SEM::Host::Entities::NDG_t<SEM::Host::Polynomials::LegendrePolynomial_t>;
using SEM::Host::Meshes::Mesh2D_t;
using SEM::Host::Solvers::Solver2D_t;

struct RefState {
    std::unique_ptr<NDG> ndg;
    std::unique_ptr<Mesh2D_t> mesh;
    std::unique_ptr<Solver2D_t> solver;
};
RefState g_ref;

constexpr std::array<double, 3> am {0, -5.0 / 9.0, -153.0 / 128.0};
constexpr std::array<double, 3> bm {0, 1.0 / 3.0, 0.75};
constexpr std::array<double, 3> gm {1.0 / 3.0, 15.0 / 16.0, 8.0 / 15.0};

void run_stage(int m, double time, double dt) {
    NDG& ndg = *g_ref.ndg;
    Mesh2D_t& mesh = *g_ref.mesh;
    const double t = time + bm[m] * dt;
    mesh.interpolate_to_boundaries(ndg.lagrange_interpolant_left_, ndg.lagrange_interpolant_right_);
    mesh.boundary_conditions(t, ndg.nodes_, ndg.weights_, ndg.barycentric_weights_);
    mesh.project_to_faces(ndg.nodes_, ndg.barycentric_weights_);
    Solver2D_t::calculate_wave_fluxes(mesh.faces_);
    mesh.project_to_elements(ndg.nodes_, ndg.weights_, ndg.barycentric_weights_);
    SEM::Host::Solvers::compute_dg_wave_derivative(mesh.n_elements_, mesh.elements_.data(), mesh.faces_.data(), ndg.weights_, ndg.derivative_matrices_hat_, ndg.lagrange_interpolant_left_, ndg.lagrange_interpolant_right_);
    if (m == 0) {
        SEM::Host::Solvers::rk3_first_step(mesh.n_elements_, mesh.elements_.data(), dt, gm[0]);
    } else {
        SEM::Host::Solvers::rk3_step(mesh.n_elements_, mesh.elements_.data(), dt, am[m], gm[m]);
    }
}

std::vector<double>& element_field(SEM::Host::Entities::Element2D_t& e, int which) {
    switch (which) {
        case 0: return e.p_;
        case 1: return e.u_;
        case 2: return e.v_;
        case 3: return e.G_p_;
        case 4: return e.G_u_;
        case 5: return e.G_v_;
        case 6: return e.p_intermediate_;
        case 7: return e.u_intermediate_;
        default: return e.v_intermediate_;
    }
}
}  // namespace

extern "C" {

void ndgref_zone_reset(long n_nodes, const double* x, const double* y) {
    ndg_mem_cgns = NdgMemZone{};
    ndg_mem_cgns.x.assign(x, x + n_nodes);
    ndg_mem_cgns.y.assign(y, y + n_nodes);
}

// type: 0 = QUAD_4, 1 = BAR_2. start/end are 1-based element numbers.
void ndgref_zone_add_section(const char* name, int type, long start, long end, const long* connectivity, long n_connectivity) {
    NdgMemSection s;
    s.name = name;
    s.type = (type == 0) ? QUAD_4 : BAR_2;
    s.start = start;
    s.end = end;
    s.connectivity.assign(connectivity, connectivity + n_connectivity);
    ndg_mem_cgns.sections.push_back(std::move(s));
}

// bc: 0 = wall, 1 = symmetry, 2 = inflow, 3 = outflow, 4 = null.
void ndgref_zone_add_boco(const char* name, int bc, const long* points, long n) {
    static const BCType_t types[] = {BCWall, BCSymmetryPlane, BCInflow, BCOutflow, BCTypeNull};
    NdgMemBoco b;
    b.name = name;
    b.type = types[bc];
    b.points.assign(points, points + n);
    ndg_mem_cgns.bocos.push_back(std::move(b));
}

void ndgref_zone_add_conn(const char* name, const long* points, const long* donor_points, long n) {
    NdgMemConn c;
    c.name = name;
    c.points.assign(points, points + n);
    c.donor_points.assign(donor_points, donor_points + n);
    ndg_mem_cgns.conns.push_back(std::move(c));
}

int ndgref_create(int initial_N, int maximum_N, long n_interpolation_points, int max_split_level, long adaptivity_interval, double tolerance_min, double tolerance_max, double cfl) {
    g_ref.mesh.reset();
    g_ref.ndg = std::make_unique<NDG>(maximum_N, static_cast<size_t>(n_interpolation_points));
    g_ref.mesh = std::make_unique<Mesh2D_t>("memory.cgns", initial_N, maximum_N, static_cast<size_t>(n_interpolation_points), max_split_level, static_cast<size_t>(adaptivity_interval), 0, tolerance_min, tolerance_max, 0.0, g_ref.ndg->nodes_, std::vector<double>{1.0});
    g_ref.solver = std::make_unique<Solver2D_t>(cfl, std::vector<double>{1.0}, 0.0);
    return 0;
}

// Same, reading a mesh file through the reference's own readers
// (Mesh2D_t::read_su2 for .su2).
int ndgref_create_file(const char* path, int initial_N, int maximum_N, long n_interpolation_points, double cfl) {
    g_ref.mesh.reset();
    g_ref.ndg = std::make_unique<NDG>(maximum_N, static_cast<size_t>(n_interpolation_points));
    g_ref.mesh = std::make_unique<Mesh2D_t>(path, initial_N, maximum_N, static_cast<size_t>(n_interpolation_points), 0, 0, 0, 1e-6, 1e-14, 0.0, g_ref.ndg->nodes_, std::vector<double>{1.0});
    g_ref.solver = std::make_unique<Solver2D_t>(cfl, std::vector<double>{1.0}, 0.0);
    return 0;
}

void ndgref_destroy() {
    g_ref.mesh.reset();
    g_ref.solver.reset();
    g_ref.ndg.reset();
}

// Tables only, without a mesh. table: 0 nodes, 1 weights, 2 barycentric,
// 3 lagrange left, 4 lagrange right, 5 lagrange derivative left,
// 6 lagrange derivative right, 7 derivative, 8 cg derivative,
// 9 derivative hat, 10 interpolation, 11 polynomials.
int ndgref_table(int N_max, long n_interpolation_points, int table, int N, double* out) {
    NDG ndg(N_max, static_cast<size_t>(n_interpolation_points));
    const std::vector<std::vector<double>>* t[] = {
        &ndg.nodes_, &ndg.weights_, &ndg.barycentric_weights_,
        &ndg.lagrange_interpolant_left_, &ndg.lagrange_interpolant_right_,
        &ndg.lagrange_interpolant_derivative_left_, &ndg.lagrange_interpolant_derivative_right_,
        &ndg.derivative_matrices_, &ndg.g_hat_derivative_matrices_, &ndg.derivative_matrices_hat_,
        &ndg.interpolation_matrices_, &ndg.polynomials_};
    const std::vector<double>& v = (*t[table])[static_cast<size_t>(N)];
    std::memcpy(out, v.data(), v.size() * sizeof(double));
    return static_cast<int>(v.size());
}

void ndgref_initial_conditions() {
    g_ref.mesh->initial_conditions(g_ref.ndg->nodes_);
}

void ndgref_counts(long* n_elements, long* n_elements_total, long* n_faces, long* n_nodes) {
    *n_elements = static_cast<long>(g_ref.mesh->n_elements_);
    *n_elements_total = static_cast<long>(g_ref.mesh->elements_.size());
    *n_faces = static_cast<long>(g_ref.mesh->faces_.size());
    *n_nodes = static_cast<long>(g_ref.mesh->nodes_.size());
}

double ndgref_get_delta_t() {
    return g_ref.solver->get_delta_t(*g_ref.mesh);
}

void ndgref_stage(int m, double time, double dt) {
    run_stage(m, time, dt);
}

// n_steps full RK3 steps, each with dt = get_delta_t(mesh), as the reference's
// time loop does. Returns the final time.
double ndgref_run(long n_steps, double time) {
    for (long s = 0; s < n_steps; ++s) {
        const double dt = g_ref.solver->get_delta_t(*g_ref.mesh);
        run_stage(0, time, dt);
        run_stage(1, time, dt);
        run_stage(2, time, dt);
        time += dt;
    }
    return time;
}

void ndgref_element_N(int* N) {
    for (size_t i = 0; i < g_ref.mesh->n_elements_; ++i) {
        N[i] = g_ref.mesh->elements_[i].N_;
    }
}

// which: 0 p, 1 u, 2 v, 3 G_p, 4 G_u, 5 G_v, 6 k_p, 7 k_u, 8 k_v. Values are
// concatenated element by element, (N+1)^2 each, index i*(N+1)+j.
long ndgref_get_field(int which, double* out) {
    long offset = 0;
    for (size_t i = 0; i < g_ref.mesh->n_elements_; ++i) {
        const std::vector<double>& v = element_field(g_ref.mesh->elements_[i], which);
        std::memcpy(out + offset, v.data(), v.size() * sizeof(double));
        offset += static_cast<long>(v.size());
    }
    return offset;
}

long ndgref_set_field(int which, const double* in) {
    long offset = 0;
    for (size_t i = 0; i < g_ref.mesh->n_elements_; ++i) {
        std::vector<double>& v = element_field(g_ref.mesh->elements_[i], which);
        std::memcpy(v.data(), in + offset, v.size() * sizeof(double));
        offset += static_cast<long>(v.size());
    }
    return offset;
}

void ndgref_get_faces(long* nodes, long* elements, long* sides, int* N, double* normal, double* tangent, double* offset, double* scale) {
    const auto& faces = g_ref.mesh->faces_;
    for (size_t f = 0; f < faces.size(); ++f) {
        for (int k = 0; k < 2; ++k) {
            nodes[2 * f + k] = static_cast<long>(faces[f].nodes_[k]);
            elements[2 * f + k] = static_cast<long>(faces[f].elements_[k]);
            sides[2 * f + k] = static_cast<long>(faces[f].elements_side_[k]);
            offset[2 * f + k] = faces[f].offset_[k];
            scale[2 * f + k] = faces[f].scale_[k];
        }
        N[f] = faces[f].N_;
        normal[2 * f] = faces[f].normal_.x();
        normal[2 * f + 1] = faces[f].normal_.y();
        tangent[2 * f] = faces[f].tangent_.x();
        tangent[2 * f + 1] = faces[f].tangent_.y();
    }
}

// All elements (domain then ghosts): nodes, N, split level, status, rotation,
// delta_xy_min and the first face of each side (-1 when the side has none).
void ndgref_get_elements(long* nodes, int* N, int* split_level, int* status, int* rotation, double* delta_xy_min, long* first_face, int* n_faces_side) {
    const auto& elements = g_ref.mesh->elements_;
    for (size_t e = 0; e < elements.size(); ++e) {
        for (int k = 0; k < 4; ++k) {
            nodes[4 * e + k] = static_cast<long>(elements[e].nodes_[k]);
            const auto& fs = elements[e].faces_[static_cast<size_t>(k)];
            n_faces_side[4 * e + k] = static_cast<int>(fs.size());
            first_face[4 * e + k] = fs.empty() ? -1 : static_cast<long>(fs[0]);
        }
        N[e] = elements[e].N_;
        split_level[e] = elements[e].split_level_;
        status[e] = static_cast<int>(elements[e].status_);
        rotation[e] = elements[e].rotation_;
        delta_xy_min[e] = elements[e].delta_xy_min_;
    }
}

void ndgref_get_nodes(double* xy) {
    const auto& nodes = g_ref.mesh->nodes_;
    for (size_t i = 0; i < nodes.size(); ++i) {
        xy[2 * i] = nodes[i].x();
        xy[2 * i + 1] = nodes[i].y();
    }
}

// Boundary lists: kind 0 wall, 1 symmetry, 2 inflow, 3 outflow,
// 4 interface origin, 5 interface origin side, 6 interface destination.
long ndgref_get_boundary(int kind, long* out) {
    Mesh2D_t& m = *g_ref.mesh;
    const std::vector<size_t>* lists[] = {&m.wall_boundaries_, &m.symmetry_boundaries_, &m.inflow_boundaries_, &m.outflow_boundaries_, &m.interfaces_origin_, &m.interfaces_origin_side_, &m.interfaces_destination_};
    const std::vector<size_t>& v = *lists[kind];
    if (out != nullptr) {
        for (size_t i = 0; i < v.size(); ++i) {
            out[i] = static_cast<long>(v[i]);
        }
    }
    return static_cast<long>(v.size());
}

// Every element's face lists, side by side (Element2D_t::faces_); returns the
// total count, writing to out when it is not NULL.
long ndgref_get_element_faces(long* out) {
    long n = 0;
    for (const auto& element : g_ref.mesh->elements_)
        for (const auto& side : element.faces_)
            for (size_t f : side) {
                if (out) out[n] = static_cast<long>(f);
                ++n;
            }
    return n;
}

void ndgref_estimate_error() {
    g_ref.mesh->estimate_error(g_ref.ndg->polynomials_);
}

void ndgref_get_error(double* p_error, double* p_sigma, int* refine, int* coarsen) {
    for (size_t i = 0; i < g_ref.mesh->n_elements_; ++i) {
        const auto& e = g_ref.mesh->elements_[i];
        p_error[i] = e.p_error_;
        p_sigma[i] = e.p_sigma_;
        refine[i] = e.refine_ ? 1 : 0;
        coarsen[i] = e.coarsen_ ? 1 : 0;
    }
}

void ndgref_adapt() {
    g_ref.mesh->adapt(g_ref.ndg->N_max_, g_ref.ndg->nodes_, g_ref.ndg->barycentric_weights_);
}

// Mesh2D_t::get_complete_solution (src/meshes/Mesh2D_t.cpp:4251-4296) at
// `time` through the reference's public interface: point arrays of
// n_elements n_interpolation_points^2 values, in the order x, y, p, u, v,
// dp_dt, du_dt, dv_dt, p/u/v analytical error (out[11], any may be NULL).
void ndgref_complete_solution(double time, double** out) {
    Mesh2D_t& mesh = *g_ref.mesh;
    NDG& ndg = *g_ref.ndg;
    const size_t K = mesh.n_elements_, PP = mesh.n_interpolation_points_ * mesh.n_interpolation_points_;
    std::vector<int> N(K), refine(K), coarsen(K), split(K), status(K), rotation(K);
    std::vector<double> pe(K), ue(K), ve(K), ps(K), us(K), vs(K);
    std::vector<double> d[6];
    for (auto& v : d) v.assign(K * PP, 0.0);
    mesh.get_complete_solution(time, ndg.nodes_, ndg.interpolation_matrices_, N, d[0], d[1], d[2], pe, ue, ve, ps, us, vs, refine, coarsen, split, d[3], d[4], d[5], status, rotation);
    const std::vector<double>* src[11] = {&mesh.x_output_, &mesh.y_output_, &mesh.p_output_, &mesh.u_output_, &mesh.v_output_, &d[0], &d[1], &d[2], &d[3], &d[4], &d[5]};
    for (int i = 0; i < 11; ++i)
        if (out[i]) std::memcpy(out[i], src[i]->data(), K * PP * sizeof(double));
}

// Solver2D_t::pre_condition (iterative = 0) or pre_condition_iterative
// (include/solvers/Solver2D_t.tpp:136-334); the progress bar goes to stdout.
void ndgref_pre_condition(long n_adaptivity_steps, long pre_condition_interval, int iterative) {
    if (iterative)
        g_ref.solver->pre_condition_iterative(*g_ref.ndg, *g_ref.mesh, static_cast<size_t>(n_adaptivity_steps), static_cast<size_t>(pre_condition_interval));
    else
        g_ref.solver->pre_condition(*g_ref.ndg, *g_ref.mesh, static_cast<size_t>(n_adaptivity_steps), static_cast<size_t>(pre_condition_interval));
}

}  // extern "C"
