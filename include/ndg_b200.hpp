/* ndg_b200.hpp: C++ host API over the C ABI of ndg_b200.h.
 *
 * The classes have the names, constructor arguments and member functions of
 * the reference's device classes on the 2D wave path:
 *   SEM::Device::Entities::NDG_t<Polynomial>   include/entities/NDG_t.cuh:11-29
 *   SEM::Device::Meshes::Mesh2D_t               include/meshes/Mesh2D_t.cuh:23-182
 *   SEM::Device::Solvers::Solver2D_t            include/solvers/Solver2D_t.cuh:14-65
 * so a driver such as the reference's src/main.cu:346-390 keeps its calls
 * after swapping `SEM::Device` for `ndg_b200`. Differences a caller sees:
 *   - tables are host vectors in the device NDG_t's packed layout (the
 *     library keeps its own device copies);
 *   - Helpers::DataWriter_t writes the reference's files without VTK (a
 *     parallel unstructured grid per output time and the .series files);
 *     Solver2D_t::solve takes it, or any output callback;
 *   - errors throw ndg_b200::Error (the reference exits);
 * Header-only; link against libndg_b200.so. */
#ifndef NDG_B200_HPP
#define NDG_B200_HPP

#include "ndg_b200.h"

#include <array>
#include <cstddef>
#include <cstdint>
#include <filesystem>
#include <functional>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

struct CUstream_st;  // cudaStream_t is CUstream_st*

namespace ndg_b200 {

class Error : public std::runtime_error {
public:
    Error(ndg_status status, const std::string& what) : std::runtime_error(what), status_(status) {}
    ndg_status status() const noexcept { return status_; }

private:
    ndg_status status_;
};

inline void check(ndg_status status, const char* call) {
    if (status != NDG_OK) throw Error(status, std::string(call) + ": " + ndg_last_error());
}

namespace Polynomials {
// Legendre-Gauss nodes (include/polynomials/LegendrePolynomial_t.cuh); the
// only family on the wave path.
struct LegendrePolynomial_t {};
}  // namespace Polynomials

namespace Entities {

// NDG_t<LegendrePolynomial_t>(N_max, n_interpolation_points, stream)
// (include/entities/NDG_t.tcu:13-72). Every table holds the orders 0..N_max
// back to back, which is the device NDG_t's packed layout: order N starts at
// N(N+1)/2 (vectors), N(N+1)(2N+1)/6 (matrices) and N(N+1)/2 *
// n_interpolation_points (interpolation matrices).
template <typename Polynomial = Polynomials::LegendrePolynomial_t>
class NDG_t {
    static_assert(std::is_same<Polynomial, Polynomials::LegendrePolynomial_t>::value,
                  "the wave path uses Legendre-Gauss nodes");

public:
    NDG_t(int N_max, size_t n_interpolation_points, CUstream_st* const& stream = nullptr)
        : N_max_(N_max), N_interpolation_points_(n_interpolation_points) {
        (void)stream;
        fill(NDG_TABLE_NODES, nodes_);
        fill(NDG_TABLE_WEIGHTS, weights_);
        fill(NDG_TABLE_BARYCENTRIC_WEIGHTS, barycentric_weights_);
        fill(NDG_TABLE_LAGRANGE_LEFT, lagrange_interpolant_left_);
        fill(NDG_TABLE_LAGRANGE_RIGHT, lagrange_interpolant_right_);
        fill(NDG_TABLE_LAGRANGE_DERIVATIVE_LEFT, lagrange_interpolant_derivative_left_);
        fill(NDG_TABLE_LAGRANGE_DERIVATIVE_RIGHT, lagrange_interpolant_derivative_right_);
        fill(NDG_TABLE_DERIVATIVE_MATRICES, derivative_matrices_);
        fill(NDG_TABLE_G_HAT_DERIVATIVE_MATRICES, g_hat_derivative_matrices_);
        fill(NDG_TABLE_DERIVATIVE_MATRICES_HAT, derivative_matrices_hat_);
        fill(NDG_TABLE_INTERPOLATION_MATRICES, interpolation_matrices_);
        fill(NDG_TABLE_POLYNOMIALS, polynomials_);
    }

    int N_max_;
    size_t N_interpolation_points_;
    std::vector<double> nodes_;
    std::vector<double> weights_;
    std::vector<double> barycentric_weights_;
    std::vector<double> lagrange_interpolant_left_;
    std::vector<double> lagrange_interpolant_right_;
    std::vector<double> lagrange_interpolant_derivative_left_;
    std::vector<double> lagrange_interpolant_derivative_right_;
    std::vector<double> derivative_matrices_;
    std::vector<double> g_hat_derivative_matrices_;
    std::vector<double> derivative_matrices_hat_;
    std::vector<double> interpolation_matrices_;
    std::vector<double> polynomials_;

private:
    void fill(ndg_table table, std::vector<double>& out) const {
        for (int N = 0; N <= N_max_; ++N) {
            int64_t count = 0;
            check(ndg_tables_compute(N_max_, static_cast<int64_t>(N_interpolation_points_), table, N, nullptr, 0, &count),
                  "ndg_tables_compute");
            const size_t at = out.size();
            out.resize(at + static_cast<size_t>(count));
            check(ndg_tables_compute(N_max_, static_cast<int64_t>(N_interpolation_points_), table, N, out.data() + at, count,
                                     &count),
                  "ndg_tables_compute");
        }
    }
};

}  // namespace Entities

namespace Helpers {

// DataWriter_t (include/helpers/DataWriter_t.h, src/helpers/DataWriter_t.cpp):
// creates the empty time series files; Mesh2D_t::write_data and
// write_complete_data add output times.
class DataWriter_t {
public:
    explicit DataWriter_t(const std::filesystem::path& output_filename) {
        check(ndg_writer_create(output_filename.string().c_str(), &w_), "ndg_writer_create");
    }
    DataWriter_t(const DataWriter_t&) = delete;
    DataWriter_t& operator=(const DataWriter_t&) = delete;
    ~DataWriter_t() {
        if (w_) ndg_writer_destroy(w_);
    }
    ndg_writer* handle() const noexcept { return w_; }

private:
    ndg_writer* w_ = nullptr;
};

}  // namespace Helpers

namespace Meshes {

// Mesh2D_t (include/meshes/Mesh2D_t.cuh:23-182): the mesh, its fields and
// the device state of one solver, on one GPU.
class Mesh2D_t {
public:
    // The reference's constructor (include/meshes/Mesh2D_t.cuh:25). The mesh
    // file is .su2 (read_su2); load balancing has nothing to do on one GPU,
    // so load_balancing_interval, load_balancing_threshold and
    // worker_weights are kept for the signature only. polynomial_nodes are
    // NDG_t::nodes_ (the library uses its own copy of the same table).
    Mesh2D_t(std::filesystem::path filename, int initial_N, int maximum_N, size_t n_interpolation_points,
             int max_split_level, size_t adaptivity_interval, size_t load_balancing_interval, double tolerance_min,
             double tolerance_max, double load_balancing_threshold, const std::vector<double>& polynomial_nodes,
             std::vector<double> worker_weights, CUstream_st* const& stream, int device = 0)
        : Mesh2D_t(device, stream) {
        (void)load_balancing_threshold;
        (void)polynomial_nodes;
        (void)worker_weights;
        const ndg_mesh_params p = params(initial_N, maximum_N, n_interpolation_points, max_split_level,
                                         adaptivity_interval, tolerance_min, tolerance_max);
        check(ndg_mesh_load_file(ctx_, filename.string().c_str(), &p, 1), "ndg_mesh_load_file");
        load_balancing_interval_ = load_balancing_interval;
        finish_load(p, 1);
    }

    // The same from a zone in memory: what read_cgns reads from a CGNS file
    // (src/meshes/Mesh2D_t.cpp:422-645), with n_instances independent
    // solutions sharing the mesh.
    Mesh2D_t(const ndg_zone& zone, int initial_N, int maximum_N, size_t n_interpolation_points, int max_split_level,
             size_t adaptivity_interval, double tolerance_min, double tolerance_max, int n_instances = 1,
             int device = 0, CUstream_st* stream = nullptr)
        : Mesh2D_t(device, stream) {
        const ndg_mesh_params p = params(initial_N, maximum_N, n_interpolation_points, max_split_level,
                                         adaptivity_interval, tolerance_min, tolerance_max);
        check(ndg_mesh_load_zone(ctx_, &zone, &p, n_instances), "ndg_mesh_load_zone");
        finish_load(p, n_instances);
    }

    Mesh2D_t(const Mesh2D_t&) = delete;
    Mesh2D_t& operator=(const Mesh2D_t&) = delete;
    Mesh2D_t(Mesh2D_t&& other) noexcept { *this = std::move(other); }
    Mesh2D_t& operator=(Mesh2D_t&& other) noexcept {
        std::swap(ctx_, other.ctx_);
        initial_N_ = other.initial_N_;
        maximum_N_ = other.maximum_N_;
        n_elements_ = other.n_elements_;
        n_elements_total_ = other.n_elements_total_;
        n_faces_ = other.n_faces_;
        n_nodes_ = other.n_nodes_;
        n_instances_ = other.n_instances_;
        field_size_ = other.field_size_;
        adaptivity_interval_ = other.adaptivity_interval_;
        load_balancing_interval_ = other.load_balancing_interval_;
        n_interpolation_points_ = other.n_interpolation_points_;
        tolerance_min_ = other.tolerance_min_;
        tolerance_max_ = other.tolerance_max_;
        return *this;
    }
    ~Mesh2D_t() {
        if (ctx_) ndg_ctx_destroy(ctx_);
    }

    int initial_N_ = 0;
    int maximum_N_ = 0;
    size_t n_elements_ = 0;        // domain elements
    size_t n_elements_total_ = 0;  // domain and ghost elements
    size_t n_faces_ = 0;
    size_t n_nodes_ = 0;
    int n_instances_ = 1;
    size_t field_size_ = 0;  // values per field and instance: sum of (N+1)^2
    size_t adaptivity_interval_ = 0;
    size_t load_balancing_interval_ = 0;
    size_t n_interpolation_points_ = 0;
    double tolerance_min_ = 0.0;
    double tolerance_max_ = 0.0;

    // Mesh2D_t::initial_conditions (src/meshes/Mesh2D_t.cu:5030): the
    // reference plane wave in every instance.
    void initial_conditions(const std::vector<double>& polynomial_nodes = {}) {
        (void)polynomial_nodes;
        check(ndg_initial_conditions(ctx_), "ndg_initial_conditions");
    }

    // Mesh2D_t::estimate_error (src/meshes/Mesh2D_t.cu:5158).
    void estimate_error(const std::vector<double>& polynomials = {}) {
        (void)polynomials;
        check(ndg_estimate_error(ctx_), "ndg_estimate_error");
    }

    // Mesh2D_t::adapt(N_max, polynomial_nodes, barycentric_weights)
    // (src/meshes/Mesh2D_t.cpp:1644-2268) from the last error estimate.
    void adapt(int N_max = 0, const std::vector<double>& polynomial_nodes = {}, const std::vector<double>& barycentric_weights = {}) {
        (void)N_max;
        (void)polynomial_nodes;
        (void)barycentric_weights;
        check(ndg_adapt(ctx_), "ndg_adapt");
        refresh_counts();
    }

    // Library-side tuning (no counterpart in the reference): the autotuner
    // of the uniform stage kernel's tile (returns the tile kept, 0 = the
    // default), the launch structure of mixed-order stages (0 one launch per
    // order group, 1 one launch over the queue of every group's tiles), and
    // the last adaptation's host wall time by phase (ms: device decisions,
    // topology rebuild, field transfer, device plan).
    int autotune(int n_launches = 20) {
        int32_t tile = 0;
        double ms = 0.0;
        check(ndg_autotune(ctx_, n_launches, &tile, &ms), "ndg_autotune");
        return tile;
    }
    void set_mixed_launch(int mode) { check(ndg_set_mixed_launch(ctx_, mode), "ndg_set_mixed_launch"); }
    std::array<double, 4> adapt_timings() const {
        std::array<double, 4> ms{};
        check(ndg_adapt_timings(ctx_, ms.data()), "ndg_adapt_timings");
        return ms;
    }

    // Fields of one instance (instance < 0: all instances back to back), in
    // the reference's element order and node layout.
    std::vector<double> get_field(ndg_field field, int instance = 0) const {
        std::vector<double> out(field_size_ * static_cast<size_t>(instance < 0 ? n_instances_ : 1));
        check(ndg_get_field(ctx_, instance, field, out.data()), "ndg_get_field");
        return out;
    }
    void set_field(ndg_field field, const std::vector<double>& values, int instance = 0) {
        const size_t want = field_size_ * static_cast<size_t>(instance < 0 ? n_instances_ : 1);
        if (values.size() != want) throw Error(NDG_ERR_INVALID_ARG, "set_field: wrong number of values");
        check(ndg_set_field(ctx_, instance, field, values.data()), "ndg_set_field");
    }

    // Per element: p_error_, p_sigma_, refine_, coarsen_ of the last estimate.
    struct ErrorEstimate {
        std::vector<double> p_error, p_sigma;
        std::vector<int32_t> refine, coarsen;
    };
    ErrorEstimate get_error(int instance = 0) const {
        ErrorEstimate e{std::vector<double>(n_elements_), std::vector<double>(n_elements_),
                        std::vector<int32_t>(n_elements_), std::vector<int32_t>(n_elements_)};
        check(ndg_get_error(ctx_, instance, e.p_error.data(), e.p_sigma.data(), e.refine.data(), e.coarsen.data()),
              "ndg_get_error");
        return e;
    }

    // Element orders N_ and minimum lengths delta_xy_min_, domain and ghosts.
    std::vector<int32_t> element_orders() const {
        std::vector<int32_t> N(n_elements_total_);
        check(ndg_mesh_get_elements(ctx_, nullptr, N.data(), nullptr, nullptr), "ndg_mesh_get_elements");
        return N;
    }

    // Mesh2D_t::get_solution / get_complete_solution (src/meshes/Mesh2D_t.cpp:4237-4296):
    // the arrays of ndg_get_solution, n_elements_ n_interpolation_points^2
    // values each; the derivatives only when the mesh keeps them.
    struct Solution {
        std::vector<double> x, y, p, u, v, dp_dt, du_dt, dv_dt, p_analytical_error, u_analytical_error, v_analytical_error;
    };
    Solution get_solution(double time = 0.0, bool complete = false, bool with_derivative = false, int instance = 0) const {
        const size_t n = n_elements_ * n_interpolation_points_ * n_interpolation_points_;
        Solution s;
        ndg_solution_output o{};
        for (auto* v : {&s.x, &s.y, &s.p, &s.u, &s.v}) v->resize(n);
        o.x = s.x.data(), o.y = s.y.data(), o.p = s.p.data(), o.u = s.u.data(), o.v = s.v.data();
        if (complete) {
            for (auto* v : {&s.p_analytical_error, &s.u_analytical_error, &s.v_analytical_error}) v->resize(n);
            o.p_analytical_error = s.p_analytical_error.data();
            o.u_analytical_error = s.u_analytical_error.data();
            o.v_analytical_error = s.v_analytical_error.data();
            if (with_derivative) {
                for (auto* v : {&s.dp_dt, &s.du_dt, &s.dv_dt}) v->resize(n);
                o.dp_dt = s.dp_dt.data(), o.du_dt = s.du_dt.data(), o.dv_dt = s.dv_dt.data();
            }
        }
        check(ndg_get_solution(ctx_, instance, time, &o), "ndg_get_solution");
        return s;
    }

    // Mesh2D_t::write_data / write_complete_data (src/meshes/Mesh2D_t.cpp:1601-1642).
    void write_data(double time, const Helpers::DataWriter_t& data_writer, int instance = 0) const {
        check(ndg_writer_write(data_writer.handle(), ctx_, instance, time, 0), "ndg_writer_write");
    }
    void write_complete_data(double time, const Helpers::DataWriter_t& data_writer, int instance = 0) const {
        check(ndg_writer_write(data_writer.handle(), ctx_, instance, time, 1), "ndg_writer_write");
    }

    void synchronize() const { check(ndg_ctx_synchronize(ctx_), "ndg_ctx_synchronize"); }

    ndg_ctx* handle() const noexcept { return ctx_; }
    // Re-reads the counts after a call that may adapt the mesh.
    void refresh() { refresh_counts(); }

private:
    Mesh2D_t(int device, CUstream_st* stream) {
        check(ndg_ctx_create(device, static_cast<void*>(stream), &ctx_), "ndg_ctx_create");
    }

    static ndg_mesh_params params(int initial_N, int maximum_N, size_t n_interpolation_points, int max_split_level,
                                  size_t adaptivity_interval, double tolerance_min, double tolerance_max) {
        ndg_mesh_params p{};
        p.initial_N = initial_N;
        p.maximum_N = maximum_N;
        p.n_interpolation_points = static_cast<int64_t>(n_interpolation_points);
        p.max_split_level = max_split_level;
        p.adaptivity_interval = static_cast<int64_t>(adaptivity_interval);
        p.tolerance_min = tolerance_min;
        p.tolerance_max = tolerance_max;
        p.cfl = 0.5;  // replaced by Solver2D_t's CFL before stepping
        return p;
    }

    void refresh_counts() {
        int64_t K = 0, total = 0, faces = 0, nodes = 0, size = 0;
        check(ndg_mesh_counts(ctx_, &K, &total, &faces, &nodes), "ndg_mesh_counts");
        check(ndg_mesh_field_size(ctx_, &size), "ndg_mesh_field_size");
        n_elements_ = static_cast<size_t>(K);
        n_elements_total_ = static_cast<size_t>(total);
        n_faces_ = static_cast<size_t>(faces);
        n_nodes_ = static_cast<size_t>(nodes);
        field_size_ = static_cast<size_t>(size);
    }

    void finish_load(const ndg_mesh_params& p, int n_instances) {
        refresh_counts();
        initial_N_ = p.initial_N;
        maximum_N_ = p.maximum_N;
        n_instances_ = n_instances;
        adaptivity_interval_ = static_cast<size_t>(p.adaptivity_interval);
        n_interpolation_points_ = static_cast<size_t>(p.n_interpolation_points);
        tolerance_min_ = p.tolerance_min;
        tolerance_max_ = p.tolerance_max;
    }

    ndg_ctx* ctx_ = nullptr;
};

}  // namespace Meshes

namespace Solvers {

// Solver2D_t(CFL, output_times, viscosity) (include/solvers/Solver2D_t.cuh:14-65).
class Solver2D_t {
public:
    // Called at every output time with the time and the mesh, after the
    // error estimate, where the reference calls write_complete_data.
    using Output = std::function<void(double time, Meshes::Mesh2D_t& mesh)>;

    Solver2D_t(double CFL, std::vector<double> output_times, double viscosity)
        : CFL_(CFL), viscosity_(viscosity), output_times_(std::move(output_times)) {}

    double CFL_;
    double viscosity_;
    std::vector<double> output_times_;

    // Solver2D_t::get_delta_t (src/solvers/Solver2D_t.cu:17-31): min over
    // elements of CFL delta_xy_min / N^2.
    double get_delta_t(Meshes::Mesh2D_t& mesh) const {
        check(ndg_set_cfl(mesh.handle(), CFL_), "ndg_set_cfl");
        double dt = 0.0;
        check(ndg_get_delta_t(mesh.handle(), &dt), "ndg_get_delta_t");
        return dt;
    }

    // Solver2D_t::solve (include/solvers/Solver2D_t.tcu:7-135): RK3 steps
    // from time 0 to output_times_.back(), the last one shortened to land
    // on it. Outputs come where the reference writes them: at the start if
    // time 0 is an output time, then after the first step whose end time t
    // satisfies e <= t < e + dt for an output time e, and at the end if no
    // output fell on the last step. With adaptivity_interval_ > 0 the error
    // is estimated and the mesh adapted after every adaptivity_interval_-th
    // step, and the step size follows the new mesh. Returns the number of
    // steps.
    template <typename Polynomial>
    size_t solve(const Entities::NDG_t<Polynomial>& NDG, Meshes::Mesh2D_t& mesh, const Output& output = {}) const {
        (void)NDG;
        if (output_times_.empty()) throw Error(NDG_ERR_INVALID_ARG, "solve: no output times");
        const double t_end = output_times_.back();
        double dt_mesh = get_delta_t(mesh);
        double time = 0.0;
        for (double e : output_times_)
            if (time >= e && time < e + dt_mesh && output) output(time, mesh);

        // The reference's steps; full steps between outputs and adaptations
        // run in one call each, the shortened last step as three stages.
        size_t steps = 0;
        int64_t pending = 0;
        double t_run = 0.0;
        bool wrote_last = false;
        auto flush = [&] {
            if (pending) check(ndg_run(mesh.handle(), pending, &t_run), "ndg_run");
            pending = 0;
        };
        while (time < t_end) {
            double dt = dt_mesh;
            const bool last = time + dt > t_end;
            if (last) dt = t_end - time;
            if (last) {
                flush();
                for (int m = 0; m < 3; ++m) check(ndg_stage(mesh.handle(), m, time, dt), "ndg_stage");
                t_run = time + dt;
            } else {
                ++pending;
            }
            time += dt;
            ++steps;
            bool write = false;
            for (double e : output_times_)
                if (time >= e && time < e + dt) {
                    write = true;
                    break;
                }
            wrote_last = write;
            if (write) {
                flush();
                mesh.estimate_error();
                if (output) output(time, mesh);
            }
            if (mesh.adaptivity_interval_ > 0 && steps % mesh.adaptivity_interval_ == 0) {
                flush();
                mesh.estimate_error();
                mesh.adapt();
                check(ndg_get_delta_t(mesh.handle(), &dt_mesh), "ndg_get_delta_t");
            }
        }
        flush();
        if (!wrote_last) {
            mesh.estimate_error();
            if (output) output(time, mesh);
        }
        return steps;
    }

    // The reference's signature: write_complete_data to data_writer at the output times.
    template <typename Polynomial>
    size_t solve(const Entities::NDG_t<Polynomial>& NDG, Meshes::Mesh2D_t& mesh, const Helpers::DataWriter_t& data_writer) const {
        return solve(NDG, mesh, Output([&data_writer](double time, Meshes::Mesh2D_t& m) { m.write_complete_data(time, data_writer); }));
    }

    // Solver2D_t::pre_condition and pre_condition_iterative
    // (include/solvers/Solver2D_t.tpp:136-334) at this solver's CFL.
    // Returns the number of steps.
    template <typename Polynomial>
    size_t pre_condition(const Entities::NDG_t<Polynomial>& NDG, Meshes::Mesh2D_t& mesh, size_t n_adaptivity_steps, size_t pre_condition_interval) const {
        return pre_condition_run(NDG, mesh, n_adaptivity_steps, pre_condition_interval, 0);
    }
    template <typename Polynomial>
    size_t pre_condition_iterative(const Entities::NDG_t<Polynomial>& NDG, Meshes::Mesh2D_t& mesh, size_t n_adaptivity_steps, size_t pre_condition_interval) const {
        return pre_condition_run(NDG, mesh, n_adaptivity_steps, pre_condition_interval, 1);
    }

private:
    template <typename Polynomial>
    size_t pre_condition_run(const Entities::NDG_t<Polynomial>& NDG, Meshes::Mesh2D_t& mesh, size_t n, size_t interval, int iterative) const {
        (void)NDG;
        (void)get_delta_t(mesh);  // sets the CFL
        int64_t steps = 0;
        check(ndg_pre_condition(mesh.handle(), static_cast<int64_t>(n), static_cast<int64_t>(interval), iterative, &steps), "ndg_pre_condition");
        mesh.refresh();
        return static_cast<size_t>(steps);
    }
};

}  // namespace Solvers
}  // namespace ndg_b200

#endif
