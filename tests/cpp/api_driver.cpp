// Drives the C++ host API (include/ndg_b200.hpp) the way the reference's
// src/main.cu:346-390 drives SEM::Device: NDG_t, Mesh2D_t from a mesh file,
// initial conditions, Solver2D_t::solve with outputs.
//
//   api_driver host  <mesh.su2> <N>                        tables and counts as JSON (no GPU)
//   api_driver solve <mesh.su2> <N> <CFL> <out.bin> <t_1> ... <t_end>
//   api_driver write <mesh.su2> <N> <CFL> <output.pvtu> <n_adapt> <interval> <t_1> ... <t_end>
//       pre_condition (n_adapt adaptations every interval steps, N_max = N + 4,
//       one split level) then solve with a DataWriter_t; prints the steps of both as JSON
//
// solve writes, little-endian: int64 steps, int64 outputs, int64 field_size,
// double dt, then per output: double time and the p, u, v fields.
#include "ndg_b200.hpp"

#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

namespace {

void print_array(const char* name, const std::vector<double>& v, bool last = false) {
    std::printf("\"%s\": [", name);
    for (size_t i = 0; i < v.size(); ++i) std::printf(i ? ", %.17g" : "%.17g", v[i]);
    std::printf("]%s", last ? "" : ", ");
}

int host_mode(const std::string& path, int N) {
    ndg_b200::Entities::NDG_t<> NDG(N, 2);
    ndg_b200::Meshes::Mesh2D_t mesh(path, N, N, 2, 0, 0, 0, 1e-6, 1e-14, 0.0, NDG.nodes_, {}, nullptr, -1);
    std::printf("{\"n_elements\": %zu, \"n_elements_total\": %zu, \"n_faces\": %zu, \"n_nodes\": %zu, \"field_size\": %zu, ",
                mesh.n_elements_, mesh.n_elements_total_, mesh.n_faces_, mesh.n_nodes_, mesh.field_size_);
    print_array("nodes", NDG.nodes_);
    print_array("weights", NDG.weights_);
    print_array("derivative_matrices_hat", NDG.derivative_matrices_hat_);
    print_array("interpolation_matrices", NDG.interpolation_matrices_);
    print_array("polynomials", NDG.polynomials_, true);
    std::printf("}\n");
    return 0;
}

int solve_mode(const std::string& path, int N, double CFL, const std::string& out, std::vector<double> times) {
    ndg_b200::Entities::NDG_t<> NDG(N, 2);
    ndg_b200::Meshes::Mesh2D_t mesh(path, N, N, 2, 0, 0, 0, 1e-6, 1e-14, 0.0, NDG.nodes_, {}, nullptr, 0);
    mesh.initial_conditions(NDG.nodes_);
    ndg_b200::Solvers::Solver2D_t solver(CFL, times, 0.0);
    struct Snapshot {
        double time;
        std::vector<double> p, u, v;
    };
    std::vector<Snapshot> outputs;
    const size_t steps = solver.solve(NDG, mesh, [&](double t, ndg_b200::Meshes::Mesh2D_t& m) {
        outputs.push_back({t, m.get_field(NDG_FIELD_P), m.get_field(NDG_FIELD_U), m.get_field(NDG_FIELD_V)});
    });
    const double dt = solver.get_delta_t(mesh);
    FILE* f = std::fopen(out.c_str(), "wb");
    if (!f) return 2;
    const int64_t header[3] = {static_cast<int64_t>(steps), static_cast<int64_t>(outputs.size()),
                               static_cast<int64_t>(mesh.field_size_)};
    std::fwrite(header, sizeof(int64_t), 3, f);
    std::fwrite(&dt, sizeof(double), 1, f);
    for (const auto& s : outputs) {
        std::fwrite(&s.time, sizeof(double), 1, f);
        std::fwrite(s.p.data(), sizeof(double), s.p.size(), f);
        std::fwrite(s.u.data(), sizeof(double), s.u.size(), f);
        std::fwrite(s.v.data(), sizeof(double), s.v.size(), f);
    }
    std::fclose(f);
    return 0;
}

int write_mode(const std::string& path, int N, double CFL, const std::string& output, size_t n_adapt, size_t interval,
               std::vector<double> times) {
    ndg_b200::Entities::NDG_t<> NDG(N + 4, 3);
    ndg_b200::Meshes::Mesh2D_t mesh(path, N, N + 4, 3, 1, 0, 0, 1e-6, 1e-14, 0.0, NDG.nodes_, {}, nullptr, 0);
    mesh.initial_conditions(NDG.nodes_);
    ndg_b200::Solvers::Solver2D_t solver(CFL, times, 0.0);
    const size_t pre = solver.pre_condition(NDG, mesh, n_adapt, interval);
    ndg_b200::Helpers::DataWriter_t writer(output);
    const size_t steps = solver.solve(NDG, mesh, writer);
    std::printf("{\"pre_condition_steps\": %zu, \"steps\": %zu, \"n_elements\": %zu}\n", pre, steps, mesh.n_elements_);
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    try {
        const std::string mode = argc > 1 ? argv[1] : "";
        if (mode == "host" && argc == 4) return host_mode(argv[2], std::atoi(argv[3]));
        if (mode == "solve" && argc >= 7) {
            std::vector<double> times;
            for (int i = 6; i < argc; ++i) times.push_back(std::strtod(argv[i], nullptr));
            return solve_mode(argv[2], std::atoi(argv[3]), std::strtod(argv[4], nullptr), argv[5], times);
        }
        if (mode == "write" && argc >= 9) {
            std::vector<double> times;
            for (int i = 8; i < argc; ++i) times.push_back(std::strtod(argv[i], nullptr));
            return write_mode(argv[2], std::atoi(argv[3]), std::strtod(argv[4], nullptr), argv[5],
                              static_cast<size_t>(std::atol(argv[6])), static_cast<size_t>(std::atol(argv[7])), times);
        }
        std::fprintf(stderr, "usage: api_driver host <mesh> <N> | solve <mesh> <N> <CFL> <out> <t_1> ... <t_end> | "
                             "write <mesh> <N> <CFL> <output> <n_adapt> <interval> <t_1> ... <t_end>\n");
        return 1;
    } catch (const ndg_b200::Error& e) {
        std::fprintf(stderr, "ndg_b200 error %d: %s\n", static_cast<int>(e.status()), e.what());
        return 3;
    }
}
