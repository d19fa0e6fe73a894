// C ABI of the output interpolation (ndg_get_solution) and of the L2 error
// against the plane wave (ndg_l2_error): gathers the per element orders,
// value offsets and corners and the orders' tables, runs the kernels of
// output.cu on the context's stream and copies the results to the caller.
#include "context.hpp"
#include "output.cuh"

#include <array>
#include <cmath>
#include <cstdint>
#include <vector>

using namespace ndg;

namespace {

// Per domain element: order, first value within a field block, corners
// (x0, y0, ..., x3, y3). Returns the largest order.
int gather_elements(const ndg_ctx* ctx, std::vector<int32_t>& N, std::vector<int64_t>& off2, std::vector<double>& corners) {
    const Topology& t = ctx->topo;
    const int64_t K = t.n_domain;
    N.resize(static_cast<size_t>(K));
    off2.resize(static_cast<size_t>(K));
    corners.resize(static_cast<size_t>(8 * K));
    int64_t o = 0;
    int max_N = 0;
    for (int64_t e = 0; e < K; ++e) {
        const size_t se = static_cast<size_t>(e);
        N[se] = t.elem_N[se];
        off2[se] = o;
        o += static_cast<int64_t>(N[se] + 1) * (N[se] + 1);
        max_N = std::max(max_N, N[se]);
        for (int v = 0; v < 4; ++v) {
            const size_t node = static_cast<size_t>(t.elem_nodes[se][static_cast<size_t>(v)]);
            corners[8 * se + 2 * static_cast<size_t>(v)] = t.node_x[node];
            corners[8 * se + 2 * static_cast<size_t>(v) + 1] = t.node_y[node];
        }
    }
    return max_N;
}

}  // namespace

extern "C" {

ndg_status ndg_get_solution(ndg_ctx* ctx, int32_t instance, double time, const ndg_solution_output* out) {
    return guarded([&] {
        require_mesh(ctx);
        require_device(ctx);
        if (!out) fail(NDG_ERR_INVALID_ARG, "out is NULL");
        if (instance < 0 || instance >= ctx->n_instances) fail(NDG_ERR_INVALID_ARG, "instance out of range");
        const int64_t P = ctx->params.n_interpolation_points;
        if (P < 2) fail(NDG_ERR_INVALID_ARG, "output needs n_interpolation_points >= 2");
        const bool want_d = out->dp_dt || out->du_dt || out->dv_dt;
        if (want_d && !ctx->keep_derivative) fail(NDG_ERR_INVALID_ARG, "time derivative output needs ndg_ctx_keep_derivative(ctx, 1) before stepping");
        if (!ctx->has_tables || ctx->tables.n_interp != P) {
            // the interpolation matrices depend on the point count; the other tables do not
            ctx->tables = build_tables(std::max(ctx->has_tables ? ctx->tables.N_max : 0, ctx->params.maximum_N), P);
            ctx->has_tables = true;
        }
        make_current(ctx);

        const int64_t K = ctx->topo.n_domain;
        std::vector<int32_t> N;
        std::vector<int64_t> off2;
        std::vector<double> corners;
        const int max_N = gather_elements(ctx, N, off2, corners);
        if (max_N > ctx->tables.N_max) fail(NDG_ERR_INVALID_ARG, "element order above the tables' N_max");
        std::vector<double> interp, nodes;
        std::vector<int64_t> interp_off(static_cast<size_t>(max_N + 1)), nodes_off(static_cast<size_t>(max_N + 1));
        for (int n = 0; n <= max_N; ++n) {
            interp_off[static_cast<size_t>(n)] = static_cast<int64_t>(interp.size());
            nodes_off[static_cast<size_t>(n)] = static_cast<int64_t>(nodes.size());
            const auto& I = ctx->tables.get(NDG_TABLE_INTERPOLATION_MATRICES, n);
            const auto& x = ctx->tables.get(NDG_TABLE_NODES, n);
            interp.insert(interp.end(), I.begin(), I.end());
            nodes.insert(nodes.end(), x.begin(), x.end());
        }

        DeviceBuffer<int32_t> dN;
        DeviceBuffer<int64_t> doff2, dioff, dnoff;
        DeviceBuffer<double> dcorners, dinterp, dnodes;
        dN.upload(N, ctx->stream);
        doff2.upload(off2, ctx->stream);
        dcorners.upload(corners, ctx->stream);
        dinterp.upload(interp, ctx->stream);
        dnodes.upload(nodes, ctx->stream);
        dioff.upload(interp_off, ctx->stream);
        dnoff.upload(nodes_off, ctx->stream);

        double* host[11] = {out->x, out->y, out->p, out->u, out->v, out->dp_dt, out->du_dt, out->dv_dt,
                            out->p_analytical_error, out->u_analytical_error, out->v_analytical_error};
        std::array<DeviceBuffer<double>, 11> dev_out;
        const size_t count = static_cast<size_t>(K * P * P);
        double* d[11] = {};
        for (int i = 0; i < 11; ++i)
            if (host[i] && count) {
                dev_out[static_cast<size_t>(i)].allocate(count);
                d[i] = dev_out[static_cast<size_t>(i)].ptr;
            }

        dev::OutputArgs a{};
        const int64_t per_inst = 3 * ctx->block;
        a.q = ctx->q.ptr + instance * per_inst;
        a.G = ctx->keep_derivative ? ctx->G.ptr + instance * per_inst : nullptr;
        a.block = ctx->block;
        a.N = dN.ptr;
        a.off2 = doff2.ptr;
        a.corners = dcorners.ptr;
        a.interp = dinterp.ptr;
        a.interp_off = dioff.ptr;
        a.nodes = dnodes.ptr;
        a.nodes_off = dnoff.ptr;
        a.K = K;
        a.n_interp = static_cast<int>(P);
        a.time = time;
        a.x = d[0], a.y = d[1], a.p = d[2], a.u = d[3], a.v = d[4];
        a.dp_dt = d[5], a.du_dt = d[6], a.dv_dt = d[7];
        a.p_err = d[8], a.u_err = d[9], a.v_err = d[10];
        check_cuda(dev::launch_output(a, max_N, ctx->stream), "output kernel launch");
        ++ctx->launches;
        for (int i = 0; i < 11; ++i)
            if (host[i] && count)
                check_cuda(cudaMemcpyAsync(host[i], d[i], count * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream), "output download");
        check_cuda(cudaStreamSynchronize(ctx->stream), "output");
    });
}

ndg_status ndg_l2_error(ndg_ctx* ctx, int32_t instance, double time, double* l2) {
    return guarded([&] {
        require_mesh(ctx);
        require_device(ctx);
        if (!l2) fail(NDG_ERR_INVALID_ARG, "l2 is NULL");
        if (instance < 0 || instance >= ctx->n_instances) fail(NDG_ERR_INVALID_ARG, "instance out of range");
        make_current(ctx);
        const int64_t K = ctx->topo.n_domain;
        std::vector<int32_t> N;
        std::vector<int64_t> off2;
        std::vector<double> corners;
        const int max_N = gather_elements(ctx, N, off2, corners);
        if (max_N > ctx->tables.N_max) fail(NDG_ERR_INVALID_ARG, "element order above the tables' N_max");
        std::vector<double> nodes, weights;
        std::vector<int64_t> vec_off(static_cast<size_t>(max_N + 1));
        for (int n = 0; n <= max_N; ++n) {
            vec_off[static_cast<size_t>(n)] = static_cast<int64_t>(nodes.size());
            const auto& x = ctx->tables.get(NDG_TABLE_NODES, n);
            const auto& w = ctx->tables.get(NDG_TABLE_WEIGHTS, n);
            nodes.insert(nodes.end(), x.begin(), x.end());
            weights.insert(weights.end(), w.begin(), w.end());
        }
        DeviceBuffer<int32_t> dN;
        DeviceBuffer<int64_t> doff2, dvoff;
        DeviceBuffer<double> dcorners, dnodes, dweights, dpartial;
        dN.upload(N, ctx->stream);
        doff2.upload(off2, ctx->stream);
        dcorners.upload(corners, ctx->stream);
        dnodes.upload(nodes, ctx->stream);
        dweights.upload(weights, ctx->stream);
        dvoff.upload(vec_off, ctx->stream);
        dpartial.allocate(static_cast<size_t>(std::max<int64_t>(3 * K, 1)));
        dev::L2Args a{};
        a.q = ctx->q.ptr + instance * 3 * ctx->block;
        a.block = ctx->block;
        a.N = dN.ptr;
        a.off2 = doff2.ptr;
        a.corners = dcorners.ptr;
        a.nodes = dnodes.ptr;
        a.weights = dweights.ptr;
        a.vec_off = dvoff.ptr;
        a.K = K;
        a.time = time;
        a.partial = dpartial.ptr;
        check_cuda(dev::launch_l2_error(a, ctx->stream), "l2 error kernel launch");
        ++ctx->launches;
        std::vector<double> partial(static_cast<size_t>(3 * K));
        if (K) check_cuda(cudaMemcpyAsync(partial.data(), dpartial.ptr, partial.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream), "l2 download");
        check_cuda(cudaStreamSynchronize(ctx->stream), "l2");
        double sum[3] = {0.0, 0.0, 0.0};
        for (int64_t e = 0; e < K; ++e)
            for (int f = 0; f < 3; ++f) sum[f] += partial[static_cast<size_t>(3 * e + f)];
        for (int f = 0; f < 3; ++f) l2[f] = std::sqrt(sum[f]);
    });
}

ndg_status ndg_writer_write(ndg_writer* writer, ndg_ctx* ctx, int32_t instance, double time, int32_t complete) {
    if (!writer || !ctx) {
        set_last_error("NULL argument");
        return NDG_ERR_INVALID_ARG;
    }
    std::vector<double> pts[11];
    std::vector<int32_t> N, split, status, rotation, refine, coarsen;
    std::vector<double> p_error, p_sigma;
    int64_t K = 0, P = 0;
    const ndg_status st = guarded([&] {
        require_mesh(ctx);
        K = ctx->topo.n_domain;
        P = ctx->params.n_interpolation_points;
        if (P < 2) fail(NDG_ERR_INVALID_ARG, "output needs n_interpolation_points >= 2");
        const size_t count = static_cast<size_t>(K * P * P);
        const int n_arrays = complete ? 11 : 5;
        for (int i = 0; i < n_arrays; ++i)
            if (i < 5 || i >= 8 || ctx->keep_derivative) pts[i].assign(count, 0.0);
        ndg_solution_output o{};
        double** dst[11] = {&o.x, &o.y, &o.p, &o.u, &o.v, &o.dp_dt, &o.du_dt, &o.dv_dt, &o.p_analytical_error, &o.u_analytical_error, &o.v_analytical_error};
        for (int i = 0; i < 11; ++i) *dst[i] = pts[i].empty() ? nullptr : pts[i].data();
        const ndg_status s = ndg_get_solution(ctx, instance, time, &o);
        if (s != NDG_OK) fail(s, ndg_last_error());
        if (complete) {
            const size_t Kt = ctx->topo.elem_N.size();
            N.assign(ctx->topo.elem_N.begin(), ctx->topo.elem_N.begin() + static_cast<std::ptrdiff_t>(K));
            split.assign(Kt, 0);
            status.assign(Kt, 0);
            rotation.assign(Kt, 0);
            ndg_status s2 = ndg_mesh_get_element_state(ctx, split.data(), status.data(), rotation.data(), nullptr);
            if (s2 != NDG_OK) fail(s2, ndg_last_error());
            if (ctx->has_error_estimate) {
                p_error.assign(static_cast<size_t>(K), 0.0);
                p_sigma.assign(static_cast<size_t>(K), 0.0);
                refine.assign(static_cast<size_t>(K), 0);
                coarsen.assign(static_cast<size_t>(K), 0);
                s2 = ndg_get_error(ctx, instance, p_error.data(), p_sigma.data(), refine.data(), coarsen.data());
                if (s2 != NDG_OK) fail(s2, ndg_last_error());
            }
        }
    });
    if (st != NDG_OK) return st;
    ndg_output_arrays a{};
    a.complete = complete ? 1 : 0;
    a.x = pts[0].data(), a.y = pts[1].data(), a.p = pts[2].data(), a.u = pts[3].data(), a.v = pts[4].data();
    auto opt = [](const std::vector<double>& v) { return v.empty() ? nullptr : v.data(); };
    auto opti = [](const std::vector<int32_t>& v) { return v.empty() ? nullptr : v.data(); };
    a.dp_dt = opt(pts[5]), a.du_dt = opt(pts[6]), a.dv_dt = opt(pts[7]);
    a.p_analytical_error = opt(pts[8]), a.u_analytical_error = opt(pts[9]), a.v_analytical_error = opt(pts[10]);
    a.N = opti(N), a.status = opti(status), a.rotation = opti(rotation), a.split_level = opti(split);
    a.rank = 0;
    a.p_error = opt(p_error), a.p_sigma = opt(p_sigma), a.refine = opti(refine), a.coarsen = opti(coarsen);
    return ndg_writer_write_arrays(writer, time, K, P, &a);
}

}  // extern "C"
