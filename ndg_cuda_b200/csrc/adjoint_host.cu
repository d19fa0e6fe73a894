// C ABI of the discrete adjoint (include/ndg_b200.h, ndg_adjoint_*): host
// orchestration of the variable-speed forward, its checkpoints, the
// recomputation of each checkpoint interval and the reverse sweep of the
// adjoint stages (adjoint_kernels.cu).
#include "adjoint.cuh"
#include "context.hpp"
#include "stage_kernels.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

struct ndg_adjoint {
    ndg_ctx* ctx = nullptr;
    int64_t mesh_version = 0;
    int N = 0;
    int64_t K = 0, Kp = 0, NN = 0, block = 0, field_size = 0;
    std::vector<double> speed;  // [K]
    std::vector<int64_t> rec_elem;
    std::vector<double> rec_xi, rec_w;
    ndg::DeviceBuffer<double> c, q, k, G, tr[2], atr[2], lq, lk, acc, ckpt, seg, d_rec_w, targets, samples, grad;
    // The backward recomputes interval j - 1 (on rstream, into seg2 or seg)
    // while the adjoint sweeps interval j (on the context's stream); qfinal
    // keeps the final state for the first adjoint stage.
    ndg::DeviceBuffer<double> seg2, qfinal;
    // The forward keeps its last interval's stage inputs in seg and its final
    // state in q; the first backward after it starts from them.
    bool last_kept = false;
    // streams of the adjoint sweep and of the recomputation, both joined to
    // the context's stream
    cudaStream_t rstream = nullptr, astream = nullptr;
    cudaEvent_t evr[2] = {nullptr, nullptr}, eva[2] = {nullptr, nullptr}, evs = nullptr;
    ndg::DeviceBuffer<float> tr_f[2], atr_f[2];  // traces of the FP32 form
    bool fp32 = false;
    ndg::dev::Receivers rec{};
    // the last forward
    bool has_forward = false;
    double dt = 0.0;
    int64_t n_steps = 0, interval = 0;
    double forward_ms = 0.0, backward_ms = 0.0;
    int64_t forward_launches = 0, backward_launches = 0;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    ~ndg_adjoint() {
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
        for (auto* e : {&evr[0], &evr[1], &eva[0], &eva[1], &evs})
            if (*e) cudaEventDestroy(*e);
        if (rstream) cudaStreamDestroy(rstream);
        if (astream) cudaStreamDestroy(astream);
    }
};

namespace ndg {
namespace {

constexpr int kAdjointMaxOrder = 12;

void require_valid(const ndg_adjoint* a) {
    if (!a) fail(NDG_ERR_INVALID_ARG, "adjoint handle is NULL");
    if (a->ctx->mesh_version != a->mesh_version) fail(NDG_ERR_INVALID_ARG, "the context's mesh changed since the adjoint problem was created");
}

// Lagrange basis of the Gauss nodes at t (barycentric form; exactly 1 at a
// node that t matches).
void lagrange_basis(const std::vector<double>& x, const std::vector<double>& bw, double t, double* out) {
    const size_t n = x.size();
    for (size_t i = 0; i < n; ++i)
        if (almost_equal(t, x[i])) {
            for (size_t j = 0; j < n; ++j) out[j] = (i == j) ? 1.0 : 0.0;
            return;
        }
    double s = 0.0;
    for (size_t i = 0; i < n; ++i) {
        out[i] = bw[i] / (t - x[i]);
        s += out[i];
    }
    for (size_t i = 0; i < n; ++i) out[i] /= s;
}

// Reference coordinates of (x, y) in a straight-sided quad (corners
// x0, y0, ..., x3, y3): Newton's method on the bilinear map. Returns false
// when the point lies outside.
bool locate(const double* cr, double x, double y, double& xi, double& eta) {
    const double xmin = std::min({cr[0], cr[2], cr[4], cr[6]}), xmax = std::max({cr[0], cr[2], cr[4], cr[6]});
    const double ymin = std::min({cr[1], cr[3], cr[5], cr[7]}), ymax = std::max({cr[1], cr[3], cr[5], cr[7]});
    const double tol = 1e-12 * std::max(xmax - xmin, ymax - ymin);
    if (x < xmin - tol || x > xmax + tol || y < ymin - tol || y > ymax + tol) return false;
    xi = 0.0;
    eta = 0.0;
    for (int it = 0; it < 50; ++it) {
        const double a0 = (1 - xi) * (1 - eta), a1 = (1 + xi) * (1 - eta), a2 = (1 + xi) * (1 + eta), a3 = (1 - xi) * (1 + eta);
        const double fx = 0.25 * (cr[0] * a0 + cr[2] * a1 + cr[4] * a2 + cr[6] * a3) - x;
        const double fy = 0.25 * (cr[1] * a0 + cr[3] * a1 + cr[5] * a2 + cr[7] * a3) - y;
        const double x_xi = 0.25 * ((1 - eta) * (cr[2] - cr[0]) + (1 + eta) * (cr[4] - cr[6]));
        const double y_xi = 0.25 * ((1 - eta) * (cr[3] - cr[1]) + (1 + eta) * (cr[5] - cr[7]));
        const double x_eta = 0.25 * ((1 - xi) * (cr[6] - cr[0]) + (1 + xi) * (cr[4] - cr[2]));
        const double y_eta = 0.25 * ((1 - xi) * (cr[7] - cr[1]) + (1 + xi) * (cr[5] - cr[3]));
        const double det = x_xi * y_eta - x_eta * y_xi;
        const double dxi = (fx * y_eta - fy * x_eta) / det, deta = (fy * x_xi - fx * y_xi) / det;
        xi -= dxi;
        eta -= deta;
        if (std::fabs(dxi) + std::fabs(deta) < 1e-15) break;
    }
    return std::fabs(xi) <= 1.0 + 1e-12 && std::fabs(eta) <= 1.0 + 1e-12;
}

// Zeroes the adjoint far traces of buffer i (both forms).
void zero_adjoint_traces(ndg_adjoint* a, int i) {
    check_cuda(cudaMemsetAsync(a->atr[i].ptr, 0, a->atr[i].count * sizeof(double), a->ctx->stream), "memset");
    check_cuda(cudaMemsetAsync(a->atr_f[i].ptr, 0, a->atr_f[i].count * sizeof(float), a->ctx->stream), "memset");
}

dev::SpeedStageArgs speed_args(ndg_adjoint* a, int m, int in, double dt) {
    ndg_ctx* c = a->ctx;
    dev::SpeedStageArgs s{};
    s.q = a->q.ptr;
    s.k = a->k.ptr;
    s.trace_in = a->tr[in].ptr;
    s.trace_out = a->tr[1 - in].ptr;
    s.trace_in_f = a->tr_f[in].ptr;
    s.trace_out_f = a->tr_f[1 - in].ptr;
    s.corners = c->corners.ptr;
    s.link = reinterpret_cast<const int2*>(c->link.ptr);
    s.normal = reinterpret_cast<const double2*>(c->normal.ptr);
    s.gscale = c->gscale.ptr;
    s.c = a->c.ptr;
    s.rk_a = kRkA[m];
    s.gdt = kRkG[m] * dt;
    s.first = m == 0;
    s.n_elements = a->K;
    s.field_stride = a->Kp;
    s.rec = a->rec;
    return s;
}

dev::AdjointStageArgs adjoint_args(ndg_adjoint* a, int in) {
    ndg_ctx* c = a->ctx;
    dev::AdjointStageArgs s{};
    s.lq = a->lq.ptr;
    s.lk = a->lk.ptr;
    s.atr_in = a->atr[in].ptr;
    s.atr_out = a->atr[1 - in].ptr;
    s.atr_in_f = a->atr_f[in].ptr;
    s.atr_out_f = a->atr_f[1 - in].ptr;
    s.acc = a->acc.ptr;
    s.corners = c->corners.ptr;
    s.link = reinterpret_cast<const int2*>(c->link.ptr);
    s.normal = reinterpret_cast<const double2*>(c->normal.ptr);
    s.gscale = c->gscale.ptr;
    s.c = a->c.ptr;
    s.n_elements = a->K;
    s.field_stride = a->Kp;
    s.rec = a->rec;
    return s;
}

void launch_traces_of_q(ndg_adjoint* a, int out, cudaStream_t stream = nullptr) {
    if (!stream) stream = a->ctx->stream;
    dev::TraceArgs t{};
    t.q = a->q.ptr;
    t.trace_out = a->tr[out].ptr;
    t.trace_out_f = a->tr_f[out].ptr;
    t.n_elements = a->K;
    t.field_stride = a->Kp;
    t.n_instances = 1;
    if (a->fp32)
        check_cuda(dev::launch_traces_f32(a->N, t, stream), "trace kernel launch");
    else
        check_cuda(dev::launch_traces(a->N, false, t, stream), "trace kernel launch");
}

// Waits for the context's stream and reports any launch or execution error.
void check_kernel_error(ndg_adjoint* a) {
    check_cuda(cudaStreamSynchronize(a->ctx->stream), "adjoint-module kernels");
    check_cuda(cudaGetLastError(), "adjoint-module kernels");
}

// Copies three host fields (field_size values each; NULL = zero) into a
// device state of three field blocks.
void upload_state(ndg_adjoint* a, double* dst, const double* const* fields) {
    cudaStream_t s = a->ctx->stream;
    check_cuda(cudaMemsetAsync(dst, 0, 3 * static_cast<size_t>(a->block) * sizeof(double), s), "memset");
    for (int f = 0; f < 3; ++f)
        if (fields[f])
            check_cuda(cudaMemcpyAsync(dst + f * a->block, fields[f], static_cast<size_t>(a->field_size) * sizeof(double), cudaMemcpyHostToDevice, s),
                       "state upload");
}

void download_field(ndg_adjoint* a, const double* src, double* out) {
    if (out) check_cuda(cudaMemcpyAsync(out, src, static_cast<size_t>(a->field_size) * sizeof(double), cudaMemcpyDeviceToHost, a->ctx->stream), "download");
}

// Runs forward steps first..last (1-based) from the state in q whose traces
// are in tr[in]; q_save (optional) receives each stage input (3 states per
// step), sample_rows (optional) the receivers' pressure after each step.
// Returns the trace buffer holding the final traces.
int run_forward(ndg_adjoint* a, int in, int64_t first, int64_t last, double* q_save, bool sample, int64_t save_every, int64_t& launches,
                cudaStream_t stream = nullptr) {
    if (!stream) stream = a->ctx->stream;
    const size_t state = 3 * static_cast<size_t>(a->block);
    for (int64_t step = first; step <= last; ++step) {
        for (int m = 0; m < 3; ++m) {
            dev::SpeedStageArgs s = speed_args(a, m, in, a->dt);
            if (q_save) s.q_save = q_save + (static_cast<size_t>(step - first) * 3 + static_cast<size_t>(m)) * state;
            if (save_every > 0 && m == 0 && (step - 1) % save_every == 0) s.q_save = a->ckpt.ptr + static_cast<size_t>((step - 1) / save_every) * state;
            if (sample && m == 2 && a->rec.n > 0) s.samples = a->samples.ptr + step * a->rec.n;
            check_cuda(dev::launch_speed_stage(a->N, a->fp32, s, stream), "speed stage launch");
            ++launches;
            in = 1 - in;
        }
    }
    return in;
}

}  // namespace
}  // namespace ndg

using namespace ndg;

extern "C" {

ndg_status ndg_adjoint_create(ndg_ctx* ctx, int32_t n_receivers, const double* receiver_xy, ndg_adjoint** out) {
    return guarded([&] {
        if (!ctx || !out) fail(NDG_ERR_INVALID_ARG, "NULL argument");
        require_mesh(ctx);
        require_device(ctx);
        if (n_receivers < 0 || n_receivers > dev::kMaxReceivers) fail(NDG_ERR_INVALID_ARG, "between 0 and 64 receivers");
        if (n_receivers > 0 && !receiver_xy) fail(NDG_ERR_INVALID_ARG, "receiver_xy is NULL");
        if (ctx->general || !fused_path_applies(ctx->topo)) fail(NDG_ERR_UNSUPPORTED, "the adjoint covers meshes of one order with conforming faces");
        if (!ctx->topo.boundary[kInflow].empty()) fail(NDG_ERR_UNSUPPORTED, "inflow boundaries make the step affine; the adjoint needs wall, symmetry, outflow or periodic sides");
        if (ctx->N < 1 || ctx->N > kAdjointMaxOrder) fail(NDG_ERR_UNSUPPORTED, "the adjoint kernels cover orders 1..12");
        make_current(ctx);
        auto a = std::make_unique<ndg_adjoint>();
        a->ctx = ctx;
        a->mesh_version = ctx->mesh_version;
        a->N = ctx->N;
        a->K = ctx->K;
        a->Kp = ctx->Kp;
        a->NN = static_cast<int64_t>(ctx->N + 1) * (ctx->N + 1);
        a->block = ctx->block;
        a->field_size = ctx->field_size;
        a->speed.assign(static_cast<size_t>(a->K), 1.0);
        // Receivers: the first element that contains the point.
        const int n = a->N + 1;
        const std::vector<double>& nodes = ctx->tables.get(NDG_TABLE_NODES, a->N);
        const std::vector<double>& bw = ctx->tables.get(NDG_TABLE_BARYCENTRIC_WEIGHTS, a->N);
        const Topology& t = ctx->topo;
        a->rec.n = n_receivers;
        a->rec_w.assign(static_cast<size_t>(std::max<int64_t>(n_receivers * a->NN, 1)), 0.0);
        for (int r = 0; r < n_receivers; ++r) {
            const double x = receiver_xy[2 * r], y = receiver_xy[2 * r + 1];
            int64_t found = -1;
            double xi = 0.0, eta = 0.0;
            for (int64_t e = 0; e < a->K && found < 0; ++e) {
                double cr[8];
                for (int v = 0; v < 4; ++v) {
                    const int64_t nd = t.elem_nodes[static_cast<size_t>(e)][static_cast<size_t>(v)];
                    cr[2 * v] = t.node_x[static_cast<size_t>(nd)];
                    cr[2 * v + 1] = t.node_y[static_cast<size_t>(nd)];
                }
                if (locate(cr, x, y, xi, eta)) found = e;
            }
            if (found < 0) fail(NDG_ERR_INVALID_ARG, "receiver " + std::to_string(r) + " lies outside the mesh");
            a->rec_elem.push_back(found);
            a->rec_xi.push_back(xi);
            a->rec_xi.push_back(eta);
            a->rec.elem[r] = static_cast<int32_t>(found);
            std::vector<double> li(static_cast<size_t>(n)), lj(static_cast<size_t>(n));
            lagrange_basis(nodes, bw, xi, li.data());
            lagrange_basis(nodes, bw, eta, lj.data());
            for (int i = 0; i < n; ++i)
                for (int j = 0; j < n; ++j) a->rec_w[static_cast<size_t>(r * a->NN + i * n + j)] = li[static_cast<size_t>(i)] * lj[static_cast<size_t>(j)];
        }
        cudaStream_t s = ctx->stream;
        a->d_rec_w.upload(a->rec_w, s);
        a->rec.w = a->d_rec_w.ptr;
        std::vector<double> cp(static_cast<size_t>(a->Kp), 1.0);
        a->c.upload(cp, s);
        const size_t state = 3 * static_cast<size_t>(a->block);
        const size_t traces = 3 * static_cast<size_t>(a->Kp) * 4 * static_cast<size_t>(n);
        a->q.allocate(state);
        a->k.allocate(state);
        a->lq.allocate(state);
        a->lk.allocate(state);
        for (int i = 0; i < 2; ++i) {
            a->tr[i].allocate(traces);
            a->atr[i].allocate(traces);
            a->tr_f[i].allocate(traces);
            a->atr_f[i].allocate(traces);
            check_cuda(cudaMemsetAsync(a->tr[i].ptr, 0, traces * sizeof(double), s), "memset");
            check_cuda(cudaMemsetAsync(a->tr_f[i].ptr, 0, traces * sizeof(float), s), "memset");
        }
        a->acc.allocate(5 * static_cast<size_t>(a->Kp));
        a->grad.allocate(static_cast<size_t>(a->Kp));
        check_cuda(dev::prepare_speed_kernels(a->N, false), "kernel attributes");
        check_cuda(dev::prepare_speed_kernels(a->N, true), "kernel attributes");
        check_cuda(dev::prepare_kernels_f32(a->N), "kernel attributes");
        check_cuda(cudaEventCreate(&a->ev[0]), "event");
        check_cuda(cudaEventCreate(&a->ev[1]), "event");
        check_cuda(cudaStreamSynchronize(s), "adjoint setup");
        *out = a.release();
    });
}

ndg_status ndg_adjoint_destroy(ndg_adjoint* adj) {
    return guarded([&] {
        if (adj) make_current(adj->ctx);
        delete adj;
    });
}

ndg_status ndg_adjoint_set_speed(ndg_adjoint* adj, const double* c) {
    return guarded([&] {
        require_valid(adj);
        if (!c) fail(NDG_ERR_INVALID_ARG, "c is NULL");
        for (int64_t e = 0; e < adj->K; ++e)
            if (!(c[e] > 0.0) || !std::isfinite(c[e])) fail(NDG_ERR_INVALID_ARG, "wave speeds must be positive and finite");
        make_current(adj->ctx);
        adj->speed.assign(c, c + adj->K);
        std::vector<double> cp(adj->speed);
        cp.resize(static_cast<size_t>(adj->Kp), 1.0);
        check_cuda(cudaMemcpyAsync(adj->c.ptr, cp.data(), cp.size() * sizeof(double), cudaMemcpyHostToDevice, adj->ctx->stream), "speed upload");
        check_cuda(cudaStreamSynchronize(adj->ctx->stream), "speed upload");
        adj->has_forward = false;
    });
}

ndg_status ndg_adjoint_set_precision(ndg_adjoint* adj, int32_t precision) {
    return guarded([&] {
        require_valid(adj);
        if (precision != NDG_FP64 && precision != NDG_FP32) fail(NDG_ERR_UNSUPPORTED, "the adjoint runs in NDG_FP64 or NDG_FP32");
        adj->fp32 = precision == NDG_FP32;
        adj->has_forward = false;
    });
}

ndg_status ndg_adjoint_delta_t(ndg_adjoint* adj, double cfl, double* delta_t) {
    return guarded([&] {
        require_valid(adj);
        if (!delta_t || !(cfl > 0.0)) fail(NDG_ERR_INVALID_ARG, "need cfl > 0 and an output");
        double dt = INFINITY;
        const double N2 = static_cast<double>(adj->N) * adj->N;
        for (int64_t e = 0; e < adj->K; ++e) dt = std::min(dt, cfl * adj->ctx->topo.delta_xy_min[static_cast<size_t>(e)] / (N2 * adj->speed[static_cast<size_t>(e)]));
        *delta_t = dt;
    });
}

ndg_status ndg_adjoint_receivers(const ndg_adjoint* adj, int64_t* element, double* xi_eta) {
    return guarded([&] {
        require_valid(adj);
        if (element) std::copy(adj->rec_elem.begin(), adj->rec_elem.end(), element);
        if (xi_eta) std::copy(adj->rec_xi.begin(), adj->rec_xi.end(), xi_eta);
    });
}

ndg_status ndg_adjoint_forward(ndg_adjoint* adj, const double* p0, const double* u0, const double* v0, const double* targets, double dt,
                               int64_t n_steps, int64_t checkpoint_interval, double* samples, double* misfit) {
    return guarded([&] {
        require_valid(adj);
        if (!p0) fail(NDG_ERR_INVALID_ARG, "p0 is NULL");
        if (!(dt > 0.0) || !std::isfinite(dt)) fail(NDG_ERR_INVALID_ARG, "dt must be positive");
        if (n_steps < 1) fail(NDG_ERR_INVALID_ARG, "n_steps must be >= 1");
        if (checkpoint_interval < 0) fail(NDG_ERR_INVALID_ARG, "checkpoint_interval must be >= 0");
        ndg_ctx* c = adj->ctx;
        make_current(c);
        cudaStream_t s = c->stream;
        const int R = adj->rec.n;
        const int64_t interval = checkpoint_interval == 0 ? n_steps : std::min(checkpoint_interval, n_steps);
        const int64_t n_ckpt = (n_steps + interval - 1) / interval;
        const size_t state = 3 * static_cast<size_t>(adj->block);
        adj->has_forward = false;
        if (adj->ckpt.count != static_cast<size_t>(n_ckpt) * state) adj->ckpt.allocate(static_cast<size_t>(n_ckpt) * state);
        const size_t rows = static_cast<size_t>(n_steps + 1) * static_cast<size_t>(std::max(R, 1));
        if (adj->samples.count != rows) adj->samples.allocate(rows);
        if (adj->targets.count != rows) adj->targets.allocate(rows);
        if (targets && R > 0)
            check_cuda(cudaMemcpyAsync(adj->targets.ptr, targets, static_cast<size_t>(n_steps + 1) * R * sizeof(double), cudaMemcpyHostToDevice, s), "target upload");
        else
            check_cuda(cudaMemsetAsync(adj->targets.ptr, 0, rows * sizeof(double), s), "memset");
        const double* fields[3] = {p0, u0, v0};
        upload_state(adj, adj->q.ptr, fields);
        adj->dt = dt;
        adj->n_steps = n_steps;
        adj->interval = interval;
        const size_t seg_values = 3 * static_cast<size_t>(interval) * state;
        if (adj->seg.count != seg_values) adj->seg.allocate(seg_values);
        int64_t launches = 0;
        check_cuda(cudaEventRecord(adj->ev[0], s), "event");
        launch_traces_of_q(adj, 0);
        ++launches;
        // Checkpoints at the starts of the intervals before the last; the
        // last interval keeps every stage input (the backward needs them
        // first, and a stage that keeps its input costs no more).
        const int64_t last_first = (n_ckpt - 1) * interval + 1;
        int in = 0;
        if (last_first > 1) in = run_forward(adj, 0, 1, last_first - 1, nullptr, true, interval, launches);
        run_forward(adj, in, last_first, n_steps, adj->seg.ptr, true, 0, launches);
        // its checkpoint too (a later backward recomputes from it): the
        // interval's first stage input
        check_cuda(cudaMemcpyAsync(adj->ckpt.ptr + static_cast<size_t>(n_ckpt - 1) * state, adj->seg.ptr, state * sizeof(double),
                                   cudaMemcpyDeviceToDevice, s),
                   "checkpoint");
        adj->last_kept = true;
        check_cuda(cudaEventRecord(adj->ev[1], s), "event");
        check_kernel_error(adj);
        float ms = 0.0f;
        check_cuda(cudaEventElapsedTime(&ms, adj->ev[0], adj->ev[1]), "event");
        adj->forward_ms = ms;
        adj->forward_launches = launches;
        // Receivers' pressure: row 0 from p0 on the host, rows 1.. from the
        // stage kernels.
        std::vector<double> smp(static_cast<size_t>(n_steps + 1) * R), tg(static_cast<size_t>(n_steps + 1) * R, 0.0);
        if (R > 0) {
            check_cuda(cudaMemcpyAsync(smp.data() + R, adj->samples.ptr + R, static_cast<size_t>(n_steps) * R * sizeof(double), cudaMemcpyDeviceToHost, s),
                       "sample download");
            check_cuda(cudaStreamSynchronize(s), "sample download");
            if (targets) std::copy(targets, targets + (n_steps + 1) * R, tg.begin());
            for (int r = 0; r < R; ++r) {
                const double* w = adj->rec_w.data() + static_cast<size_t>(r * adj->NN);
                const double* p = p0 + adj->rec_elem[static_cast<size_t>(r)] * adj->NN;
                double v = 0.0;
                for (int64_t i = 0; i < adj->NN; ++i) v = std::fma(w[i], p[i], v);
                smp[static_cast<size_t>(r)] = v;
            }
        }
        double J = 0.0;
        for (int64_t nstep = 1; nstep <= n_steps; ++nstep)
            for (int r = 0; r < R; ++r) {
                const double d = smp[static_cast<size_t>(nstep * R + r)] - tg[static_cast<size_t>(nstep * R + r)];
                J += d * d;
            }
        if (misfit) *misfit = 0.5 * dt * J;
        if (samples && R > 0) std::copy(smp.begin(), smp.end(), samples);
        adj->has_forward = true;
    });
}

ndg_status ndg_adjoint_backward(ndg_adjoint* adj, double* grad_p0, double* grad_u0, double* grad_v0, double* grad_c) {
    return guarded([&] {
        require_valid(adj);
        if (!adj->has_forward) fail(NDG_ERR_INVALID_ARG, "ndg_adjoint_backward needs a forward solve first (on the current speeds)");
        ndg_ctx* c = adj->ctx;
        make_current(c);
        cudaStream_t s = c->stream;
        const size_t state = 3 * static_cast<size_t>(adj->block);
        const int64_t I = adj->interval, n = adj->n_steps, n_ckpt = (n + I - 1) / I;
        const int R = adj->rec.n;
        const size_t seg_values = 3 * static_cast<size_t>(I) * state;
        if (adj->seg.count != seg_values) adj->seg.allocate(seg_values);
        if (adj->qfinal.count != state) adj->qfinal.allocate(state);
        // A second interval buffer lets the recomputation of interval j - 1
        // overlap the adjoint sweep of interval j; without the memory for it
        // the intervals run one after the other on one buffer.
        bool overlap = n_ckpt > 1;
        if (overlap && adj->seg2.count != seg_values) {
            try {
                adj->seg2.allocate(seg_values);
            } catch (const Error&) {
                cudaGetLastError();
                overlap = false;
            }
        }
        if (!adj->rstream) {
            check_cuda(cudaStreamCreateWithFlags(&adj->rstream, cudaStreamNonBlocking), "cudaStreamCreate");
            check_cuda(cudaStreamCreateWithFlags(&adj->astream, cudaStreamNonBlocking), "cudaStreamCreate");
            for (auto* e : {&adj->evr[0], &adj->evr[1], &adj->eva[0], &adj->eva[1], &adj->evs})
                check_cuda(cudaEventCreateWithFlags(e, cudaEventDisableTiming), "cudaEventCreate");
        }
        cudaStream_t r = overlap ? adj->rstream : s;
        cudaStream_t as = overlap ? adj->astream : s;
        // the last interval's buffer is seg (where the forward kept it)
        const int last_buf = static_cast<int>((n_ckpt - 1) % 2);
        double* buf[2];
        buf[last_buf] = adj->seg.ptr;
        buf[1 - last_buf] = overlap ? adj->seg2.ptr : adj->seg.ptr;
        const bool kept = adj->last_kept;
        adj->last_kept = false;  // this backward overwrites seg and q
        check_cuda(cudaMemsetAsync(adj->lq.ptr, 0, state * sizeof(double), s), "memset");
        check_cuda(cudaMemsetAsync(adj->lk.ptr, 0, state * sizeof(double), s), "memset");
        check_cuda(cudaMemsetAsync(adj->acc.ptr, 0, adj->acc.count * sizeof(double), s), "memset");
        zero_adjoint_traces(adj, 0);
        int64_t launches = 0;
        int ain = 0;
        check_cuda(cudaEventRecord(adj->ev[0], s), "event");
        if (kept) check_cuda(cudaMemcpyAsync(adj->qfinal.ptr, adj->q.ptr, state * sizeof(double), cudaMemcpyDeviceToDevice, s), "final state");
        if (overlap) {
            check_cuda(cudaEventRecord(adj->evs, s), "event");
            check_cuda(cudaStreamWaitEvent(r, adj->evs, 0), "stream wait");
            check_cuda(cudaStreamWaitEvent(as, adj->evs, 0), "stream wait");
        }
        // Recomputes interval j from its checkpoint, keeping every stage
        // input, into buf[j % 2] (on stream r).
        auto recompute = [&](int64_t j) {
            const int64_t first = j * I + 1, last = std::min((j + 1) * I, n);
            check_cuda(cudaMemcpyAsync(adj->q.ptr, adj->ckpt.ptr + static_cast<size_t>(j) * state, state * sizeof(double), cudaMemcpyDeviceToDevice, r),
                       "checkpoint restore");
            launch_traces_of_q(adj, 0, r);
            ++launches;
            run_forward(adj, 0, first, last, buf[j % 2], false, 0, launches, r);
            if (j == n_ckpt - 1)
                check_cuda(cudaMemcpyAsync(adj->qfinal.ptr, adj->q.ptr, state * sizeof(double), cudaMemcpyDeviceToDevice, r), "final state");
            if (overlap) check_cuda(cudaEventRecord(adj->evr[j % 2], r), "event");
        };
        if (kept) {
            if (overlap) check_cuda(cudaEventRecord(adj->evr[(n_ckpt - 1) % 2], s), "event");
        } else {
            recompute(n_ckpt - 1);
        }
        for (int64_t j = n_ckpt - 1; j >= 0; --j) {
            const int64_t first = j * I + 1, last = std::min((j + 1) * I, n);
            if (overlap) {
                if (j >= 1) {
                    // interval j - 1 reuses the buffer of interval j + 1
                    if (j + 1 <= n_ckpt - 1) check_cuda(cudaStreamWaitEvent(r, adj->eva[(j + 1) % 2], 0), "stream wait");
                    recompute(j - 1);
                }
                check_cuda(cudaStreamWaitEvent(as, adj->evr[j % 2], 0), "stream wait");
            } else if (j < n_ckpt - 1) {
                recompute(j);
            }
            if (j == n_ckpt - 1) {
                // The misfit's derivative at the final state, and the first
                // adjoint far traces.
                dev::AdjointStageArgs a = adjoint_args(adj, ain);
                a.qs = adj->qfinal.ptr;
                a.rk_a = 0.0;
                a.gdt = 0.0;
                a.gdt_next = kRkG[2] * adj->dt;
                a.inject = R > 0;
                a.target = adj->targets.ptr + n * R;
                a.wdt = adj->dt;
                check_cuda(dev::launch_adjoint_stage(adj->N, adj->fp32, a, as), "adjoint stage launch");
                ++launches;
                ain = 1 - ain;
            }
            for (int64_t step = last; step >= first; --step) {
                for (int m = 2; m >= 0; --m) {
                    dev::AdjointStageArgs a = adjoint_args(adj, ain);
                    a.qs = buf[j % 2] + (static_cast<size_t>(step - first) * 3 + static_cast<size_t>(m)) * state;
                    a.rk_a = kRkA[m];
                    a.gdt = kRkG[m] * adj->dt;
                    a.gdt_next = kRkG[m > 0 ? m - 1 : 2] * adj->dt;
                    a.inject = (m == 0 && step - 1 >= 1 && R > 0) ? 1 : 0;
                    a.target = adj->targets.ptr + (step - 1) * R;
                    a.wdt = adj->dt;
                    check_cuda(dev::launch_adjoint_stage(adj->N, adj->fp32, a, as), "adjoint stage launch");
                    ++launches;
                    ain = 1 - ain;
                }
            }
            if (overlap) check_cuda(cudaEventRecord(adj->eva[j % 2], as), "event");
        }
        if (overlap) {
            // the adjoint stream's last event covers the recomputations it waited for
            check_cuda(cudaEventRecord(adj->evs, as), "event");
            check_cuda(cudaStreamWaitEvent(s, adj->evs, 0), "stream wait");
        }
        check_cuda(dev::launch_speed_gradient(adj->acc.ptr, reinterpret_cast<const int2*>(c->link.ptr), adj->K, adj->grad.ptr, s), "gradient kernel");
        ++launches;
        check_cuda(cudaEventRecord(adj->ev[1], s), "event");
        check_kernel_error(adj);
        float ms = 0.0f;
        check_cuda(cudaEventElapsedTime(&ms, adj->ev[0], adj->ev[1]), "event");
        adj->backward_ms = ms;
        adj->backward_launches = launches;
        download_field(adj, adj->lq.ptr, grad_p0);
        download_field(adj, adj->lq.ptr + adj->block, grad_u0);
        download_field(adj, adj->lq.ptr + 2 * adj->block, grad_v0);
        if (grad_c) check_cuda(cudaMemcpyAsync(grad_c, adj->grad.ptr, static_cast<size_t>(adj->K) * sizeof(double), cudaMemcpyDeviceToHost, s), "download");
        check_cuda(cudaStreamSynchronize(s), "download");
    });
}

ndg_status ndg_adjoint_operator(ndg_adjoint* adj, const double* x, const double* y, double* Lx, double* LTy, double* dc) {
    return guarded([&] {
        require_valid(adj);
        if (!x || !y) fail(NDG_ERR_INVALID_ARG, "x and y are required");
        ndg_ctx* c = adj->ctx;
        make_current(c);
        cudaStream_t s = c->stream;
        const size_t state = 3 * static_cast<size_t>(adj->block);
        const int64_t fs = adj->field_size;
        const double* xf[3] = {x, x + fs, x + 2 * fs};
        const double* yf[3] = {y, y + fs, y + 2 * fs};
        const double* none[3] = {nullptr, nullptr, nullptr};
        if (adj->G.count != state) adj->G.allocate(state);
        adj->has_forward = false;  // q, k and the traces are reused
        // L x: one stage with gdt = 0 from q = x, keeping G.
        upload_state(adj, adj->q.ptr, xf);
        launch_traces_of_q(adj, 0);
        dev::SpeedStageArgs f = speed_args(adj, 0, 0, 0.0);
        f.gdt = 0.0;
        f.G_out = adj->G.ptr;
        check_cuda(dev::launch_speed_stage(adj->N, adj->fp32, f, s), "speed stage launch");
        // L^T y: publish the adjoint far traces of y (mu = 0, mu' = lq = y),
        // then one adjoint stage with mu = lk = y, lq = 0 and qs = x.
        zero_adjoint_traces(adj, 0);
        check_cuda(cudaMemsetAsync(adj->acc.ptr, 0, adj->acc.count * sizeof(double), s), "memset");
        upload_state(adj, adj->lq.ptr, yf);
        upload_state(adj, adj->lk.ptr, none);
        dev::AdjointStageArgs a = adjoint_args(adj, 0);
        a.qs = adj->q.ptr;
        a.gdt_next = 1.0;
        check_cuda(dev::launch_adjoint_stage(adj->N, adj->fp32, a, s), "adjoint stage launch");
        check_cuda(cudaMemsetAsync(adj->acc.ptr, 0, adj->acc.count * sizeof(double), s), "memset");
        upload_state(adj, adj->lq.ptr, none);
        upload_state(adj, adj->lk.ptr, yf);
        a = adjoint_args(adj, 1);
        a.qs = adj->q.ptr;
        check_cuda(dev::launch_adjoint_stage(adj->N, adj->fp32, a, s), "adjoint stage launch");
        check_cuda(dev::launch_speed_gradient(adj->acc.ptr, reinterpret_cast<const int2*>(c->link.ptr), adj->K, adj->grad.ptr, s), "gradient kernel");
        check_kernel_error(adj);
        for (int ff = 0; ff < 3; ++ff) {
            if (Lx) download_field(adj, adj->G.ptr + ff * adj->block, Lx + ff * fs);
            if (LTy) download_field(adj, adj->lq.ptr + ff * adj->block, LTy + ff * fs);
        }
        if (dc) check_cuda(cudaMemcpyAsync(dc, adj->grad.ptr, static_cast<size_t>(adj->K) * sizeof(double), cudaMemcpyDeviceToHost, s), "download");
        check_cuda(cudaStreamSynchronize(s), "download");
    });
}

ndg_status ndg_adjoint_timings(const ndg_adjoint* adj, double* forward_ms, double* backward_ms, int64_t* forward_launches, int64_t* backward_launches) {
    return guarded([&] {
        require_valid(adj);
        if (forward_ms) *forward_ms = adj->forward_ms;
        if (backward_ms) *backward_ms = adj->backward_ms;
        if (forward_launches) *forward_launches = adj->forward_launches;
        if (backward_launches) *backward_launches = adj->backward_launches;
    });
}

ndg_status ndg_adjoint_time_stage(ndg_adjoint* adj, int32_t which, int32_t n_launches, double* avg_ms) {
    return guarded([&] {
        require_valid(adj);
        if (which < 0 || which > 2 || n_launches < 1 || !avg_ms) fail(NDG_ERR_INVALID_ARG, "bad stage timing request");
        if (!(adj->dt > 0.0) || adj->seg.count == 0) fail(NDG_ERR_INVALID_ARG, "stage timing needs a forward and a backward first");
        ndg_ctx* c = adj->ctx;
        make_current(c);
        cudaStream_t s = c->stream;
        std::vector<cudaEvent_t> ev(static_cast<size_t>(2 * n_launches));
        for (auto& e : ev) check_cuda(cudaEventCreate(&e), "cudaEventCreate");
        launch_traces_of_q(adj, 0);
        int in = 0;
        for (int i = 0; i < n_launches; ++i) {
            check_cuda(cudaEventRecord(ev[static_cast<size_t>(2 * i)], s), "cudaEventRecord");
            if (which < 2) {
                dev::SpeedStageArgs a = speed_args(adj, 1, in, adj->dt);
                if (which == 1) a.q_save = adj->seg.ptr;
                check_cuda(dev::launch_speed_stage(adj->N, adj->fp32, a, s), "speed stage launch");
            } else {
                dev::AdjointStageArgs a = adjoint_args(adj, in);
                a.qs = adj->seg.ptr;
                a.rk_a = kRkA[1];
                a.gdt = kRkG[1] * adj->dt;
                a.gdt_next = kRkG[0] * adj->dt;
                check_cuda(dev::launch_adjoint_stage(adj->N, adj->fp32, a, s), "adjoint stage launch");
            }
            check_cuda(cudaEventRecord(ev[static_cast<size_t>(2 * i + 1)], s), "cudaEventRecord");
            in = 1 - in;
        }
        check_cuda(cudaStreamSynchronize(s), "stage timing");
        check_kernel_error(adj);
        double total = 0.0;
        for (int i = 0; i < n_launches; ++i) {
            float ms = 0.0f;
            check_cuda(cudaEventElapsedTime(&ms, ev[static_cast<size_t>(2 * i)], ev[static_cast<size_t>(2 * i + 1)]), "cudaEventElapsedTime");
            total += ms;
        }
        for (auto& e : ev) cudaEventDestroy(e);
        *avg_ms = total / n_launches;
        adj->has_forward = false;  // the state advanced
    });
}

}  // extern "C"
