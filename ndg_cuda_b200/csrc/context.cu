// C ABI of the library (include/ndg_b200.h): contexts, tables, meshes,
// fields and time stepping. Host orchestration only; the arithmetic is in
// stage_kernels.cu.
#include "context.hpp"
#include "estimator.cuh"
#include "general_kernels.cuh"
#include "stage_kernels.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <new>
#include <string>
#include <vector>

namespace ndg {

namespace {
thread_local std::string g_last_error;
}

void set_last_error(const std::string& message) { g_last_error = message; }

[[noreturn]] void fail(ndg_status status, const std::string& message) { throw Error{status, message}; }

}  // namespace ndg

namespace ndg {
namespace {

bool strict(const ndg_ctx* c) { return c->precision == NDG_FP64_STRICT; }

void drop_graphs(ndg_ctx* c) {
    for (auto& g : c->graph) {
        if (g) cudaGraphExecDestroy(g);
        g = nullptr;
    }
}

// Reads the kernels' error word (set when a bounded wait in a stage kernel
// gave up); synchronises the stream.
void check_device_error(ndg_ctx* c) {
    if (!c->error.ptr) return;
    unsigned err = 0;
    check_cuda(cudaMemcpyAsync(&err, c->error.ptr, sizeof(err), cudaMemcpyDeviceToHost, c->stream), "error word readback");
    check_cuda(cudaStreamSynchronize(c->stream), "error word readback");
    if (err) {
        check_cuda(cudaMemsetAsync(c->error.ptr, 0, sizeof(unsigned), c->stream), "memset");
        fail(NDG_ERR_TIMEOUT, "a stage kernel gave up waiting for its tile copies; the state is not valid");
    }
}

dev::StageArgs stage_args(ndg_ctx* c, int m, int in) {
    dev::StageArgs a{};
    a.q = c->q.ptr;
    a.k = c->k.ptr;
    a.trace_in = c->tr[in].ptr;
    a.trace_out = c->tr[1 - in].ptr;
    a.trace_in_f = c->tr32[in].ptr;
    a.trace_out_f = c->tr32[1 - in].ptr;
    a.G_out = c->keep_derivative ? c->G.ptr : nullptr;
    a.corners = c->corners.ptr;
    a.link = reinterpret_cast<const int2*>(c->link.ptr);
    a.normal = reinterpret_cast<const double2*>(c->normal.ptr);
    a.gscale = c->gscale.ptr;
    a.inflow = reinterpret_cast<const double4*>(c->inflow.ptr);
    a.step = c->step.ptr;
    a.rk_a = kRkA[m];
    a.rk_b = kRkB[m];
    a.rk_g = kRkG[m];
    a.first = m == 0;
    a.n_elements = c->K;
    a.field_stride = c->Kp;
    a.n_instances = c->n_instances;
    a.error = c->error.ptr;
    a.tc64 = c->tc64.ptr;
    a.tc32 = c->tc32.ptr;
    return a;
}

dev::GeneralStage general_args(ndg_ctx* c, int m, int in) {
    dev::GeneralStage a{};
    a.m = c->gmesh;
    a.q = c->q.ptr;
    a.k = c->k.ptr;
    a.G_out = c->keep_derivative ? c->G.ptr : nullptr;
    a.etr = c->getr[in].ptr;
    a.etr_out = c->getr[1 - in].ptr;
    a.etr_f = c->getr32[in].ptr;
    a.etr_out_f = c->getr32[1 - in].ptr;
    a.sflux = c->gsflux.ptr;
    a.sflux_f = c->gsflux32.ptr;
    a.side_slots = c->side_slots;
    a.step = c->step.ptr;
    a.rk_a = kRkA[m];
    a.rk_b = kRkB[m];
    a.rk_g = kRkG[m];
    a.first = m == 0;
    a.n_instances = c->n_instances;
    return a;
}

// Kernel launches of one stage of the general path: ghost traces, then the
// fused stage of every order group.
bool fp32(const ndg_ctx* c) { return c->precision == NDG_FP32; }

// The order groups a stage launches.
const std::vector<dev::OrderGroup>& stage_groups(const ndg_ctx* c) { return c->groups; }

// Whether an order group runs split (side_flux_kernel, then the
// conforming-element kernel over its side fluxes) rather than fused: always
// in launch mode 2; in mode 0 where the group (times the instances) has at
// least kSplitMinElements elements and its order has no conforming part. A
// remainder beside a conforming part runs in parallel with it, which hides
// its latency, and small groups are one short wave either way. Measured
// (ms per step, DOF-stage updates/s), fused against split by this rule:
// the mixed p-adapted 128² mesh FP64 0.2709 → 0.2502, FP32 0.2092 →
// 0.2045; the hp refining run (about 30 meshes) FP64 4.71e10 → 4.81e10,
// FP32 6.16e10 → 6.27e10. Splitting every group cost the hp run 4% (FP64)
// and 5% (FP32).
constexpr int64_t kSplitMinElements = 2048;
bool split_group(const ndg_ctx* c, const dev::OrderGroup& og) {
    if (og.conforming || c->mixed_launch == 1) return false;
    if (c->mixed_launch == 2) return true;
    const bool has_conforming_part =
        std::any_of(c->groups.begin(), c->groups.end(), [&](const dev::OrderGroup& other) { return other.conforming && other.N == og.N; });
    return !has_conforming_part && og.count * c->n_instances >= kSplitMinElements;
}

int64_t general_stage_launches(const ndg_ctx* c) {
    const int64_t ghosts = c->gmesh.n_total > c->gmesh.n_domain ? 1 : 0;
    if (c->mixed_launch == 1) return (c->queue.n_tiles > 0 ? 1 : 0) + ghosts;
    const auto& groups = stage_groups(c);
    const int64_t split = std::count_if(groups.begin(), groups.end(), [&](const dev::OrderGroup& og) { return split_group(c, og); });
    return static_cast<int64_t>(groups.size()) + split + ghosts;
}

// Side streams and events for the concurrent order groups (created once,
// before any capture).
void ensure_aux_streams(ndg_ctx* c) {
    const size_t most = std::max(c->groups.size(), c->whole_groups.size());
    const size_t want = most > 1 ? most - 1 : 0;
    while (c->aux_streams.size() < want) {
        cudaStream_t st;
        check_cuda(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "cudaStreamCreate");
        c->aux_streams.push_back(st);
    }
    while (c->aux_events.size() < want + 1) {
        cudaEvent_t ev;
        check_cuda(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "cudaEventCreate");
        c->aux_events.push_back(ev);
    }
}

// One stage of the mixed-order path: the ghost traces on the context's
// stream, then the order groups forked onto side streams (group 0 stays on
// the stream) and joined back.
cudaError_t issue_general_stage(ndg_ctx* c, int m, int in) {
    const dev::GeneralStage a = general_args(c, m, in);
    cudaError_t err = dev::launch_general_ghosts(a, strict(c), fp32(c), c->stream);
    if (c->mixed_launch == 1) return err == cudaSuccess ? dev::launch_general_queue(a, c->queue, strict(c), fp32(c), c->stream) : err;
    const std::vector<dev::OrderGroup>& groups = stage_groups(c);
    const size_t G = groups.size();
    if (err != cudaSuccess || G == 0) return err;
    // Group 0 goes before the forks, except in the FP32 form on a mesh whose
    // orders all run whole (no conforming group): the order in which the
    // branches reach the GPU changes how their CTAs share the SMs, and these
    // were the faster orders on the hp-adaptive mesh (FP64 and FP32) and on
    // the mixed p-adapted mesh (FP32: 0.220 against 0.257 ms per step).
    const bool first0 = !fp32(c) || std::any_of(groups.begin(), groups.end(), [](const dev::OrderGroup& og) { return og.conforming != 0; });
    if (G > 1 && (err = cudaEventRecord(c->aux_events[0], c->stream)) != cudaSuccess) return err;
    // A split group runs its element side fluxes first (side_flux_kernel),
    // then the conforming-element kernel over them (split_group).
    const auto group = [&](size_t g) {
        dev::OrderGroup og = groups[g];
        og.split = split_group(c, og) ? 1 : 0;
        return og;
    };
    if (first0 && (err = dev::launch_general_group(a, group(0), strict(c), fp32(c), c->stream)) != cudaSuccess) return err;
    for (size_t g = 1; g < G && err == cudaSuccess; ++g) {
        cudaStream_t st = c->aux_streams[g - 1];
        if ((err = cudaStreamWaitEvent(st, c->aux_events[0], 0)) != cudaSuccess) break;
        if ((err = dev::launch_general_group(a, group(g), strict(c), fp32(c), st)) != cudaSuccess) break;
        err = cudaEventRecord(c->aux_events[g], st);
    }
    if (!first0 && err == cudaSuccess) err = dev::launch_general_group(a, group(0), strict(c), fp32(c), c->stream);
    for (size_t g = 1; g < G && err == cudaSuccess; ++g) err = cudaStreamWaitEvent(c->stream, c->aux_events[g], 0);
    return err;
}

cudaError_t issue_stage(ndg_ctx* c, int m, int in) {
    if (c->general) return issue_general_stage(c, m, in);
    if (fp32(c)) {
        if (c->tile[1]) return dev::launch_stage_variant_fp32(c->N, c->tile[1], stage_args(c, m, in), c->stream);
        return dev::launch_stage_f32(c->N, stage_args(c, m, in), c->stream);
    }
    if (!strict(c) && c->tile[0]) return dev::launch_stage_variant_fp64(c->N, c->tile[0], stage_args(c, m, in), c->stream);
    return dev::launch_stage(c->N, strict(c), stage_args(c, m, in), c->stream);
}

// The FP32 form on a mixed-order mesh allocates its trace buffers the first
// time it runs (before any capture).
void require_form(ndg_ctx* c) {
    if (c->general && std::any_of(c->groups.begin(), c->groups.end(), [&](const dev::OrderGroup& og) { return split_group(c, og); })) {
        // The split groups' side fluxes, written before they are read in every stage.
        const size_t count = c->getr[0].count;
        if (c->gsflux.count != count) c->gsflux.allocate(count);
        if (fp32(c) && c->gsflux32.count != count) c->gsflux32.allocate(count);
    }
    if (c->general && fp32(c)) {
        const size_t count = c->getr[0].count;
        for (auto& t : c->getr32)
            if (t.count != count) {
                t.allocate(count);
                check_cuda(cudaMemsetAsync(t.ptr, 0, count * sizeof(float), c->stream), "memset");
            }
    }
}

void launch_stage(ndg_ctx* c, int m) {
    require_form(c);
    check_cuda(issue_stage(c, m, c->cur), "stage kernel launch");
    c->cur = 1 - c->cur;
    c->launches += c->general ? general_stage_launches(c) : 1;
}

// The tile candidates of the context's form (FP64 or FP32).
std::vector<int> tile_candidates(const ndg_ctx* c) {
    int buf[16];
    const int n = fp32(c) ? dev::tile_candidates_fp32(c->N, buf, 16) : dev::tile_candidates_fp64(c->N, buf, 16);
    return std::vector<int>(buf, buf + n);
}

void set_tile(ndg_ctx* c, int epb) {
    if (epb != 0) {
        const std::vector<int> cand = tile_candidates(c);
        if (std::find(cand.begin(), cand.end(), epb) == cand.end()) fail(NDG_ERR_INVALID_ARG, "not a candidate tile of this order and form");
        check_cuda(fp32(c) ? dev::prepare_stage_variant_fp32(c->N, epb) : dev::prepare_stage_variant_fp64(c->N, epb), "kernel attributes");
    }
    c->tile[fp32(c) ? 1 : 0] = epb;
    drop_graphs(c);
}

void ensure_traces(ndg_ctx* c) {
    if (c->traces_valid) return;
    if (c->general) {
        require_form(c);
        dev::GeneralStage g = general_args(c, 0, c->cur);
        check_cuda(dev::launch_general_traces(g, c->whole_groups.data(), static_cast<int>(c->whole_groups.size()), strict(c), fp32(c), c->stream),
                   "trace kernel launch");
        c->launches += static_cast<int64_t>(c->whole_groups.size());
        c->traces_valid = true;
        return;
    }
    dev::TraceArgs a{};
    a.q = c->q.ptr;
    a.trace_out = c->tr[c->cur].ptr;
    a.link = reinterpret_cast<const int2*>(c->link.ptr);  // far-slot layout of the stage kernels
    a.n_elements = c->K;
    a.field_stride = c->Kp;
    a.n_instances = c->n_instances;
    if (fp32(c)) {
        // FP32 traces are allocated the first time the form runs on this mesh.
        const size_t count = c->tr[0].count;
        for (auto& t : c->tr32)
            if (t.count != count) t.allocate(count);
        a.trace_out_f = c->tr32[c->cur].ptr;
        check_cuda(dev::prepare_kernels_f32(c->N), "kernel attributes");
        check_cuda(dev::launch_traces_f32(c->N, a, c->stream), "trace kernel launch");
    } else {
        check_cuda(dev::launch_traces(c->N, strict(c), a, c->stream), "trace kernel launch");
    }
    ++c->launches;
    c->traces_valid = true;
}

void set_step(ndg_ctx* c, double time, double dt, double t_end) {
    const double host[4] = {time, dt, c->dt_mesh, t_end};
    check_cuda(cudaMemcpyAsync(c->step.ptr, host, sizeof(host), cudaMemcpyHostToDevice, c->stream), "step upload");
    check_cuda(cudaStreamSynchronize(c->stream), "step upload");
}

// One RK3 step as a CUDA graph: the three stages and the time update. The
// uniform path alternates two trace buffers, so it has one graph per parity;
// the general path has one.
void ensure_graphs(ndg_ctx* c) {
    require_form(c);
    const int n_graphs = 2;
    if (c->graph[0] && (n_graphs == 1 || c->graph[1])) return;
    for (int parity = 0; parity < n_graphs; ++parity) {
        cudaGraph_t g = nullptr;
        check_cuda(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal), "graph capture");
        cudaError_t err = cudaSuccess;
        for (int m = 0; m < 3 && err == cudaSuccess; ++m) err = issue_stage(c, m, (parity + m) & 1);
        if (err == cudaSuccess) err = dev::launch_end_step(c->step.ptr, c->stream);
        cudaError_t end = cudaStreamEndCapture(c->stream, &g);
        check_cuda(err, "graph capture launch");
        check_cuda(end, "graph capture end");
        cudaGraphExec_t exec = nullptr;
        err = cudaGraphInstantiate(&exec, g, 0);
        cudaGraphDestroy(g);
        check_cuda(err, "graph instantiate");
        c->graph[parity] = exec;
    }
}

void run_steps(ndg_ctx* c, int64_t n_steps) {
    ensure_traces(c);
    ensure_graphs(c);
    const int64_t per_step = 3 * (c->general ? general_stage_launches(c) : 1) + 1;
    for (int64_t s = 0; s < n_steps; ++s) {
        check_cuda(cudaGraphLaunch(c->graph[c->cur], c->stream), "graph launch");
        c->cur = 1 - c->cur;  // three stages flip the trace buffer an odd number of times
        c->launches += per_step;
    }
}

double* field_ptr(ndg_ctx* c, int32_t field, int instance) {
    const int64_t per_inst = 3 * c->block;
    if (field >= NDG_FIELD_P && field <= NDG_FIELD_V) return c->q.ptr + instance * per_inst + field * c->block;
    if (field >= NDG_FIELD_K_P && field <= NDG_FIELD_K_V) return c->k.ptr + instance * per_inst + (field - NDG_FIELD_K_P) * c->block;
    if (field >= NDG_FIELD_G_P && field <= NDG_FIELD_G_V) {
        if (!c->keep_derivative) fail(NDG_ERR_INVALID_ARG, "time derivative fields need ndg_ctx_keep_derivative(ctx, 1) before stepping");
        return c->G.ptr + instance * per_inst + (field - NDG_FIELD_G_P) * c->block;
    }
    fail(NDG_ERR_INVALID_ARG, "unknown field");
}

// CFL step of the fixed mesh, reduced on the device (Solver2D_t.cu:17-31).
void compute_dt_mesh(ndg_ctx* c, double cfl) {
    check_cuda(dev::launch_delta_t(c->dxy.ptr, c->elem_N.ptr, c->K, cfl, c->step.ptr + 2, c->stream), "delta_t kernel");
    ++c->launches;
    check_cuda(cudaMemcpyAsync(&c->dt_mesh, c->step.ptr + 2, sizeof(double), cudaMemcpyDeviceToHost, c->stream), "delta_t readback");
    check_cuda(cudaStreamSynchronize(c->stream), "delta_t");
    c->params.cfl = cfl;
}

// Field layout of a topology: per domain element its order and first
// value within a field block, the block size and the values per field seen
// through the API. The uniform path pads the element count to even.
struct Layout {
    bool general = false;
    int64_t block = 0, field_size = 0;
    std::vector<int32_t> N;
    std::vector<int64_t> off2;
};

Layout layout_of(const Topology& t) {
    Layout l;
    l.general = !fused_path_applies(t);
    const int64_t K = t.n_domain;
    l.N.assign(t.elem_N.begin(), t.elem_N.begin() + static_cast<std::ptrdiff_t>(K));
    l.off2.resize(static_cast<size_t>(K));
    int64_t o = 0;
    for (int64_t e = 0; e < K; ++e) {
        l.off2[static_cast<size_t>(e)] = o;
        o += static_cast<int64_t>(l.N[static_cast<size_t>(e)] + 1) * (l.N[static_cast<size_t>(e)] + 1);
    }
    l.field_size = o;
    if (l.general) {
        l.block = o + (o & 1);
    } else {
        const int64_t NN = static_cast<int64_t>(l.N[0] + 1) * (l.N[0] + 1);
        l.block = (K + (K & 1)) * NN;
    }
    return l;
}

// Uploads what the stage kernels of the current topology read: the side
// plan of the uniform path or the arrays of the general path.
void upload_plan(ndg_ctx* c, const Layout& l) {
    const size_t inst = static_cast<size_t>(c->n_instances);
    c->general = l.general;
    c->block = l.block;
    c->field_size = l.field_size;
    c->K = c->topo.n_domain;
    c->Kp = c->K + (c->K & 1);
    c->N = *std::max_element(l.N.begin(), l.N.end());
    c->tile[0] = c->tile[1] = 0;
    const size_t K = static_cast<size_t>(c->K);
    if (!l.general) {
        if (c->N > kMaxOrder) fail(NDG_ERR_UNSUPPORTED, "orders above 16 have no compiled kernel");
        SidePlan plan = build_side_plan(c->topo, c->tables);
        // Tiles copy an even number of elements: pad the per-element arrays
        // to the even element count (the pad element has no sides).
        const size_t Kpad = static_cast<size_t>(c->Kp);
        plan.corners.resize(8 * Kpad, 0.0);
        plan.link.resize(8 * Kpad, static_cast<int32_t>(kZero << 2));
        plan.normal.resize(8 * Kpad, 0.0);
        plan.gscale.resize(4 * Kpad, 0.0);
        plan.inflow_xy.resize(16 * Kpad, 0.0);
        const size_t n = static_cast<size_t>(c->N + 1);
        c->tr[0].allocate(inst * 3 * static_cast<size_t>(c->Kp) * 4 * n);
        c->tr[1].allocate(inst * 3 * static_cast<size_t>(c->Kp) * 4 * n);
        check_cuda(cudaMemsetAsync(c->tr[0].ptr, 0, c->tr[0].count * sizeof(double), c->stream), "memset");
        check_cuda(cudaMemsetAsync(c->tr[1].ptr, 0, c->tr[1].count * sizeof(double), c->stream), "memset");
        c->corners.upload(plan.corners, c->stream);
        c->normal.upload(plan.normal, c->stream);
        c->gscale.upload(plan.gscale, c->stream);
        c->inflow.upload(plan.inflow_xy, c->stream);
        c->link.upload(plan.link, c->stream);
        c->tc64.upload(dev::tc_lane_table_fp64(c->N), c->stream);
        c->tc32.upload(dev::tc_lane_table_fp32(c->N), c->stream);
        check_cuda(dev::prepare_kernels(c->N, false), "kernel attributes");
        check_cuda(dev::prepare_kernels(c->N, true), "kernel attributes");
        c->groups.clear();
        c->whole_groups.clear();
    } else {
        for (int Ne : c->topo.elem_N)
            if (Ne < 1 || Ne > kMaxOrder) fail(NDG_ERR_UNSUPPORTED, "element orders must lie in 1..16");
        c->tr[0].release();
        c->tr[1].release();
        c->tr32[0].release();
        c->tr32[1].release();
        if (4 * c->topo.n_domain >= (int64_t{1} << 31)) fail(NDG_ERR_UNSUPPORTED, "mixed-order meshes hold fewer than 2^29 elements");
        c->gplan = build_general_plan(c->topo, c->has_tables ? &c->tables : nullptr);
        const GeneralPlan& g = c->gplan;
        c->g_eN.upload(g.eN, c->stream);
        c->g_off2.upload_reuse(g.off2, c->stream);
        c->g_off1.upload_reuse(g.off1, c->stream);
        c->g_enodes.upload_reuse(g.enodes, c->stream);
        c->g_sface_start.upload_reuse(g.sface_start, c->stream);
        c->g_sface.upload_reuse(g.sface, c->stream);
        c->g_corners.upload_reuse(g.corners, c->stream);
        c->g_node_xy.upload_reuse(g.node_xy, c->stream);
        c->g_fN.upload(g.fN, c->stream);
        c->g_foff.upload_reuse(g.foff, c->stream);
        c->g_fnodes.upload_reuse(g.fnodes, c->stream);
        c->g_felem.upload_reuse(g.felem, c->stream);
        c->g_fside.upload_reuse(g.fside, c->stream);
        c->g_fnormal.upload_reuse(g.fnormal, c->stream);
        c->g_ftangent.upload_reuse(g.ftangent, c->stream);
        c->g_foffset.upload_reuse(g.foffset, c->stream);
        c->g_fscale.upload_reuse(g.fscale, c->stream);
        c->g_gkind.upload_reuse(g.gkind, c->stream);
        c->g_gscale.upload_reuse(g.gscale, c->stream);
        c->g_gsrc.upload_reuse(g.gsrc, c->stream);
        c->g_gsrc_side.upload_reuse(g.gsrc_side, c->stream);
        c->g_fbase.upload_reuse(g.fbase, c->stream);
        c->g_fsN.upload(g.fsN, c->stream);
        c->g_sw_off.upload_reuse(g.sw_off, c->stream);
        c->g_sm_off.upload_reuse(g.sm_off, c->stream);
        c->g_fw_off.upload_reuse(g.fw_off, c->stream);
        c->g_fm_off.upload_reuse(g.fm_off, c->stream);
        c->g_sw.reserve(static_cast<size_t>(std::max<int64_t>(g.sw_total, 1)));
        c->g_fw.reserve(static_cast<size_t>(std::max<int64_t>(g.fw_total, 1)));
        c->g_smatch.reserve(static_cast<size_t>(std::max<int64_t>(g.sm_total, 1)));
        c->g_fmatch.reserve(static_cast<size_t>(std::max<int64_t>(g.fm_total, 1)));
        c->g_pslot_start.upload_reuse(g.pslot_start, c->stream);
        c->g_slot_desc.upload_reuse(g.slot_desc, c->stream);
        c->g_slot_normal.upload_reuse(g.slot_normal, c->stream);
        c->g_pside_mode.upload_reuse(g.pside_mode, c->stream);
        c->g_slot_side.upload_reuse(g.slot_side, c->stream);
        c->g_cnb.upload_reuse(g.cnb, c->stream);
        c->g_crole.upload_reuse(g.crole, c->stream);
        c->g_cnormal.upload_reuse(g.cnormal, c->stream);
        c->g_slot_src.reserve(static_cast<size_t>(std::max<int64_t>(2 * g.n_slots, 1)));
        c->g_pq_start.upload_reuse(g.pq_start, c->stream);
        c->g_pq_N.upload(g.pq_N, c->stream);
        c->g_pq_scale.upload_reuse(g.pq_scale, c->stream);
        c->g_pq_woff.upload_reuse(g.pq_woff, c->stream);
        c->g_pq_moff.upload_reuse(g.pq_moff, c->stream);
        c->g_poff2.upload_reuse(g.poff2, c->stream);
        c->g_poff1.upload_reuse(g.poff1, c->stream);
        c->g_pcorners.upload_reuse(g.pcorners, c->stream);
        c->g_gq_start.upload_reuse(g.gq_start, c->stream);
        c->g_gq_face.upload_reuse(g.gq_face, c->stream);
        c->g_gq_fs.upload_reuse(g.gq_fs, c->stream);
        c->g_gq_base.upload_reuse(g.gq_base, c->stream);
        c->g_gq_N.upload(g.gq_N, c->stream);
        c->g_gq_woff.upload_reuse(g.gq_woff, c->stream);
        c->g_gq_moff.upload_reuse(g.gq_moff, c->stream);
        c->g_gframe.upload_reuse(g.gframe, c->stream);
        c->g_gdirect.upload_reuse(g.gdirect, c->stream);
        std::vector<int64_t> ids;
        for (const auto& grp : g.groups) ids.insert(ids.end(), grp.second.begin(), grp.second.end());
        c->g_ids.upload_reuse(ids, c->stream);
        // Where most of an order's elements are conforming (the plan lists
        // them last), they and the rest are groups of their own, run by their
        // own kernels as concurrent branches; the rest, latency-bound on
        // their dependent loads, come first in the list. Where few are, the split
        // only adds a branch beside the fused launch (measured slower), and
        // the order stays one group (group_conforming 0).
        c->groups.clear();
        c->whole_groups.clear();
        std::vector<dev::OrderGroup> conforming_parts;
        int64_t at = 0;
        for (size_t gi = 0; gi < g.groups.size(); ++gi) {
            const int64_t total = static_cast<int64_t>(g.groups[gi].second.size()), nconf = g.group_conforming[gi];
            dev::OrderGroup og;
            og.N = g.groups[gi].first;
            og.ids = c->g_ids.ptr + at;
            og.first = at;
            og.count = total;
            if (total > 0) c->whole_groups.push_back(og);
            og.count = total - nconf;
            if (og.count > 0) c->groups.push_back(og);
            og.ids += total - nconf;
            og.first += total - nconf;
            og.count = nconf;
            og.conforming = 1;
            if (nconf > 0) conforming_parts.push_back(og);
            at += total;
            check_cuda(dev::prepare_general_kernels(g.groups[gi].first, g.side_slots), "kernel attributes");
        }
        c->groups.insert(c->groups.end(), conforming_parts.begin(), conforming_parts.end());
        // The stage queue: the groups' tiles, largest order first, and the
        // shared memory of the largest tile in either form.
        {
            std::vector<const dev::OrderGroup*> by_N;
            for (const auto& og : c->whole_groups) by_N.push_back(&og);
            std::stable_sort(by_N.begin(), by_N.end(), [](const dev::OrderGroup* x, const dev::OrderGroup* y) { return x->N > y->N; });
            std::vector<dev::QueueTile> tiles;
            size_t smem = 0;
            for (const dev::OrderGroup* og : by_N) {
                const int epb = dev::general_tile_elements(og->N);
                for (int64_t b = 0; b < og->count; b += epb) tiles.push_back(dev::QueueTile{og->N, og->first, og->count, b});
                smem = std::max({smem, dev::general_tile_bytes(og->N, g.side_slots, false), dev::general_tile_bytes(og->N, g.side_slots, true)});
            }
            c->g_queue.upload_reuse(tiles, c->stream);
            c->queue = dev::StageQueue{};
            c->queue.tiles = c->g_queue.ptr;
            c->queue.n_tiles = static_cast<int64_t>(tiles.size());
            c->queue.smem_bytes = smem;
            check_cuda(dev::prepare_general_queue(smem), "queue kernel attributes");
        }
        c->getr[0].allocate(inst * 3 * static_cast<size_t>(g.trace_total));
        c->getr[1].allocate(inst * 3 * static_cast<size_t>(g.trace_total));
        check_cuda(cudaMemsetAsync(c->getr[0].ptr, 0, c->getr[0].count * sizeof(double), c->stream), "memset");
        check_cuda(cudaMemsetAsync(c->getr[1].ptr, 0, c->getr[1].count * sizeof(double), c->stream), "memset");
        c->side_slots = static_cast<int>(g.side_slots);
        ensure_aux_streams(c);
        dev::GeneralMesh& M = c->gmesh;
        M = dev::GeneralMesh{};
        M.n_domain = g.n_domain;
        M.n_total = g.n_total;
        M.n_faces = g.n_faces;
        M.trace_total = g.trace_total;
        M.face_total = g.face_total;
        M.block = g.block;
        M.max_n = 1;
        for (int Ne : g.eN) M.max_n = std::max(M.max_n, Ne + 1);
        for (int Nf : g.fN) M.max_n = std::max(M.max_n, Nf + 1);
        M.eN = c->g_eN.ptr;
        M.off2 = c->g_off2.ptr;
        M.off1 = c->g_off1.ptr;
        M.enodes = c->g_enodes.ptr;
        M.sface_start = c->g_sface_start.ptr;
        M.sface = c->g_sface.ptr;
        M.corners = c->g_corners.ptr;
        M.node_xy = c->g_node_xy.ptr;
        M.fN = c->g_fN.ptr;
        M.foff = c->g_foff.ptr;
        M.fnodes = c->g_fnodes.ptr;
        M.felem = c->g_felem.ptr;
        M.fside = c->g_fside.ptr;
        M.fnormal = c->g_fnormal.ptr;
        M.ftangent = c->g_ftangent.ptr;
        M.foffset = c->g_foffset.ptr;
        M.fscale = c->g_fscale.ptr;
        M.gkind = c->g_gkind.ptr;
        M.gscale = c->g_gscale.ptr;
        M.gsrc = c->g_gsrc.ptr;
        M.gsrc_side = c->g_gsrc_side.ptr;
        M.fbase = c->g_fbase.ptr;
        M.fsN = c->g_fsN.ptr;
        M.sw_off = c->g_sw_off.ptr;
        M.sm_off = c->g_sm_off.ptr;
        M.fw_off = c->g_fw_off.ptr;
        M.fm_off = c->g_fm_off.ptr;
        M.sw = c->g_sw.ptr;
        M.smatch = c->g_smatch.ptr;
        M.fw = c->g_fw.ptr;
        M.fmatch = c->g_fmatch.ptr;
        M.n_slots = g.n_slots;
        M.pslot_start = c->g_pslot_start.ptr;
        M.slot_desc = c->g_slot_desc.ptr;
        M.slot_normal = c->g_slot_normal.ptr;
        M.slot_src = c->g_slot_src.ptr;
        M.pside_mode = c->g_pside_mode.ptr;
        M.slot_side = c->g_slot_side.ptr;
        M.cnb = c->g_cnb.ptr;
        M.crole = c->g_crole.ptr;
        M.cnormal = c->g_cnormal.ptr;
        M.pq_start = c->g_pq_start.ptr;
        M.pq_N = c->g_pq_N.ptr;
        M.pq_scale = c->g_pq_scale.ptr;
        M.pq_woff = c->g_pq_woff.ptr;
        M.pq_moff = c->g_pq_moff.ptr;
        M.poff2 = c->g_poff2.ptr;
        M.poff1 = c->g_poff1.ptr;
        M.pcorners = c->g_pcorners.ptr;
        M.gq_start = c->g_gq_start.ptr;
        M.gq_face = c->g_gq_face.ptr;
        M.gq_fs = c->g_gq_fs.ptr;
        M.gq_base = c->g_gq_base.ptr;
        M.gq_N = c->g_gq_N.ptr;
        M.gq_woff = c->g_gq_woff.ptr;
        M.gq_moff = c->g_gq_moff.ptr;
        M.gframe = c->g_gframe.ptr;
        M.gdirect = c->g_gdirect.ptr;
        check_cuda(dev::launch_general_weights(M, c->g_sw.ptr, c->g_smatch.ptr, c->g_fw.ptr, c->g_fmatch.ptr, c->g_slot_src.ptr, c->stream),
                   "mortar weights");
        c->launches += 4;
        // The uniform-path corners also serve the initial condition of a
        // general mesh.
        c->corners.upload(g.corners, c->stream);
    }
    std::vector<double> dxy(c->topo.delta_xy_min.begin(), c->topo.delta_xy_min.begin() + static_cast<std::ptrdiff_t>(K));
    c->dxy.upload(dxy, c->stream);
    c->elem_N.upload(l.N, c->stream);
    c->p_error.allocate(inst * K);
    c->p_sigma.allocate(inst * K);
    c->refine.allocate(inst * K);
    c->coarsen.allocate(inst * K);
    c->has_error_estimate = false;
    c->traces_valid = false;
    c->cur = 0;
    drop_graphs(c);
}

void load_mesh(ndg_ctx* c, Topology&& topo, const ndg_mesh_params& p, int32_t n_instances) {
    if (n_instances < 1) fail(NDG_ERR_INVALID_ARG, "n_instances must be >= 1");
    if (p.initial_N < 1 || p.initial_N > p.maximum_N) fail(NDG_ERR_INVALID_ARG, "need 1 <= initial_N <= maximum_N");
    if (!(p.cfl > 0.0)) fail(NDG_ERR_INVALID_ARG, "cfl must be positive");
    if (!c->has_tables || c->tables.N_max < p.maximum_N) {
        c->tables = build_tables(p.maximum_N, p.n_interpolation_points > 1 ? p.n_interpolation_points : 2);
        c->has_tables = true;
        if (c->device >= 0) {
            check_cuda(dev::upload_tables(c->tables), "table upload");
            check_cuda(dev::upload_general_tables(c->tables), "table upload");
            check_cuda(dev::upload_polynomials(c->tables), "table upload");
        }
    }
    compute_geometry(topo, c->tables);
    init_adaptivity_state(topo);
    c->topo = std::move(topo);
    c->params = p;
    c->n_instances = n_instances;
    const Layout l = layout_of(c->topo);
    c->N = p.initial_N;
    c->K = c->topo.n_domain;
    c->field_size = l.field_size;
    c->Kp = c->K + (c->K & 1);
    c->block = l.block;
    c->has_mesh = true;
    ++c->mesh_version;
    c->traces_valid = false;
    c->cur = 0;
    drop_graphs(c);
    if (c->device < 0) return;

    const size_t inst = static_cast<size_t>(n_instances);
    c->q.allocate(inst * 3 * static_cast<size_t>(l.block));
    c->k.allocate(inst * 3 * static_cast<size_t>(l.block));
    c->G.release();
    if (c->keep_derivative) c->G.allocate(inst * 3 * static_cast<size_t>(l.block));
    c->error.allocate(1);
    c->step.allocate(4);
    check_cuda(cudaMemsetAsync(c->q.ptr, 0, c->q.count * sizeof(double), c->stream), "memset");
    check_cuda(cudaMemsetAsync(c->k.ptr, 0, c->k.count * sizeof(double), c->stream), "memset");
    check_cuda(cudaMemsetAsync(c->error.ptr, 0, sizeof(unsigned), c->stream), "memset");
    upload_plan(c, l);
    compute_dt_mesh(c, p.cfl);
}

// The adaptation's decisions on the device (adapt_device.cu), from the
// estimate in ctx->refine / ctx->p_sigma (instance 0): uploads the topology
// the kernels read, runs them and downloads their compact results.
AdaptDecisions device_decisions(ndg_ctx* c) {
    const Topology& t = c->topo;
    const int64_t E = static_cast<int64_t>(t.elem_N.size()), K = t.n_domain, F = static_cast<int64_t>(t.face_N.size());
    std::vector<int64_t> enodes(static_cast<size_t>(4 * E)), sstart(static_cast<size_t>(4 * E + 1), 0), sface;
    for (int64_t e = 0; e < E; ++e)
        for (size_t s = 0; s < 4; ++s) {
            enodes[static_cast<size_t>(4 * e) + s] = t.elem_nodes[static_cast<size_t>(e)][s];
            const auto& l = t.elem_faces[static_cast<size_t>(e)][s];
            sface.insert(sface.end(), l.begin(), l.end());
            sstart[static_cast<size_t>(4 * e) + s + 1] = static_cast<int64_t>(sface.size());
        }
    std::vector<int64_t> fnodes(static_cast<size_t>(2 * F)), felem(static_cast<size_t>(2 * F)), fside(static_cast<size_t>(2 * F));
    for (int64_t f = 0; f < F; ++f)
        for (size_t k = 0; k < 2; ++k) {
            fnodes[static_cast<size_t>(2 * f) + k] = t.face_nodes[static_cast<size_t>(f)][k];
            felem[static_cast<size_t>(2 * f) + k] = t.face_elems[static_cast<size_t>(f)][k];
            fside[static_cast<size_t>(2 * f) + k] = t.face_sides[static_cast<size_t>(f)][k];
        }
    const size_t n_if = t.if_origin.size();
    std::vector<int64_t> ifs(3 * n_if), bnd;
    for (size_t i = 0; i < n_if; ++i) {
        ifs[i] = t.if_origin[i];
        ifs[n_if + i] = t.if_origin_side[i];
        ifs[2 * n_if + i] = t.if_destination[i];
    }
    for (const auto& l : t.boundary) bnd.insert(bnd.end(), l.begin(), l.end());
    std::vector<double> xy(2 * t.node_x.size());
    for (size_t i = 0; i < t.node_x.size(); ++i) {
        xy[2 * i] = t.node_x[i];
        xy[2 * i + 1] = t.node_y[i];
    }
    const std::vector<int32_t> split(t.elem_split.begin(), t.elem_split.begin() + K);
    c->av_split.upload_reuse(split, c->stream);
    c->av_enodes.upload_reuse(enodes, c->stream);
    c->av_sface_start.upload_reuse(sstart, c->stream);
    c->av_sface.upload_reuse(sface, c->stream);
    c->av_fnodes.upload_reuse(fnodes, c->stream);
    c->av_felem.upload_reuse(felem, c->stream);
    c->av_fside.upload_reuse(fside, c->stream);
    c->av_if.upload_reuse(ifs, c->stream);
    c->av_boundary.upload_reuse(bnd, c->stream);
    c->av_node_xy.upload_reuse(xy, c->stream);
    c->ad_code.reserve(static_cast<size_t>(E));
    c->ad_add.reserve(static_cast<size_t>(4 * E));
    c->ad_frefine.reserve(static_cast<size_t>(std::max<int64_t>(F, 1)));
    c->ad_split_flags.reserve(static_cast<size_t>(std::max<int64_t>(K, 1)));
    c->ad_split_prefix.reserve(static_cast<size_t>(K + 1));
    c->ad_refined_prefix.reserve(static_cast<size_t>(F + 1));
    c->ad_scan.reserve(static_cast<size_t>(dev::adapt_scan_scratch(std::max(K, F))));
    dev::AdaptView v;
    v.n_domain = K;
    v.n_total = E;
    v.n_faces = F;
    v.n_interfaces = static_cast<int64_t>(n_if);
    v.n_boundary = static_cast<int64_t>(bnd.size());
    v.max_split = c->params.max_split_level;
    v.split = c->av_split.ptr;
    v.enodes = c->av_enodes.ptr;
    v.sface_start = c->av_sface_start.ptr;
    v.sface = c->av_sface.ptr;
    v.fnodes = c->av_fnodes.ptr;
    v.felem = c->av_felem.ptr;
    v.fside = c->av_fside.ptr;
    v.if_origin = c->av_if.ptr;
    v.if_origin_side = c->av_if.ptr + n_if;
    v.if_destination = c->av_if.ptr + 2 * n_if;
    v.boundary = c->av_boundary.ptr;
    v.node_xy = c->av_node_xy.ptr;
    dev::AdaptOutputs o;
    o.code = c->ad_code.ptr;
    o.add = c->ad_add.ptr;
    o.frefine = c->ad_frefine.ptr;
    o.split_flags = c->ad_split_flags.ptr;
    o.split_prefix = c->ad_split_prefix.ptr;
    o.refined_prefix = c->ad_refined_prefix.ptr;
    o.scan_sums = c->ad_scan.ptr;
    check_cuda(dev::launch_adapt_decisions(v, c->refine.ptr, c->p_sigma.ptr, o, c->stream), "adaptation decision kernels");
    c->launches += 9;
    AdaptDecisions d;
    d.code.resize(static_cast<size_t>(E));
    d.add.resize(static_cast<size_t>(4 * E));
    d.face_split.resize(static_cast<size_t>(F));
    d.split_prefix.resize(static_cast<size_t>(K + 1));
    d.split_face_prefix.resize(static_cast<size_t>(F + 1));
    check_cuda(cudaMemcpyAsync(d.code.data(), o.code, d.code.size(), cudaMemcpyDeviceToHost, c->stream), "decision download");
    check_cuda(cudaMemcpyAsync(d.add.data(), o.add, d.add.size(), cudaMemcpyDeviceToHost, c->stream), "decision download");
    if (F > 0) check_cuda(cudaMemcpyAsync(d.face_split.data(), o.frefine, d.face_split.size(), cudaMemcpyDeviceToHost, c->stream), "decision download");
    check_cuda(cudaMemcpyAsync(d.split_prefix.data(), o.split_prefix, d.split_prefix.size() * sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream),
               "decision download");
    check_cuda(cudaMemcpyAsync(d.split_face_prefix.data(), o.refined_prefix, d.split_face_prefix.size() * sizeof(int64_t), cudaMemcpyDeviceToHost,
                               c->stream),
               "decision download");
    check_cuda(cudaStreamSynchronize(c->stream), "adaptation decisions");
    return d;
}

// Mesh2D_t::adapt from per-element refine flags and decay rates; moves the
// fields of a device context to the new mesh. With `dec` (device contexts)
// the flags are dec's bits and the topology rebuild takes dec's decisions
// and counts.
void adapt_mesh(ndg_ctx* ctx, const int32_t* refine_in, const double* sigma_in, const AdaptDecisions* dec = nullptr) {
    if (std::none_of(refine_in, refine_in + ctx->topo.n_domain, [](int32_t r) { return r != 0; })) {
        // Mesh2D_t::adapt changes nothing without a refine flag
        ctx->has_error_estimate = false;
        return;
    }
    const std::vector<int32_t> refine(refine_in, refine_in + ctx->topo.n_domain);
    const std::vector<double> sigma(sigma_in, sigma_in + ctx->topo.n_domain);
    const auto t_topo = std::chrono::steady_clock::now();
    if (!dec) ctx->adapt_ms[0] = 0.0;
    const Layout before = layout_of(ctx->topo);
    Topology topo = ctx->topo;
    // Mesh2D_t::adapt: element splitting when any element splits, the
    // p-only branch otherwise.
    std::vector<ElementSource> sources;
    const bool split = h_adapt(topo, ctx->tables, refine.data(), sigma.data(), ctx->params.maximum_N, ctx->params.max_split_level, sources, dec);
    if (!split && !p_adapt(topo, refine.data(), sigma.data(), ctx->params.maximum_N, ctx->params.max_split_level)) {
        ctx->has_error_estimate = false;
        return;
    }
    const Layout after = layout_of(topo);
    ++ctx->mesh_version;
    const auto t_transfer = std::chrono::steady_clock::now();
    ctx->adapt_ms[1] = std::chrono::duration<double, std::milli>(t_transfer - t_topo).count();
    if (ctx->device < 0) {
        // Host-only context: the topology alone.
        ctx->topo = std::move(topo);
        ctx->K = ctx->topo.n_domain;
        ctx->Kp = ctx->K + (ctx->K & 1);
        ctx->field_size = after.field_size;
        ctx->block = after.block;
        ctx->has_error_estimate = false;
        return;
    }
    // Per new domain element: its source element's order and offset, and
    // for children the node coordinates in the parent.
    const size_t K_new = static_cast<size_t>(topo.n_domain);
    std::vector<int32_t> oNv(K_new), mode(K_new);
    std::vector<int64_t> oOffv(K_new), coord_off(K_new, 0);
    std::vector<double> coords;
    for (size_t e = 0; e < K_new; ++e) {
        const int64_t old = split ? sources[e].old : static_cast<int64_t>(e);
        oNv[e] = before.N[static_cast<size_t>(old)];
        oOffv[e] = before.off2[static_cast<size_t>(old)];
        mode[e] = split ? sources[e].kind : (oNv[e] == after.N[e] ? 0 : 1);
        if (mode[e] == 2) {
            std::vector<double> c;
            child_coordinates(sources[e], ctx->tables.get(NDG_TABLE_NODES, after.N[e]), c);
            coord_off[e] = static_cast<int64_t>(coords.size());
            coords.insert(coords.end(), c.begin(), c.end());
        }
    }
    // Transfer the fields to the new elements, then switch the topology
    // and the device plan.
    DeviceBuffer<int32_t> oN, nN, dMode;
    DeviceBuffer<int64_t> oOff, nOff, dCoordOff;
    DeviceBuffer<double> dCoords;
    oN.upload(oNv, ctx->stream);
    nN.upload(after.N, ctx->stream);
    oOff.upload(oOffv, ctx->stream);
    nOff.upload(after.off2, ctx->stream);
    dMode.upload(mode, ctx->stream);
    dCoordOff.upload(coord_off, ctx->stream);
    dCoords.upload(coords, ctx->stream);
    dev::Transfer t{};
    t.mode = dMode.ptr;
    t.coords = dCoords.ptr;
    t.coord_off = dCoordOff.ptr;
    t.old_block = before.block;
    t.new_block = after.block;
    t.n_fields = 3;
    t.n_instances = ctx->n_instances;
    t.n_elements = static_cast<int64_t>(K_new);
    t.old_N = oN.ptr;
    t.new_N = nN.ptr;
    t.old_off2 = oOff.ptr;
    t.new_off2 = nOff.ptr;
    const size_t values = static_cast<size_t>(ctx->n_instances) * 3 * static_cast<size_t>(after.block);
    DeviceBuffer<double> q2, k2, G2;
    q2.allocate(values);
    k2.allocate(values);
    check_cuda(cudaMemsetAsync(q2.ptr, 0, values * sizeof(double), ctx->stream), "memset");
    check_cuda(cudaMemsetAsync(k2.ptr, 0, values * sizeof(double), ctx->stream), "memset");
    t.src = ctx->q.ptr;
    t.dst = q2.ptr;
    check_cuda(dev::launch_transfer(t, ctx->stream), "transfer kernel");
    t.src = ctx->k.ptr;
    t.dst = k2.ptr;
    t.zero_changed = 1;
    check_cuda(dev::launch_transfer(t, ctx->stream), "transfer kernel");
    ctx->launches += 2;
    if (ctx->keep_derivative) {
        G2.allocate(values);
        check_cuda(cudaMemsetAsync(G2.ptr, 0, values * sizeof(double), ctx->stream), "memset");
        t.src = ctx->G.ptr;
        t.dst = G2.ptr;
        t.zero_changed = 0;
        check_cuda(dev::launch_transfer(t, ctx->stream), "transfer kernel");
        ++ctx->launches;
    }
    check_cuda(cudaStreamSynchronize(ctx->stream), "transfer");
    ctx->q.swap(q2);
    ctx->k.swap(k2);
    if (ctx->keep_derivative) ctx->G.swap(G2);
    const auto t_plan = std::chrono::steady_clock::now();
    ctx->adapt_ms[2] = std::chrono::duration<double, std::milli>(t_plan - t_transfer).count();
    ctx->topo = std::move(topo);
    upload_plan(ctx, after);
    compute_dt_mesh(ctx, ctx->params.cfl);
    ctx->adapt_ms[3] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_plan).count();
}

// Legendre-decay error estimate of every element and instance
// (Mesh2D_t::estimate_error), one launch per order group.
void estimate(ndg_ctx* ctx) {
    dev::EstimatorArgs a{};
    a.q = ctx->q.ptr;
    a.p_error = ctx->p_error.ptr;
    a.p_sigma = ctx->p_sigma.ptr;
    a.refine = ctx->refine.ptr;
    a.coarsen = ctx->coarsen.ptr;
    a.tolerance_min = ctx->params.tolerance_min;
    a.tolerance_max = ctx->params.tolerance_max;
    a.n_elements = ctx->K;
    a.block = ctx->block;
    a.n_instances = ctx->n_instances;
    if (ctx->general) {
        a.off2 = ctx->g_off2.ptr;
        for (const auto& g : ctx->groups) {
            a.N = g.N;
            a.count = g.count;
            a.ids = g.ids;
            check_cuda(dev::launch_estimate_error(a, ctx->stream), "estimator kernel launch");
            ++ctx->launches;
        }
    } else {
        a.N = ctx->N;
        a.count = ctx->K;
        check_cuda(dev::launch_estimate_error(a, ctx->stream), "estimator kernel launch");
        ++ctx->launches;
    }
    ctx->has_error_estimate = true;
}

// Mesh2D_t::adapt from the last estimate of instance 0 (or flags the caller
// placed there): the decisions on the device, the topology rebuilt from them.
void adapt_from_estimate(ndg_ctx* ctx) {
    const auto t0 = std::chrono::steady_clock::now();
    const AdaptDecisions dec = device_decisions(ctx);
    ctx->adapt_ms[0] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    const size_t K = static_cast<size_t>(ctx->K);
    std::vector<int32_t> refine(K);
    std::vector<double> sigma(K);
    for (size_t e = 0; e < K; ++e) {
        refine[e] = dec.code[e] & 1u;
        sigma[e] = (dec.code[e] & 2u) ? 1.0 : 0.0;  // only its comparison with 1 decides
    }
    adapt_mesh(ctx, refine.data(), sigma.data(), &dec);
}

void copy_table(const Tables& t, int32_t table, int32_t N, double* out, int64_t capacity, int64_t* count) {
    if (table < 0 || table > 11) fail(NDG_ERR_INVALID_ARG, "unknown table");
    if (N < 0 || N > t.N_max) fail(NDG_ERR_INVALID_ARG, "order outside the tables");
    const auto& v = t.get(static_cast<ndg_table>(table), N);
    if (count) *count = static_cast<int64_t>(v.size());
    if (out) {
        if (capacity < static_cast<int64_t>(v.size())) fail(NDG_ERR_INVALID_ARG, "output buffer too small");
        std::memcpy(out, v.data(), v.size() * sizeof(double));
    }
}

}  // namespace

// Mesh2D_t::initial_conditions on every instance (the device must be current).
void set_initial_conditions(ndg_ctx* ctx) {
    if (ctx->general) {
        check_cuda(dev::launch_general_initial_conditions(general_args(ctx, 0, ctx->cur), ctx->groups.data(), static_cast<int>(ctx->groups.size()), ctx->stream),
                   "initial condition kernel");
        ctx->launches += static_cast<int64_t>(ctx->groups.size());
    } else {
        check_cuda(dev::launch_initial_conditions(ctx->q.ptr, ctx->k.ptr, ctx->corners.ptr, ctx->N, ctx->K, ctx->Kp, ctx->n_instances, ctx->stream),
                   "initial condition kernel");
        ++ctx->launches;
    }
    if (ctx->keep_derivative) check_cuda(cudaMemsetAsync(ctx->G.ptr, 0, ctx->G.count * sizeof(double), ctx->stream), "memset");
    ctx->traces_valid = false;
}

}  // namespace ndg

using namespace ndg;

extern "C" {

const char* ndg_last_error(void) { return g_last_error.c_str(); }

const char* ndg_version(void) { return "ndg_b200 0.1.0 (sm_100a)"; }

ndg_status ndg_ctx_create(int32_t device, void* stream, ndg_ctx** out) {
    return guarded([&] {
        if (!out) fail(NDG_ERR_INVALID_ARG, "out is NULL");
        auto c = std::make_unique<ndg_ctx>();
        c->device = device;
        if (device >= 0) {
            int count = 0;
            check_cuda(cudaGetDeviceCount(&count), "cudaGetDeviceCount");
            if (device >= count) fail(NDG_ERR_INVALID_ARG, "no such device");
            check_cuda(cudaSetDevice(device), "cudaSetDevice");
            if (stream) {
                c->stream = static_cast<cudaStream_t>(stream);
            } else {
                check_cuda(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking), "cudaStreamCreate");
                c->own_stream = true;
            }
        }
        *out = c.release();
    });
}

ndg_status ndg_ctx_destroy(ndg_ctx* ctx) {
    return guarded([&] {
        if (!ctx) return;
        if (ctx->device >= 0) {
            cudaSetDevice(ctx->device);
            cudaStreamSynchronize(ctx->stream);
        }
        delete ctx;
    });
}

ndg_status ndg_ctx_set_precision(ndg_ctx* ctx, int32_t precision) {
    return guarded([&] {
        if (!ctx) fail(NDG_ERR_INVALID_ARG, "ctx is NULL");
        if (precision != NDG_FP64 && precision != NDG_FP64_STRICT && precision != NDG_FP32) fail(NDG_ERR_INVALID_ARG, "unknown precision");
        if (ctx->precision != precision) {
            drop_graphs(ctx);
            ctx->traces_valid = false;  // the forms keep their traces in different buffers
        }
        ctx->precision = precision;
    });
}

ndg_status ndg_set_mixed_launch(ndg_ctx* ctx, int32_t mode) {
    return guarded([&] {
        if (!ctx) fail(NDG_ERR_INVALID_ARG, "ctx is NULL");
        if (mode < 0 || mode > 2)
            fail(NDG_ERR_INVALID_ARG, "mode is 0 (one launch per order group), 1 (one queue launch per stage) or 2 (order groups split into side fluxes and element tiles)");
        ctx->mixed_launch = mode;
        drop_graphs(ctx);
    });
}

ndg_status ndg_ctx_keep_derivative(ndg_ctx* ctx, int32_t enable) {
    return guarded([&] {
        if (!ctx) fail(NDG_ERR_INVALID_ARG, "ctx is NULL");
        make_current(ctx);
        ctx->keep_derivative = enable != 0;
        drop_graphs(ctx);
        if (ctx->has_mesh && ctx->device >= 0) {
            if (ctx->keep_derivative) {
                ctx->G.allocate(static_cast<size_t>(3 * ctx->block * ctx->n_instances));
                check_cuda(cudaMemsetAsync(ctx->G.ptr, 0, ctx->G.count * sizeof(double), ctx->stream), "memset");
            } else {
                ctx->G.release();
            }
        }
    });
}

ndg_status ndg_ctx_synchronize(ndg_ctx* ctx) {
    return guarded([&] {
        if (!ctx) fail(NDG_ERR_INVALID_ARG, "ctx is NULL");
        if (ctx->device >= 0) {
            make_current(ctx);
            check_cuda(cudaStreamSynchronize(ctx->stream), "synchronize");
            check_device_error(ctx);
        }
    });
}

ndg_status ndg_tables_build(ndg_ctx* ctx, int32_t N_max, int64_t n_interp) {
    return guarded([&] {
        if (!ctx) fail(NDG_ERR_INVALID_ARG, "ctx is NULL");
        make_current(ctx);
        ctx->tables = build_tables(N_max, n_interp);
        ctx->has_tables = true;
        if (ctx->device >= 0) {
            check_cuda(dev::upload_tables(ctx->tables), "table upload");
            check_cuda(dev::upload_polynomials(ctx->tables), "table upload");
        }
    });
}

ndg_status ndg_tables_get(const ndg_ctx* ctx, int32_t table, int32_t N, double* out, int64_t capacity, int64_t* count) {
    return guarded([&] {
        if (!ctx || !ctx->has_tables) fail(NDG_ERR_INVALID_ARG, "no tables built");
        copy_table(ctx->tables, table, N, out, capacity, count);
    });
}

ndg_status ndg_tables_compute(int32_t N_max, int64_t n_interp, int32_t table, int32_t N, double* out, int64_t capacity, int64_t* count) {
    return guarded([&] {
        const Tables t = build_tables(N_max, n_interp);
        copy_table(t, table, N, out, capacity, count);
    });
}

ndg_status ndg_mesh_load_zone(ndg_ctx* ctx, const ndg_zone* zone, const ndg_mesh_params* params, int32_t n_instances) {
    return guarded([&] {
        if (!ctx || !zone || !params) fail(NDG_ERR_INVALID_ARG, "NULL argument");
        make_current(ctx);
        load_mesh(ctx, build_topology(*zone, params->initial_N), *params, n_instances);
    });
}

ndg_status ndg_mesh_load_file(ndg_ctx* ctx, const char* path, const ndg_mesh_params* params, int32_t n_instances) {
    return guarded([&] {
        if (!ctx || !path || !params) fail(NDG_ERR_INVALID_ARG, "NULL argument");
        make_current(ctx);
        std::string p(path);
        std::string ext = p.size() >= 4 ? p.substr(p.size() - 4) : "";
        for (auto& ch : ext) ch = static_cast<char>(std::tolower(static_cast<unsigned char>(ch)));
        if (ext == ".su2") {
            load_mesh(ctx, read_su2(p, params->initial_N), *params, n_instances);
        } else if (p.size() >= 5 && (p.substr(p.size() - 5) == ".cgns" || p.substr(p.size() - 5) == ".CGNS")) {
            fail(NDG_ERR_UNSUPPORTED, "this build has no CGNS library; pass the zone arrays to ndg_mesh_load_zone");
        } else {
            fail(NDG_ERR_INVALID_ARG, "extension not recognised (.su2 or .cgns)");
        }
    });
}

ndg_status ndg_mesh_counts(const ndg_ctx* ctx, int64_t* n_elements, int64_t* n_elements_total, int64_t* n_faces, int64_t* n_nodes) {
    return guarded([&] {
        require_mesh(ctx);
        if (n_elements) *n_elements = ctx->topo.n_domain;
        if (n_elements_total) *n_elements_total = static_cast<int64_t>(ctx->topo.elem_nodes.size());
        if (n_faces) *n_faces = static_cast<int64_t>(ctx->topo.face_nodes.size());
        if (n_nodes) *n_nodes = static_cast<int64_t>(ctx->topo.node_x.size());
    });
}

ndg_status ndg_mesh_get_faces(const ndg_ctx* ctx, int64_t* nodes, int64_t* elements, int64_t* sides, int32_t* N, double* normal, double* tangent, double* offset, double* scale) {
    return guarded([&] {
        require_mesh(ctx);
        const auto& t = ctx->topo;
        for (size_t f = 0; f < t.face_nodes.size(); ++f) {
            for (size_t k = 0; k < 2; ++k) {
                if (nodes) nodes[2 * f + k] = t.face_nodes[f][k];
                if (elements) elements[2 * f + k] = t.face_elems[f][k];
                if (sides) sides[2 * f + k] = t.face_sides[f][k];
                if (normal) normal[2 * f + k] = t.face_normal[f][k];
                if (tangent) tangent[2 * f + k] = t.face_tangent[f][k];
                if (offset) offset[2 * f + k] = t.face_offset[f][k];
                if (scale) scale[2 * f + k] = t.face_scale[f][k];
            }
            if (N) N[f] = t.face_N[f];
        }
    });
}

ndg_status ndg_mesh_get_elements(const ndg_ctx* ctx, int64_t* nodes, int32_t* N, double* delta_xy_min, int64_t* first_face) {
    return guarded([&] {
        require_mesh(ctx);
        const auto& t = ctx->topo;
        for (size_t e = 0; e < t.elem_nodes.size(); ++e) {
            for (size_t k = 0; k < 4; ++k) {
                if (nodes) nodes[4 * e + k] = t.elem_nodes[e][k];
                if (first_face) first_face[4 * e + k] = t.elem_face[e][k];
            }
            if (N) N[e] = t.elem_N[e];
            if (delta_xy_min) delta_xy_min[e] = t.delta_xy_min[e];
        }
    });
}

ndg_status ndg_mesh_get_boundary(const ndg_ctx* ctx, int32_t list, int64_t* out, int64_t capacity, int64_t* count) {
    return guarded([&] {
        require_mesh(ctx);
        const auto& t = ctx->topo;
        const std::vector<int64_t>* v = nullptr;
        switch (list) {
            case NDG_LIST_WALL: v = &t.boundary[kWall]; break;
            case NDG_LIST_SYMMETRY: v = &t.boundary[kSymmetry]; break;
            case NDG_LIST_INFLOW: v = &t.boundary[kInflow]; break;
            case NDG_LIST_OUTFLOW: v = &t.boundary[kOutflow]; break;
            case NDG_LIST_INTERFACE_ORIGIN: v = &t.if_origin; break;
            case NDG_LIST_INTERFACE_ORIGIN_SIDE: v = &t.if_origin_side; break;
            case NDG_LIST_INTERFACE_DESTINATION: v = &t.if_destination; break;
            default: fail(NDG_ERR_INVALID_ARG, "unknown boundary list");
        }
        if (count) *count = static_cast<int64_t>(v->size());
        if (out) {
            if (capacity < static_cast<int64_t>(v->size())) fail(NDG_ERR_INVALID_ARG, "output buffer too small");
            std::memcpy(out, v->data(), v->size() * sizeof(int64_t));
        }
    });
}

ndg_status ndg_mesh_get_element_state(const ndg_ctx* ctx, int32_t* split_level, int32_t* status, int32_t* rotation, int32_t* n_faces_side) {
    return guarded([&] {
        require_mesh(ctx);
        const auto& t = ctx->topo;
        for (size_t e = 0; e < t.elem_N.size(); ++e) {
            if (split_level) split_level[e] = t.elem_split[e];
            if (status) status[e] = t.elem_status[e];
            if (rotation) rotation[e] = t.elem_rotation[e];
            if (n_faces_side)
                for (size_t s = 0; s < 4; ++s) n_faces_side[4 * e + s] = static_cast<int32_t>(t.elem_faces[e][s].size());
        }
    });
}

ndg_status ndg_mesh_get_element_faces(const ndg_ctx* ctx, int64_t* out, int64_t capacity, int64_t* count) {
    return guarded([&] {
        require_mesh(ctx);
        int64_t n = 0;
        for (const auto& sides : ctx->topo.elem_faces)
            for (const auto& list : sides) n += static_cast<int64_t>(list.size());
        if (count) *count = n;
        if (!out) return;
        if (capacity < n) fail(NDG_ERR_INVALID_ARG, "output buffer too small");
        int64_t i = 0;
        for (const auto& sides : ctx->topo.elem_faces)
            for (const auto& list : sides)
                for (int64_t f : list) out[i++] = f;
    });
}

ndg_status ndg_mesh_get_nodes(const ndg_ctx* ctx, double* xy) {
    return guarded([&] {
        require_mesh(ctx);
        for (size_t i = 0; i < ctx->topo.node_x.size(); ++i) {
            xy[2 * i] = ctx->topo.node_x[i];
            xy[2 * i + 1] = ctx->topo.node_y[i];
        }
    });
}

ndg_status ndg_mesh_field_size(const ndg_ctx* ctx, int64_t* n_values) {
    return guarded([&] {
        require_mesh(ctx);
        *n_values = ctx->field_size;
    });
}


ndg_status ndg_initial_conditions(ndg_ctx* ctx) {
    return guarded([&] {
        require_mesh(ctx);
        require_device(ctx);
        make_current(ctx);
        set_initial_conditions(ctx);
    });
}

ndg_status ndg_set_field(ndg_ctx* ctx, int32_t instance, int32_t field, const double* values) {
    return guarded([&] {
        require_mesh(ctx);
        require_device(ctx);
        if (!values) fail(NDG_ERR_INVALID_ARG, "values is NULL");
        if (instance >= ctx->n_instances) fail(NDG_ERR_INVALID_ARG, "instance out of range");
        make_current(ctx);
        const int first = instance < 0 ? 0 : instance;
        const int last = instance < 0 ? ctx->n_instances : instance + 1;
        for (int i = first; i < last; ++i) {
            double* dst = field_ptr(ctx, field, i);
            check_cuda(cudaMemcpyAsync(dst, values + (i - first) * ctx->field_size, static_cast<size_t>(ctx->field_size) * sizeof(double),
                                       cudaMemcpyHostToDevice, ctx->stream),
                       "field upload");
        }
        if (field <= NDG_FIELD_V) ctx->traces_valid = false;
    });
}

ndg_status ndg_get_field(ndg_ctx* ctx, int32_t instance, int32_t field, double* values) {
    return guarded([&] {
        require_mesh(ctx);
        require_device(ctx);
        if (!values) fail(NDG_ERR_INVALID_ARG, "values is NULL");
        if (instance >= ctx->n_instances) fail(NDG_ERR_INVALID_ARG, "instance out of range");
        make_current(ctx);
        const int first = instance < 0 ? 0 : instance;
        const int last = instance < 0 ? ctx->n_instances : instance + 1;
        for (int i = first; i < last; ++i) {
            const double* src = field_ptr(ctx, field, i);
            check_cuda(cudaMemcpyAsync(values + (i - first) * ctx->field_size, src, static_cast<size_t>(ctx->field_size) * sizeof(double),
                                       cudaMemcpyDeviceToHost, ctx->stream),
                       "field download");
        }
        check_cuda(cudaStreamSynchronize(ctx->stream), "field download");
        check_device_error(ctx);
    });
}

ndg_status ndg_get_delta_t(ndg_ctx* ctx, double* delta_t) {
    return guarded([&] {
        require_mesh(ctx);
        require_device(ctx);
        if (!delta_t) fail(NDG_ERR_INVALID_ARG, "delta_t is NULL");
        *delta_t = ctx->dt_mesh;
    });
}

ndg_status ndg_set_cfl(ndg_ctx* ctx, double cfl) {
    return guarded([&] {
        require_mesh(ctx);
        require_device(ctx);
        if (!(cfl > 0.0) || !std::isfinite(cfl)) fail(NDG_ERR_INVALID_ARG, "cfl must be positive and finite");
        make_current(ctx);
        compute_dt_mesh(ctx, cfl);
    });
}

ndg_status ndg_stage(ndg_ctx* ctx, int32_t m, double time, double dt) {
    return guarded([&] {
        require_mesh(ctx);
        require_device(ctx);
        if (m < 0 || m > 2) fail(NDG_ERR_INVALID_ARG, "stage index must be 0, 1 or 2");
        make_current(ctx);
        set_step(ctx, time, dt, std::numeric_limits<double>::infinity());
        ensure_traces(ctx);
        launch_stage(ctx, m);
    });
}

ndg_status ndg_run(ndg_ctx* ctx, int64_t n_steps, double* time) {
    return guarded([&] {
        require_mesh(ctx);
        require_device(ctx);
        if (n_steps < 0) fail(NDG_ERR_INVALID_ARG, "n_steps must be >= 0");
        make_current(ctx);
        const double t0 = time ? *time : 0.0;
        set_step(ctx, t0, ctx->dt_mesh, std::numeric_limits<double>::infinity());
        run_steps(ctx, n_steps);
        // The device advances time by the same FP64 additions.
        double t = t0;
        for (int64_t s = 0; s < n_steps; ++s) t += ctx->dt_mesh;
        if (time) *time = t;
    });
}

ndg_status ndg_solve(ndg_ctx* ctx, double t_end, double* time, int64_t* n_steps) {
    return guarded([&] {
        require_mesh(ctx);
        require_device(ctx);
        make_current(ctx);
        const int64_t interval = ctx->params.adaptivity_interval;
        if (interval > 0 && ctx->n_instances != 1) fail(NDG_ERR_UNSUPPORTED, "adaptation needs a single instance (the mesh is shared)");
        // The reference loop (Solver2D_t.tcu:35-110): the last step is
        // shortened to land on t_end, and after every adaptivity_interval-th
        // step the error is estimated and the mesh adapted. Steps between
        // adaptations run as graph launches.
        double t = time ? *time : 0.0;
        int64_t steps = 0;
        while (t < t_end) {
            const int64_t limit = interval > 0 ? interval - steps % interval : std::numeric_limits<int64_t>::max();
            const double c0 = t;
            int64_t n = 0;
            while (t < t_end && n < limit) {
                double dt = ctx->dt_mesh;
                if (t + dt > t_end) dt = t_end - t;
                t += dt;
                ++n;
            }
            const double dt0 = (c0 + ctx->dt_mesh > t_end) ? t_end - c0 : ctx->dt_mesh;
            set_step(ctx, c0, dt0, t_end);
            run_steps(ctx, n);
            steps += n;
            if (interval > 0 && n == limit) {
                estimate(ctx);
                adapt_from_estimate(ctx);
            }
        }
        if (time) *time = t;
        if (n_steps) *n_steps = steps;
    });
}

ndg_status ndg_pre_condition(ndg_ctx* ctx, int64_t n_adaptivity_steps, int64_t pre_condition_interval, int32_t iterative, int64_t* n_steps) {
    return guarded([&] {
        require_mesh(ctx);
        require_device(ctx);
        if (pre_condition_interval <= 0) fail(NDG_ERR_INVALID_ARG, "pre-condition needs a positive pre_condition_interval");
        if (n_adaptivity_steps < 0) fail(NDG_ERR_INVALID_ARG, "n_adaptivity_steps must be >= 0");
        if (n_adaptivity_steps > 0 && ctx->n_instances != 1) fail(NDG_ERR_UNSUPPORTED, "adaptation needs a single instance (the mesh is shared)");
        make_current(ctx);
        // Solver2D_t.tpp:136-334: full steps of the current mesh's dt; an
        // estimate and an adaptation after every pre_condition_interval-th
        // step; the initial conditions once at the end (sequential) or after
        // every adaptation with the time restarted (iterative).
        double t = 0.0;
        int64_t steps = 0;
        for (int64_t a = 0; a < n_adaptivity_steps; ++a) {
            set_step(ctx, t, ctx->dt_mesh, std::numeric_limits<double>::infinity());
            run_steps(ctx, pre_condition_interval);
            for (int64_t s = 0; s < pre_condition_interval; ++s) t += ctx->dt_mesh;
            steps += pre_condition_interval;
            estimate(ctx);
            adapt_from_estimate(ctx);
            if (iterative) {
                set_initial_conditions(ctx);
                t = 0.0;
            }
        }
        if (!iterative) set_initial_conditions(ctx);
        if (n_steps) *n_steps = steps;
    });
}

ndg_status ndg_time_stage(ndg_ctx* ctx, int32_t m, int32_t n_launches, double* avg_ms) {
    return guarded([&] {
        require_mesh(ctx);
        require_device(ctx);
        if (m < 0 || m > 2 || n_launches < 1 || !avg_ms) fail(NDG_ERR_INVALID_ARG, "bad stage timing request");
        make_current(ctx);
        ensure_traces(ctx);
        std::vector<cudaEvent_t> ev(static_cast<size_t>(2 * n_launches));
        for (auto& e : ev) check_cuda(cudaEventCreate(&e), "cudaEventCreate");
        for (int i = 0; i < n_launches; ++i) {
            check_cuda(cudaEventRecord(ev[static_cast<size_t>(2 * i)], ctx->stream), "cudaEventRecord");
            launch_stage(ctx, m);
            check_cuda(cudaEventRecord(ev[static_cast<size_t>(2 * i + 1)], ctx->stream), "cudaEventRecord");
        }
        check_cuda(cudaStreamSynchronize(ctx->stream), "stage timing");
        check_device_error(ctx);
        double total = 0.0;
        for (int i = 0; i < n_launches; ++i) {
            float ms = 0.0f;
            check_cuda(cudaEventElapsedTime(&ms, ev[static_cast<size_t>(2 * i)], ev[static_cast<size_t>(2 * i + 1)]), "cudaEventElapsedTime");
            total += ms;
        }
        for (auto& e : ev) cudaEventDestroy(e);
        *avg_ms = total / n_launches;
    });
}

ndg_status ndg_tile_candidates(const ndg_ctx* ctx, int32_t* out, int32_t capacity, int32_t* count, int32_t* default_tile) {
    return guarded([&] {
        require_mesh(ctx);
        if (ctx->general) fail(NDG_ERR_UNSUPPORTED, "tiles are tuned for meshes of one order");
        const std::vector<int> cand = tile_candidates(ctx);
        if (count) *count = static_cast<int32_t>(cand.size());
        if (out) {
            if (capacity < static_cast<int32_t>(cand.size())) fail(NDG_ERR_INVALID_ARG, "output buffer too small");
            std::copy(cand.begin(), cand.end(), out);
        }
        if (default_tile) *default_tile = dev::elements_per_block(ctx->N);
    });
}

ndg_status ndg_set_tile(ndg_ctx* ctx, int32_t elements_per_block) {
    return guarded([&] {
        require_mesh(ctx);
        require_device(ctx);
        if (ctx->general) fail(NDG_ERR_UNSUPPORTED, "tiles are tuned for meshes of one order");
        if (strict(ctx) && elements_per_block != 0) fail(NDG_ERR_UNSUPPORTED, "the strict form keeps its default tile");
        make_current(ctx);
        set_tile(ctx, elements_per_block);
    });
}

ndg_status ndg_autotune(ndg_ctx* ctx, int32_t n_launches, int32_t* elements_per_block, double* best_ms) {
    return guarded([&] {
        require_mesh(ctx);
        require_device(ctx);
        if (n_launches < 1) fail(NDG_ERR_INVALID_ARG, "n_launches must be >= 1");
        make_current(ctx);
        const int form = fp32(ctx) ? 1 : 0;
        if (ctx->general || strict(ctx)) {
            // mixed-order meshes and the strict form keep their tiles
            if (elements_per_block) *elements_per_block = 0;
            if (best_ms) *best_ms = 0.0;
            return;
        }
        // Time on a copy of the state, then restore it.
        const size_t values = ctx->q.count;
        DeviceBuffer<double> q0, k0;
        q0.allocate(values);
        k0.allocate(values);
        check_cuda(cudaMemcpyAsync(q0.ptr, ctx->q.ptr, values * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream), "state copy");
        check_cuda(cudaMemcpyAsync(k0.ptr, ctx->k.ptr, values * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream), "state copy");
        std::vector<int> cand = tile_candidates(ctx);
        cand.insert(cand.begin(), 0);  // the default tile
        cudaEvent_t e0, e1;
        check_cuda(cudaEventCreate(&e0), "cudaEventCreate");
        check_cuda(cudaEventCreate(&e1), "cudaEventCreate");
        int best = 0;
        double best_t = INFINITY;
        for (int epb : cand) {
            set_tile(ctx, epb);
            ensure_traces(ctx);
            launch_stage(ctx, 1);  // warm-up
            check_cuda(cudaEventRecord(e0, ctx->stream), "cudaEventRecord");
            for (int i = 0; i < n_launches; ++i) launch_stage(ctx, 1);
            check_cuda(cudaEventRecord(e1, ctx->stream), "cudaEventRecord");
            check_cuda(cudaStreamSynchronize(ctx->stream), "autotune");
            float ms = 0.0f;
            check_cuda(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime");
            const double t = ms / n_launches;
            if (t < best_t) {
                best_t = t;
                best = epb;
            }
            // restart every candidate from the same state
            check_cuda(cudaMemcpyAsync(ctx->q.ptr, q0.ptr, values * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream), "state restore");
            check_cuda(cudaMemcpyAsync(ctx->k.ptr, k0.ptr, values * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream), "state restore");
            ctx->traces_valid = false;
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        check_device_error(ctx);
        set_tile(ctx, best);
        ctx->tile[form] = best;
        check_cuda(cudaStreamSynchronize(ctx->stream), "autotune");
        if (elements_per_block) *elements_per_block = best;
        if (best_ms) *best_ms = best_t;
    });
}

ndg_status ndg_estimate_error(ndg_ctx* ctx) {
    return guarded([&] {
        require_mesh(ctx);
        require_device(ctx);
        make_current(ctx);
        estimate(ctx);
    });
}

ndg_status ndg_get_error(ndg_ctx* ctx, int32_t instance, double* p_error, double* p_sigma, int32_t* refine, int32_t* coarsen) {
    return guarded([&] {
        require_mesh(ctx);
        require_device(ctx);
        if (!ctx->has_error_estimate) fail(NDG_ERR_INVALID_ARG, "call ndg_estimate_error first");
        if (instance < 0 || instance >= ctx->n_instances) fail(NDG_ERR_INVALID_ARG, "instance out of range");
        make_current(ctx);
        const size_t off = static_cast<size_t>(instance) * static_cast<size_t>(ctx->K);
        const size_t K = static_cast<size_t>(ctx->K);
        if (p_error) check_cuda(cudaMemcpyAsync(p_error, ctx->p_error.ptr + off, K * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream), "error download");
        if (p_sigma) check_cuda(cudaMemcpyAsync(p_sigma, ctx->p_sigma.ptr + off, K * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream), "error download");
        if (refine) check_cuda(cudaMemcpyAsync(refine, ctx->refine.ptr + off, K * sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream), "error download");
        if (coarsen) check_cuda(cudaMemcpyAsync(coarsen, ctx->coarsen.ptr + off, K * sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream), "error download");
        check_cuda(cudaStreamSynchronize(ctx->stream), "error download");
    });
}

ndg_status ndg_adapt(ndg_ctx* ctx) {
    return guarded([&] {
        require_mesh(ctx);
        require_device(ctx);
        if (!ctx->has_error_estimate) fail(NDG_ERR_INVALID_ARG, "call ndg_estimate_error first");
        if (ctx->n_instances != 1) fail(NDG_ERR_UNSUPPORTED, "adaptation needs a single instance (the mesh is shared)");
        make_current(ctx);
        adapt_from_estimate(ctx);
    });
}

ndg_status ndg_adapt_flags(ndg_ctx* ctx, const int32_t* refine, const double* p_sigma) {
    return guarded([&] {
        require_mesh(ctx);
        if (!refine || !p_sigma) fail(NDG_ERR_INVALID_ARG, "refine and p_sigma must not be NULL");
        if (ctx->n_instances != 1) fail(NDG_ERR_UNSUPPORTED, "adaptation needs a single instance (the mesh is shared)");
        make_current(ctx);
        if (ctx->device < 0) {
            adapt_mesh(ctx, refine, p_sigma);  // host-only context: the topology alone, decided on the host
            return;
        }
        // Device contexts take the caller's flags through the device decisions.
        const size_t K = static_cast<size_t>(ctx->K);
        check_cuda(cudaMemcpyAsync(ctx->refine.ptr, refine, K * sizeof(int32_t), cudaMemcpyHostToDevice, ctx->stream), "flag upload");
        check_cuda(cudaMemcpyAsync(ctx->p_sigma.ptr, p_sigma, K * sizeof(double), cudaMemcpyHostToDevice, ctx->stream), "flag upload");
        adapt_from_estimate(ctx);
        ctx->has_error_estimate = false;
    });
}

ndg_status ndg_adapt_timings(const ndg_ctx* ctx, double* ms) {
    return guarded([&] {
        if (!ctx || !ms) fail(NDG_ERR_INVALID_ARG, "NULL argument");
        for (int i = 0; i < 4; ++i) ms[i] = ctx->adapt_ms[i];
    });
}

ndg_status ndg_launch_count(const ndg_ctx* ctx, int64_t* launches) {
    return guarded([&] {
        if (!ctx || !launches) fail(NDG_ERR_INVALID_ARG, "NULL argument");
        *launches = ctx->launches;
    });
}

}  // extern "C"
