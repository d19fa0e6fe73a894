// Internal host types of the C ABI shared by context.cu (contexts, meshes,
// stepping) and adjoint_host.cu (adjoint problems): device buffers, CUDA
// error mapping, the RK3 coefficients and the solver context itself.
#pragma once

#include "general_kernels.cuh"
#include "ndg_internal.hpp"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <exception>
#include <new>
#include <string>
#include <vector>

namespace ndg {

inline void check_cuda(cudaError_t err, const char* what) {
    if (err != cudaSuccess) {
        const ndg_status st = (err == cudaErrorMemoryAllocation) ? NDG_ERR_OOM : NDG_ERR_CUDA;
        fail(st, std::string(what) + ": " + cudaGetErrorString(err));
    }
}

template <typename T>
struct DeviceBuffer {
    T* ptr = nullptr;
    size_t count = 0;
    DeviceBuffer() = default;
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    void swap(DeviceBuffer& o) noexcept {
        std::swap(ptr, o.ptr);
        std::swap(count, o.count);
    }
    void upload(const std::vector<T>& v, cudaStream_t stream) {
        allocate(std::max<size_t>(v.size(), 1));
        if (!v.empty()) check_cuda(cudaMemcpyAsync(ptr, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, stream), "mesh upload");
    }
    // At least n values, keeping the allocation when it is large enough
    // (scratch reused from call to call; grows by half again when it is not).
    void reserve(size_t n) {
        if (n <= count && ptr) return;
        allocate(std::max<size_t>(n + n / 2, 1));
    }
    void upload_reuse(const std::vector<T>& v, cudaStream_t stream) {
        reserve(std::max<size_t>(v.size(), 1));
        if (!v.empty()) check_cuda(cudaMemcpyAsync(ptr, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, stream), "mesh upload");
    }
    void allocate(size_t n) {
        release();
        if (n == 0) return;
        check_cuda(cudaMalloc(reinterpret_cast<void**>(&ptr), n * sizeof(T)), "cudaMalloc");
        count = n;
    }
    void release() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        count = 0;
    }
    ~DeviceBuffer() { release(); }
};

// Williamson low-storage RK3 coefficients (include/solvers/Solver2D_t.tpp:16-18).
inline constexpr double kRkA[3] = {0, -5.0 / 9.0, -153.0 / 128.0};
inline constexpr double kRkB[3] = {0, 1.0 / 3.0, 0.75};
inline constexpr double kRkG[3] = {1.0 / 3.0, 15.0 / 16.0, 8.0 / 15.0};

}  // namespace ndg

struct ndg_ctx {
    int device = -1;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int precision = NDG_FP64;
    bool keep_derivative = false;

    bool has_tables = false;
    ndg::Tables tables;

    bool has_mesh = false;
    ndg::Topology topo;
    ndg_mesh_params params{};
    int n_instances = 1;
    int N = 0;
    int64_t K = 0;
    int64_t field_size = 0;  // values per field and instance seen through the API: K (N+1)^2
    int64_t Kp = 0;          // elements per device field block: K rounded up to even
    int64_t block = 0;       // values per device field block: Kp (N+1)^2

    ndg::DeviceBuffer<double> q, k, G, tr[2], corners, normal, gscale, inflow, dxy, step, scratch;
    ndg::DeviceBuffer<float> tr32[2];  // traces of the FP32 form
    ndg::DeviceBuffer<double> tc64;    // per-lane tables of the tensor-core stage passes (order N)
    ndg::DeviceBuffer<float> tc32;
    ndg::DeviceBuffer<int32_t> link, elem_N;
    ndg::DeviceBuffer<unsigned> error;
    ndg::DeviceBuffer<double> p_error, p_sigma;
    ndg::DeviceBuffer<int32_t> refine, coarsen;
    // The adaptation's decisions on the device (adapt_device.cu): a copy of
    // the topology they read, uploaded at each adaptation, and their outputs.
    ndg::DeviceBuffer<int32_t> av_split;
    ndg::DeviceBuffer<int64_t> av_enodes, av_sface_start, av_sface, av_fnodes, av_felem, av_fside, av_if, av_boundary;
    ndg::DeviceBuffer<double> av_node_xy;
    ndg::DeviceBuffer<uint8_t> ad_code, ad_add, ad_frefine, ad_split_flags;
    ndg::DeviceBuffer<int64_t> ad_split_prefix, ad_refined_prefix, ad_scan;
    // Host wall time of the last adaptation by phase, in ms: decisions on
    // the device, topology rebuild, field transfer, device plan.
    double adapt_ms[4] = {0, 0, 0, 0};
    bool has_error_estimate = false;
    int cur = 0;
    bool traces_valid = false;
    double dt_mesh = 0.0;

    // Mixed-order meshes (after adaptation) run the general stage path.
    bool general = false;
    ndg::GeneralPlan gplan;
    ndg::DeviceBuffer<int32_t> g_eN, g_fN, g_gkind, g_gsrc_side;
    ndg::DeviceBuffer<int64_t> g_off2, g_off1, g_enodes, g_sface_start, g_sface, g_foff, g_fnodes, g_felem, g_fside, g_gsrc, g_ids;
    ndg::DeviceBuffer<double> g_corners, g_node_xy, g_fnormal, g_ftangent, g_foffset, g_fscale, g_gscale;
    ndg::DeviceBuffer<double> getr[2];  // element side traces, double-buffered between stages
    ndg::DeviceBuffer<float> getr32[2]; // the same in the FP32 form (allocated when it first runs)
    ndg::DeviceBuffer<double> gsflux;   // element side fluxes of the split launch (mixed launch 2, allocated when it first runs)
    ndg::DeviceBuffer<float> gsflux32;
    int side_slots = 1;                 // largest sum of (face order + 1) over one element side
    ndg::DeviceBuffer<int64_t> g_sw_off, g_sm_off, g_fw_off, g_fm_off, g_fbase;  // mortar weight offsets, face-side trace bases
    ndg::DeviceBuffer<int32_t> g_fsN;                                            // face-side element orders
    ndg::DeviceBuffer<double> g_sw, g_fw;                              // mortar weights
    ndg::DeviceBuffer<int32_t> g_smatch, g_fmatch;                     // mortar node matches
    ndg::DeviceBuffer<int64_t> g_pslot_start, g_slot_desc, g_slot_src;  // face-node slots of the sides, list order
    ndg::DeviceBuffer<double> g_slot_normal;
    ndg::DeviceBuffer<int32_t> g_pside_mode, g_slot_side;
    ndg::DeviceBuffer<int64_t> g_cnb;  // conforming position sides: neighbour trace base, role, face normal
    ndg::DeviceBuffer<int32_t> g_crole;
    ndg::DeviceBuffer<double> g_cnormal;
    ndg::DeviceBuffer<int64_t> g_pq_start, g_pq_woff, g_pq_moff;        // mortar side entries, list order
    ndg::DeviceBuffer<int32_t> g_pq_N;
    ndg::DeviceBuffer<double> g_pq_scale;
    ndg::DeviceBuffer<int64_t> g_poff2, g_poff1;                       // offsets and corners in list order
    ndg::DeviceBuffer<double> g_pcorners;
    ndg::DeviceBuffer<int64_t> g_gq_start, g_gq_face, g_gq_base, g_gq_woff, g_gq_moff;  // ghost side-0 gathers
    ndg::DeviceBuffer<int32_t> g_gq_fs, g_gq_N;
    ndg::DeviceBuffer<double> g_gframe;
    ndg::DeviceBuffer<int64_t> g_gdirect;
    std::vector<ndg::dev::OrderGroup> groups;        // mostly-conforming orders split (conforming parts last)
    std::vector<ndg::dev::OrderGroup> whole_groups;  // one group per order: first traces and the stage queue
    ndg::dev::GeneralMesh gmesh;
    // Mixed-order stages: one launch per order group as concurrent graph
    // branches (mixed_launch 0, the default), or one launch per stage over
    // the stage queue, every tile of every group (mixed_launch 1).
    ndg::DeviceBuffer<ndg::dev::QueueTile> g_queue;
    ndg::dev::StageQueue queue;
    int mixed_launch = 0;

    // Streams and events on which the order groups of a mixed-order stage
    // run concurrently (forked from and joined to `stream`).
    std::vector<cudaStream_t> aux_streams;
    std::vector<cudaEvent_t> aux_events;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    int64_t launches = 0;
    // Incremented whenever the topology or its device plan changes (load,
    // adaptation): objects built on the mesh (adjoint problems) check it.
    int64_t mesh_version = 0;
    // Elements per CTA of the uniform stage kernel chosen by the autotuner
    // (or by hand) for the FP64 and FP32 forms; 0 = the default tile.
    int tile[2] = {0, 0};

    ~ndg_ctx() {
        for (auto& g : graph)
            if (g) cudaGraphExecDestroy(g);
        for (auto& e : aux_events) cudaEventDestroy(e);
        for (auto& st : aux_streams) cudaStreamDestroy(st);
        if (own_stream && stream) cudaStreamDestroy(stream);
    }
};

namespace ndg {

inline void require_device(const ndg_ctx* c) {
    if (c->device < 0) fail(NDG_ERR_INVALID_ARG, "this call needs a GPU context (device >= 0)");
}

inline void require_mesh(const ndg_ctx* c) {
    if (!c->has_mesh) fail(NDG_ERR_INVALID_ARG, "no mesh loaded");
}

inline void make_current(const ndg_ctx* c) {
    if (c->device >= 0) check_cuda(cudaSetDevice(c->device), "cudaSetDevice");
}

// Runs f, converting an ndg::Error (or an allocation failure) into a status
// and the thread's last-error message.
template <typename F>
ndg_status guarded(F&& f) {
    try {
        f();
        set_last_error("");
        return NDG_OK;
    } catch (const Error& e) {
        set_last_error(e.message);
        return e.status;
    } catch (const std::bad_alloc&) {
        set_last_error("host allocation failed");
        return NDG_ERR_OOM;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return NDG_ERR_INVALID_ARG;
    }
}

}  // namespace ndg
