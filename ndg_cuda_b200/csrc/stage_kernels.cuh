// Device entry points of the fused stage kernels (stage_kernels.cu).
#pragma once

#include "ndg_internal.hpp"

#include <cuda_runtime.h>

#include <vector>

namespace ndg {
namespace dev {

// Arguments of one RK3 stage over all elements and instances.
// Layouts (FP64): q, k, G_out: [instance][field p,u,v][field_stride][(N+1)^2];
// traces: [instance][field][field_stride][side][N+1], where field_stride is
// the element count rounded up to even; per element side: link, normal,
// gscale, inflow ([element][side]); corners: [element][8].
struct StageArgs {
    double* q;
    double* k;
    const double* trace_in;
    double* trace_out;
    const float* trace_in_f;  // FP32 form: traces kept in FP32
    float* trace_out_f;
    double* G_out;  // optional copy of the stage's time derivative
    const double* corners;
    const int2* link;
    const double2* normal;
    const double* gscale;
    const double4* inflow;
    const double* step;  // {time, dt, dt_mesh, t_end}
    unsigned* error;     // set when a bounded wait gives up
    const double* tc64;  // per-lane tables of the tensor-core passes (TcTable64 / TcTable32 of the order)
    const float* tc32;
    double rk_a, rk_b, rk_g;
    int first;
    int64_t n_elements;
    int64_t field_stride;
    int n_instances;
};

// Side traces of q. With link (the side plan of the uniform stage kernels)
// each interior side's trace goes into the far slots of the neighbour across
// it (neighbour side lk.y & 3, node N - m), the layout the stage kernels
// read; without, into the element's own slots [element][side][node].
struct TraceArgs {
    const double* q;
    double* trace_out;
    float* trace_out_f;  // FP32 form
    int64_t n_elements;
    int64_t field_stride;
    int n_instances;
    const int2* link = nullptr;
};

cudaError_t prepare_kernels(int N, bool strict);
cudaError_t launch_stage(int N, bool strict, const StageArgs& a, cudaStream_t stream);
cudaError_t launch_traces(int N, bool strict, const TraceArgs& a, cudaStream_t stream);
// FP32 form: volume, surface and flux arithmetic in FP32, traces in FP32, the
// RK update of q and k in FP64.
cudaError_t prepare_kernels_f32(int N);
cudaError_t launch_stage_f32(int N, const StageArgs& a, cudaStream_t stream);
cudaError_t launch_traces_f32(int N, const TraceArgs& a, cudaStream_t stream);
cudaError_t launch_initial_conditions(double* q, double* k, const double* corners, int N, int64_t K, int64_t Kp, int n_instances, cudaStream_t stream);
cudaError_t launch_delta_t(const double* delta_xy_min, const int* elem_N, int64_t K, double cfl, double* out, cudaStream_t stream);
cudaError_t launch_end_step(double* step, cudaStream_t stream);
cudaError_t upload_tables(const Tables& t);
// Host copy of the order-N coefficients uploaded by upload_tables: Dhat
// ((N+1)^2), nodes, Lagrange values at -1 and +1, weights, 1/weights.
void host_coefficients(int N, double* dhat, double* xn, double* lm, double* lp, double* w, double* iw);
int elements_per_block(int N);
// Candidate tiles of the autotuner (stage_variants_fp64.cu, _fp32.cu): the
// feasible elements-per-CTA values of order N, and the stage kernel with
// one of them (FP64 default rounding, or the FP32 form).
int tile_candidates_fp64(int N, int* out, int max);
int tile_candidates_fp32(int N, int* out, int max);
cudaError_t prepare_stage_variant_fp64(int N, int epb);
cudaError_t prepare_stage_variant_fp32(int N, int epb);
cudaError_t launch_stage_variant_fp64(int N, int epb, const StageArgs& a, cudaStream_t stream);
cudaError_t launch_stage_variant_fp32(int N, int epb, const StageArgs& a, cudaStream_t stream);
// Tile codes at or above kTensorTile select the tensor-core contraction
// variant with (code - kTensorTile) elements per CTA.
constexpr int kTensorTile = 100;
// Per-lane tables of the tensor-core passes of order N (stage_common.cuh).
std::vector<double> tc_lane_table_fp64(int N);
std::vector<float> tc_lane_table_fp32(int N);

}  // namespace dev
}  // namespace ndg
