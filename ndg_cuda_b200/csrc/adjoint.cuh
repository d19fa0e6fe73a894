// Device entry points of the variable-speed forward stage and of its
// discrete adjoint (adjoint_kernels.cu), for meshes of one order with
// conforming faces (the uniform path's side plan) and no inflow sides.
//
// The operator: a wave speed c_e > 0 per element in
//   p_t + c (u_x + v_y) = 0,   u_t + c p_x = 0,   v_t + c p_y = 0,
// i.e. the reference's fluxes (Solver2D_t.cpp:31-37) times c_e inside
// element e, and its upwind face flux (Solver2D_t.cpp:48-63, w = p +- u.n)
// times the face speed (c_left + c_right) / 2. With c = 1 it is the
// reference's operator.
//
// Layouts as the stage kernels: fields [field p,u,v][Kp][(N+1)^2], traces
// and adjoint traces [field][Kp][side][N+1]; per element side link, normal
// and gscale of the side plan; speeds [Kp] (the pad element's speed is 1).
//
// Two arithmetic forms. FP64: everything in FP64. FP32: traces, fluxes,
// metrics, the volume term and their transposes in FP32 (traces and adjoint
// traces stored in FP32); the states q, k, lq, lk, the RK updates, the
// misfit and the gradient accumulators stay FP64.
#pragma once

#include "ndg_internal.hpp"

#include <cuda_runtime.h>

#include <cstdint>

namespace ndg {
namespace dev {

constexpr int kMaxReceivers = 64;

// Receivers: the element holding each one and its (N+1)^2 interpolation
// weights (Lagrange basis products at its reference coordinates).
struct Receivers {
    int n = 0;
    int32_t elem[kMaxReceivers];
    const double* w = nullptr;  // [n][(N+1)^2]
};

// One RK3 stage of the variable-speed operator:
//   G = L(c) q,  k = a k + G (k = G when first),  q += gdt k.
struct SpeedStageArgs {
    double* q;
    double* k;
    const double* trace_in;  // side traces of q (the previous stage's output)
    double* trace_out;       // side traces of the new q
    const float* trace_in_f;  // the same in the FP32 form
    float* trace_out_f;
    double* q_save;          // optional: copy of the stage input q
    double* G_out;           // optional: copy of G
    double* samples;         // optional: receivers' pressure of the new q
    const double* corners;
    const int2* link;
    const double2* normal;
    const double* gscale;
    const double* c;
    double rk_a, gdt;
    int first;
    int64_t n_elements, field_stride;
    Receivers rec;
};

// One stage of the adjoint, in reverse order. With mu = lk + gdt lq (the
// adjoint of the stage's k update):
//   lq += L(c)^T mu,  lk = a mu,
//   acc[e] += d/dc of (mu . L(c) qs) split as [volume, side 0..3],
// then, when inject, lq += wdt (P_r qs - target_r) P_r^T on the pressure
// (the misfit's derivative at the state qs), and the adjoint far traces of
// the next stage's mu' = lk + gdt_next lq are published to atr_out.
struct AdjointStageArgs {
    double* lq;
    double* lk;
    const double* qs;      // the forward stage's input
    const double* atr_in;  // neighbours' adjoint far traces of mu
    double* atr_out;       // this element's adjoint far traces of mu'
    const float* atr_in_f;  // the same in the FP32 form
    float* atr_out_f;
    double* acc;           // [Kp][5]
    const double* corners;
    const int2* link;
    const double2* normal;
    const double* gscale;
    const double* c;
    const double* target;  // [n receivers], when inject
    double rk_a, gdt, gdt_next, wdt;
    int inject;
    int64_t n_elements, field_stride;
    Receivers rec;
};

cudaError_t prepare_speed_kernels(int N, bool fp32);
cudaError_t launch_speed_stage(int N, bool fp32, const SpeedStageArgs& a, cudaStream_t stream);
cudaError_t launch_adjoint_stage(int N, bool fp32, const AdjointStageArgs& a, cudaStream_t stream);
// grad_c[e] = acc[e][0] + sum over sides of acc[e][1+s] (boundary sides) or
// (acc[e][1+s] + acc[nb][1+s']) / 2 (sides shared with element nb, side s').
cudaError_t launch_speed_gradient(const double* acc, const int2* link, int64_t K, double* grad_c, cudaStream_t stream);
int adjoint_elements_per_block(int N, bool fp32);

}  // namespace dev
}  // namespace ndg
