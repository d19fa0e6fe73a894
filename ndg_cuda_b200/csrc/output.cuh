// Output interpolation of the solution on the device (Mesh2D_t::get_solution
// and get_complete_solution; see output.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace ndg {
namespace dev {

struct OutputArgs {
    const double* q;         // field blocks of p, u, v of one instance (block values apart)
    const double* G;         // time derivative blocks of the same instance, or null
    int64_t block;           // values per field block
    const int32_t* N;        // [K] order of each domain element
    const int64_t* off2;     // [K] first value of each element within a field block
    const double* corners;   // [K][8] x0, y0, x1, y1, x2, y2, x3, y3
    const double* interp;    // interpolation matrices, order by order
    const int64_t* interp_off;  // [N_max + 1] first value of order N's n_interp x (N + 1) matrix
    const double* nodes;     // Gauss nodes, order by order
    const int64_t* nodes_off;   // [N_max + 1] first node of order N
    int64_t K;
    int n_interp;
    double time;             // time of the analytic solution
    // outputs, K n_interp^2 values each (point (i, j) of element e at
    // e n_interp^2 + i n_interp + j); any may be null
    double *x, *y, *p, *u, *v, *dp_dt, *du_dt, *dv_dt, *p_err, *u_err, *v_err;
};

cudaError_t launch_output(const OutputArgs& a, int max_N, cudaStream_t stream);

// L2 error against the reference plane wave at `time`: per domain element
// and field, sum_ij w_i w_j J_ij (q_ij - g_ij)^2 into partial[3 e + f].
struct L2Args {
    const double* q;          // field blocks of p, u, v of one instance
    int64_t block;
    const int32_t* N;
    const int64_t* off2;
    const double* corners;    // [K][8]
    const double* nodes;      // Gauss nodes, order by order
    const double* weights;    // Gauss weights, order by order
    const int64_t* vec_off;   // [N_max + 1] first node of order N in nodes / weights
    int64_t K;
    double time;
    double* partial;          // [K][3]
};

cudaError_t launch_l2_error(const L2Args& a, cudaStream_t stream);

}  // namespace dev
}  // namespace ndg
