// Device entry points of the error estimator (estimator.cu).
#pragma once

#include "ndg_internal.hpp"

#include <cuda_runtime.h>

namespace ndg {
namespace dev {

// One launch covers `count` elements of order N. q: [instance][field][block]
// with element e at off2[e] (e (N+1)^2 when off2 is null); outputs
// [instance][n_elements] at the element numbers ids[] (0 .. count-1 when
// ids is null).
struct EstimatorArgs {
    const double* q;
    double* p_error;
    double* p_sigma;
    int* refine;
    int* coarsen;
    double tolerance_min;
    double tolerance_max;
    int64_t count;
    int64_t n_elements;
    int64_t block;
    const int64_t* ids;
    const int64_t* off2;
    int n_instances;
    int N;
};

cudaError_t upload_polynomials(const Tables& t);
cudaError_t launch_estimate_error(const EstimatorArgs& a, cudaStream_t stream);

}  // namespace dev
}  // namespace ndg
