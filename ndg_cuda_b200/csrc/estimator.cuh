// Device entry points of the error estimator (estimator.cu).
#pragma once

#include "ndg_internal.hpp"

#include <cuda_runtime.h>

namespace ndg {
namespace dev {

// Layouts: q as in StageArgs ([instance][field][field_stride][(N+1)^2]);
// outputs [instance][element].
struct EstimatorArgs {
    const double* q;
    double* p_error;
    double* p_sigma;
    int* refine;
    int* coarsen;
    double tolerance_min;
    double tolerance_max;
    int64_t n_elements;
    int64_t field_stride;
    int n_instances;
    int N;
};

cudaError_t upload_polynomials(const Tables& t);
cudaError_t launch_estimate_error(const EstimatorArgs& a, cudaStream_t stream);

}  // namespace dev
}  // namespace ndg
