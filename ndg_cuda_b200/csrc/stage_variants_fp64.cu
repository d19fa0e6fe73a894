// Autotuner candidate tiles of the FP64 stage kernel (stage_variants.cuh).
#include "stage_variants.cuh"

namespace ndg {
namespace dev {

int tile_candidates_fp64(int N, int* out, int max) {
#define NDG_CALL(n) return variant_candidates<false, n>(out, max)
    NDG_VARIANT_ORDERS(NDG_CALL)
#undef NDG_CALL
    return 0;
}

cudaError_t prepare_stage_variant_fp64(int N, int epb) {
#define NDG_CALL(n) return variant_prepare_n<false, n>(epb)
    NDG_VARIANT_ORDERS(NDG_CALL)
#undef NDG_CALL
    return cudaErrorInvalidValue;
}

cudaError_t launch_stage_variant_fp64(int N, int epb, const StageArgs& a, cudaStream_t stream) {
#define NDG_CALL(n) return variant_launch_n<false, n>(epb, a, stream)
    NDG_VARIANT_ORDERS(NDG_CALL)
#undef NDG_CALL
    return cudaErrorInvalidValue;
}

}  // namespace dev
}  // namespace ndg
