// Tensor-core variants of the FP64 stage kernel (the contraction passes on
// DMMA m16n8k4; stage_templates.cuh): tile codes kTensorTile + E for
// E = 2, 4, 8 elements per CTA, orders kTensorMinOrder and up.
#include "stage_variants.cuh"

namespace ndg {
namespace dev {

int tile_candidates_tc64(int N, int* out, int max) {
    if (max <= 0) return 0;
#define NDG_CALL(n) return variant_candidates<false, n, true>(out, max)
    NDG_VARIANT_ORDERS(NDG_CALL)
#undef NDG_CALL
    return 0;
}

cudaError_t prepare_stage_variant_tc64(int N, int epb) {
#define NDG_CALL(n) return variant_prepare_n<false, n, true>(epb)
    NDG_VARIANT_ORDERS(NDG_CALL)
#undef NDG_CALL
    return cudaErrorInvalidValue;
}

cudaError_t launch_stage_variant_tc64(int N, int epb, const StageArgs& a, cudaStream_t stream) {
#define NDG_CALL(n) return variant_launch_n<false, n, true>(epb, a, stream)
    NDG_VARIANT_ORDERS(NDG_CALL)
#undef NDG_CALL
    return cudaErrorInvalidValue;
}

}  // namespace dev
}  // namespace ndg
