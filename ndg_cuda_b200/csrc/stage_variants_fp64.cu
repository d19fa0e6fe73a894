// Autotuner candidate tiles of the FP64 stage kernel (stage_variants.cuh):
// the SIMT tiles here, the tensor-core tiles (codes kTensorTile + E) in
// stage_variants_tc64.cu.
#include "stage_variants.cuh"

namespace ndg {
namespace dev {

int tile_candidates_tc64(int N, int* out, int max);
cudaError_t prepare_stage_variant_tc64(int N, int epb);
cudaError_t launch_stage_variant_tc64(int N, int epb, const StageArgs& a, cudaStream_t stream);

namespace {
int simt_candidates(int N, int* out, int max) {
#define NDG_CALL(n) return variant_candidates<false, n, false>(out, max)
    NDG_VARIANT_ORDERS(NDG_CALL)
#undef NDG_CALL
    return 0;
}
}  // namespace

int tile_candidates_fp64(int N, int* out, int max) {
    const int c = simt_candidates(N, out, max);
    return c + tile_candidates_tc64(N, out + c, max - c);
}

cudaError_t prepare_stage_variant_fp64(int N, int epb) {
    if (epb >= kTensorTile) return prepare_stage_variant_tc64(N, epb - kTensorTile);
#define NDG_CALL(n) return variant_prepare_n<false, n, false>(epb)
    NDG_VARIANT_ORDERS(NDG_CALL)
#undef NDG_CALL
    return cudaErrorInvalidValue;
}

cudaError_t launch_stage_variant_fp64(int N, int epb, const StageArgs& a, cudaStream_t stream) {
    if (epb >= kTensorTile) return launch_stage_variant_tc64(N, epb - kTensorTile, a, stream);
#define NDG_CALL(n) return variant_launch_n<false, n, false>(epb, a, stream)
    NDG_VARIANT_ORDERS(NDG_CALL)
#undef NDG_CALL
    return cudaErrorInvalidValue;
}

}  // namespace dev
}  // namespace ndg
