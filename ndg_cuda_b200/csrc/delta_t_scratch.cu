// CFL time step over caller-owned device arrays, with no memory allocation
// (ndg_delta_t_from_device in include/ndg_b200.h).
//
// This is a variant of the time-step reduction that ndg_get_delta_t runs at
// mesh load: the same per-element value cfl * delta_xy_min / N^2, rounded the
// same way, reduced to its minimum. Instead of one block over the whole mesh
// it runs one block per 1024 elements, so it needs a place for the blocks'
// partial minima. That place is a fixed array in the library's own device
// image, not memory the call allocates. It serves callers that cannot
// allocate device memory at the point where they need the step: a code that
// hands the solver views into device arrays it manages through its own pool
// and gives the library no memory budget of its own, or a time loop where a
// cudaMalloc/cudaFree pair would synchronise the whole device every step.
//
// Limits and sharing:
//  * at most kMaxElements = 4,194,304 elements per call (a 2048 x 2048
//    mesh); more is rejected with NDG_ERR_INVALID_ARG before any launch;
//  * one scratch array per device, shared by every call on that device: the
//    header (completion counter and result) is cleared on the caller's stream
//    at the start of each call, the partial minima need no clearing. Two
//    calls on the same device that overlap in time (from different host
//    threads, or on different streams) race on the array; callers must
//    serialise them;
//  * every call looks up the array's device address for the current device
//    (cudaGetSymbolAddress), so no address is kept between calls: after the
//    device's context is torn down and rebuilt, the next call finds the
//    array where the reloaded module put it. The first lookup on a device
//    also loads the library's kernels there; make that first call before any
//    stream capture begins on the device;
//  * every call waits for its stream (cudaStreamSynchronize) before it
//    returns, since the result is returned in host memory.
#include "ndg_internal.hpp"

#include <cuda_runtime.h>

#include <cstdint>

namespace {

constexpr int kThreads = 256;
constexpr int kPerThread = 4;
constexpr int64_t kElementsPerBlock = static_cast<int64_t>(kThreads) * kPerThread;
constexpr int kMaxBlocks = 4096;
constexpr int64_t kMaxElements = kElementsPerBlock * kMaxBlocks;
// Header: 256 bytes, double 0 holds the completion counter (as an unsigned),
// double 1 the result. The partial minima follow.
constexpr int kHeaderDoubles = 32;
constexpr int kScratchDoubles = kHeaderDoubles + kMaxBlocks;  // 33,024 bytes

}  // namespace

// The scratch array. Host code reaches it only through the address that
// cudaGetSymbolAddress returns for the current device.
static __device__ __align__(256) double g_delta_t_scratch[kScratchDoubles];

namespace ndg {
namespace {

__device__ __forceinline__ double warp_min(double v) {
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Block b reduces elements [1024 b, 1024 (b+1)) into scratch[header + b]; the
// last block to finish reduces the partials into scratch[1]. Element values
// and fmin are those of delta_t_kernel, so the minimum is bit-identical.
__global__ void __launch_bounds__(kThreads) delta_t_scratch_kernel(const double* __restrict__ delta_xy_min,
                                                                   const int* __restrict__ elem_N, int64_t K,
                                                                   double cfl, double* scratch) {
    __shared__ double block_min[kThreads / 32];
    __shared__ int is_last;
    const double inf = __longlong_as_double(0x7FF0000000000000ll);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double v = inf;
    const int64_t base = static_cast<int64_t>(blockIdx.x) * kElementsPerBlock;
    for (int j = 0; j < kPerThread; ++j) {
        const int64_t e = base + j * kThreads + threadIdx.x;
        if (e < K) {
            const int Ne = elem_N[e];
            v = fmin(v, __ddiv_rn(__dmul_rn(cfl, delta_xy_min[e]), static_cast<double>(Ne * Ne)));
        }
    }
    v = warp_min(v);
    if (lane == 0) block_min[warp] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = block_min[0];
        for (int w = 1; w < kThreads / 32; ++w) m = fmin(m, block_min[w]);
        scratch[kHeaderDoubles + blockIdx.x] = m;
        __threadfence();
        const unsigned done = atomicAdd(reinterpret_cast<unsigned*>(scratch), 1u);
        is_last = (done == gridDim.x - 1) ? 1 : 0;
    }
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    v = inf;
    for (int b = threadIdx.x; b < static_cast<int>(gridDim.x); b += kThreads) v = fmin(v, __ldcg(scratch + kHeaderDoubles + b));
    v = warp_min(v);
    if (lane == 0) block_min[warp] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = block_min[0];
        for (int w = 1; w < kThreads / 32; ++w) m = fmin(m, block_min[w]);
        scratch[1] = m;
    }
}

// The device address of the scratch array on the current device, looked up
// on every call: a cached address could outlive the context it came from.
double* scratch_for_current_device() {
    double* ptr = nullptr;
    const cudaError_t err = cudaGetSymbolAddress(reinterpret_cast<void**>(&ptr), g_delta_t_scratch);
    if (err != cudaSuccess || !ptr)
        fail(NDG_ERR_CUDA, std::string("scratch address lookup: ") + cudaGetErrorString(err));
    return ptr;
}

// The kernel dereferences both arrays, so host pointers that the device
// cannot reach are refused here rather than faulting there.
void require_device_pointer(const void* p, int device, const char* name) {
    if (!p) fail(NDG_ERR_INVALID_ARG, std::string(name) + " is NULL");
    cudaPointerAttributes attr{};
    const cudaError_t err = cudaPointerGetAttributes(&attr, p);
    if (err != cudaSuccess) fail(NDG_ERR_CUDA, std::string("pointer attributes of ") + name + ": " + cudaGetErrorString(err));
    if (attr.type == cudaMemoryTypeUnregistered)
        fail(NDG_ERR_INVALID_ARG, std::string(name) + " is not device-accessible memory");
    if (attr.type == cudaMemoryTypeDevice && attr.device != device)
        fail(NDG_ERR_INVALID_ARG, std::string(name) + " lives on another device than the current one");
}

}  // namespace
}  // namespace ndg

extern "C" ndg_status ndg_delta_t_from_device(const double* delta_xy_min, const int32_t* elem_N, int64_t n_elements,
                                              double cfl, void* stream, double* delta_t) {
    using namespace ndg;
    try {
        if (!delta_t) fail(NDG_ERR_INVALID_ARG, "delta_t is NULL");
        if (n_elements < 1) fail(NDG_ERR_INVALID_ARG, "n_elements must be at least 1");
        if (n_elements > kMaxElements)
            fail(NDG_ERR_INVALID_ARG, "n_elements exceeds the scratch limit of 4194304 elements per call");
        int device = -1;
        cudaError_t err = cudaGetDevice(&device);
        if (err != cudaSuccess) fail(NDG_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(err));
        require_device_pointer(delta_xy_min, device, "delta_xy_min");
        require_device_pointer(elem_N, device, "elem_N");
        const cudaStream_t s = static_cast<cudaStream_t>(stream);
        if (s) {
            int stream_device = -1;
            err = cudaStreamGetDevice(s, &stream_device);
            if (err != cudaSuccess) fail(NDG_ERR_INVALID_ARG, std::string("stream: ") + cudaGetErrorString(err));
            if (stream_device != device) fail(NDG_ERR_INVALID_ARG, "stream belongs to another device than the current one");
        }
        double* scratch = scratch_for_current_device();
        err = cudaMemsetAsync(scratch, 0, kHeaderDoubles * sizeof(double), s);
        if (err != cudaSuccess) fail(NDG_ERR_CUDA, std::string("scratch clear: ") + cudaGetErrorString(err));
        const unsigned blocks = static_cast<unsigned>((n_elements + kElementsPerBlock - 1) / kElementsPerBlock);
        delta_t_scratch_kernel<<<blocks, kThreads, 0, s>>>(delta_xy_min, elem_N, n_elements, cfl, scratch);
        err = cudaGetLastError();
        if (err != cudaSuccess) fail(NDG_ERR_CUDA, std::string("delta_t kernel: ") + cudaGetErrorString(err));
        err = cudaMemcpyAsync(delta_t, scratch + 1, sizeof(double), cudaMemcpyDeviceToHost, s);
        if (err != cudaSuccess) fail(NDG_ERR_CUDA, std::string("delta_t readback: ") + cudaGetErrorString(err));
        err = cudaStreamSynchronize(s);
        if (err != cudaSuccess) fail(NDG_ERR_CUDA, std::string("delta_t: ") + cudaGetErrorString(err));
        set_last_error("");
        return NDG_OK;
    } catch (const Error& e) {
        set_last_error(e.message);
        return e.status;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return NDG_ERR_INVALID_ARG;
    }
}
