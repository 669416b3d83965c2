// selftest.cu - exhaustive check of the library's short-path correctly
// rounded reciprocal (rcp_rn, gm1b_common.cuh) against CUDA's __frcp_rn on
// all 2^32 binary32 words.  A run takes a few milliseconds on a B200; the
// kernels that use rcp_rn are word-identical to __frcp_rn exactly when this
// reports zero mismatches.
#include "gm1b_common.cuh"

namespace gm1b {
namespace {

__global__ void __launch_bounds__(256) reciprocal_selftest_kernel(unsigned long long *counts, unsigned *first) {
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    unsigned long long bad = 0, fast = 0;
    for (unsigned long long w = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; w < (1ull << 32);
         w += stride) {
        const float b = __uint_as_float((unsigned)w);
        const float ab = fabsf(b);
        if (ab >= 0x1p-125f && ab <= 0x1p125f) ++fast;
        if (__float_as_uint(rcp_rn(b)) != __float_as_uint(__frcp_rn(b))) {
            ++bad;
            atomicMin(first, (unsigned)w);
        }
    }
    if (bad) atomicAdd(counts, bad);
    atomicAdd(counts + 1, fast);
}

}  // namespace
}  // namespace gm1b

using namespace gm1b;

extern "C" int32_t gm1b_selftest_reciprocal(unsigned long long *device_counts, uint32_t *device_first_mismatch,
                                            void *stream) {
    if (device_counts == nullptr || device_first_mismatch == nullptr) {
        gm1b_set_error("gm1b_selftest_reciprocal: need the two device result buffers");
        return GM1B_ERR_ARGUMENT;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (cudaMemsetAsync(device_counts, 0, 2 * sizeof(unsigned long long), st) != cudaSuccess ||
        cudaMemsetAsync(device_first_mismatch, 0xff, sizeof(uint32_t), st) != cudaSuccess) {
        cudaGetLastError();
        gm1b_set_error("gm1b_selftest_reciprocal: result reset failed");
        return GM1B_ERR_CUDA;
    }
    reciprocal_selftest_kernel<<<148 * 8, 256, 0, st>>>(device_counts, device_first_mismatch);
    const cudaError_t e = cudaPeekAtLastError();
    if (e != cudaSuccess) {
        cudaGetLastError();
        gm1b_set_error("gm1b_selftest_reciprocal: %s", cudaGetErrorString(e));
        return GM1B_ERR_CUDA;
    }
    return GM1B_OK;
}
