// selftest.cu -- device-side self-checks exposed through the C ABI.
//
// fr_selftest_philox runs the engine's Philox4x32-10 (frmath.cuh) and cuRAND's
// curand_Philox4x32_10 on the same counters and keys, so a test can check the generator that
// drives every sample against an independent device implementation of the published algorithm.
#include <curand_philox4x32_x.h>

#include <vector>

#include "fresnel_b200.h"
#include "frmath.cuh"

namespace {

__global__ void k_philox(const uint32_t* in, uint32_t n, uint32_t* ours, uint32_t* theirs)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const uint32_t* a = in + 6 * size_t(i);
    fr::U4 r = fr::philox(a[0], a[1], a[2], a[3], a[4], a[5]);
    ours[4 * size_t(i) + 0] = r.x;
    ours[4 * size_t(i) + 1] = r.y;
    ours[4 * size_t(i) + 2] = r.z;
    ours[4 * size_t(i) + 3] = r.w;
    uint4 c = make_uint4(a[0], a[1], a[2], a[3]);
    uint2 k = make_uint2(a[4], a[5]);
    uint4 t = curand_Philox4x32_10(c, k);
    theirs[4 * size_t(i) + 0] = t.x;
    theirs[4 * size_t(i) + 1] = t.y;
    theirs[4 * size_t(i) + 2] = t.z;
    theirs[4 * size_t(i) + 3] = t.w;
}

}  // namespace

extern "C" FR_API fr_status fr_selftest_philox(const uint32_t* in, uint32_t n, uint32_t* ours,
                                               uint32_t* curand_out)
{
    if (!in || !ours || !curand_out || n == 0)
        return FR_ERR_INVALID;
    int avail = 0;
    fr_get_num_available_devices(&avail);
    if (avail == 0)
        return FR_ERR_UNSUPPORTED;
    uint32_t *d_in = nullptr, *d_a = nullptr, *d_b = nullptr;
    size_t nin = size_t(n) * 6 * sizeof(uint32_t), nout = size_t(n) * 4 * sizeof(uint32_t);
    fr_status st = FR_OK;
    if (cudaMalloc(&d_in, nin) != cudaSuccess || cudaMalloc(&d_a, nout) != cudaSuccess ||
        cudaMalloc(&d_b, nout) != cudaSuccess) {
        st = FR_ERR_OUT_OF_MEMORY;
    } else if (cudaMemcpy(d_in, in, nin, cudaMemcpyHostToDevice) != cudaSuccess) {
        st = FR_ERR_CUDA;
    } else {
        k_philox<<<(n + 255) / 256, 256>>>(d_in, n, d_a, d_b);
        if (cudaMemcpy(ours, d_a, nout, cudaMemcpyDeviceToHost) != cudaSuccess ||
            cudaMemcpy(curand_out, d_b, nout, cudaMemcpyDeviceToHost) != cudaSuccess)
            st = FR_ERR_CUDA;
    }
    cudaFree(d_in);
    cudaFree(d_a);
    cudaFree(d_b);
    return st;
}
