// probe.cu — copy-bandwidth probe of the device this library runs on.
//
// aefdtd_probe_copy_bandwidth copies the first half of a device buffer into
// the second half `reps` times (16-byte loads and stores, L2-cached) and
// reports bytes read plus written per second. Over a buffer smaller than the
// 126 MB L2 the copy runs out of L2 after the first pass: that is the ceiling
// against which the batches (whose subsets are sized to stay in L2) are
// measured. Over a buffer far larger than L2 it is an HBM copy.
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/aefdtd.h"

namespace {

__global__ void copy_halves(const float4 *__restrict__ src, float4 *__restrict__ dst, size_t n, int reps) {
    for (int r = 0; r < reps; ++r)
        for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
            float4 v = __ldcg(src + i);
            v.x += 1.0f;
            __stcg(dst + i, v);
        }
}

}  // namespace

extern "C" aefdtd_status aefdtd_probe_copy_bandwidth(int32_t device, size_t bytes, int32_t reps, double *gbs) {
    if (!gbs || reps < 1 || bytes < 4096) return AEFDTD_BAD_ARG;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return AEFDTD_NO_DEVICE;
    }
    if (device < 0 || device >= n) return AEFDTD_BAD_ARG;
    int prev = 0;
    cudaGetDevice(&prev);
    if (cudaSetDevice(device) != cudaSuccess) {
        cudaGetLastError();
        return AEFDTD_CUDA_ERROR;
    }
    aefdtd_status st = AEFDTD_OK;
    void *buf = nullptr;
    cudaStream_t s = nullptr;
    cudaEvent_t a = nullptr, b = nullptr;
    const size_t half = (bytes / 2) / 16;   // float4 elements per half
    int sms = 0;
    if (cudaMalloc(&buf, 2 * half * 16) != cudaSuccess) {
        st = AEFDTD_OOM;
    } else if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
               cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess ||
               cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess ||
               cudaMemsetAsync(buf, 0, 2 * half * 16, s) != cudaSuccess) {
        st = AEFDTD_CUDA_ERROR;
    } else {
        const float4 *src = static_cast<const float4 *>(buf);
        float4 *dst = static_cast<float4 *>(buf) + half;
        const int grid = sms * 8;
        copy_halves<<<grid, 256, 0, s>>>(src, dst, half, 1);   // warm-up: brings the buffer into L2 when it fits
        cudaEventRecord(a, s);
        copy_halves<<<grid, 256, 0, s>>>(src, dst, half, reps);
        cudaEventRecord(b, s);
        float ms = 0;
        if (cudaEventSynchronize(b) != cudaSuccess || cudaEventElapsedTime(&ms, a, b) != cudaSuccess || ms <= 0)
            st = AEFDTD_CUDA_ERROR;
        else
            *gbs = double(2 * half * 16) * reps / (ms * 1e-3) / 1e9;
    }
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    if (s) cudaStreamDestroy(s);
    if (buf) cudaFree(buf);
    cudaGetLastError();
    cudaSetDevice(prev);
    return st;
}
