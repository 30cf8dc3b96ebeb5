// plane_static.cu — per-plane field sums that allocate no device memory.
//
// aefdtd_plane_sums_static sums up to AEFDTD_STATIC_MAX_PLANES whole x-y
// planes of three field arrays the caller already holds on the device
// (for instance the Ex, Ey, Ez arrays from aefdtd_field_device_ptr), in FP64,
// into an output array the caller also owns. It is the same two-stage
// reduction the stepping path uses for the transmission-plane sums: stage 1
// gives each plane the same number of blocks and the same chunking, thread
// striding and tree order, stage 2 adds the block partials in block order.
// So, for the plane and weight the stepping path used, the result matches
// slots 9..11 of aefdtd_get_plane_sums bit for bit.
//
// Who needs this: a process that has sized its device memory up front (a
// batch of simulations admitted up to a fixed share of HBM, or a serving loop
// whose footprint must not grow per request) cannot let a diagnostic call
// allocate: the allocation may fail once memory is fully committed, and
// freeing memory synchronises the device, stalling every stream. Here the
// stage-1 partials live in one file-scope device array instead of a buffer
// allocated per call or per handle.
//
// Scratch: g_plane_scratch, 96 KiB (AEFDTD_STATIC_MAX_PLANES planes x 64
// blocks x 3 components x 8 bytes), held by every device that loads this
// library until the process exits. Every call shares it; stage 1 overwrites
// each partial it reads later, so nothing needs clearing between calls. Two
// calls whose kernels overlap on one device (different streams, or different
// host threads) race on it and may return each other's sums: serialise them.
//
// Set-up: every call resolves the array's address on the current device with
// cudaGetSymbolAddress and checks the result. The first call on a device also
// loads this library's device code there; make that first call before any
// stream capture on the device.
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdint>
#include <cstdio>

#include "../../include/aefdtd.h"
#include "aefdtd_dev.hpp"

namespace aefdtd {
namespace {

constexpr int kStaticPlanes = AEFDTD_STATIC_MAX_PLANES;

static __device__ __align__(256) double g_plane_scratch[kStaticPlanes * kPlaneBlocks * 3];

struct StaticPlaneArgs {
    const void *f[3];
    long long NxNy;
    int n, nbp, n_planes;
    double w;
    int planes[kStaticPlanes];
};

// Stage 1: block (b, p) sums its chunk of plane p, partial[(p*nbp + b)*3 + c].
template <typename T>
__global__ void __launch_bounds__(kPlaneThreads)
plane_sums_static_partial(const __grid_constant__ StaticPlaneArgs a, double *partial) {
    const int b = blockIdx.x, p = blockIdx.y;
    const T *f0 = static_cast<const T *>(a.f[0]), *f1 = static_cast<const T *>(a.f[1]);
    const T *f2 = static_cast<const T *>(a.f[2]);
    const long long base = (long long)a.planes[p] * a.NxNy;
    const int per = (a.n + a.nbp - 1) / a.nbp;
    const int q0 = b * per, q1 = min(a.n, q0 + per);
    // every multiply and add rounded separately, as in the stepping path's
    // plane_partial, so that no contraction into a fused multiply-add can
    // change the last bit for weights other than 1
    double s0 = 0, s1 = 0, s2 = 0;
    for (int q = q0 + threadIdx.x; q < q1; q += blockDim.x) {
        s0 = __dadd_rn(s0, __dmul_rn((double)f0[base + q], a.w));
        s1 = __dadd_rn(s1, __dmul_rn((double)f1[base + q], a.w));
        s2 = __dadd_rn(s2, __dmul_rn((double)f2[base + q], a.w));
    }
    __shared__ double red[3][kPlaneThreads];
    red[0][threadIdx.x] = s0;
    red[1][threadIdx.x] = s1;
    red[2][threadIdx.x] = s2;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            red[0][threadIdx.x] += red[0][threadIdx.x + s];
            red[1][threadIdx.x] += red[1][threadIdx.x + s];
            red[2][threadIdx.x] += red[2][threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x < 3) partial[((long long)p * a.nbp + b) * 3 + threadIdx.x] = red[threadIdx.x][0];
}

// Stage 2: out[p*3 + c] = sum of plane p's partials in block order.
__global__ void plane_sums_static_reduce(const double *partial, int nbp, double *out) {
    const int p = blockIdx.x, c = threadIdx.x;
    if (c >= 3) return;
    double s = 0;
    for (int b = 0; b < nbp; ++b) s += partial[((long long)p * nbp + b) * 3 + c];
    out[p * 3 + c] = s;
}

// Address of g_plane_scratch on the current device, resolved on every call:
// after a cudaDeviceReset (or a new primary context) the module is loaded
// again at another address, so a cached pointer would go stale. Once the
// module is loaded on the device the lookup is cheap; the first lookup loads
// it, which is why the first call on a device should come before any stream
// capture there.
cudaError_t scratch_address(double **out) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_plane_scratch);
    if (e != cudaSuccess) return e;
    *out = static_cast<double *>(p);
    return cudaSuccess;
}

aefdtd_status report(char *buf, size_t len, aefdtd_status st, const char *fmt, ...) {
    if (buf && len > 0) {
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, len, fmt, ap);
        va_end(ap);
    }
    return st;
}

// Device pointer on device `dev` with the given alignment, else a message.
const char *check_device_ptr(const void *p, int dev, size_t align) {
    if (!p) return "is null";
    if (reinterpret_cast<uintptr_t>(p) % align) return "is misaligned for its element type";
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return "is not a CUDA pointer";
    }
    if (at.type != cudaMemoryTypeDevice && at.type != cudaMemoryTypeManaged) return "is not device memory";
    if (at.device != dev) return "belongs to another device than the current one";
    return nullptr;
}

}  // namespace
}  // namespace aefdtd

using namespace aefdtd;

extern "C" aefdtd_status aefdtd_plane_sums_static(const void *const *fields, int32_t precision, int32_t nx,
                                                  int32_t ny, int32_t nz, const int32_t *planes, int32_t n_planes,
                                                  double weight, double *out, void *stream, char *errbuf,
                                                  size_t errbuf_len) {
    if (errbuf && errbuf_len > 0) errbuf[0] = '\0';
    if (!fields || !planes) return report(errbuf, errbuf_len, AEFDTD_BAD_ARG, "fields and planes must not be null");
    if (precision != AEFDTD_FP64 && precision != AEFDTD_FP32)
        return report(errbuf, errbuf_len, AEFDTD_BAD_ARG, "precision must be AEFDTD_FP64 or AEFDTD_FP32");
    if (nx < 1 || ny < 1 || nz < 1 || (long long)nx * ny > INT32_MAX)
        return report(errbuf, errbuf_len, AEFDTD_BAD_ARG, "grid %d x %d x %d: each size must be >= 1 and nx*ny < 2^31",
                      nx, ny, nz);
    if (n_planes < 1 || n_planes > kStaticPlanes)
        return report(errbuf, errbuf_len, AEFDTD_BAD_ARG,
                      "n_planes = %d: the static scratch holds 1 to %d planes per call", n_planes, kStaticPlanes);
    StaticPlaneArgs a{};
    for (int p = 0; p < n_planes; ++p) {
        if (planes[p] < 0 || planes[p] >= nz)
            return report(errbuf, errbuf_len, AEFDTD_BAD_ARG, "planes[%d] = %d is outside [0, %d)", p, planes[p], nz);
        a.planes[p] = planes[p];
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return report(errbuf, errbuf_len, AEFDTD_NO_DEVICE, "cudaGetDevice: %s", cudaGetErrorString(e));
    }
    const size_t elem = precision == AEFDTD_FP64 ? 8 : 4;
    for (int c = 0; c < 3; ++c) {
        if (const char *why = check_device_ptr(fields[c], dev, elem))
            return report(errbuf, errbuf_len, AEFDTD_BAD_ARG, "fields[%d] %s", c, why);
        a.f[c] = fields[c];
    }
    if (const char *why = check_device_ptr(out, dev, 8))
        return report(errbuf, errbuf_len, AEFDTD_BAD_ARG, "out %s", why);
    double *scratch = nullptr;
    e = scratch_address(&scratch);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return report(errbuf, errbuf_len, AEFDTD_CUDA_ERROR, "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
    }
    a.NxNy = (long long)nx * ny;
    a.n = nx * ny;
    a.nbp = a.n >= kPlaneBlocks * kPlaneThreads ? kPlaneBlocks : (a.n + kPlaneThreads - 1) / kPlaneThreads;
    a.n_planes = n_planes;
    a.w = weight;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const dim3 grid(a.nbp, n_planes);
    if (precision == AEFDTD_FP64)
        plane_sums_static_partial<double><<<grid, kPlaneThreads, 0, s>>>(a, scratch);
    else
        plane_sums_static_partial<float><<<grid, kPlaneThreads, 0, s>>>(a, scratch);
    plane_sums_static_reduce<<<n_planes, 32, 0, s>>>(scratch, a.nbp, out);
    e = cudaGetLastError();
    if (e != cudaSuccess)
        return report(errbuf, errbuf_len, AEFDTD_CUDA_ERROR, "kernel launch: %s", cudaGetErrorString(e));
    return AEFDTD_OK;
}
