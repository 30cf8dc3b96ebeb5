// mbar.cuh — shared-memory mbarriers and bulk copies (sm_100a inline PTX),
// shared by the tensor-core DFT (dft_tc.cu) and the staged interior
// half-steps (interior_tma.cuh).
//
// Every wait is bounded: it gives up after `limit` SM cycles (or when an
// abort flag is raised) and the caller reports AEFDTD_TIMEOUT through the
// device error flag instead of spinning forever.
#pragma once
#include <cstdint>

namespace aefdtd {
namespace mbar {

__device__ __forceinline__ uint32_t saddr(const void *p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ void init(uint64_t *b, uint32_t n) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(saddr(b)), "r"(n) : "memory");
}
// makes the initialised barriers visible to the async (bulk-copy) proxy
__device__ __forceinline__ void fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void expect_tx(uint64_t *b, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(saddr(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void arrive(uint64_t *b) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(saddr(b)) : "memory");
}
__device__ __forceinline__ bool try_wait(uint64_t *b, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(saddr(b)), "r"(parity)
        : "memory");
    return ok != 0;
}
// waits for the phase of parity `parity` to complete; false after `limit` cycles
__device__ __forceinline__ bool wait(uint64_t *b, uint32_t parity, long long limit) {
    if (try_wait(b, parity)) return true;
    const long long t0 = clock64();
    while (!try_wait(b, parity))
        if (clock64() - t0 > limit) return false;
    return true;
}
// as wait(), and also false as soon as *abort is set by another warp of the CTA
__device__ __forceinline__ bool wait_or_abort(uint64_t *b, uint32_t parity, long long limit, const volatile int *abort) {
    if (try_wait(b, parity)) return true;
    const long long t0 = clock64();
    while (!try_wait(b, parity))
        if (*abort || clock64() - t0 > limit) return false;
    return true;
}
// untiled bulk copy global -> shared (16-byte aligned addresses, size a multiple of 16)
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *b) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(saddr(dst)), "l"(src), "r"(bytes), "r"(saddr(b))
                 : "memory");
}
// tiled 3-D tensor copy global -> shared of the box at (x, y, z); x times the
// element size must be a multiple of 16 bytes (negative or out-of-range
// coordinates read zeros)
__device__ __forceinline__ void tensor_g2s_3d(void *dst, const void *tmap, int x, int y, int z, uint64_t *b) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
        ::"r"(saddr(dst)), "l"(tmap), "r"(x), "r"(y), "r"(z), "r"(saddr(b))
        : "memory");
}
__device__ __forceinline__ void prefetch_tmap(const void *tmap) {
    asm volatile("prefetch.tensormap [%0];" ::"l"(tmap) : "memory");
}

}  // namespace mbar
}  // namespace aefdtd
