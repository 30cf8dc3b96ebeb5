// FP32 instantiation of the fused time-step kernels (leapfrog.cuh); contraction allowed.
#include "kernels.hpp"
#include "leapfrog.cuh"

namespace aefdtd {
void launch_fused_group(const FusedArgs<float, uint8_t> &a, const int4 *items, int off, int n, int g, int ty,
                        cudaStream_t s) {
    launch_fused_group_impl(a, items, off, n, g, ty, s);
}
void launch_fused_group(const FusedArgs<float, uint16_t> &a, const int4 *items, int off, int n, int g, int ty,
                        cudaStream_t s) {
    launch_fused_group_impl(a, items, off, n, g, ty, s);
}
}  // namespace aefdtd
