// FP64 instantiation of the fused time-step kernels (leapfrog.cuh).
// Built with --fmad=false: every multiply and add rounds separately, in the
// reference's order.
#include "kernels.hpp"
#include "leapfrog.cuh"

namespace aefdtd {
void launch_fused_group(const FusedArgs<double, uint8_t> &a, const int4 *items, int off, int n, int g, int ty,
                        cudaStream_t s) {
    launch_fused_group_impl(a, items, off, n, g, ty, s);
}
void launch_fused_group(const FusedArgs<double, uint16_t> &a, const int4 *items, int off, int n, int g, int ty,
                        cudaStream_t s) {
    launch_fused_group_impl(a, items, off, n, g, ty, s);
}
}  // namespace aefdtd
