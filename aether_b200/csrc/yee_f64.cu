// FP64 instantiation of the fused half-step kernels. Built with --fmad=false
// so that every multiply and add rounds separately, in the reference's order.
#include "kernels.hpp"
#include "yee.cuh"

namespace aefdtd {
void launch_e_interior(const StepArgs<double, uint8_t> &a, const int4 *items, int n, cudaStream_t s) {
    if (n > 0) e_interior<double, uint8_t><<<n, dim3(kTileX, kTileY), 0, s>>>(a, items);
}
void launch_e_boundary(const StepArgs<double, uint8_t> &a, const int4 *items, int n, cudaStream_t s) {
    if (n > 0) e_boundary<double, uint8_t><<<n, dim3(kTileX, kTileY), 0, s>>>(a, items);
}
void launch_h_interior(const StepArgs<double, uint8_t> &a, const int4 *items, int n, cudaStream_t s) {
    if (n > 0) h_interior<double, uint8_t><<<n, dim3(kTileX, kTileY), 0, s>>>(a, items);
}
void launch_h_boundary(const StepArgs<double, uint8_t> &a, const int4 *items, int n, cudaStream_t s) {
    if (n > 0) h_boundary<double, uint8_t><<<n, dim3(kTileX, kTileY), 0, s>>>(a, items);
}
void launch_e_interior(const StepArgs<double, uint16_t> &a, const int4 *items, int n, cudaStream_t s) {
    if (n > 0) e_interior<double, uint16_t><<<n, dim3(kTileX, kTileY), 0, s>>>(a, items);
}
void launch_e_boundary(const StepArgs<double, uint16_t> &a, const int4 *items, int n, cudaStream_t s) {
    if (n > 0) e_boundary<double, uint16_t><<<n, dim3(kTileX, kTileY), 0, s>>>(a, items);
}
void launch_h_interior(const StepArgs<double, uint16_t> &a, const int4 *items, int n, cudaStream_t s) {
    if (n > 0) h_interior<double, uint16_t><<<n, dim3(kTileX, kTileY), 0, s>>>(a, items);
}
void launch_h_boundary(const StepArgs<double, uint16_t> &a, const int4 *items, int n, cudaStream_t s) {
    if (n > 0) h_boundary<double, uint16_t><<<n, dim3(kTileX, kTileY), 0, s>>>(a, items);
}
}  // namespace aefdtd
