// FP32 instantiation of the fused half-step kernels (contraction allowed).
#include "kernels.hpp"
#include "yee.cuh"

namespace aefdtd {
void launch_e_interior(const StepArgs<float, uint8_t> &a, const int4 *items, int n, cudaStream_t s) {
    if (n > 0) e_interior<float, uint8_t><<<n, dim3(kTileX, kTileY), 0, s>>>(a, items);
}
void launch_e_boundary(const StepArgs<float, uint8_t> &a, const int4 *items, int n, cudaStream_t s) {
    if (n > 0) e_boundary<float, uint8_t><<<n, dim3(kTileX, kTileY), 0, s>>>(a, items);
}
void launch_h_interior(const StepArgs<float, uint8_t> &a, const int4 *items, int n, cudaStream_t s) {
    if (n > 0) h_interior<float, uint8_t><<<n, dim3(kTileX, kTileY), 0, s>>>(a, items);
}
void launch_h_boundary(const StepArgs<float, uint8_t> &a, const int4 *items, int n, cudaStream_t s) {
    if (n > 0) h_boundary<float, uint8_t><<<n, dim3(kTileX, kTileY), 0, s>>>(a, items);
}
void launch_e_interior(const StepArgs<float, uint16_t> &a, const int4 *items, int n, cudaStream_t s) {
    if (n > 0) e_interior<float, uint16_t><<<n, dim3(kTileX, kTileY), 0, s>>>(a, items);
}
void launch_e_boundary(const StepArgs<float, uint16_t> &a, const int4 *items, int n, cudaStream_t s) {
    if (n > 0) e_boundary<float, uint16_t><<<n, dim3(kTileX, kTileY), 0, s>>>(a, items);
}
void launch_h_interior(const StepArgs<float, uint16_t> &a, const int4 *items, int n, cudaStream_t s) {
    if (n > 0) h_interior<float, uint16_t><<<n, dim3(kTileX, kTileY), 0, s>>>(a, items);
}
void launch_h_boundary(const StepArgs<float, uint16_t> &a, const int4 *items, int n, cudaStream_t s) {
    if (n > 0) h_boundary<float, uint16_t><<<n, dim3(kTileX, kTileY), 0, s>>>(a, items);
}
}  // namespace aefdtd
