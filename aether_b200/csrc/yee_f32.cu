// FP32 instantiation of the fused half-step kernels (contraction allowed).
#include "kernels.hpp"
#include "yee.cuh"

namespace aefdtd {
void launch_e(const StepArgs<float, uint8_t> &a, dim3 g, dim3 b, cudaStream_t s) { e_half_step<<<g, b, 0, s>>>(a); }
void launch_e(const StepArgs<float, uint16_t> &a, dim3 g, dim3 b, cudaStream_t s) { e_half_step<<<g, b, 0, s>>>(a); }
void launch_h(const StepArgs<float, uint8_t> &a, dim3 g, dim3 b, cudaStream_t s) { h_half_step<<<g, b, 0, s>>>(a); }
void launch_h(const StepArgs<float, uint16_t> &a, dim3 g, dim3 b, cudaStream_t s) { h_half_step<<<g, b, 0, s>>>(a); }
}  // namespace aefdtd
