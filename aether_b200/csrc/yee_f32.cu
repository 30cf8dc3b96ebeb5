// FP32 instantiation of the fused half-step kernels (contraction allowed).
#include "kernels.hpp"
#include "yee.cuh"

namespace aefdtd {
void launch_e_group(const StepArgs<float, uint8_t> &a, const int4 *items, const WorkSplit &w, int g, cudaStream_t s) {
    launch_e_group_impl(a, items, w, g, s);
}
void launch_h_group(const StepArgs<float, uint8_t> &a, const int4 *items, const WorkSplit &w, int g, cudaStream_t s) {
    launch_h_group_impl(a, items, w, g, s);
}
void launch_e_group(const StepArgs<float, uint16_t> &a, const int4 *items, const WorkSplit &w, int g, cudaStream_t s) {
    launch_e_group_impl(a, items, w, g, s);
}
void launch_h_group(const StepArgs<float, uint16_t> &a, const int4 *items, const WorkSplit &w, int g, cudaStream_t s) {
    launch_h_group_impl(a, items, w, g, s);
}
void launch_e_group_batch(const StepArgs<float, uint8_t> *args, int q, const int4 *items, const WorkSplit &w, int g,
                          cudaStream_t s) {
    launch_e_group_batch_impl(args, q, items, w, g, s);
}
void launch_h_group_batch(const StepArgs<float, uint8_t> *args, int q, const int4 *items, const WorkSplit &w, int g,
                          cudaStream_t s) {
    launch_h_group_batch_impl(args, q, items, w, g, s);
}
void launch_e_group_batch(const StepArgs<float, uint16_t> *args, int q, const int4 *items, const WorkSplit &w, int g,
                          cudaStream_t s) {
    launch_e_group_batch_impl(args, q, items, w, g, s);
}
void launch_h_group_batch(const StepArgs<float, uint16_t> *args, int q, const int4 *items, const WorkSplit &w, int g,
                          cudaStream_t s) {
    launch_h_group_batch_impl(args, q, items, w, g, s);
}
}  // namespace aefdtd
