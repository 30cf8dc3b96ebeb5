// FP32 instantiation of the fused half-step kernels (contraction allowed).
#include "kernels.hpp"
#include "yee.cuh"
#include "batch_persist.cuh"

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
cudaError_t launch_persist(const PersistArgs<float, uint8_t> &p, int grid, int ty, cudaStream_t s) {
    return launch_persist_impl(p, grid, ty, s);
}
template <> int persist_capacity<float, uint8_t>(int ty) { return persist_capacity_impl<float, uint8_t>(ty); }
cudaError_t launch_persist(const PersistArgs<float, uint16_t> &p, int grid, int ty, cudaStream_t s) {
    return launch_persist_impl(p, grid, ty, s);
}
template <> int persist_capacity<float, uint16_t>(int ty) { return persist_capacity_impl<float, uint16_t>(ty); }
}  // namespace aefdtd
