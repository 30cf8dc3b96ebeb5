// Sensor-path kernels. Built with --fmad=false: with one buffered step the
// DFT update is the reference's acc + coeff*t exactly.
#include "kernels.hpp"
#include "sensors.cuh"

namespace aefdtd {
void launch_plane_sums(const PlaneSumArgs<double> &a, cudaStream_t s) { plane_sums<<<1, 512, 0, s>>>(a); }
void launch_plane_sums(const PlaneSumArgs<float> &a, cudaStream_t s) { plane_sums<<<1, 512, 0, s>>>(a); }
void launch_gather(const GatherArgs<double> &a, cudaStream_t s) {
    const int P = a.span1 * a.span2;
    dft_gather<<<(P + 255) / 256, 256, 0, s>>>(a);
}
void launch_gather(const GatherArgs<float> &a, cudaStream_t s) {
    const int P = a.span1 * a.span2;
    dft_gather<<<(P + 255) / 256, 256, 0, s>>>(a);
}
void launch_phasors(const PhasorArgs &a, cudaStream_t s) {
    const int n = a.nk * a.nl;
    dft_phasors<<<(n + 255) / 256, 256, 0, s>>>(a);
}
template <typename T> static void acc_impl(const AccumArgs<T> &a, cudaStream_t s) {
    dim3 g((a.P + 127) / 128, (a.nl + kDftFTile - 1) / kDftFTile, 6);
    dft_accumulate<<<g, 128, 0, s>>>(a);
}
void launch_accumulate(const AccumArgs<double> &a, cudaStream_t s) { acc_impl(a, s); }
void launch_accumulate(const AccumArgs<float> &a, cudaStream_t s) { acc_impl(a, s); }
void launch_flux(const FluxArgs &a, cudaStream_t s) { flux_reduce<<<a.nl, 256, 0, s>>>(a); }
}  // namespace aefdtd
