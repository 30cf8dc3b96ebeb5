// Sensor-path kernels. Contraction is allowed: the SIMT DFT accumulates its
// K-step partial sums with FMA starting from zero, so with one buffered step
// the update is still the reference's acc + round(coeff*t) exactly.
#include "kernels.hpp"
#include "sensors.cuh"

#include <algorithm>

namespace aefdtd {
// Part 0: plane-sum and gather blocks; part 1: gather blocks only.
template <typename T> static int step_impl(const SensorStepArgs<T> &a, cudaStream_t s) {
    int nb = a.nbp;
    for (int g = 0; g < a.ng; ++g) nb = std::max(nb, a.g[g].block0 + a.g[g].nblocks);
    if (a.part) nb -= a.nbp;
    if (nb > 0) sensor_step<<<nb, kPlaneThreads, 0, s>>>(a);
    return nb > 0;
}
int launch_sensor_step(const SensorStepArgs<double> &a, cudaStream_t s) { return step_impl(a, s); }
int launch_sensor_step(const SensorStepArgs<float> &a, cudaStream_t s) { return step_impl(a, s); }
template <typename T> static int map_impl(const MapStepArgs<T> &a, cudaStream_t s) {
    int nb = 0;
    for (int m = 0; m < a.nm; ++m) nb = std::max(nb, a.m[m].block0 + a.m[m].nblocks);
    if (nb > 0) fieldmap_step<<<nb, kPlaneThreads, 0, s>>>(a);
    return nb > 0;
}
int launch_fieldmap_step(const MapStepArgs<double> &a, cudaStream_t s) { return map_impl(a, s); }
template <typename T> static void ccft_impl(const CcFtArgs<T> &a, cudaStream_t s) {
    if (a.np > 0) completion_ft_step<<<(a.np + kPlaneThreads - 1) / kPlaneThreads, kPlaneThreads, 0, s>>>(a);
}
void launch_completion_ft(const CcFtArgs<double> &a, cudaStream_t s) { ccft_impl(a, s); }
void launch_completion_ft(const CcFtArgs<float> &a, cudaStream_t s) { ccft_impl(a, s); }
int launch_fieldmap_step(const MapStepArgs<float> &a, cudaStream_t s) { return map_impl(a, s); }
void launch_plane_reduce(const double *partial, int nbp, const StepScalars *sc, double *out, int steps,
                         cudaStream_t s) {
    if (steps > 0) plane_sums_reduce<<<steps, 32, 0, s>>>(partial, nbp, sc, out);
}
void launch_phasors(const PhasorArgs &a, cudaStream_t s) {
    const int n = a.nk * a.nl;
    dft_phasors<<<(n + 255) / 256, 256, 0, s>>>(a);
}
template <typename T> static void acc_impl(const AccumArgs<T> &a, cudaStream_t s) {
    const dim3 g((a.P + 63) / 64, (a.nl + 63) / 64, 6);
    if (a.mma) {
        constexpr int smem = dft_mma_smem<T>();
        static bool attr = false;   // one instantiation per T
        if (!attr) {
            cudaFuncSetAttribute(dft_accumulate_mma<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
            attr = true;
        }
        dft_accumulate_mma<<<g, 256, smem, s>>>(a);
        return;
    }
    constexpr int smem = dft_acc_smem<T>();
    static bool attr = false;   // one instantiation per T
    if (!attr) {
        cudaFuncSetAttribute(dft_accumulate<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        attr = true;
    }
    dft_accumulate<<<g, 256, smem, s>>>(a);
}
void launch_accumulate(const AccumArgs<double> &a, cudaStream_t s) { acc_impl(a, s); }
void launch_accumulate(const AccumArgs<float> &a, cudaStream_t s) { acc_impl(a, s); }
void launch_flux(const FluxArgs &a, cudaStream_t s) { flux_reduce<<<a.nl, 256, 0, s>>>(a); }
template <typename T> static void plane_batch_impl(const SensorStepArgs<T> *args, const int2 *blk, int nblk, int q,
                                                   cudaStream_t s) {
    if (nblk > 0) plane_partial_batch<T><<<nblk, kPlaneThreads, 0, s>>>(args, blk, q);
}
void launch_plane_partial_batch(const SensorStepArgs<double> *args, const int2 *blk, int nblk, int q, cudaStream_t s) {
    plane_batch_impl(args, blk, nblk, q, s);
}
void launch_plane_partial_batch(const SensorStepArgs<float> *args, const int2 *blk, int nblk, int q, cudaStream_t s) {
    plane_batch_impl(args, blk, nblk, q, s);
}
void launch_plane_reduce_batch(const SensorStepArgs<double> *args, int n_inst, int steps, cudaStream_t s) {
    if (n_inst > 0 && steps > 0) plane_sums_reduce_batch<double><<<dim3(steps, n_inst), 32, 0, s>>>(args);
}
void launch_plane_reduce_batch(const SensorStepArgs<float> *args, int n_inst, int steps, cudaStream_t s) {
    if (n_inst > 0 && steps > 0) plane_sums_reduce_batch<float><<<dim3(steps, n_inst), 32, 0, s>>>(args);
}
void launch_energy_partial(const double *Ex, const double *Ey, const double *Ez, long long N, int nb, double *part,
                           cudaStream_t s) {
    energy_partial<double><<<nb, kPlaneThreads, 0, s>>>(Ex, Ey, Ez, N, nb, part);
}
void launch_energy_partial(const float *Ex, const float *Ey, const float *Ez, long long N, int nb, double *part,
                           cudaStream_t s) {
    energy_partial<float><<<nb, kPlaneThreads, 0, s>>>(Ex, Ey, Ez, N, nb, part);
}
void launch_energy_reduce(const double *part, int nb, const StepScalars *sc, double *hist, int steps, cudaStream_t s) {
    if (steps > 0) energy_reduce<<<steps, 32, 0, s>>>(part, nb, sc, hist);
}
}  // namespace aefdtd
