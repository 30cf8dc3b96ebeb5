// kernels.hpp — host-callable launchers of the device kernels. Each .cu unit
// instantiates the templates for its precision.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "aefdtd_dev.hpp"

namespace aefdtd {

// yee_f64.cu (compiled with --fmad=false) and yee_f32.cu
void launch_e(const StepArgs<double, uint8_t> &a, dim3 g, dim3 b, cudaStream_t s);
void launch_e(const StepArgs<double, uint16_t> &a, dim3 g, dim3 b, cudaStream_t s);
void launch_h(const StepArgs<double, uint8_t> &a, dim3 g, dim3 b, cudaStream_t s);
void launch_h(const StepArgs<double, uint16_t> &a, dim3 g, dim3 b, cudaStream_t s);
void launch_e(const StepArgs<float, uint8_t> &a, dim3 g, dim3 b, cudaStream_t s);
void launch_e(const StepArgs<float, uint16_t> &a, dim3 g, dim3 b, cudaStream_t s);
void launch_h(const StepArgs<float, uint8_t> &a, dim3 g, dim3 b, cudaStream_t s);
void launch_h(const StepArgs<float, uint16_t> &a, dim3 g, dim3 b, cudaStream_t s);

// sensors.cu (compiled with --fmad=false)
void launch_plane_sums(const PlaneSumArgs<double> &a, cudaStream_t s);
void launch_plane_sums(const PlaneSumArgs<float> &a, cudaStream_t s);
void launch_gather(const GatherArgs<double> &a, cudaStream_t s);
void launch_gather(const GatherArgs<float> &a, cudaStream_t s);
void launch_phasors(const PhasorArgs &a, cudaStream_t s);
void launch_accumulate(const AccumArgs<double> &a, cudaStream_t s);
void launch_accumulate(const AccumArgs<float> &a, cudaStream_t s);
void launch_flux(const FluxArgs &a, cudaStream_t s);

}  // namespace aefdtd
