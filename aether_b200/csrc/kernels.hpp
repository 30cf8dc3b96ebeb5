// kernels.hpp — host-callable launchers of the device kernels. Each .cu unit
// instantiates the templates for its precision.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "aefdtd_dev.hpp"


namespace aefdtd {

// yee_f64.cu (compiled with --fmad=false) and yee_f32.cu: group g of an E or
// H half-step's WorkSplit, one 32 x tile_y CTA per item (nothing when empty);
// the batch forms take a device array of per-instance arguments.
#define AEFDTD_DECL_YEE(T, Tid)                                                                          \
    void launch_e_group(const StepArgs<T, Tid> &a, const int4 *items, const WorkSplit &w, int g,        \
                        cudaStream_t s);                                                                  \
    void launch_h_group(const StepArgs<T, Tid> &a, const int4 *items, const WorkSplit &w, int g,        \
                        cudaStream_t s);                                                                  \
    void launch_e_group_batch(const StepArgs<T, Tid> *args, int q, const int4 *items, const WorkSplit &w, \
                              int g, cudaStream_t s);                                                     \
    void launch_h_group_batch(const StepArgs<T, Tid> *args, int q, const int4 *items, const WorkSplit &w, \
                              int g, cudaStream_t s);
// leapfrog_f64.cu (--fmad=false) and leapfrog_f32.cu: fused group g
// (kFused*) of one time step, items [off, off + n), CTAs of 32 x (ty + 2) threads
#define AEFDTD_DECL_FUSED(T, Tid)                                                                      \
    void launch_fused_group(const FusedArgs<T, Tid> &a, const int4 *items, int off, int n, int g, int ty, \
                            cudaStream_t s);
AEFDTD_DECL_FUSED(double, uint8_t)
AEFDTD_DECL_FUSED(double, uint16_t)
AEFDTD_DECL_FUSED(float, uint8_t)
AEFDTD_DECL_FUSED(float, uint16_t)
#undef AEFDTD_DECL_FUSED
// yee_f64.cu (--fmad=false) and yee_f32.cu: the persistent batch kernel
// (batch_persist.cuh), one cooperative launch of `grid` CTAs of 32 x ty
// threads; persist_capacity: such CTAs resident on the current device at once
template <typename T, typename Tid> int persist_capacity(int ty);
#define AEFDTD_DECL_PERSIST(T, Tid)                                                                    \
    cudaError_t launch_persist(const PersistArgs<T, Tid> &p, int grid, int ty, cudaStream_t s);        \
    template <> int persist_capacity<T, Tid>(int ty);
AEFDTD_DECL_PERSIST(double, uint8_t)
AEFDTD_DECL_PERSIST(double, uint16_t)
AEFDTD_DECL_PERSIST(float, uint8_t)
AEFDTD_DECL_PERSIST(float, uint16_t)
#undef AEFDTD_DECL_PERSIST
AEFDTD_DECL_YEE(double, uint8_t)
AEFDTD_DECL_YEE(double, uint16_t)
AEFDTD_DECL_YEE(float, uint8_t)
AEFDTD_DECL_YEE(float, uint16_t)
#undef AEFDTD_DECL_YEE

// sensors.cu (compiled with --fmad=false)
// one part (a.part) of a step's sensor work; returns the launches issued
int launch_sensor_step(const SensorStepArgs<double> &a, cudaStream_t s);
int launch_sensor_step(const SensorStepArgs<float> &a, cudaStream_t s);
void launch_plane_reduce(const double *partial, int nbp, const StepScalars *sc, double *out, int steps,
                         cudaStream_t s);
// completion sensor, FT mode: step a.q of every probe
void launch_completion_ft(const CcFtArgs<double> &a, cudaStream_t s);
void launch_completion_ft(const CcFtArgs<float> &a, cudaStream_t s);
// single-wavelength field sensors: one part (a.part) of step a.q; returns the launches issued
int launch_fieldmap_step(const MapStepArgs<double> &a, cudaStream_t s);
int launch_fieldmap_step(const MapStepArgs<float> &a, cudaStream_t s);
// batch members: plane-sum partials of step q (blk: block -> (instance, block)),
// and the reduction of `steps` steps of every instance into its history
void launch_plane_partial_batch(const SensorStepArgs<double> *args, const int2 *blk, int nblk, int q, cudaStream_t s);
void launch_plane_partial_batch(const SensorStepArgs<float> *args, const int2 *blk, int nblk, int q, cudaStream_t s);
void launch_plane_reduce_batch(const SensorStepArgs<double> *args, int n_inst, int steps, cudaStream_t s);
void launch_plane_reduce_batch(const SensorStepArgs<float> *args, int n_inst, int steps, cudaStream_t s);
// completion sensor (energy mode): per-step grid energy partials, and their
// reduction for `steps` steps into hist[sc[0].step + q]
void launch_energy_partial(const double *Ex, const double *Ey, const double *Ez, long long N, int nb, double *part,
                           cudaStream_t s);
void launch_energy_partial(const float *Ex, const float *Ey, const float *Ez, long long N, int nb, double *part,
                           cudaStream_t s);
void launch_energy_reduce(const double *part, int nb, const StepScalars *sc, double *hist, int steps, cudaStream_t s);
void launch_phasors(const PhasorArgs &a, cudaStream_t s);
void launch_accumulate(const AccumArgs<double> &a, cudaStream_t s);
void launch_accumulate(const AccumArgs<float> &a, cudaStream_t s);
void launch_flux(const FluxArgs &a, cudaStream_t s);

// oblique.cu (compiled with --fmad=false): the oblique driver's incident sums
// and its per-step R/T sums (block partials of step a.q, then the reduction
// of `steps` steps into hist[sc[0].step + q][18]); the sums return launches issued
void launch_obl_incident(const OblIncArgs &a, cudaStream_t s);
int launch_obl_sums(const OblSumArgs<double> &a, int nb, cudaStream_t s);
int launch_obl_sums(const OblSumArgs<float> &a, int nb, cudaStream_t s);
void launch_obl_reduce(const double *partial, int nb, const StepScalars *sc, double *hist, int steps, cudaStream_t s);

// dft_tc.cu: FP32 DFT blocks on the tensor cores (tcgen05, 3xTF32)
void launch_phasors_tc(const DftTcPhasorArgs &a, cudaStream_t s);
void launch_accumulate_tc(const DftTcArgs &a, cudaStream_t s);

}  // namespace aefdtd
