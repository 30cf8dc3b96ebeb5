// pulse.cuh — the incident pulse of the normal-incidence plane sums
// (ChpIn::PulseE*, chpin.cpp:44-90) in FP64, shared by the sensor kernels
// (sensors.cuh) and the persistent batch kernel (batch_persist.cuh).
#pragma once

#include <cuda_runtime.h>

#include "aefdtd_dev.hpp"

namespace aefdtd {

// Plane-sum arithmetic rounds every multiply and add separately (explicit
// _rn operations), so every kernel that inlines it gives the same bits.
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }

__device__ __forceinline__ double pulse_eval(const PulseDev &P, double A0, double x, double y, double z, double t) {
    const double p = dadd(dadd(dmul(P.kx, x), dmul(P.ky, y)), dmul(P.kz, z));
    const double a = dsub(p, dmul(P.omega, t));
    const double b = dadd(dsub(dmul(1.0 / P.k, p), dmul(299792458.0, t) / P.n_ind), P.C1) / P.dz;
    return dmul(dmul(A0, exp(-dmul(b, b))), cos(a));
}

}  // namespace aefdtd
