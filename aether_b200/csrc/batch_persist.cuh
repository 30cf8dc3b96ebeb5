// batch_persist.cuh — one persistent launch advances every member of a batch
// subset by a chunk of time steps.
//
// The split path of a batch (batch.cpp) launches each work-item group of each
// half-step separately; on the L2-resident unit cells of a parameter sweep
// every such launch is short and the step time is mostly launch, fork/join
// and ramp latency. Here one cooperative launch runs all half-steps of the
// chunk (the loop of normal_incidence.cpp:325-436 for every member at once).
//
// Units. Each member's grid is cut into units: a band of tile rows (all x
// tiles of tile_y rows) times one z-chunk of its work items. CTA b owns the
// units b, b + grid, ... for the whole launch and walks the half-steps in
// order (E of step q, then H of step q), each over all of its units.
//
// Waits. A unit's E update reads H of its own cells, of the row below (y-1)
// and of the plane below (z-1); its H update reads E of the row above and of
// the plane above (fdtd_core.cpp:363-969; both wrap). So before E of step q a
// unit waits until its y-1 and z-1 units have finished H of step q-1, and
// before H of step q until its y+1 and z+1 units have finished E of step q.
// These are also the only units that read the values the unit is about to
// overwrite, in the half-step it waits for, so the same waits order the
// overwrites. Each unit has a progress counter (half-steps finished in this
// launch): the owning CTA's barrier, then an acq_rel fence and a store by its
// first thread publish it; the waiting CTA's first thread reads it with an
// acquire load, and the CTA's barrier passes that on to its other threads,
// whose loads of neighbour fields are ordinary cached loads (yee.cuh,
// ldf<true>), never the read-only path.
// Waits only ever look back one half-step and every CTA finishes a half-step
// before starting the next, so with all CTAs resident (cooperative launch)
// every wait ends. Each wait is still bounded: one that runs out raises the
// device error flag and the abort flag, and every CTA leaves at its next wait.
//
// Cells are updated by the split kernels' bodies (yee.cuh) with coherent
// field loads, so FP64 fields are bit-identical to the split path and to the
// reference core. The normal-mode plane sums (normal_incidence.cpp:387-415)
// are summed per band: the unit holding the band's reflection plane adds its
// six terms, the unit holding the transmission plane the other six, right
// after its E update; the bands are added in order after the launch.
#pragma once

#include "pulse.cuh"

namespace aefdtd {

__device__ __forceinline__ int ps_ld_acquire(const int *p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
// The release orders every store of the CTA before it: they precede it
// through the CTA barrier (fence.acq_rel at gpu scope, then a relaxed store).
__device__ __forceinline__ void ps_st_release(int *p, int v) {
    asm volatile("fence.acq_rel.gpu;\n\tst.relaxed.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// First thread of a CTA: until units a and b have both finished `need`
// half-steps. False when the bound ran out or another CTA gave up.
__device__ __forceinline__ bool ps_wait(const int *prog, int a, int b, int need, long long limit,
                                        const volatile int *abort) {
    if (ps_ld_acquire(prog + a) >= need && ps_ld_acquire(prog + b) >= need) return true;
    const long long t0 = clock64();
    for (;;) {
        __nanosleep(32);
        if (ps_ld_acquire(prog + a) >= need && ps_ld_acquire(prog + b) >= need) return true;
        if (*abort) return false;
        if (clock64() - t0 > limit) return false;
    }
}

template <typename T, typename Tid>
__device__ __forceinline__ void ps_e_item(const StepArgs<T, Tid> &a, int q, int4 b) {
    const int4 it = make_int4(b.x, b.y, b.z & 0xffff, b.z >> 16);
    switch (b.w) {
        case kGroupInterior: e_interior_body<T, Tid, 2, false, true>(a, q, it); break;
        case kGroupPmlZ: e_interior_body<T, Tid, 2, true, true>(a, q, it); break;
        case kGroupDisp: e_boundary_body<T, Tid, kFDisp, true>(a, q, it); break;
        case kGroupPmlXY: e_boundary_body<T, Tid, kFPmlXY | kFPmlZ, true>(a, q, it); break;
        default: e_boundary_body<T, Tid, kFAll, true>(a, q, it); break;
    }
}
template <typename T, typename Tid>
__device__ __forceinline__ void ps_h_item(const StepArgs<T, Tid> &a, int q, int4 b) {
    const int4 it = make_int4(b.x, b.y, b.z & 0xffff, b.z >> 16);
    switch (b.w) {
        case kGroupInterior: h_interior_body<T, Tid, 2, false, true>(a, q, it); break;
        case kGroupPmlZ: h_interior_body<T, Tid, 2, true, true>(a, q, it); break;
        case kGroupPmlXY: h_boundary_body<T, Tid, kFPmlXY | kFPmlZ, true>(a, q, it); break;
        default: h_boundary_body<T, Tid, kFAll, true>(a, q, it); break;
    }
}

constexpr int kPsMaxThreads = 256;

// Six plane-sum terms of rows [j0, j1) at step q: the reflection plane kr
// (half 0: incident Ex, Ey, Ez and E minus incident) or the transmission plane
// kt (half 1: incident and E), each tapered, into part[0..5]. The per-cell
// operations are plane_partial's (sensors.cuh).
template <typename T>
__device__ __forceinline__ void ps_band_sums(const SensorStepArgs<T> &a, int j0, int j1, int q, int half,
                                             double *part, double (*red)[kPsMaxThreads], double *pv) {
    const int nt = blockDim.x * blockDim.y, t = threadIdx.x + blockDim.x * threadIdx.y;
    const double Dx2 = a.Dx / 2.0, Dy2 = a.Dy / 2.0, Dz2 = a.Dz / 2.0;
    const int k = half ? a.kt : a.kr;
    const double z0 = k * a.Dz;
    const double tb = a.sc[q].tb, tap = a.sc[q].taper;
    const bool uniform = a.P.kx == 0.0 && a.P.ky == 0.0;
    if (uniform) {
        if (t < 3) {
            const double A0 = t == 0 ? a.P.Ex0 : t == 1 ? a.P.Ey0 : a.P.Ez0;
            pv[t] = pulse_eval(a.P, A0, t == 0 ? Dx2 : 0.0, t == 1 ? Dy2 : 0.0, z0 + (t == 2 ? Dz2 : 0.0), tb);
        }
        __syncthreads();
    }
    double acc[6] = {0, 0, 0, 0, 0, 0};
    const long long o = (long long)k * a.NxNy;
    for (int c = j0 * a.Nx + t; c < j1 * a.Nx; c += nt) {
        const int i = c % a.Nx, j = c / a.Nx;
        double bx, by, bz;
        if (uniform) {
            bx = pv[0]; by = pv[1]; bz = pv[2];
        } else {
            const double x = i * a.Dx, y = j * a.Dy;
            bx = pulse_eval(a.P, a.P.Ex0, x + Dx2, y, z0, tb);
            by = pulse_eval(a.P, a.P.Ey0, x, y + Dy2, z0, tb);
            bz = pulse_eval(a.P, a.P.Ez0, x, y, z0 + Dz2, tb);
        }
        const double ex = (double)a.Ex[c + o], ey = (double)a.Ey[c + o], ez = (double)a.Ez[c + o];
        acc[0] = dadd(acc[0], dmul(bx, tap));
        acc[1] = dadd(acc[1], dmul(by, tap));
        acc[2] = dadd(acc[2], dmul(bz, tap));
        if (half == 0) {
            acc[3] = dadd(acc[3], dmul(dsub(ex, bx), tap));
            acc[4] = dadd(acc[4], dmul(dsub(ey, by), tap));
            acc[5] = dadd(acc[5], dmul(dsub(ez, bz), tap));
        } else {
            acc[3] = dadd(acc[3], dmul(ex, tap));
            acc[4] = dadd(acc[4], dmul(ey, tap));
            acc[5] = dadd(acc[5], dmul(ez, tap));
        }
    }
#pragma unroll
    for (int c = 0; c < 6; ++c) red[c][t] = acc[c];
    __syncthreads();
    for (int s = nt / 2; s > 0; s >>= 1) {
        if (t < s)
#pragma unroll
            for (int c = 0; c < 6; ++c) red[c][t] += red[c][t + s];
        __syncthreads();
    }
    if (t < 6) part[t] = red[t][0];
}

template <typename T, typename Tid>
__global__ void __launch_bounds__(kPsMaxThreads, sizeof(T) == 8 ? 1 : 2)
    batch_persist(const __grid_constant__ PersistArgs<T, Tid> P) {
    __shared__ double red[6][kPsMaxThreads];
    __shared__ double pv[3];
    __shared__ int go;
    const bool lead = threadIdx.x == 0 && threadIdx.y == 0;
    volatile int *abort = P.flags + 1;
    for (int q = 0; q < P.steps; ++q) {
        for (int half = 0; half < 2; ++half) {
            const int h = 2 * q + half;   // this half-step; the waits need h finished before it
            for (int u = blockIdx.x; u < P.nunits; u += gridDim.x) {
                const PsUnit &U = P.units[u];
                if (lead) {
                    const bool ok = ps_wait(P.prog, U.nb[2 * half], U.nb[2 * half + 1], h, P.wait_cycles, abort);
                    if (!ok) {
                        *abort = 1;
                        atomicExch(P.flags, 1);
                    }
                    go = ok;
                }
                __syncthreads();
                if (!go) return;
                if (half == 0) {
                    const StepArgs<T, Tid> &a = P.ea[U.m];
                    for (int k = 0; k < U.e_n; ++k) ps_e_item<T, Tid>(a, q, P.items[U.e_off + k]);
                    if (U.planes) {
                        __syncthreads();
                        const SensorStepArgs<T> &s = P.sa[U.m];
                        double *part = s.partial + ((long long)q * s.nbp + U.band) * 12;
                        if (U.planes & 1) ps_band_sums(s, U.j0, U.j1, q, 0, part, red, pv);
                        if (U.planes & 2) {
                            __syncthreads();
                            ps_band_sums(s, U.j0, U.j1, q, 1, part + 6, red, pv);
                        }
                    }
                } else {
                    const StepArgs<T, Tid> &a = P.ha[U.m];
                    for (int k = 0; k < U.h_n; ++k) ps_h_item<T, Tid>(a, q, P.items[U.h_off + k]);
                }
                __syncthreads();
                if (lead && !(P.withhold && u == 0)) ps_st_release(P.prog + u, h + 1);
            }
        }
    }
}

template <typename T, typename Tid>
cudaError_t launch_persist_impl(const PersistArgs<T, Tid> &p, int grid, int ty, cudaStream_t s) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(32, ty);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, batch_persist<T, Tid>, p);
}

// CTAs of 32 x ty threads that fit on the device at once
template <typename T, typename Tid> int persist_capacity_impl(int ty) {
    int dev = 0, sms = 0, per = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, batch_persist<T, Tid>, 32 * ty, 0) != cudaSuccess) return 0;
    return per * sms;
}

}  // namespace aefdtd
