// sensors.cuh — device kernels of the sensor path.
//
//  * plane_sums: the normal-incidence R/T plane sums of one step
//    (normal_incidence.cpp:378-415), with the analytic incident pulse
//    (ChpIn::PulseE*, chpin.cpp:44-90) evaluated per cell in FP64.
//  * dft_gather: interpolated plane samples of one step into the K-step
//    sample buffer (SensorFieldHolder::update_t_interp, sensors.cpp:601-644,
//    with FDTD::local_E*/H*, fdtd_utils.cpp:457-507).
//  * dft_phasors / dft_accumulate: the buffered DFT of K steps,
//    acc[c][l][p] += sum_k S[k][c][p] * W_c[k][l] with
//    W_E = taper_E * exp(i w_l step Dt), W_H = taper_H * exp(i w_l (step+1/2) Dt)
//    (SensorFieldHolder::FT_comp, sensors.cpp:456-479; tapering from
//    Sensor::feed, sensors.cpp:232-243). With one buffered step the sum is the
//    reference's per-step update exactly.
//  * flux: Spect_Poynting::treat (s_spec_power.cpp:44-119) in FP64.
#pragma once

#include <cuda_runtime.h>

#include "aefdtd_dev.hpp"
#include "pulse.cuh"

namespace aefdtd {

// Block b of the plane-sum partials of step q (scalars a.sc[q]) into part[b*12 + c].
template <typename T>
__device__ __forceinline__ void plane_partial(const SensorStepArgs<T> &a, int b, int q, double *part) {
    double acc[12];
#pragma unroll
    for (int c = 0; c < 12; ++c) acc[c] = 0;
    const int n = a.Nx * a.Ny;
    const int per = (n + a.nbp - 1) / a.nbp;
    const int q0 = b * per, q1 = min(n, q0 + per);
    const double Dx2 = a.Dx / 2.0, Dy2 = a.Dy / 2.0, Dz2 = a.Dz / 2.0;
    const double zr = a.kr * a.Dz, zt = a.kt * a.Dz;
    const double tb = a.sc[q].tb, tap = a.sc[q].taper;
    // With kx = ky = 0 (normal incidence) the phase kx x + ky y + kz z is
    // exactly kz z, so the six pulse values are the same at every cell of the
    // planes: evaluate them once per block.
    const bool uniform = a.P.kx == 0.0 && a.P.ky == 0.0;
    __shared__ double pv[6];
    if (uniform) {
        const int t = threadIdx.x;
        if (t < 6) {
            const double A0 = (t % 3 == 0) ? a.P.Ex0 : (t % 3 == 1) ? a.P.Ey0 : a.P.Ez0;
            const double z = (t < 3 ? zr : zt) + (t % 3 == 2 ? Dz2 : 0.0);
            pv[t] = pulse_eval(a.P, A0, (t % 3 == 0) ? Dx2 : 0.0, (t % 3 == 1) ? Dy2 : 0.0, z, tb);
        }
        __syncthreads();
    }
    for (int c = q0 + threadIdx.x; c < q1; c += blockDim.x) {
        const int i = c % a.Nx, j = c / a.Nx;
        const double x = i * a.Dx, y = j * a.Dy;
        double bx, by, bz, tx, ty, tz;
        if (uniform) {
            bx = pv[0]; by = pv[1]; bz = pv[2]; tx = pv[3]; ty = pv[4]; tz = pv[5];
        } else {
            bx = pulse_eval(a.P, a.P.Ex0, x + Dx2, y, zr, tb);
            by = pulse_eval(a.P, a.P.Ey0, x, y + Dy2, zr, tb);
            bz = pulse_eval(a.P, a.P.Ez0, x, y, zr + Dz2, tb);
            tx = pulse_eval(a.P, a.P.Ex0, x + Dx2, y, zt, tb);
            ty = pulse_eval(a.P, a.P.Ey0, x, y + Dy2, zt, tb);
            tz = pulse_eval(a.P, a.P.Ez0, x, y, zt + Dz2, tb);
        }
        const long long ir = c + a.kr * a.NxNy, it = c + a.kt * a.NxNy;
        acc[0] = dadd(acc[0], dmul(bx, tap));
        acc[1] = dadd(acc[1], dmul(by, tap));
        acc[2] = dadd(acc[2], dmul(bz, tap));
        acc[3] = dadd(acc[3], dmul(dsub((double)a.Ex[ir], bx), tap));
        acc[4] = dadd(acc[4], dmul(dsub((double)a.Ey[ir], by), tap));
        acc[5] = dadd(acc[5], dmul(dsub((double)a.Ez[ir], bz), tap));
        acc[6] = dadd(acc[6], dmul(tx, tap));
        acc[7] = dadd(acc[7], dmul(ty, tap));
        acc[8] = dadd(acc[8], dmul(tz, tap));
        acc[9] = dadd(acc[9], dmul((double)a.Ex[it], tap));
        acc[10] = dadd(acc[10], dmul((double)a.Ey[it], tap));
        acc[11] = dadd(acc[11], dmul((double)a.Ez[it], tap));
    }
    __shared__ double red[12][kPlaneThreads];
#pragma unroll
    for (int c = 0; c < 12; ++c) red[c][threadIdx.x] = acc[c];
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s)
#pragma unroll
            for (int c = 0; c < 12; ++c) red[c][threadIdx.x] += red[c][threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x < 12) part[b * 12 + threadIdx.x] = red[threadIdx.x][0];
}

// Fields interpolated to the node of cell (i, j, k): FDTD::local_E*/local_H*
// (fdtd_utils.cpp:457-507), periodic wrap at the upper faces. A: any argument
// struct with the grid sizes and the six field pointers.
template <typename T, typename A>
__device__ __forceinline__ void local_e(const A &a, int i, int j, int k, T f[3]) {
    const int ip = (i + 1 == a.Nx) ? 0 : i + 1;
    const int jp = (j + 1 == a.Ny) ? 0 : j + 1;
    const int kp = (k + 1 == a.Nz) ? 0 : k + 1;
    auto I = [&](int x, int y, int z) { return x + (long long)y * a.Nx + (long long)z * a.NxNy; };
    f[0] = (a.Ex[I(i, j, k)] + a.Ex[I(i, jp, k)] + a.Ex[I(i, j, kp)] + a.Ex[I(i, jp, kp)]) / T(4.0);
    f[1] = (a.Ey[I(i, j, k)] + a.Ey[I(ip, j, k)] + a.Ey[I(i, j, kp)] + a.Ey[I(ip, j, kp)]) / T(4.0);
    f[2] = (a.Ez[I(i, j, k)] + a.Ez[I(ip, j, k)] + a.Ez[I(i, jp, k)] + a.Ez[I(ip, jp, k)]) / T(4.0);
}
template <typename T, typename A>
__device__ __forceinline__ void local_h(const A &a, int i, int j, int k, T f[3]) {
    const int ip = (i + 1 == a.Nx) ? 0 : i + 1;
    const int jp = (j + 1 == a.Ny) ? 0 : j + 1;
    const int kp = (k + 1 == a.Nz) ? 0 : k + 1;
    auto I = [&](int x, int y, int z) { return x + (long long)y * a.Nx + (long long)z * a.NxNy; };
    f[0] = (a.Hx[I(i, j, k)] + a.Hx[I(ip, j, k)]) / T(2.0);
    f[1] = (a.Hy[I(i, j, k)] + a.Hy[I(i, jp, k)]) / T(2.0);
    f[2] = (a.Hz[I(i, j, k)] + a.Hz[I(i, j, kp)]) / T(2.0);
}

template <typename T>
__device__ __forceinline__ void gather_one(const SensorStepArgs<T> &a, const GatherDesc &g, int b) {
    const int q = (b - g.block0) * blockDim.x + threadIdx.x;
    if (q >= g.P) return;
    const int u = q % g.span1, v = q / g.span1;
    int i, j, k;
    if (g.type <= 1) { i = g.x1; j = g.y1 + u; k = g.z1 + v; }
    else if (g.type <= 3) { i = g.x1 + u; j = g.y1; k = g.z1 + v; }
    else { i = g.x1 + u; j = g.y1 + v; k = g.z1; }
    T *S = static_cast<T *>(g.S);
    T f[3];
    if (a.part == 0) local_e(a, i, j, k, f);
    else local_h(a, i, j, k, f);
    const int c0 = a.part ? 3 : 0;
#pragma unroll
    for (int c = 0; c < 3; ++c) S[(c0 + c) * (long long)g.P + q] = f[c];
}

// One cell (or map point) of a single-wavelength field sensor for step q.
// Plane maps (FieldMap::FT_compute, s_fieldmap.cpp:352-423): F at the plane,
// or summed along the normal over span3 planes in order (cumulative), then
// acc += e^{i w t Dt} F per component. Blocks (FieldBlock::FT_E*/FT_H*,
// :113-173, 191-228): acc += F e^{i w t Dt} (E, part 0) or e^{i w (t+1/2) Dt}
// (H, part 1). Points (FieldPoint::deep_feed, :711-719): E into row t - step0.
// Products and sums in FP64 with round-to-nearest intrinsics: the reference's
// complex x real product is two real products, the += two real sums.
template <typename T>
__device__ __forceinline__ void map_one(const MapStepArgs<T> &a, const MapDesc &m, int b) {
    const int p = (b - m.block0) * blockDim.x + threadIdx.x;
    if (p >= m.P) return;
    const double *cf = a.coef + ((size_t)a.q * kMaxMaps + m.slot) * 4;
    T f[3];
    if (m.kind == kMapPoint) {
        const int row = a.sc[a.q].step - m.step0;
        if (row < 0 || row >= m.cap) return;
        local_e(a, m.x1, m.y1, m.z1, f);
#pragma unroll
        for (int c = 0; c < 3; ++c) m.acc[(size_t)row * 3 + c] = (double)f[c];
        return;
    }
    double2 *acc = reinterpret_cast<double2 *>(m.acc);
    if (m.kind == kMapBlock) {
        const int i = m.x1 + p % m.span1, j = m.y1 + (p / m.span1) % m.span2, k = m.z1 + p / (m.span1 * m.span2);
        if (a.part == 0) local_e(a, i, j, k, f);
        else local_h(a, i, j, k, f);
        const double cr = cf[2 * a.part], ci = cf[2 * a.part + 1];
        acc += (size_t)(3 * a.part) * m.P + p;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            double2 v = acc[(size_t)c * m.P];
            v.x = dadd(v.x, dmul(cr, (double)f[c]));
            v.y = dadd(v.y, dmul(ci, (double)f[c]));
            acc[(size_t)c * m.P] = v;
        }
        return;
    }
    const int u = p % m.span1, v = p / m.span1;
    double S[3] = {0.0, 0.0, 0.0};
    for (int kk = 0; kk < m.span3; ++kk) {
        int i, j, k;
        if (m.type == 0) { i = m.x1 + kk; j = m.y1 + u; k = m.z1 + v; }
        else if (m.type == 1) { i = m.x1 + u; j = m.y1 + kk; k = m.z1 + v; }
        else { i = m.x1 + u; j = m.y1 + v; k = m.z1 + kk; }
        if (m.mag) local_h(a, i, j, k, f);
        else local_e(a, i, j, k, f);
#pragma unroll
        for (int c = 0; c < 3; ++c) S[c] = dadd(S[c], (double)f[c]);
    }
    const double cr = cf[0], ci = cf[1];
    acc += p;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        double2 w = acc[(size_t)c * m.P];
        w.x = dadd(w.x, dmul(cr, S[c]));
        w.y = dadd(w.y, dmul(ci, S[c]));
        acc[(size_t)c * m.P] = w;
    }
}

// One step of the FT-mode completion sensor: one thread per probe.
template <typename T>
__global__ void __launch_bounds__(kPlaneThreads) completion_ft_step(const __grid_constant__ CcFtArgs<T> a) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.np) return;
    T f[3];
    local_e(a, a.pts[3 * p], a.pts[3 * p + 1], a.pts[3 * p + 2], f);
    const double2 c = a.coef[(size_t)a.q * a.np + p];
    const int offset = (a.sc[a.q].step - a.step0) % a.n_avg;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        double2 v = a.acc[3 * p + d];
        v.x = dadd(v.x, dmul((double)f[d], c.x));
        v.y = dadd(v.y, dmul((double)f[d], c.y));
        a.acc[3 * p + d] = v;
        a.ring[((size_t)d * a.np + p) * a.n_avg + offset] = v.x;
        a.ring[((size_t)(3 + d) * a.np + p) * a.n_avg + offset] = v.y;
    }
    // a batch member's check step: this probe's ring as the check will read it
    const int slot = a.sc[a.q].snap;
    if (a.snap && slot >= 0) {
        const size_t per = (size_t)a.np * a.n_avg;
        for (int d = 0; d < 6; ++d)
            for (int j = 0; j < a.n_avg; ++j)
                a.snap[((size_t)slot * 6 + d) * per + (size_t)p * a.n_avg + j] = a.ring[((size_t)d * a.np + p) * a.n_avg + j];
    }
}

template <typename T>
__global__ void __launch_bounds__(kPlaneThreads) fieldmap_step(const __grid_constant__ MapStepArgs<T> a) {
    const int b = blockIdx.x;
    for (int s = 0; s < a.nm; ++s)
        if (b >= a.m[s].block0 && b < a.m[s].block0 + a.m[s].nblocks) {
            map_one(a, a.m[s], b);
            return;
        }
}

// One step of the sensors, in two launches. Part 0 (blocks [0, nbp) plane-sum
// partials, then the gather blocks) reads E only and may run beside the H
// half-step of the same step; part 1 (the gather blocks, block index offset by
// nbp) reads H only and may run beside the next E half-step.
template <typename T>
__global__ void __launch_bounds__(kPlaneThreads) sensor_step(const __grid_constant__ SensorStepArgs<T> a) {
    const int b = blockIdx.x + (a.part ? a.nbp : 0);
    if (b < a.nbp) {
        plane_partial(a, b, a.q, a.partial);
        return;
    }
    for (int s = 0; s < a.ng; ++s)
        if (b >= a.g[s].block0 && b < a.g[s].block0 + a.g[s].nblocks) {
            gather_one(a, a.g[s], b);
            return;
        }
}

// Plane sums of L steps from their block partials, block q summing step q's
// partials in block order; out[(sc[0].step + q) * 12 + c].
__global__ void plane_sums_reduce(const double *partial, int nbp, const StepScalars *sc, double *out) {
    const int q = blockIdx.x, c = threadIdx.x;
    if (c >= 12) return;
    double s = 0;
    const double *p = partial + (long long)q * nbp * 12;
    for (int b = 0; b < nbp; ++b) s += p[b * 12 + c];
    out[((long long)sc[0].step + q) * 12 + c] = s;
}

// Batched plane sums (normal-mode members of a batch, no sample gathers):
// block -> (instance, block of that instance) from blk; partials of step q at
// args[inst].partial + q * nbp * 12.
template <typename T>
__global__ void __launch_bounds__(kPlaneThreads)
plane_partial_batch(const SensorStepArgs<T> *__restrict__ args, const int2 *__restrict__ blk, int q) {
    const int2 m = blk[blockIdx.x];
    const SensorStepArgs<T> &a = args[m.x];
    plane_partial(a, m.y, q, a.partial + (long long)q * a.nbp * 12);
}

// grid (L, instances): instance x's step q sums into x.out[(sc[0].step + q) * 12 + c]
template <typename T>
__global__ void plane_sums_reduce_batch(const SensorStepArgs<T> *__restrict__ args) {
    const SensorStepArgs<T> &a = args[blockIdx.y];
    const int q = blockIdx.x, c = threadIdx.x;
    if (c >= 12 || a.nbp == 0) return;
    double s = 0;
    const double *p = a.partial + (long long)q * a.nbp * 12;
    for (int b = 0; b < a.nbp; ++b) s += p[b * 12 + c];
    a.out[((long long)a.sc[0].step + q) * 12 + c] = s;
}

// Completion sensor, energy mode (CompletionSensor::deep_feed,
// s_completion.cpp:177-190): sum of Ex^2 + Ey^2 + Ez^2 over the grid after a
// step. Block b of nb sums a contiguous chunk (threads strided, then a tree);
// the partials of step q go to part[q * nb + b] and are added in block order.
template <typename T>
__global__ void __launch_bounds__(kPlaneThreads)
energy_partial(const T *__restrict__ Ex, const T *__restrict__ Ey, const T *__restrict__ Ez, long long N, int nb,
               double *part) {
    const int b = blockIdx.x;
    const long long per = (N + nb - 1) / nb;
    const long long q0 = b * per, q1 = min(N, q0 + per);
    double s = 0;
    for (long long c = q0 + threadIdx.x; c < q1; c += blockDim.x) {
        const double ex = (double)Ex[c], ey = (double)Ey[c], ez = (double)Ez[c];
        s = dadd(s, dadd(dadd(dmul(ex, ex), dmul(ey, ey)), dmul(ez, ez)));
    }
    __shared__ double red[kPlaneThreads];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] = dadd(red[threadIdx.x], red[threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0) part[b] = red[0];
}

// grid L: step q's energy into hist[sc[0].step + q]
__global__ void energy_reduce(const double *part, int nb, const StepScalars *sc, double *hist) {
    if (threadIdx.x != 0) return;
    const int q = blockIdx.x;
    double s = 0;
    for (int b = 0; b < nb; ++b) s = dadd(s, part[(long long)q * nb + b]);
    hist[(long long)sc[0].step + q] = s;
}

// s_curve (src/common/mathUT.cpp:1186-1193)
__device__ __forceinline__ double s_curve_dev(double x, double xmin, double xmax) {
    const double u = (x - xmin) / (xmax - xmin);
    if (u <= 0) return 0;
    if (u >= 1.0) return 1.0;
    return u * u * (3.0 - 2.0 * u);
}

__global__ void dft_phasors(PhasorArgs a) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.nk * a.nl) return;
    const int kk = t / a.nl, l = t % a.nl;
    const int step = (a.step_ptr ? *a.step_ptr : 0) + a.step_add + kk;
    // tapering_E/H in effect at `step` were set after feeding step-1.
    double tE = 1.0, tH = 1.0;
    if (step - 1 >= a.Nt - a.Ntap && step >= 1) {
        tE = s_curve_dev(step - 1, a.Nt - 1.0, a.Nt - a.Ntap);
        tH = s_curve_dev(step - 1 + 0.5, a.Nt - 1.0, a.Nt - a.Ntap);
    }
    const double w = a.w[l];
    double sE, cE, sH, cH;
    sincos(w * step * a.Dt, &sE, &cE);
    sincos(w * (step + 0.5) * a.Dt, &sH, &cH);
    a.WE[t] = make_double2(tE * cE, tE * sE);
    a.WH[t] = make_double2(tH * cH, tH * sH);
}




// cp.async of BYTES (4, 8 or 16) from global to shared memory; an invalid
// source writes zeros (source size 0; the address is not read).
template <int BYTES> __device__ __forceinline__ void cp_async_zfill(void *smem, const void *gmem, bool valid) {
    const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
    const uint32_t n = valid ? BYTES : 0;
    if constexpr (BYTES == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(gmem), "r"(n) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;" ::"r"(d), "l"(gmem), "n"(BYTES), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_commit_group() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait_group() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// One DFT block of one component: acc[c][l][p] += sum_k S[k][c][p] W_c[k][l],
// as a tiled FP64 product. A CTA of 256 threads takes 64 points x 64
// wavelengths; each thread keeps a 4-point x 4-wavelength block of complex
// partial sums in registers (32 FMA per 8 shared-memory loads of one
// wavefront each). The K steps
// arrive in slices of kDftKSlice samples and phasors, double-buffered with
// cp.async so that the next slice loads while this one is multiplied; the
// CTA's 64 x 64 accumulator tile is copied into shared memory at the start
// (its latency hidden behind the products), the partial sums are added there
// and the tile is written back with coalesced stores. Partial sums start
// from zero and add the steps in order with FMA, then are added to the
// accumulators once, so a one-step block is the reference's
// acc + round(coeff * t) exactly.
// grid: (ceil(P / 64), ceil(nl / 64), 6); dynamic shared memory dft_acc_smem<T>()
constexpr int kDftKSlice = 16;
template <typename T> constexpr int dft_acc_smem() {
    return 64 * 64 * 16 + 2 * kDftKSlice * 64 * (int)sizeof(T) + 2 * kDftKSlice * 64 * 16;
}
template <typename T>
__global__ void __launch_bounds__(256, 2) dft_accumulate(AccumArgs<T> a) {
    extern __shared__ __align__(16) unsigned char dft_sm[];
    double2 *sAcc = reinterpret_cast<double2 *>(dft_sm);                                       // [64 l][64 p]
    double2 *sW = reinterpret_cast<double2 *>(dft_sm + 64 * 64 * 16);                          // [2][K][64 l]
    T *sS = reinterpret_cast<T *>(dft_sm + 64 * 64 * 16 + 2 * kDftKSlice * 64 * 16);           // [2][K][64 p]
    const int tid = threadIdx.x;
    const int p0 = blockIdx.x * 64, l0 = blockIdx.y * 64, c = blockIdx.z;
    const double2 *W = (c < 3) ? a.WE : a.WH;
    // points p0 + tp + 16 i (a half-warp's sample loads are one contiguous
    // 128-byte line), wavelengths l0 + 4 tl + f (two per warp: broadcast)
    const int tp = tid & 15, tl = tid >> 4;
    const int ns = (a.nk + kDftKSlice - 1) / kDftKSlice;
    auto stage = [&](int sl) {
        if (sl < ns) {
            const int kt = sl * kDftKSlice, b = sl & 1;
            for (int t = tid; t < kDftKSlice * 64; t += 256) {
                const int kk = t >> 6, x = t & 63;
                const bool kin = kt + kk < a.nk;
                const bool sv = kin && p0 + x < a.P, wv = kin && l0 + x < a.nl;
                cp_async_zfill<(int)sizeof(T)>(&sS[(b * kDftKSlice + kk) * 64 + x],
                                               sv ? a.S + ((long long)(kt + kk) * 6 + c) * a.P + p0 + x : a.S, sv);
                cp_async_zfill<16>(&sW[(b * kDftKSlice + kk) * 64 + x],
                                   wv ? W + (long long)(kt + kk) * a.nl + l0 + x : W, wv);
            }
        }
        cp_async_commit_group();   // empty groups keep the count uniform
    };
    stage(0);
    stage(1);
    // the accumulator tile, behind the first two slices
    for (int t = tid; t < 64 * 64; t += 256) {
        const int l = t >> 6, x = t & 63;
        const bool in = l0 + l < a.nl && p0 + x < a.P;
        cp_async_zfill<16>(&sAcc[t], in ? a.acc + ((long long)c * a.nl + l0 + l) * a.P + p0 + x : a.acc, in);
    }
    cp_async_commit_group();
    double re[4][4], im[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int f = 0; f < 4; ++f) { re[i][f] = 0; im[i][f] = 0; }
    for (int sl = 0; sl < ns; ++sl) {
        // groups so far: slices 0, 1, the tile, then slices 2 .. sl + 1
        if (sl < 2) cp_async_wait_group<2>();
        else cp_async_wait_group<1>();
        __syncthreads();
        const int kn = min(kDftKSlice, a.nk - sl * kDftKSlice), b = sl & 1;
        const T *S = sS + b * kDftKSlice * 64;
        const double2 *Wb = sW + b * kDftKSlice * 64;
        // threads whose wavelengths are all past nl (the last tile) leave the FP64 pipe to others
        for (int kk = 0; kk < (l0 + 4 * tl < a.nl ? kn : 0); ++kk) {
            double sv[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) sv[i] = (double)S[kk * 64 + tp + 16 * i];
            double2 wv[4];
#pragma unroll
            for (int f = 0; f < 4; ++f) wv[f] = Wb[kk * 64 + 4 * tl + f];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int f = 0; f < 4; ++f) {
                    re[i][f] = fma(sv[i], wv[f].x, re[i][f]);
                    im[i][f] = fma(sv[i], wv[f].y, im[i][f]);
                }
        }
        __syncthreads();   // the buffer is free for slice sl + 2
        stage(sl + 2);
    }
    cp_async_wait_group<0>();
    __syncthreads();
#pragma unroll
    for (int f = 0; f < 4; ++f)
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            double2 &v = sAcc[(4 * tl + f) * 64 + tp + 16 * i];
            v.x = v.x + re[i][f];
            v.y = v.y + im[i][f];
        }
    __syncthreads();
    for (int t = tid; t < 64 * 64; t += 256) {
        const int l = t >> 6, x = t & 63;
        if (l0 + l < a.nl && p0 + x < a.P) a.acc[((long long)c * a.nl + l0 + l) * a.P + p0 + x] = sAcc[t];
    }
}

// The same DFT block on the FP64 tensor path (mma.sync m8n8k4 f64; the
// tcgen05 MMA has no FP64 kind): per component the real product
// D[P x 2 nl] += S[P x K] W[K x 2 nl], columns (Re, Im) of each wavelength.
// A CTA of 8 warps takes 64 points x 64 wavelengths (128 columns); each warp
// 32 points x 32 columns as 4 x 4 tiles of 8 x 8, i.e. 16 accumulators of two
// doubles per thread. Samples and phasors arrive in slices of
// kDftMmaSlice steps, three buffers deep with cp.async (one barrier per
// slice, two slices in flight); the accumulator tile is copied to shared
// memory at the start, and the block's sums are added there and written
// back with coalesced stores, as in dft_accumulate. Rows of the staged
// slices are padded so that a fragment load (4 steps x 8 consecutive
// points or columns) takes two wavefronts without bank conflicts. Warps
// whose columns are all past nl skip their products. Products and sums are
// FP64; within a group of four steps the order of the sums is the MMA's, so
// spectra agree with dft_accumulate to rounding (a one-step block is still
// round(s * w) added once).
// grid: (ceil(P / 64), ceil(nl / 64), 6); dynamic shared memory dft_mma_smem<T>()
constexpr int kDftMmaSlice = 8;
constexpr int kDftMmaBufs = 3;
constexpr int kDftSRow = 72;    // doubles per staged sample row (64 points + pad)
constexpr int kDftWRow = 136;   // doubles per staged phasor row (128 columns + pad)
template <typename T> constexpr int dft_mma_smem() {
    return 64 * 64 * 16 + kDftMmaBufs * kDftMmaSlice * kDftWRow * 8 +
           kDftMmaBufs * kDftMmaSlice * kDftSRow * (int)sizeof(T);
}
__device__ __forceinline__ void mma_f64_m8n8k4(double &d0, double &d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}
template <typename T>
__global__ void __launch_bounds__(256, 2) dft_accumulate_mma(AccumArgs<T> a) {
    extern __shared__ __align__(16) unsigned char dft_sm[];
    double2 *sAcc = reinterpret_cast<double2 *>(dft_sm);                                   // [64 l][64 p]
    double *sW = reinterpret_cast<double *>(dft_sm + 64 * 64 * 16);                        // [bufs][K][kDftWRow]
    T *sS = reinterpret_cast<T *>(dft_sm + 64 * 64 * 16 + kDftMmaBufs * kDftMmaSlice * kDftWRow * 8);  // [bufs][K][kDftSRow]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int p0 = blockIdx.x * 64, l0 = blockIdx.y * 64, c = blockIdx.z;
    const double2 *W = (c < 3) ? a.WE : a.WH;
    const int ns = (a.nk + kDftMmaSlice - 1) / kDftMmaSlice;
    auto stage = [&](int sl) {
        if (sl < ns) {
            const int kt = sl * kDftMmaSlice, b = sl % kDftMmaBufs;
            for (int t = tid; t < kDftMmaSlice * 64; t += 256) {
                const int kk = t >> 6, x = t & 63;
                const bool kin = kt + kk < a.nk;
                const bool sv = kin && p0 + x < a.P, wv = kin && l0 + x < a.nl;
                cp_async_zfill<(int)sizeof(T)>(&sS[(b * kDftMmaSlice + kk) * kDftSRow + x],
                                               sv ? a.S + ((long long)(kt + kk) * 6 + c) * a.P + p0 + x : a.S, sv);
                cp_async_zfill<16>(&sW[(b * kDftMmaSlice + kk) * kDftWRow + 2 * x],
                                   wv ? W + (long long)(kt + kk) * a.nl + l0 + x : W, wv);
            }
        }
        cp_async_commit_group();   // empty groups keep the count uniform
    };
    stage(0);
    stage(1);
    for (int t = tid; t < 64 * 64; t += 256) {
        const int l = t >> 6, x = t & 63;
        const bool in = l0 + l < a.nl && p0 + x < a.P;
        cp_async_zfill<16>(&sAcc[t], in ? a.acc + ((long long)c * a.nl + l0 + l) * a.P + p0 + x : a.acc, in);
    }
    cp_async_commit_group();
    const int m0 = (warp & 1) * 32, n0 = (warp >> 1) * 32;   // warp tile: points m0.., columns n0..
    const bool live = l0 + n0 / 2 < a.nl;
    const int fr = lane & 3, fc = lane >> 2;                 // fragment: step row / point or column
    double d[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) { d[i][j][0] = 0; d[i][j][1] = 0; }
    for (int sl = 0; sl < ns; ++sl) {
        // groups so far: slices 0, 1, the tile, then slices 2 .. sl + 1
        if (sl < 2) cp_async_wait_group<2>();
        else cp_async_wait_group<1>();
        __syncthreads();   // slice sl visible; every warp is past slice sl - 1
        stage(sl + 2);     // into the buffer slice sl - 1 used
        if (!live) continue;
        const int b = sl % kDftMmaBufs;
        const T *S = sS + b * kDftMmaSlice * kDftSRow;
        const double *Wb = sW + b * kDftMmaSlice * kDftWRow;
#pragma unroll
        for (int k4 = 0; k4 < kDftMmaSlice; k4 += 4) {
            double af[4], bf[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) af[i] = (double)S[(k4 + fr) * kDftSRow + m0 + 8 * i + fc];
#pragma unroll
            for (int j = 0; j < 4; ++j) bf[j] = Wb[(k4 + fr) * kDftWRow + n0 + 8 * j + fc];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) mma_f64_m8n8k4(d[i][j][0], d[i][j][1], af[i], bf[j]);
        }
    }
    cp_async_wait_group<0>();
    __syncthreads();
    // D fragment: row (point) m0 + 8 i + lane / 4, columns n0 + 8 j + 2 (lane % 4) + {0, 1}
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            double2 &v = sAcc[((n0 + 8 * j) / 2 + fr) * 64 + m0 + 8 * i + fc];
            v.x = v.x + d[i][j][0];
            v.y = v.y + d[i][j][1];
        }
    __syncthreads();
    for (int t = tid; t < 64 * 64; t += 256) {
        const int l = t >> 6, x = t & 63;
        if (l0 + l < a.nl && p0 + x < a.P) a.acc[((long long)c * a.nl + l0 + l) * a.P + p0 + x] = sAcc[t];
    }
}

// One block per wavelength; deterministic reduction.
__global__ void __launch_bounds__(256) flux_reduce(FluxArgs a) {
    const int l = blockIdx.x;
    double sx = 0, sy = 0, sz = 0;
    const double2 *ex = a.acc + ((long long)0 * a.nl + l) * a.P, *ey = a.acc + ((long long)1 * a.nl + l) * a.P;
    const double2 *ez = a.acc + ((long long)2 * a.nl + l) * a.P, *hx = a.acc + ((long long)3 * a.nl + l) * a.P;
    const double2 *hy = a.acc + ((long long)4 * a.nl + l) * a.P, *hz = a.acc + ((long long)5 * a.nl + l) * a.P;
    for (int p = threadIdx.x; p < a.P; p += blockDim.x) {
        const double2 Ex = ex[p], Ey = ey[p], Ez = ez[p], Hx = hx[p], Hy = hy[p], Hz = hz[p];
        // Re(A*conj(B)) = A.re*B.re + A.im*B.im
        sx += (Ey.x * Hz.x + Ey.y * Hz.y) - (Ez.x * Hy.x + Ez.y * Hy.y);
        sy += (Ez.x * Hx.x + Ez.y * Hx.y) - (Ex.x * Hz.x + Ex.y * Hz.y);
        sz += (Ex.x * Hy.x + Ex.y * Hy.y) - (Ey.x * Hx.x + Ey.y * Hx.y);
    }
    __shared__ double red[3][256];
    red[0][threadIdx.x] = sx;
    red[1][threadIdx.x] = sy;
    red[2][threadIdx.x] = sz;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            red[0][threadIdx.x] += red[0][threadIdx.x + s];
            red[1][threadIdx.x] += red[1][threadIdx.x + s];
            red[2][threadIdx.x] += red[2][threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double Sx = red[0][0] * a.area_factor, Sy = red[1][0] * a.area_factor, Sz = red[2][0] * a.area_factor;
        double r = 0;
        switch (a.type) {
            case 0: r = Sx; break;
            case 1: r = -Sx; break;
            case 2: r = Sy; break;
            case 3: r = -Sy; break;
            case 4: r = Sz; break;
            case 5: r = -Sz; break;
        }
        a.out[l] = r;
    }
}

}  // namespace aefdtd
