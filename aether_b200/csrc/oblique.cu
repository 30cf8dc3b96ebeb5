// Kernels of the oblique driver (FDTD_oblique_biphase_comp,
// oblique_biphase.cpp:29-330). Compiled with --fmad=false: the products and
// sums follow the reference's std::complex<double> order term by term.
#include "kernels.hpp"

#include <algorithm>

namespace aefdtd {

constexpr int kOblThreads = 256;

// One thread per (step, part): the step's sum over the spectral lines in line
// order. part 0: Bloch_Wideband::inject_E's H sums, e^{-i(kz (z2 - 1/2) Dz +
// w Dt (t - 1/2 + t_offset))}; part 1: inject_H's E sums at (z2, t); part 2:
// get_E at z = zs_s Dz and time (t + 1/2) Dt, the z component a half cell up.
// e^{-ix} is (cos x, -sin x), as std::exp gives for (-0, -x).
__global__ void __launch_bounds__(kOblThreads) obl_incident(const OblIncArgs a) {
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= 3 * a.n) return;
    const int t = a.t0 + id / 3, part = id % 3;
    double2 s0 = make_double2(0, 0), s1 = s0, s2 = s0;
    if (part == 0) {
        const double zz = __dsub_rn((double)a.z2, 0.5);
        const double tt = __dadd_rn(__dsub_rn((double)t, 0.5), (double)a.t_offset);
        for (int l = 0; l < a.nl; ++l) {
            const double x = __dadd_rn(__dmul_rn(__dmul_rn(a.kz[l], zz), a.Dz), __dmul_rn(__dmul_rn(a.w[l], a.Dt), tt));
            double sn, cs;
            sincos(-x, &sn, &cs);
            const double hx = a.hb[2 * l], hy = a.hb[2 * l + 1];
            s0.x = __dadd_rn(s0.x, __dmul_rn(hx, cs)); s0.y = __dadd_rn(s0.y, __dmul_rn(hx, sn));
            s1.x = __dadd_rn(s1.x, __dmul_rn(hy, cs)); s1.y = __dadd_rn(s1.y, __dmul_rn(hy, sn));
        }
        double *o = a.out + (size_t)t * 14;
        o[0] = s0.x; o[1] = s0.y; o[2] = s1.x; o[3] = s1.y;
    } else if (part == 1) {
        const double tt = (double)(t + a.t_offset);
        for (int l = 0; l < a.nl; ++l) {
            const double x = __dadd_rn(__dmul_rn(__dmul_rn(a.kz[l], (double)a.z2), a.Dz),
                                       __dmul_rn(__dmul_rn(a.w[l], a.Dt), tt));
            double sn, cs;
            sincos(-x, &sn, &cs);
            const double ex = a.eb[3 * l], ey = a.eb[3 * l + 1];
            s0.x = __dadd_rn(s0.x, __dmul_rn(ex, cs)); s0.y = __dadd_rn(s0.y, __dmul_rn(ex, sn));
            s1.x = __dadd_rn(s1.x, __dmul_rn(ey, cs)); s1.y = __dadd_rn(s1.y, __dmul_rn(ey, sn));
        }
        double *o = a.out + (size_t)t * 14 + 4;
        o[0] = s0.x; o[1] = s0.y; o[2] = s1.x; o[3] = s1.y;
    } else {
        const double z = __dmul_rn((double)a.zs_s, a.Dz);
        const double zh = __dadd_rn(z, a.Dz / 2.0);
        const double tb = __dmul_rn(__dadd_rn((double)t, 0.5), a.Dt);
        const double tt = __dadd_rn(tb, __dmul_rn(a.Dt, (double)a.t_offset));
        for (int l = 0; l < a.nl; ++l) {
            const double wt = __dmul_rn(a.w[l], tt);
            const double x = __dadd_rn(__dmul_rn(a.kz[l], z), wt);
            const double xz = __dadd_rn(__dmul_rn(a.kz[l], zh), wt);
            double sn, cs, snz, csz;
            sincos(-x, &sn, &cs);
            sincos(-xz, &snz, &csz);
            const double ex = a.eb[3 * l], ey = a.eb[3 * l + 1], ez = a.eb[3 * l + 2];
            s0.x = __dadd_rn(s0.x, __dmul_rn(ex, cs)); s0.y = __dadd_rn(s0.y, __dmul_rn(ex, sn));
            s1.x = __dadd_rn(s1.x, __dmul_rn(ey, cs)); s1.y = __dadd_rn(s1.y, __dmul_rn(ey, sn));
            s2.x = __dadd_rn(s2.x, __dmul_rn(ez, csz)); s2.y = __dadd_rn(s2.y, __dmul_rn(ez, snz));
        }
        double *o = a.out + (size_t)t * 14 + 8;
        o[0] = s0.x; o[1] = s0.y; o[2] = s1.x; o[3] = s1.y; o[4] = s2.x; o[5] = s2.y;
    }
}

// Block partials of step q's R/T sums (oblique_biphase.cpp:300-327), 18
// doubles: BR x, y, z, R x, y, z, T x, y, z as (re, im). The incident field at
// a cell is Re(E_c e^{+i k.r}) (Bloch_Wideband::get_E); every term is a real
// field value times the cell's complex e^{-i k.r}.
template <typename T>
__global__ void __launch_bounds__(kOblThreads) obl_sums(const OblSumArgs<T> a) {
    __shared__ double red[18][kOblThreads];
    double acc[18];
#pragma unroll
    for (int c = 0; c < 18; ++c) acc[c] = 0;
    const long long P = a.NxNy;
    const double *v = a.inc + (size_t)a.sc[a.q].step * 14 + 8;
    const double2 *mx = a.mk, *my = a.mk + P, *mz = a.mk + 2 * P;
    const double2 *px = a.ph, *py = a.ph + P, *pz = a.ph + 2 * P;
    const long long r0 = (long long)a.kr * P, r1 = (long long)(a.kr - 1) * P;
    const long long t0 = (long long)a.kt * P, t1 = (long long)(a.kt - 1) * P;
    auto add = [&](int c, double f, double2 m) {
        acc[c] = __dadd_rn(acc[c], __dmul_rn(f, m.x));
        acc[c + 1] = __dadd_rn(acc[c + 1], __dmul_rn(f, m.y));
    };
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < P; p += (long long)gridDim.x * blockDim.x) {
        const double2 kx = mx[p], ky = my[p], kz = mz[p];
        const double2 ex = px[p], ey = py[p], ez = pz[p];
        add(0, __dsub_rn(__dmul_rn(v[0], ex.x), __dmul_rn(v[1], ex.y)), kx);
        add(2, __dsub_rn(__dmul_rn(v[2], ey.x), __dmul_rn(v[3], ey.y)), ky);
        add(4, __dsub_rn(__dmul_rn(v[4], ez.x), __dmul_rn(v[5], ez.y)), kz);
        add(6, (double)a.Ex[r0 + p], kx);
        add(8, (double)a.Ey[r0 + p], ky);
        add(10, __dmul_rn(0.5, __dadd_rn((double)a.Ez[r1 + p], (double)a.Ez[r0 + p])), kz);
        add(12, (double)a.Ex[t0 + p], kx);
        add(14, (double)a.Ey[t0 + p], ky);
        add(16, __dmul_rn(0.5, __dadd_rn((double)a.Ez[t0 + p], (double)a.Ez[t1 + p])), kz);
    }
#pragma unroll
    for (int c = 0; c < 18; ++c) red[c][threadIdx.x] = acc[c];
    __syncthreads();
    for (int s = kOblThreads / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s)
#pragma unroll
            for (int c = 0; c < 18; ++c) red[c][threadIdx.x] = __dadd_rn(red[c][threadIdx.x], red[c][threadIdx.x + s]);
        __syncthreads();
    }
    if (threadIdx.x < 18) a.partial[(size_t)blockIdx.x * 18 + threadIdx.x] = red[threadIdx.x][0];
}

// R/T sums of `steps` steps from their block partials, in block order.
__global__ void obl_reduce(const double *partial, int nb, const StepScalars *sc, double *hist) {
    const int q = blockIdx.x, c = threadIdx.x;
    if (c >= 18) return;
    const double *p = partial + (size_t)q * nb * 18;
    double s = 0;
    for (int b = 0; b < nb; ++b) s = __dadd_rn(s, p[(size_t)b * 18 + c]);
    hist[(size_t)(sc[0].step + q) * 18 + c] = s;
}

void launch_obl_incident(const OblIncArgs &a, cudaStream_t s) {
    const int n = 3 * a.n;
    if (n > 0) obl_incident<<<(n + kOblThreads - 1) / kOblThreads, kOblThreads, 0, s>>>(a);
}
template <typename T> static int sums_impl(const OblSumArgs<T> &a, int nb, cudaStream_t s) {
    obl_sums<<<nb, kOblThreads, 0, s>>>(a);
    return 1;
}
int launch_obl_sums(const OblSumArgs<double> &a, int nb, cudaStream_t s) { return sums_impl(a, nb, s); }
int launch_obl_sums(const OblSumArgs<float> &a, int nb, cudaStream_t s) { return sums_impl(a, nb, s); }
void launch_obl_reduce(const double *partial, int nb, const StepScalars *sc, double *hist, int steps, cudaStream_t s) {
    if (steps > 0) obl_reduce<<<steps, 32, 0, s>>>(partial, nb, sc, hist);
}

}  // namespace aefdtd
