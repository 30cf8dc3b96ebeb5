// yee.cuh — fused E and H half-step kernels.
//
// The E half-step fuses, per cell, the six phases of FDTD::update_E
// (src/finite_differences/FDTD/core/fdtd_core.cpp:1163-1218 driving
// fdtd_threads.cpp:32-150): recursive-convolution "ante" update with E^n
// (mats_RC.cpp:21-36), the Yee curl update (fdtd_core.cpp:363-541), the RC
// apply (mats_RC.cpp:38-50), the CPML psi updates and PEC planes in the
// reference's order (fdtd_pml.cpp:504-735), then the normal-mode plane
// injection (normal_incidence.cpp:338-342) or Oscillator boxes
// (sc_oscillator.cpp:34-67). The H half-step fuses advHx/Hy/Hz
// (fdtd_core.cpp:546-698), app_pml_H* (fdtd_pml.cpp:737-929) and the H plane
// injection (normal_incidence.cpp:353-357). Every phase of the reference only
// reads the other field family plus the cell's own state, so fusing them per
// cell is exact.
//
// Work decomposition. The grid is cut into work items: a 32 x 4 tile of
// (i, j) columns times a z-chunk. A CTA of 32 x 4 threads takes one item;
// each thread owns one column and marches the chunk along z, carrying the z-1
// (E) or z+1 (H) plane in registers, with x and y neighbours through L1. The
// host (runtime.cpp, build_work) tags every item with the features its cells
// need -- CPML or PEC on x/y, CPML or PEC on z, dispersive poles, plane
// injection or source boxes -- and sorts the items of each half-step into
// groups, each run by a kernel compiled for exactly those features:
//   * interior items (no feature): the curl update only, U z-planes per
//     iteration with all loads of the U planes issued before any store, so
//     each thread keeps U planes of reads in flight;
//   * z-CPML items: the same loop with the psi_z recursions and z PEC planes
//     (PZ instantiation of the interior kernels);
//   * x/y-CPML items (with or without z-CPML): the boundary kernel for
//     kFPmlXY | kFPmlZ (about 50 registers instead of 120);
//   * dispersive items and the rest (every phase): the boundary kernel
//     instantiated for feature sets kFDisp and kFAll.
// All groups of a half-step together cover each cell exactly once.
//
// FP64 instantiation (compiled with --fmad=false): operation order equals the
// reference's expression order, so results are bit-identical to the CPU
// core. FP32 instantiation: FP32 fields and state; CPML b and RC Crec are
// applied as (b-1) and (Crec-1) to keep their small decrements exact.
#pragma once

#include <cuda_runtime.h>
#include <type_traits>

#include "aefdtd_dev.hpp"

namespace aefdtd {

template <typename T> struct Exact { static constexpr bool value = std::is_same<T, double>::value; };

constexpr int kTileX = 32;
constexpr int kTileY = 4;   // default tile height (the batch autotuner may choose 2 or 8)

// psi_new = b*psi + c*diff (FP64, reference order) or psi + ((b-1)*psi + c*diff) (FP32)
template <typename T> __device__ __forceinline__ T cpml_rec(T b, T psi, T c, T diff) {
    if constexpr (Exact<T>::value) return b * psi + c * diff;
    else return psi + (b * psi + c * diff);
}

// L2 prefetch hint for the line holding p (no register result, no wait).
__device__ __forceinline__ void prefetch_l2(const void *p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

// Loads of the other field family (and of the oblique driver's other grid).
// Within one half-step launch those arrays do not change, so they go through
// the read-only path. In the persistent batch kernel (batch_persist.cuh) other
// CTAs rewrite them during the launch: Coh selects ordinary cached loads
// (ld.global.ca), which the kernel's acquire of a neighbour's progress counter
// orders after that neighbour's stores; read-only-path data may stay stale.
template <bool Coh, typename X> __device__ __forceinline__ X ldf(const X *p) {
    if constexpr (Coh) return __ldca(p);
    else return __ldg(p);
}

// Boundary-item features (bit mask per item; a kernel compiled for set F may
// run any item whose mask is a subset of F).
constexpr unsigned kFPmlXY = 1;   // a cell in an x or y CPML range or PEC plane
constexpr unsigned kFPmlZ = 2;    // a cell in a z CPML range or PEC plane
constexpr unsigned kFDisp = 4;    // a cell of a dispersive (recursive-convolution) material
constexpr unsigned kFMisc = 8;    // the injection plane or an oscillator box
constexpr unsigned kFAll = 15;

// ---- interior items: curl update only -----------------------------------
// Kernel bodies take the arguments by reference (from the parameter bank for
// one simulation, from a device array for a batch), the step's table index q
// and the item (x0, y0, k0, k1). A CTA is 32 x TY threads for tiles of 32 x
// TY columns (TY = 2, 4 or 8, chosen per launch).
// PZ: the item may also hold z-CPML planes and the z = 0 PEC plane (and no
// other feature): the psi_z recursions and PEC of app_pml_Ex/Ey
// (fdtd_pml.cpp:504-735) are applied after the curl update, in the general
// kernel's order.
template <typename T, typename Tid, int U, bool PZ = false, bool Coh = false>
__device__ __forceinline__ void e_interior_body(const StepArgs<T, Tid> &a, int q, int4 it) {
    // coefficients through the read-only path: short-lived CTAs skip a table fill and barrier
    const int i = it.x + threadIdx.x, j = it.y + threadIdx.y;
    if (i >= a.Nx || j >= a.Ny) return;
    const long long NxNy = a.NxNy;
    const int im = (i == 0) ? a.Nx - 1 : i - 1;
    const int jm = (j == 0) ? a.Ny - 1 : j - 1;
    const long long col = i + (long long)j * a.Nx;
    const long long colx = im + (long long)j * a.Nx;
    const long long coly = i + (long long)jm * a.Nx;
    const long long colm = i + (long long)j * a.mpitch;
    const long long mNxNy = (long long)a.mpitch * a.Ny;
    const T *__restrict__ Hx = a.Hx;
    const T *__restrict__ Hy = a.Hy;
    const T *__restrict__ Hz = a.Hz;
    T *__restrict__ Ex = a.Ex;
    T *__restrict__ Ey = a.Ey;
    T *__restrict__ Ez = a.Ez;
    const Tid *__restrict__ mat = a.mat;
    const MatCoef<T> *__restrict__ coef = a.coef;
    const T ikx = __ldg(a.ikx + i), iky = __ldg(a.iky + j);
    const int kmi = (it.z == 0) ? a.Nz - 1 : it.z - 1;
    T hx_km = ldf<Coh>(Hx + col + kmi * NxNy);
    T hy_km = ldf<Coh>(Hy + col + kmi * NxNy);
    if (a.prefetch & 1) {
        // every plane of the item into L2 up front: only the first iteration
        // waits on DRAM; the y-1 row lines are fetched by row 0 only
        for (int k = it.z; k < it.w; ++k) {
            const long long o = (long long)k * NxNy;
            prefetch_l2(Hx + col + o); prefetch_l2(Hy + col + o); prefetch_l2(Hz + col + o);
            prefetch_l2(Hz + colx + o); prefetch_l2(Hy + colx + o);
            if (threadIdx.y == 0) { prefetch_l2(Hz + coly + o); prefetch_l2(Hx + coly + o); }
            prefetch_l2(Ex + col + o); prefetch_l2(Ey + col + o); prefetch_l2(Ez + col + o);
            prefetch_l2(mat + colm + (long long)k * mNxNy);
            if constexpr (PZ) {
                if (a.pz && ((k >= 1 && k < a.pml_zm) || (k >= a.Nz - a.pml_zp + 1))) {
                    const int zn = (k < a.pml_zm) ? k : k - (a.Nz - a.pml_zp) + a.pml_zm;
                    prefetch_l2(a.psi_z0 + col + (long long)zn * NxNy);
                    prefetch_l2(a.psi_z1 + col + (long long)zn * NxNy);
                }
            }
        }
    }
    for (int k = it.z; k < it.w; k += U) {
        T hx[U], hy[U], hz[U], hz_jm[U], hx_jm[U], hz_im[U], hy_im[U], ex[U], ey[U], ez[U];
        int m[U];
        T p0[U], p1[U], bzv[U], czv[U];
        bool zeu[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            // planes past the chunk end re-read its last plane (not stored)
            const long long o = (long long)min(k + u, it.w - 1) * NxNy;
            hx[u] = ldf<Coh>(Hx + col + o); hy[u] = ldf<Coh>(Hy + col + o); hz[u] = ldf<Coh>(Hz + col + o);
            hz_jm[u] = ldf<Coh>(Hz + coly + o); hx_jm[u] = ldf<Coh>(Hx + coly + o);
            hz_im[u] = ldf<Coh>(Hz + colx + o); hy_im[u] = ldf<Coh>(Hy + colx + o);
            ex[u] = Ex[col + o]; ey[u] = Ey[col + o]; ez[u] = Ez[col + o];
            m[u] = __ldg(mat + colm + (long long)min(k + u, it.w - 1) * mNxNy);
            if constexpr (PZ) {
                // E-side z range [1, pml_zm) and [Nz - pml_zp + 1, Nz) (fdtd_pml.cpp:547,559)
                const int kk = min(k + u, it.w - 1);
                zeu[u] = a.pz && ((kk >= 1 && kk < a.pml_zm) || (kk >= a.Nz - a.pml_zp + 1));
                if (zeu[u]) {
                    const int zn = (kk < a.pml_zm) ? kk : kk - (a.Nz - a.pml_zp) + a.pml_zm;
                    const long long pz = col + (long long)zn * NxNy;
                    p0[u] = a.psi_z0[pz];
                    p1[u] = a.psi_z1[pz];
                    bzv[u] = __ldg(a.bz + kk);
                    czv[u] = __ldg(a.cz + kk);
                }
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const MatCoef<T> *cp = coef + m[u];
            const T C1 = __ldg(&cp->C1), C2x = __ldg(&cp->C2x), C2y = __ldg(&cp->C2y), C2z = __ldg(&cp->C2z);
            const int kk = min(k + u, it.w - 1);
            const T ikz = __ldg(a.ikz + kk);
            const T hxm = u ? hx[u - 1] : hx_km, hym = u ? hy[u - 1] : hy_km;
            T nex = (C1 * ex[u] + (C2y * iky) * (hz[u] - hz_jm[u])) - (C2z * ikz) * (hy[u] - hym);
            T ney = (C1 * ey[u] + (C2z * ikz) * (hx[u] - hxm)) - (C2x * ikx) * (hz[u] - hz_im[u]);
            const T nez = (C1 * ez[u] + (C2x * ikx) * (hy[u] - hy_im[u])) - (C2y * iky) * (hx[u] - hx_jm[u]);
            if constexpr (PZ) {
                if (zeu[u]) {
                    const T C4 = __ldg(&cp->C4);
                    const T ps0 = cpml_rec(bzv[u], p0[u], czv[u], hy[u] - hym);   // Ex: PsiExz
                    nex -= C4 * ps0;
                    const T ps1 = cpml_rec(bzv[u], p1[u], czv[u], hx[u] - hxm);   // Ey: PsiEyz
                    ney += C4 * ps1;
                    if (k + u < it.w) {
                        const int zn = (kk < a.pml_zm) ? kk : kk - (a.Nz - a.pml_zp) + a.pml_zm;
                        const long long pz = col + (long long)zn * NxNy;
                        a.psi_z0[pz] = ps0;
                        a.psi_z1[pz] = ps1;
                    }
                }
                if (a.pz && kk == 0) { nex = 0; ney = 0; }
            }
            if (k + u < it.w) {
                const long long id = col + (long long)kk * NxNy;
                Ex[id] = nex; Ey[id] = ney; Ez[id] = nez;
            }
        }
        hx_km = hx[U - 1];
        hy_km = hy[U - 1];
    }
}

// PZ: as for E, with the H-side z range, psi recursions and z = Nz-1 PEC of
// app_pml_Hx/Hy (fdtd_pml.cpp:737-929).
template <typename T, typename Tid, int U, bool PZ = false, bool Coh = false>
__device__ __forceinline__ void h_interior_body(const StepArgs<T, Tid> &a, int q, int4 it) {
    const int i = it.x + threadIdx.x, j = it.y + threadIdx.y;
    if (i >= a.Nx || j >= a.Ny) return;
    const long long NxNy = a.NxNy;
    const int ip = (i == a.Nx - 1) ? 0 : i + 1;
    const int jp = (j == a.Ny - 1) ? 0 : j + 1;
    const long long col = i + (long long)j * a.Nx;
    const long long colx = ip + (long long)j * a.Nx;
    const long long coly = i + (long long)jp * a.Nx;
    const T *__restrict__ Ex = a.Ex;
    const T *__restrict__ Ey = a.Ey;
    const T *__restrict__ Ez = a.Ez;
    T *__restrict__ Hx = a.Hx;
    T *__restrict__ Hy = a.Hy;
    T *__restrict__ Hz = a.Hz;
    const T ax = a.dtdmx * __ldg(a.ikx + i);
    const T ay = a.dtdmy * __ldg(a.iky + j);
    T ex = ldf<Coh>(Ex + col + it.z * NxNy);
    T ey = ldf<Coh>(Ey + col + it.z * NxNy);
    if (a.prefetch & 1) {
        // every plane of the item (and the E plane above it) into L2 up front;
        // the y+1 row lines are fetched by the last row only
        for (int k = it.z; k < it.w; ++k) {
            const int kp = (k == a.Nz - 1) ? 0 : k + 1;
            const long long o = (long long)k * NxNy, op = (long long)kp * NxNy;
            prefetch_l2(Ex + col + op); prefetch_l2(Ey + col + op); prefetch_l2(Ez + col + o);
            prefetch_l2(Ez + colx + o); prefetch_l2(Ey + colx + o);
            if (threadIdx.y == blockDim.y - 1) { prefetch_l2(Ez + coly + o); prefetch_l2(Ex + coly + o); }
            prefetch_l2(Hx + col + o); prefetch_l2(Hy + col + o); prefetch_l2(Hz + col + o);
            if constexpr (PZ) {
                if (a.pz && ((k < a.pml_zm) || (k >= a.Nz - a.pml_zp && k < a.Nz - 1))) {
                    const int zn = (k < a.pml_zm) ? k : k - (a.Nz - a.pml_zp) + a.pml_zm;
                    prefetch_l2(a.psi_z0 + col + (long long)zn * NxNy);
                    prefetch_l2(a.psi_z1 + col + (long long)zn * NxNy);
                }
            }
        }
    }
    for (int k = it.z; k < it.w; k += U) {
        T ex_kp[U], ey_kp[U], ez[U], ez_jp[U], ex_jp[U], ez_ip[U], ey_ip[U], hx[U], hy[U], hz[U];
        T p0[U], p1[U], bzv[U], czv[U];
        bool zhu[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int kk = min(k + u, it.w - 1);
            const int kp = (kk == a.Nz - 1) ? 0 : kk + 1;
            const long long o = (long long)kk * NxNy, op = (long long)kp * NxNy;
            ex_kp[u] = ldf<Coh>(Ex + col + op); ey_kp[u] = ldf<Coh>(Ey + col + op);
            ez[u] = ldf<Coh>(Ez + col + o);
            ez_jp[u] = ldf<Coh>(Ez + coly + o); ex_jp[u] = ldf<Coh>(Ex + coly + o);
            ez_ip[u] = ldf<Coh>(Ez + colx + o); ey_ip[u] = ldf<Coh>(Ey + colx + o);
            hx[u] = Hx[col + o]; hy[u] = Hy[col + o]; hz[u] = Hz[col + o];
            if constexpr (PZ) {
                // H-side z range [0, pml_zm) and [Nz - pml_zp, Nz - 1) (fdtd_pml.cpp:775,784)
                zhu[u] = a.pz && ((kk < a.pml_zm) || (kk >= a.Nz - a.pml_zp && kk < a.Nz - 1));
                if (zhu[u]) {
                    const int zn = (kk < a.pml_zm) ? kk : kk - (a.Nz - a.pml_zp) + a.pml_zm;
                    const long long pz = col + (long long)zn * NxNy;
                    p0[u] = a.psi_z0[pz];
                    p1[u] = a.psi_z1[pz];
                    bzv[u] = __ldg(a.bz + kk);
                    czv[u] = __ldg(a.cz + kk);
                }
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int kk = min(k + u, it.w - 1);
            const T az = a.dtdmz * __ldg(a.ikz + kk);
            const T exk = u ? ex_kp[u - 1] : ex, eyk = u ? ey_kp[u - 1] : ey;
            T nhx = hx[u] + (az * (ey_kp[u] - eyk) - ay * (ez_jp[u] - ez[u]));
            T nhy = hy[u] + (ax * (ez_ip[u] - ez[u]) - az * (ex_kp[u] - exk));
            const T nhz = hz[u] + (ay * (ex_jp[u] - exk) - ax * (ey_ip[u] - eyk));
            if constexpr (PZ) {
                if (zhu[u]) {
                    const T ps0 = cpml_rec(bzv[u], p0[u], czv[u], ey_kp[u] - eyk);   // Hx: PsiHxz
                    nhx += a.dtm * ps0;
                    const T ps1 = cpml_rec(bzv[u], p1[u], czv[u], ex_kp[u] - exk);   // Hy: PsiHyz
                    nhy -= a.dtm * ps1;
                    if (k + u < it.w) {
                        const int zn = (kk < a.pml_zm) ? kk : kk - (a.Nz - a.pml_zp) + a.pml_zm;
                        const long long pz = col + (long long)zn * NxNy;
                        a.psi_z0[pz] = ps0;
                        a.psi_z1[pz] = ps1;
                    }
                }
                if (a.pz && kk == a.Nz - 1) { nhx = 0; nhy = 0; }
            }
            if (k + u < it.w) {
                const long long id = col + (long long)kk * NxNy;
                Hx[id] = nhx; Hy[id] = nhy; Hz[id] = nhz;
            }
        }
        ex = ex_kp[U - 1];
        ey = ey_kp[U - 1];
    }
}

// Bloch wrap of the oblique driver (oblique_biphase.cpp:211-290): the value
// past the x or y edge is the wrapped cell's complex field (real grid +
// i imaginary grid) times the Bloch phase c + i d; the real grid takes the
// real part, the imaginary grid the imaginary part, in std::complex order.
template <typename T>
__device__ __forceinline__ T bloch_ghost(int bloch, T own, T other, double c, double d) {
    const T tc = (T)c, td = (T)d;
    return bloch == 1 ? own * tc - other * td : other * td + own * tc;
}

// ---- boundary items: the phases of feature set F ---------------------------
template <typename T, typename Tid, unsigned F, bool Coh = false>
__device__ __forceinline__ void e_boundary_body(const StepArgs<T, Tid> &a, int q, int4 it) {
    const int i = it.x + threadIdx.x, j = it.y + threadIdx.y;
    if (i >= a.Nx || j >= a.Ny) return;
    const int k0 = it.z, k1 = it.w;
    const long long NxNy = a.NxNy;
    const int im = (i == 0) ? a.Nx - 1 : i - 1;
    const int jm = (j == 0) ? a.Ny - 1 : j - 1;
    const long long col = i + (long long)j * a.Nx;
    const long long colx = im + (long long)j * a.Nx;
    const long long coly = i + (long long)jm * a.Nx;
    const long long colm = i + (long long)j * a.mpitch;
    const long long mNxNy = (long long)a.mpitch * a.Ny;
    const T *__restrict__ Hx = a.Hx;
    const T *__restrict__ Hy = a.Hy;
    const T *__restrict__ Hz = a.Hz;
    T *__restrict__ Ex = a.Ex;
    T *__restrict__ Ey = a.Ey;
    T *__restrict__ Ez = a.Ez;
    const T ikx = __ldg(a.ikx + i);
    const T iky = __ldg(a.iky + j);

    // E-side CPML index ranges: [1, pml_m) and [N - pml_p + 1, N) (fdtd_pml.cpp:518,527,547,559)
    bool xe = false, ye = false;
    int xn = 0, yn = 0;
    const int nxs = a.pml_xm + a.pml_xp, nys = a.pml_ym + a.pml_yp;
    T bxi = 0, cxi = 0, byj = 0, cyj = 0;
    if constexpr ((F & kFPmlXY) != 0) {
        xe = a.px && ((i >= 1 && i < a.pml_xm) || (i >= a.Nx - a.pml_xp + 1));
        ye = a.py && ((j >= 1 && j < a.pml_ym) || (j >= a.Ny - a.pml_yp + 1));
        xn = (i < a.pml_xm) ? i : i - (a.Nx - a.pml_xp) + a.pml_xm;
        yn = (j < a.pml_ym) ? j : j - (a.Ny - a.pml_yp) + a.pml_ym;
        if (xe) { bxi = __ldg(a.bx + i); cxi = __ldg(a.cx + i); }
        if (ye) { byj = __ldg(a.by + j); cyj = __ldg(a.cy + j); }
    }

    if constexpr (F == (kFPmlXY | kFPmlZ)) {
        // CPML items: every plane of the item (fields, ids, psi slabs) into L2 up front
        if (a.prefetch & 2)
            for (int k = k0; k < k1; ++k) {
                const long long o = (long long)k * NxNy;
                prefetch_l2(Hx + col + o); prefetch_l2(Hy + col + o); prefetch_l2(Hz + col + o);
                prefetch_l2(Hz + colx + o); prefetch_l2(Hy + colx + o);
                if (threadIdx.y == 0) { prefetch_l2(Hz + coly + o); prefetch_l2(Hx + coly + o); }
                prefetch_l2(Ex + col + o); prefetch_l2(Ey + col + o); prefetch_l2(Ez + col + o);
                prefetch_l2(a.mat + colm + (long long)k * mNxNy);
                if (xe) {
                    const long long px = xn + (long long)j * nxs + (long long)k * nxs * a.Ny;
                    prefetch_l2(a.psi_x0 + px); prefetch_l2(a.psi_x1 + px);
                }
                if (ye) {
                    const long long py = i + (long long)yn * a.Nx + (long long)k * a.Nx * nys;
                    prefetch_l2(a.psi_y0 + py); prefetch_l2(a.psi_y1 + py);
                }
                if (a.pz && ((k >= 1 && k < a.pml_zm) || (k >= a.Nz - a.pml_zp + 1))) {
                    const int zn = (k < a.pml_zm) ? k : k - (a.Nz - a.pml_zp) + a.pml_zm;
                    prefetch_l2(a.psi_z0 + col + (long long)zn * NxNy);
                    prefetch_l2(a.psi_z1 + col + (long long)zn * NxNy);
                }
            }
    }
    const int kmi = (k0 == 0) ? a.Nz - 1 : k0 - 1;
    T hx_km = ldf<Coh>(Hx + col + kmi * NxNy);
    T hy_km = ldf<Coh>(Hy + col + kmi * NxNy);

    for (int k = k0; k < k1; ++k) {
        const long long id = col + k * NxNy;
        const T hx = ldf<Coh>(Hx + id), hy = ldf<Coh>(Hy + id), hz = ldf<Coh>(Hz + id);
        T hz_jm = ldf<Coh>(Hz + coly + k * NxNy), hx_jm = ldf<Coh>(Hx + coly + k * NxNy);
        T hz_im = ldf<Coh>(Hz + colx + k * NxNy), hy_im = ldf<Coh>(Hy + colx + k * NxNy);
        if constexpr ((F & kFMisc) != 0) {
            // oblique driver: H ghosts past the y = 0 and x = 0 edges (set before update_E)
            if (a.bloch) {
                if (j == 0) {
                    hz_jm = bloch_ghost(a.bloch, hz_jm, ldf<Coh>(a.oHz + coly + k * NxNy), a.byr, a.byi);
                    hx_jm = bloch_ghost(a.bloch, hx_jm, ldf<Coh>(a.oHx + coly + k * NxNy), a.byr, a.byi);
                }
                if (i == 0) {
                    hz_im = bloch_ghost(a.bloch, hz_im, ldf<Coh>(a.oHz + colx + k * NxNy), a.bxr, a.bxi);
                    hy_im = bloch_ghost(a.bloch, hy_im, ldf<Coh>(a.oHy + colx + k * NxNy), a.bxr, a.bxi);
                }
            }
        }
        const T ex = Ex[id], ey = Ey[id], ez = Ez[id];
        const int m = __ldg(a.mat + colm + k * mNxNy);
        const MatCoef<T> c = a.coef[m];
        const T ikz = __ldg(a.ikz + k);

        // Recursive-convolution "ante" with E^n; sums of Re(psi) per component.
        T s0 = 0, s1 = 0, s2 = 0;
        int np_m = 0;
        if constexpr ((F & kFDisp) != 0) {
            np_m = a.disp ? __ldg(&a.disp[m].np) : 0;
            if (np_m > 0) {
                const DispInfo d = a.disp[m];
                const long long q = (i - d.x1) + (long long)(j - d.y1) * d.xs + (long long)(k - d.z1) * d.xs * d.ys;
                Cplx<T> *__restrict__ P = a.psi + d.psi_off + q;
                const T ev[3] = {ex, ey, ez};
                // up to four poles at a time: every psi load issued before any
                // store, then the updates in pole order (the sums keep the
                // reference's order over poles)
                for (int p0 = 0; p0 < d.np; p0 += 4) {
                    const int pn = min(4, d.np - p0);
                    Cplx<T> v[4][3], cr[4], dc[4];
#pragma unroll
                    for (int p = 0; p < 4; ++p)
                        if (p < pn) {
                            cr[p] = a.crec[d.pole_off + p0 + p];
                            dc[p] = a.dchi[d.pole_off + p0 + p];
#pragma unroll
                            for (int dd = 0; dd < 3; ++dd) v[p][dd] = P[(long long)(3 * (p0 + p) + dd) * d.box];
                        }
#pragma unroll
                    for (int p = 0; p < 4; ++p)
                        if (p < pn) {
#pragma unroll
                            for (int dd = 0; dd < 3; ++dd) {
                                Cplx<T> r;
                                if constexpr (Exact<T>::value) {
                                    // Crec*psi + Dchi*E with std::complex<double> rounding order
                                    r.re = (cr[p].re * v[p][dd].re - cr[p].im * v[p][dd].im) + dc[p].re * ev[dd];
                                    r.im = (cr[p].re * v[p][dd].im + cr[p].im * v[p][dd].re) + dc[p].im * ev[dd];
                                } else {
                                    // (Crec-1) stored: psi + ((Crec-1)*psi + Dchi*E)
                                    r.re = v[p][dd].re + ((cr[p].re * v[p][dd].re - cr[p].im * v[p][dd].im) + dc[p].re * ev[dd]);
                                    r.im = v[p][dd].im + ((cr[p].re * v[p][dd].im + cr[p].im * v[p][dd].re) + dc[p].im * ev[dd]);
                                }
                                P[(long long)(3 * (p0 + p) + dd) * d.box] = r;
                                if (dd == 0) s0 = s0 + r.re;
                                else if (dd == 1) s1 = s1 + r.re;
                                else s2 = s2 + r.re;
                            }
                        }
                }
            }
        }

        const T dHz_y = hz - hz_jm, dHy_z = hy - hy_km;
        const T dHx_z = hx - hx_km, dHz_x = hz - hz_im;
        const T dHy_x = hy - hy_im, dHx_y = hx - hx_jm;
        T nex = (c.C1 * ex + (c.C2y * iky) * dHz_y) - (c.C2z * ikz) * dHy_z;
        T ney = (c.C1 * ey + (c.C2z * ikz) * dHx_z) - (c.C2x * ikx) * dHz_x;
        T nez = (c.C1 * ez + (c.C2x * ikx) * dHy_x) - (c.C2y * iky) * dHx_y;
        if constexpr ((F & kFDisp) != 0) {
            if (np_m > 0) {
                nex += c.C3 * s0;
                ney += c.C3 * s1;
                nez += c.C3 * s2;
            }
        }

        // CPML and PEC planes in app_pml_Ex / Ey / Ez order. Every psi value the
        // cell needs is loaded before any is stored (the six arrays are distinct),
        // so the loads are in flight together.
        bool ze = false;
        int zn = 0;
        T bzk = 0, czk = 0;
        if constexpr ((F & kFPmlZ) != 0) {
            ze = a.pz && ((k >= 1 && k < a.pml_zm) || (k >= a.Nz - a.pml_zp + 1));
            zn = (k < a.pml_zm) ? k : k - (a.Nz - a.pml_zp) + a.pml_zm;
            if (ze) { bzk = __ldg(a.bz + k); czk = __ldg(a.cz + k); }
        }
        const long long oy = i + (long long)yn * a.Nx + (long long)k * a.Nx * nys;
        const long long ox = xn + (long long)j * nxs + (long long)k * nxs * a.Ny;
        const long long oz = col + (long long)zn * NxNy;
        T qy0 = 0, qy1 = 0, qx0 = 0, qx1 = 0, qz0 = 0, qz1 = 0;
        if constexpr ((F & kFPmlXY) != 0) {
            if (ye) { qy0 = a.psi_y0[oy]; qy1 = a.psi_y1[oy]; }
            if (xe) { qx0 = a.psi_x0[ox]; qx1 = a.psi_x1[ox]; }
        }
        if constexpr ((F & kFPmlZ) != 0) {
            if (ze) { qz0 = a.psi_z0[oz]; qz1 = a.psi_z1[oz]; }
        }
        // Ex: y block, then z block
        if constexpr ((F & kFPmlXY) != 0) {
            if (ye) {
                const T ps = cpml_rec(byj, qy0, cyj, dHz_y);
                a.psi_y0[oy] = ps;
                nex += c.C4 * ps;
            }
            if (a.py && j == 0) nex = 0;
        }
        if constexpr ((F & kFPmlZ) != 0) {
            if (ze) {
                const T ps = cpml_rec(bzk, qz0, czk, dHy_z);
                a.psi_z0[oz] = ps;
                nex -= c.C4 * ps;
            }
            if (a.pz && k == 0) nex = 0;
        }
        // Ey: x block, then z block
        if constexpr ((F & kFPmlXY) != 0) {
            if (xe) {
                const T ps = cpml_rec(bxi, qx0, cxi, dHz_x);
                a.psi_x0[ox] = ps;
                ney -= c.C4 * ps;
            }
            if (a.px && i == 0) ney = 0;
        }
        if constexpr ((F & kFPmlZ) != 0) {
            if (ze) {
                const T ps = cpml_rec(bzk, qz1, czk, dHx_z);
                a.psi_z1[oz] = ps;
                ney += c.C4 * ps;
            }
            if (a.pz && k == 0) ney = 0;
        }
        // Ez: x block, then y block
        if constexpr ((F & kFPmlXY) != 0) {
            if (xe) {
                const T ps = cpml_rec(bxi, qx1, cxi, dHy_x);
                a.psi_x1[ox] = ps;
                nez += c.C4 * ps;
            }
            if (a.px && i == 0) nez = 0;
            if (ye) {
                const T ps = cpml_rec(byj, qy1, cyj, dHx_y);
                a.psi_y1[oy] = ps;
                nez -= c.C4 * ps;
            }
            if (a.py && j == 0) nez = 0;
        }

        if constexpr ((F & kFMisc) != 0) {
            // Normal-incidence plane injection after update_E (normal_incidence.cpp:338-342)
            if (k == a.kinj) {
                nex = nex - (T)a.sc[q].inj_eA;
                ney = ney + (T)a.sc[q].inj_eB;
            }
            // Bloch_Wideband::inject_E after update_E (sc_bloch.cpp:216-250): the
            // step's complex H sums times the column's phase, real or imaginary part
            if (k == a.kobl) {
                const double *v = a.obl_inc + (size_t)a.sc[q].step * 14;
                const double2 px = a.obl_px[col], py = a.obl_py[col];
                const double hyr = v[2] * px.x - v[3] * px.y, hyi = v[2] * px.y + v[3] * px.x;
                const double hxr = v[0] * py.x - v[1] * py.y, hxi = v[0] * py.y + v[1] * py.x;
                nex = nex - (T)(a.obl_coef * (a.bloch == 1 ? hyr : hyi));
                ney = ney + (T)(a.obl_coef * (a.bloch == 1 ? hxr : hxi));
            }
            // Oscillator boxes after update_E (sc_oscillator.cpp:43-63)
            for (int s = 0; s < a.nsrc; ++s) {
                const int *b = a.src_box[s];
                if (i >= b[0] && i < b[1] && j >= b[2] && j < b[3] && k >= b[4] && k < b[5]) {
                    const T v = (T)a.sc[q].src[s];
                    if (a.src_comp[s] == 0) nex += v;
                    else if (a.src_comp[s] == 1) ney += v;
                    else nez += v;
                }
            }
        }

        Ex[id] = nex;
        Ey[id] = ney;
        Ez[id] = nez;
        hx_km = hx;
        hy_km = hy;
    }
}

template <typename T, typename Tid, unsigned F, bool Coh = false>
__device__ __forceinline__ void h_boundary_body(const StepArgs<T, Tid> &a, int q, int4 it) {
    const int i = it.x + threadIdx.x, j = it.y + threadIdx.y;
    if (i >= a.Nx || j >= a.Ny) return;
    const int k0 = it.z, k1 = it.w;
    const long long NxNy = a.NxNy;
    const int ip = (i == a.Nx - 1) ? 0 : i + 1;
    const int jp = (j == a.Ny - 1) ? 0 : j + 1;
    const long long col = i + (long long)j * a.Nx;
    const long long colx = ip + (long long)j * a.Nx;
    const long long coly = i + (long long)jp * a.Nx;
    const T *__restrict__ Ex = a.Ex;
    const T *__restrict__ Ey = a.Ey;
    const T *__restrict__ Ez = a.Ez;
    T *__restrict__ Hx = a.Hx;
    T *__restrict__ Hy = a.Hy;
    T *__restrict__ Hz = a.Hz;
    const T ax = a.dtdmx * __ldg(a.ikx + i);
    const T ay = a.dtdmy * __ldg(a.iky + j);

    // H-side CPML index ranges: [0, pml_m) and [N - pml_p, N - 1) (fdtd_pml.cpp:750,756,775,784)
    bool xh = false, yh = false;
    int xn = 0, yn = 0;
    const int nxs = a.pml_xm + a.pml_xp, nys = a.pml_ym + a.pml_yp;
    T bxi = 0, cxi = 0, byj = 0, cyj = 0;
    if constexpr ((F & kFPmlXY) != 0) {
        xh = a.px && ((i < a.pml_xm) || (i >= a.Nx - a.pml_xp && i < a.Nx - 1));
        yh = a.py && ((j < a.pml_ym) || (j >= a.Ny - a.pml_yp && j < a.Ny - 1));
        xn = (i < a.pml_xm) ? i : i - (a.Nx - a.pml_xp) + a.pml_xm;
        yn = (j < a.pml_ym) ? j : j - (a.Ny - a.pml_yp) + a.pml_ym;
        if (xh) { bxi = __ldg(a.bx + i); cxi = __ldg(a.cx + i); }
        if (yh) { byj = __ldg(a.by + j); cyj = __ldg(a.cy + j); }
    }

    if constexpr (F == (kFPmlXY | kFPmlZ)) {
        if (a.prefetch & 2)
            for (int k = k0; k < k1; ++k) {
                const int kp = (k == a.Nz - 1) ? 0 : k + 1;
                const long long o = (long long)k * NxNy, op = (long long)kp * NxNy;
                prefetch_l2(Ex + col + op); prefetch_l2(Ey + col + op); prefetch_l2(Ez + col + o);
                prefetch_l2(Ez + colx + o); prefetch_l2(Ey + colx + o);
                if (threadIdx.y == blockDim.y - 1) { prefetch_l2(Ez + coly + o); prefetch_l2(Ex + coly + o); }
                prefetch_l2(Hx + col + o); prefetch_l2(Hy + col + o); prefetch_l2(Hz + col + o);
                if (xh) {
                    const long long px = xn + (long long)j * nxs + (long long)k * nxs * a.Ny;
                    prefetch_l2(a.psi_x0 + px); prefetch_l2(a.psi_x1 + px);
                }
                if (yh) {
                    const long long py = i + (long long)yn * a.Nx + (long long)k * a.Nx * nys;
                    prefetch_l2(a.psi_y0 + py); prefetch_l2(a.psi_y1 + py);
                }
                if (a.pz && ((k < a.pml_zm) || (k >= a.Nz - a.pml_zp && k < a.Nz - 1))) {
                    const int zn = (k < a.pml_zm) ? k : k - (a.Nz - a.pml_zp) + a.pml_zm;
                    prefetch_l2(a.psi_z0 + col + (long long)zn * NxNy);
                    prefetch_l2(a.psi_z1 + col + (long long)zn * NxNy);
                }
            }
    }
    T ex = ldf<Coh>(Ex + col + k0 * NxNy);
    T ey = ldf<Coh>(Ey + col + k0 * NxNy);

    for (int k = k0; k < k1; ++k) {
        const long long id = col + k * NxNy;
        const int kp = (k == a.Nz - 1) ? 0 : k + 1;
        const T ex_kp = ldf<Coh>(Ex + col + kp * NxNy), ey_kp = ldf<Coh>(Ey + col + kp * NxNy);
        const T ez = ldf<Coh>(Ez + id);
        T ez_jp = ldf<Coh>(Ez + coly + k * NxNy), ex_jp = ldf<Coh>(Ex + coly + k * NxNy);
        T ez_ip = ldf<Coh>(Ez + colx + k * NxNy), ey_ip = ldf<Coh>(Ey + colx + k * NxNy);
        if constexpr ((F & kFMisc) != 0) {
            // oblique driver: E ghosts past the y = Ny-1 and x = Nx-1 edges (set after inject_E)
            if (a.bloch) {
                if (j == a.Ny - 1) {
                    ez_jp = bloch_ghost(a.bloch, ez_jp, ldf<Coh>(a.oEz + coly + k * NxNy), a.byr, a.byi);
                    ex_jp = bloch_ghost(a.bloch, ex_jp, ldf<Coh>(a.oEx + coly + k * NxNy), a.byr, a.byi);
                }
                if (i == a.Nx - 1) {
                    ez_ip = bloch_ghost(a.bloch, ez_ip, ldf<Coh>(a.oEz + colx + k * NxNy), a.bxr, a.bxi);
                    ey_ip = bloch_ghost(a.bloch, ey_ip, ldf<Coh>(a.oEy + colx + k * NxNy), a.bxr, a.bxi);
                }
            }
        }
        const T hx = Hx[id], hy = Hy[id], hz = Hz[id];
        const T az = a.dtdmz * __ldg(a.ikz + k);

        const T dEy_z = ey_kp - ey, dEz_y = ez_jp - ez;
        const T dEz_x = ez_ip - ez, dEx_z = ex_kp - ex;
        const T dEx_y = ex_jp - ex, dEy_x = ey_ip - ey;
        T nhx = hx + (az * dEy_z - ay * dEz_y);
        T nhy = hy + (ax * dEz_x - az * dEx_z);
        T nhz = hz + (ay * dEx_y - ax * dEy_x);

        bool zh = false;
        int zn = 0;
        T bzk = 0, czk = 0;
        if constexpr ((F & kFPmlZ) != 0) {
            zh = a.pz && ((k < a.pml_zm) || (k >= a.Nz - a.pml_zp && k < a.Nz - 1));
            zn = (k < a.pml_zm) ? k : k - (a.Nz - a.pml_zp) + a.pml_zm;
            if (zh) { bzk = __ldg(a.bz + k); czk = __ldg(a.cz + k); }
        }
        // every psi load of the cell before any store (distinct arrays)
        const long long oy = i + (long long)yn * a.Nx + (long long)k * a.Nx * nys;
        const long long ox = xn + (long long)j * nxs + (long long)k * nxs * a.Ny;
        const long long oz = col + (long long)zn * NxNy;
        T qy0 = 0, qy1 = 0, qx0 = 0, qx1 = 0, qz0 = 0, qz1 = 0;
        if constexpr ((F & kFPmlXY) != 0) {
            if (yh) { qy0 = a.psi_y0[oy]; qy1 = a.psi_y1[oy]; }
            if (xh) { qx0 = a.psi_x0[ox]; qx1 = a.psi_x1[ox]; }
        }
        if constexpr ((F & kFPmlZ) != 0) {
            if (zh) { qz0 = a.psi_z0[oz]; qz1 = a.psi_z1[oz]; }
        }
        // Hx: y block, then z block
        if constexpr ((F & kFPmlXY) != 0) {
            if (yh) {
                const T ps = cpml_rec(byj, qy0, cyj, dEz_y);
                a.psi_y0[oy] = ps;
                nhx -= a.dtm * ps;
            }
            if (a.py && j == a.Ny - 1) nhx = 0;
        }
        if constexpr ((F & kFPmlZ) != 0) {
            if (zh) {
                const T ps = cpml_rec(bzk, qz0, czk, dEy_z);
                a.psi_z0[oz] = ps;
                nhx += a.dtm * ps;
            }
            if (a.pz && k == a.Nz - 1) nhx = 0;
        }
        // Hy: x block, then z block
        if constexpr ((F & kFPmlXY) != 0) {
            if (xh) {
                const T ps = cpml_rec(bxi, qx0, cxi, dEz_x);
                a.psi_x0[ox] = ps;
                nhy += a.dtm * ps;
            }
            if (a.px && i == a.Nx - 1) nhy = 0;
        }
        if constexpr ((F & kFPmlZ) != 0) {
            if (zh) {
                const T ps = cpml_rec(bzk, qz1, czk, dEx_z);
                a.psi_z1[oz] = ps;
                nhy -= a.dtm * ps;
            }
            if (a.pz && k == a.Nz - 1) nhy = 0;
        }
        // Hz: x block, then y block
        if constexpr ((F & kFPmlXY) != 0) {
            if (xh) {
                const T ps = cpml_rec(bxi, qx1, cxi, dEy_x);
                a.psi_x1[ox] = ps;
                nhz -= a.dtm * ps;
            }
            if (a.px && i == a.Nx - 1) nhz = 0;
            if (yh) {
                const T ps = cpml_rec(byj, qy1, cyj, dEx_y);
                a.psi_y1[oy] = ps;
                nhz += a.dtm * ps;
            }
            if (a.py && j == a.Ny - 1) nhz = 0;
        }

        if constexpr ((F & kFMisc) != 0) {
            // H plane injection after update_H (normal_incidence.cpp:353-357)
            if (k == a.kinj) {
                nhx = nhx + (T)a.sc[q].inj_hA;
                nhy = nhy - (T)a.sc[q].inj_hB;
            }
            // Bloch_Wideband::inject_H (sc_bloch.cpp:252-285): dtdmz times the
            // step's complex E sums times the column's phase
            if (k == a.kobl) {
                const double *v = a.obl_inc + (size_t)a.sc[q].step * 14 + 4;
                const double2 px = a.obl_px[col], py = a.obl_py[col];
                const double exr = v[0] * px.x - v[1] * px.y, exi = v[0] * px.y + v[1] * px.x;
                const double eyr = v[2] * py.x - v[3] * py.y, eyi = v[2] * py.y + v[3] * py.x;
                nhx = nhx + (T)(a.obl_coef * (a.bloch == 1 ? eyr : eyi));
                nhy = nhy - (T)(a.obl_coef * (a.bloch == 1 ? exr : exi));
            }
        }
        Hx[id] = nhx;
        Hy[id] = nhy;
        Hz[id] = nhz;
        ex = ex_kp;
        ey = ey_kp;
    }
}

// ---- interior items, two cells per thread along x ------------------------
// The same curl updates (and PZ phases) on items of 64 x TY columns: each
// thread owns columns i0 = x0 + 2 lane and i0 + 1 and moves both with 8-byte
// (FP32) or 16-byte (FP64) loads. The x-1 (E) or x+1 (H) neighbour of the
// pair comes from the adjacent lane by a warp shuffle; the lane at the tile
// edge loads it, with the periodic wrap. Needs Nx even (vector alignment).
// An item whose x0 carries kHalfItem covers 32 columns (the other half of its
// 64-column tile belongs to another group). Per cell the arithmetic and its
// order are those of the one-cell bodies.
template <typename T> struct Vec2;
template <> struct Vec2<float> { using type = float2; };
template <> struct Vec2<double> { using type = double2; };
template <typename Tid> struct IdPair;
template <> struct IdPair<uint8_t> { using type = uchar2; };
template <> struct IdPair<uint16_t> { using type = ushort2; };
constexpr unsigned kFullMask = 0xffffffffu;

template <typename V, typename P> __device__ __forceinline__ V ldg2(const P *p) {
    return __ldg(reinterpret_cast<const V *>(p));
}
template <typename V, typename P> __device__ __forceinline__ V ld2(const P *p) { return *reinterpret_cast<const V *>(p); }
template <typename V, typename P> __device__ __forceinline__ void st2(P *p, V v) { *reinterpret_cast<V *>(p) = v; }

// PY: the item's cells may also lie in a y-CPML range or on the j = 0 PEC
// plane, but in no x-CPML range: the y psi recursions and PEC of app_pml_Ex
// and app_pml_Ez (fdtd_pml.cpp:504-735) are applied in the general kernel's
// order (Ex: y block, then z block; Ez: y block).
template <typename T, typename Tid, bool PZ, bool PY = false>
__device__ __forceinline__ void e_interior_v2_body(const StepArgs<T, Tid> &a, int q, int4 it) {
    using T2 = typename Vec2<T>::type;
    using I2 = typename IdPair<Tid>::type;
    const int lane = threadIdx.x;
    const int j = it.y + threadIdx.y;
    if (j >= a.Ny) return;                          // a whole warp: one row
    // lanes past the item (kHalfItem: 32 columns) or the grid read valid
    // memory, feed the shuffles and store nothing
    const int i0 = (it.x & ~kHalfItem) + 2 * lane;
    const bool act = i0 < a.Nx && ((it.x & kHalfItem) == 0 || lane < 16);
    const int ic = i0 < a.Nx ? i0 : a.Nx - 2;
    const long long NxNy = a.NxNy;
    const int jm = (j == 0) ? a.Ny - 1 : j - 1;
    const int im = (ic == 0) ? a.Nx - 1 : ic - 1;   // used by lane 0 only
    const long long col = ic + (long long)j * a.Nx;
    const long long coly = ic + (long long)jm * a.Nx;
    const long long colx = im + (long long)j * a.Nx;
    const long long colm = ic + (long long)j * a.mpitch;
    const long long mNxNy = (long long)a.mpitch * a.Ny;
    const T *__restrict__ Hx = a.Hx;
    const T *__restrict__ Hy = a.Hy;
    const T *__restrict__ Hz = a.Hz;
    T *__restrict__ Ex = a.Ex;
    T *__restrict__ Ey = a.Ey;
    T *__restrict__ Ez = a.Ez;
    const MatCoef<T> *__restrict__ coef = a.coef;
    const T2 ikx = ldg2<T2>(a.ikx + ic);
    const T iky = __ldg(a.iky + j);
    const int kmi = (it.z == 0) ? a.Nz - 1 : it.z - 1;
    T2 hx_km = ldg2<T2>(Hx + col + kmi * NxNy);
    T2 hy_km = ldg2<T2>(Hy + col + kmi * NxNy);
    // E-side y range [1, pml_ym) and [Ny - pml_yp + 1, Ny) (fdtd_pml.cpp:518,527); one row per warp
    bool ye = false;
    int yn = 0;
    T byj = 0, cyj = 0;
    const int nys = a.pml_ym + a.pml_yp;
    if constexpr (PY) {
        ye = a.py && ((j >= 1 && j < a.pml_ym) || (j >= a.Ny - a.pml_yp + 1));
        yn = (j < a.pml_ym) ? j : j - (a.Ny - a.pml_yp) + a.pml_ym;
        if (ye) { byj = __ldg(a.by + j); cyj = __ldg(a.cy + j); }
    }
    if (a.prefetch & 1) {
        for (int k = it.z; k < it.w; ++k) {
            const long long o = (long long)k * NxNy;
            prefetch_l2(Hx + col + o); prefetch_l2(Hy + col + o); prefetch_l2(Hz + col + o);
            if (lane == 0) { prefetch_l2(Hz + colx + o); prefetch_l2(Hy + colx + o); }
            if (threadIdx.y == 0) { prefetch_l2(Hz + coly + o); prefetch_l2(Hx + coly + o); }
            prefetch_l2(Ex + col + o); prefetch_l2(Ey + col + o); prefetch_l2(Ez + col + o);
            prefetch_l2(a.mat + colm + (long long)k * mNxNy);
            if constexpr (PZ) {
                if (a.pz && ((k >= 1 && k < a.pml_zm) || (k >= a.Nz - a.pml_zp + 1))) {
                    const int zn = (k < a.pml_zm) ? k : k - (a.Nz - a.pml_zp) + a.pml_zm;
                    prefetch_l2(a.psi_z0 + col + (long long)zn * NxNy);
                    prefetch_l2(a.psi_z1 + col + (long long)zn * NxNy);
                }
            }
            if constexpr (PY) {
                if (ye) {
                    const long long oy = ic + (long long)yn * a.Nx + (long long)k * a.Nx * nys;
                    prefetch_l2(a.psi_y0 + oy);
                    prefetch_l2(a.psi_y1 + oy);
                }
            }
        }
    }
    for (int k = it.z; k < it.w; ++k) {
        const long long o = (long long)k * NxNy;
        T2 qy0, qy1;
        long long oy = 0;
        if constexpr (PY) {
            if (ye) {
                oy = ic + (long long)yn * a.Nx + (long long)k * a.Nx * nys;
                qy0 = ld2<T2>(a.psi_y0 + oy);
                qy1 = ld2<T2>(a.psi_y1 + oy);
            }
        }
        const T2 hx = ldg2<T2>(Hx + col + o), hy = ldg2<T2>(Hy + col + o), hz = ldg2<T2>(Hz + col + o);
        const T2 hz_jm = ldg2<T2>(Hz + coly + o), hx_jm = ldg2<T2>(Hx + coly + o);
        T hz_edge = 0, hy_edge = 0;
        if (lane == 0) { hz_edge = __ldg(Hz + colx + o); hy_edge = __ldg(Hy + colx + o); }
        const T2 ex = ld2<T2>(Ex + col + o), ey = ld2<T2>(Ey + col + o), ez = ld2<T2>(Ez + col + o);
        const I2 mm = ldg2<I2>(a.mat + colm + (long long)k * mNxNy);
        T2 p0, p1;
        T bzk = 0, czk = 0;
        bool ze = false;
        long long pzi = 0;
        if constexpr (PZ) {
            // E-side z range [1, pml_zm) and [Nz - pml_zp + 1, Nz) (fdtd_pml.cpp:547,559)
            ze = a.pz && ((k >= 1 && k < a.pml_zm) || (k >= a.Nz - a.pml_zp + 1));
            if (ze) {
                const int zn = (k < a.pml_zm) ? k : k - (a.Nz - a.pml_zp) + a.pml_zm;
                pzi = col + (long long)zn * NxNy;
                p0 = ld2<T2>(a.psi_z0 + pzi);
                p1 = ld2<T2>(a.psi_z1 + pzi);
                bzk = __ldg(a.bz + k);
                czk = __ldg(a.cz + k);
            }
        }
        // x-1 neighbours: column i0 - 1 from the previous lane, or loaded at the edge
        const T hz_up = __shfl_up_sync(kFullMask, hz.y, 1), hy_up = __shfl_up_sync(kFullMask, hy.y, 1);
        const T hz_im0 = lane == 0 ? hz_edge : hz_up, hy_im0 = lane == 0 ? hy_edge : hy_up;
        const MatCoef<T> *ca = coef + mm.x, *cb = coef + mm.y;
        const T C1a = __ldg(&ca->C1), C2xa = __ldg(&ca->C2x), C2ya = __ldg(&ca->C2y), C2za = __ldg(&ca->C2z);
        const T C1b = __ldg(&cb->C1), C2xb = __ldg(&cb->C2x), C2yb = __ldg(&cb->C2y), C2zb = __ldg(&cb->C2z);
        const T ikz = __ldg(a.ikz + k);
        T2 ne, nf, ng;   // Ex, Ey, Ez of the pair
        ne.x = (C1a * ex.x + (C2ya * iky) * (hz.x - hz_jm.x)) - (C2za * ikz) * (hy.x - hy_km.x);
        nf.x = (C1a * ey.x + (C2za * ikz) * (hx.x - hx_km.x)) - (C2xa * ikx.x) * (hz.x - hz_im0);
        ng.x = (C1a * ez.x + (C2xa * ikx.x) * (hy.x - hy_im0)) - (C2ya * iky) * (hx.x - hx_jm.x);
        ne.y = (C1b * ex.y + (C2yb * iky) * (hz.y - hz_jm.y)) - (C2zb * ikz) * (hy.y - hy_km.y);
        nf.y = (C1b * ey.y + (C2zb * ikz) * (hx.y - hx_km.y)) - (C2xb * ikx.y) * (hz.y - hz.x);
        ng.y = (C1b * ez.y + (C2xb * ikx.y) * (hy.y - hy.x)) - (C2yb * iky) * (hx.y - hx_jm.y);
        if constexpr (PY) {
            // Ex: y block (before the z block); Ez: y block (no x block here)
            if (ye) {
                const T C4a = __ldg(&ca->C4), C4b = __ldg(&cb->C4);
                T2 ps0, ps1;
                ps0.x = cpml_rec(byj, qy0.x, cyj, hz.x - hz_jm.x);   // Ex: PsiExy
                ps0.y = cpml_rec(byj, qy0.y, cyj, hz.y - hz_jm.y);
                ne.x += C4a * ps0.x;
                ne.y += C4b * ps0.y;
                ps1.x = cpml_rec(byj, qy1.x, cyj, hx.x - hx_jm.x);   // Ez: PsiEzy
                ps1.y = cpml_rec(byj, qy1.y, cyj, hx.y - hx_jm.y);
                ng.x -= C4a * ps1.x;
                ng.y -= C4b * ps1.y;
                if (act) {
                    st2<T2>(a.psi_y0 + oy, ps0);
                    st2<T2>(a.psi_y1 + oy, ps1);
                }
            }
            if (a.py && j == 0) { ne.x = 0; ne.y = 0; ng.x = 0; ng.y = 0; }
        }
        if constexpr (PZ) {
            if (ze) {
                const T C4a = __ldg(&ca->C4), C4b = __ldg(&cb->C4);
                T2 ps0, ps1;
                ps0.x = cpml_rec(bzk, p0.x, czk, hy.x - hy_km.x);   // Ex: PsiExz
                ps0.y = cpml_rec(bzk, p0.y, czk, hy.y - hy_km.y);
                ne.x -= C4a * ps0.x;
                ne.y -= C4b * ps0.y;
                ps1.x = cpml_rec(bzk, p1.x, czk, hx.x - hx_km.x);   // Ey: PsiEyz
                ps1.y = cpml_rec(bzk, p1.y, czk, hx.y - hx_km.y);
                nf.x += C4a * ps1.x;
                nf.y += C4b * ps1.y;
                if (act) {
                    st2<T2>(a.psi_z0 + pzi, ps0);
                    st2<T2>(a.psi_z1 + pzi, ps1);
                }
            }
            if (a.pz && k == 0) { ne.x = 0; ne.y = 0; nf.x = 0; nf.y = 0; }
        }
        if (act) {
            st2<T2>(Ex + col + o, ne);
            st2<T2>(Ey + col + o, nf);
            st2<T2>(Ez + col + o, ng);
        }
        hx_km = hx;
        hy_km = hy;
    }
}

// PY: as for E, with the H-side y range, psi recursions and j = Ny - 1 PEC of
// app_pml_Hx and app_pml_Hz (fdtd_pml.cpp:737-1164).
template <typename T, typename Tid, bool PZ, bool PY = false>
__device__ __forceinline__ void h_interior_v2_body(const StepArgs<T, Tid> &a, int q, int4 it) {
    using T2 = typename Vec2<T>::type;
    const int lane = threadIdx.x;
    const int j = it.y + threadIdx.y;
    if (j >= a.Ny) return;
    const int i0 = (it.x & ~kHalfItem) + 2 * lane;
    const bool act = i0 < a.Nx && ((it.x & kHalfItem) == 0 || lane < 16);
    const int ic = i0 < a.Nx ? i0 : a.Nx - 2;
    // x+1 neighbour of the pair's second cell: the next lane's first, or loaded
    // (last lane, or the grid end with its periodic wrap)
    const bool edge = lane == 31 || ic + 2 >= a.Nx;
    const int ipn = (ic + 2 >= a.Nx) ? ic + 2 - a.Nx : ic + 2;
    const long long NxNy = a.NxNy;
    const int jp = (j == a.Ny - 1) ? 0 : j + 1;
    const long long col = ic + (long long)j * a.Nx;
    const long long colx = ipn + (long long)j * a.Nx;
    const long long coly = ic + (long long)jp * a.Nx;
    const T *__restrict__ Ex = a.Ex;
    const T *__restrict__ Ey = a.Ey;
    const T *__restrict__ Ez = a.Ez;
    T *__restrict__ Hx = a.Hx;
    T *__restrict__ Hy = a.Hy;
    T *__restrict__ Hz = a.Hz;
    const T2 ikx = ldg2<T2>(a.ikx + ic);
    T2 ax;
    ax.x = a.dtdmx * ikx.x;
    ax.y = a.dtdmx * ikx.y;
    const T ay = a.dtdmy * __ldg(a.iky + j);
    T2 ex = ldg2<T2>(Ex + col + it.z * NxNy);
    T2 ey = ldg2<T2>(Ey + col + it.z * NxNy);
    // H-side y range [0, pml_ym) and [Ny - pml_yp, Ny - 1) (fdtd_pml.cpp:783,792); one row per warp
    bool yh = false;
    int yn = 0;
    T byj = 0, cyj = 0;
    const int nys = a.pml_ym + a.pml_yp;
    if constexpr (PY) {
        yh = a.py && ((j < a.pml_ym) || (j >= a.Ny - a.pml_yp && j < a.Ny - 1));
        yn = (j < a.pml_ym) ? j : j - (a.Ny - a.pml_yp) + a.pml_ym;
        if (yh) { byj = __ldg(a.by + j); cyj = __ldg(a.cy + j); }
    }
    if (a.prefetch & 1) {
        for (int k = it.z; k < it.w; ++k) {
            const int kp = (k == a.Nz - 1) ? 0 : k + 1;
            const long long o = (long long)k * NxNy, op = (long long)kp * NxNy;
            prefetch_l2(Ex + col + op); prefetch_l2(Ey + col + op); prefetch_l2(Ez + col + o);
            if (edge) { prefetch_l2(Ez + colx + o); prefetch_l2(Ey + colx + o); }
            if (threadIdx.y == blockDim.y - 1) { prefetch_l2(Ez + coly + o); prefetch_l2(Ex + coly + o); }
            prefetch_l2(Hx + col + o); prefetch_l2(Hy + col + o); prefetch_l2(Hz + col + o);
            if constexpr (PZ) {
                if (a.pz && ((k < a.pml_zm) || (k >= a.Nz - a.pml_zp && k < a.Nz - 1))) {
                    const int zn = (k < a.pml_zm) ? k : k - (a.Nz - a.pml_zp) + a.pml_zm;
                    prefetch_l2(a.psi_z0 + col + (long long)zn * NxNy);
                    prefetch_l2(a.psi_z1 + col + (long long)zn * NxNy);
                }
            }
            if constexpr (PY) {
                if (yh) {
                    const long long oy = ic + (long long)yn * a.Nx + (long long)k * a.Nx * nys;
                    prefetch_l2(a.psi_y0 + oy);
                    prefetch_l2(a.psi_y1 + oy);
                }
            }
        }
    }
    for (int k = it.z; k < it.w; ++k) {
        const int kp = (k == a.Nz - 1) ? 0 : k + 1;
        const long long o = (long long)k * NxNy, op = (long long)kp * NxNy;
        T2 qy0, qy1;
        long long oy = 0;
        if constexpr (PY) {
            if (yh) {
                oy = ic + (long long)yn * a.Nx + (long long)k * a.Nx * nys;
                qy0 = ld2<T2>(a.psi_y0 + oy);
                qy1 = ld2<T2>(a.psi_y1 + oy);
            }
        }
        const T2 ex_kp = ldg2<T2>(Ex + col + op), ey_kp = ldg2<T2>(Ey + col + op);
        const T2 ez = ldg2<T2>(Ez + col + o);
        const T2 ez_jp = ldg2<T2>(Ez + coly + o), ex_jp = ldg2<T2>(Ex + coly + o);
        T ez_edge = 0, ey_edge = 0;
        if (edge) { ez_edge = __ldg(Ez + colx + o); ey_edge = __ldg(Ey + colx + o); }
        const T2 hx = ld2<T2>(Hx + col + o), hy = ld2<T2>(Hy + col + o), hz = ld2<T2>(Hz + col + o);
        T2 p0, p1;
        T bzk = 0, czk = 0;
        bool zh = false;
        long long pzi = 0;
        if constexpr (PZ) {
            // H-side z range [0, pml_zm) and [Nz - pml_zp, Nz - 1) (fdtd_pml.cpp:775,784)
            zh = a.pz && ((k < a.pml_zm) || (k >= a.Nz - a.pml_zp && k < a.Nz - 1));
            if (zh) {
                const int zn = (k < a.pml_zm) ? k : k - (a.Nz - a.pml_zp) + a.pml_zm;
                pzi = col + (long long)zn * NxNy;
                p0 = ld2<T2>(a.psi_z0 + pzi);
                p1 = ld2<T2>(a.psi_z1 + pzi);
                bzk = __ldg(a.bz + k);
                czk = __ldg(a.cz + k);
            }
        }
        const T ez_dn = __shfl_down_sync(kFullMask, ez.x, 1), ey_dn = __shfl_down_sync(kFullMask, ey.x, 1);
        const T ez_ip1 = edge ? ez_edge : ez_dn, ey_ip1 = edge ? ey_edge : ey_dn;
        const T az = a.dtdmz * __ldg(a.ikz + k);
        T2 nh, ni, nk;   // Hx, Hy, Hz of the pair
        nh.x = hx.x + (az * (ey_kp.x - ey.x) - ay * (ez_jp.x - ez.x));
        ni.x = hy.x + (ax.x * (ez.y - ez.x) - az * (ex_kp.x - ex.x));
        nk.x = hz.x + (ay * (ex_jp.x - ex.x) - ax.x * (ey.y - ey.x));
        nh.y = hx.y + (az * (ey_kp.y - ey.y) - ay * (ez_jp.y - ez.y));
        ni.y = hy.y + (ax.y * (ez_ip1 - ez.y) - az * (ex_kp.y - ex.y));
        nk.y = hz.y + (ay * (ex_jp.y - ex.y) - ax.y * (ey_ip1 - ey.y));
        if constexpr (PY) {
            // Hx: y block (before the z block); Hz: y block (no x block here)
            if (yh) {
                T2 ps0, ps1;
                ps0.x = cpml_rec(byj, qy0.x, cyj, ez_jp.x - ez.x);   // Hx: PsiHxy
                ps0.y = cpml_rec(byj, qy0.y, cyj, ez_jp.y - ez.y);
                nh.x -= a.dtm * ps0.x;
                nh.y -= a.dtm * ps0.y;
                ps1.x = cpml_rec(byj, qy1.x, cyj, ex_jp.x - ex.x);   // Hz: PsiHzy
                ps1.y = cpml_rec(byj, qy1.y, cyj, ex_jp.y - ex.y);
                nk.x += a.dtm * ps1.x;
                nk.y += a.dtm * ps1.y;
                if (act) {
                    st2<T2>(a.psi_y0 + oy, ps0);
                    st2<T2>(a.psi_y1 + oy, ps1);
                }
            }
            if (a.py && j == a.Ny - 1) { nh.x = 0; nh.y = 0; nk.x = 0; nk.y = 0; }
        }
        if constexpr (PZ) {
            if (zh) {
                T2 ps0, ps1;
                ps0.x = cpml_rec(bzk, p0.x, czk, ey_kp.x - ey.x);   // Hx: PsiHxz
                ps0.y = cpml_rec(bzk, p0.y, czk, ey_kp.y - ey.y);
                nh.x += a.dtm * ps0.x;
                nh.y += a.dtm * ps0.y;
                ps1.x = cpml_rec(bzk, p1.x, czk, ex_kp.x - ex.x);   // Hy: PsiHyz
                ps1.y = cpml_rec(bzk, p1.y, czk, ex_kp.y - ex.y);
                ni.x -= a.dtm * ps1.x;
                ni.y -= a.dtm * ps1.y;
                if (act) {
                    st2<T2>(a.psi_z0 + pzi, ps0);
                    st2<T2>(a.psi_z1 + pzi, ps1);
                }
            }
            if (a.pz && k == a.Nz - 1) { nh.x = 0; nh.y = 0; ni.x = 0; ni.y = 0; }
        }
        if (act) {
            st2<T2>(Hx + col + o, nh);
            st2<T2>(Hy + col + o, ni);
            st2<T2>(Hz + col + o, nk);
        }
        ex = ex_kp;
        ey = ey_kp;
    }
}

// ---- kernels -----------------------------------------------------------------
// Register caps: at most 256 threads per CTA; the interior kernels keep the
// register budget of 12 (U = 1, FP32) or 8 resident 128-thread CTAs per SM.
template <typename T, int U, bool PZ = false> struct InteriorBounds {
    static constexpr int kMinBlocks = PZ ? (sizeof(T) == 8 ? 2 : 3) : ((U == 1 && sizeof(T) == 4) ? 6 : 4);   // per 256 threads
    // batched forms keep the member's arguments in registers too
    static constexpr int kMinBlocksBatch = sizeof(T) == 8 ? 2 : 3;
    // two cells per thread: FP64 pairs need about 80 registers
    static constexpr int kMinBlocksVec2 = PZ ? (sizeof(T) == 8 ? 2 : 3) : (sizeof(T) == 8 ? 3 : 4);
};
constexpr int kMaxTileThreads = 256;

template <typename T, typename Tid, int U, bool PZ = false>
__global__ void __launch_bounds__(kMaxTileThreads, InteriorBounds<T, U, PZ>::kMinBlocks)
e_interior(const __grid_constant__ StepArgs<T, Tid> a, const int4 *__restrict__ items) {
    e_interior_body<T, Tid, U, PZ>(a, a.q, items[blockIdx.x]);
}
template <typename T, typename Tid, int U, bool PZ = false>
__global__ void __launch_bounds__(kMaxTileThreads, InteriorBounds<T, U, PZ>::kMinBlocks)
h_interior(const __grid_constant__ StepArgs<T, Tid> a, const int4 *__restrict__ items) {
    h_interior_body<T, Tid, U, PZ>(a, a.q, items[blockIdx.x]);
}
template <typename T, typename Tid, unsigned F>
__global__ void __launch_bounds__(kMaxTileThreads) e_boundary(const __grid_constant__ StepArgs<T, Tid> a,
                                                              const int4 *__restrict__ items) {
    e_boundary_body<T, Tid, F>(a, a.q, items[blockIdx.x]);
}
template <typename T, typename Tid, unsigned F>
__global__ void __launch_bounds__(kMaxTileThreads) h_boundary(const __grid_constant__ StepArgs<T, Tid> a,
                                                              const int4 *__restrict__ items) {
    h_boundary_body<T, Tid, F>(a, a.q, items[blockIdx.x]);
}

template <typename T, typename Tid, bool PZ>
__global__ void __launch_bounds__(kMaxTileThreads, InteriorBounds<T, 2, PZ>::kMinBlocksVec2)
e_interior_v2(const __grid_constant__ StepArgs<T, Tid> a, const int4 *__restrict__ items) {
    e_interior_v2_body<T, Tid, PZ>(a, a.q, items[blockIdx.x]);
}
template <typename T, typename Tid, bool PZ>
__global__ void __launch_bounds__(kMaxTileThreads, InteriorBounds<T, 2, PZ>::kMinBlocksVec2)
h_interior_v2(const __grid_constant__ StepArgs<T, Tid> a, const int4 *__restrict__ items) {
    h_interior_v2_body<T, Tid, PZ>(a, a.q, items[blockIdx.x]);
}

// y-CPML items without x-CPML cells: two cells per thread, y and z psi
template <typename T, typename Tid>
__global__ void __launch_bounds__(kMaxTileThreads, InteriorBounds<T, 2, true>::kMinBlocksVec2)
e_pmly_v2(const __grid_constant__ StepArgs<T, Tid> a, const int4 *__restrict__ items) {
    e_interior_v2_body<T, Tid, true, true>(a, a.q, items[blockIdx.x]);
}
template <typename T, typename Tid>
__global__ void __launch_bounds__(kMaxTileThreads, InteriorBounds<T, 2, true>::kMinBlocksVec2)
h_pmly_v2(const __grid_constant__ StepArgs<T, Tid> a, const int4 *__restrict__ items) {
    h_interior_v2_body<T, Tid, true, true>(a, a.q, items[blockIdx.x]);
}

// Batched forms: item (x0, y0, k0 | k1 << 16, instance), arguments of the
// instance from a device array, q the step's index in every member's table.
__device__ __forceinline__ int4 batch_item(int4 b) { return make_int4(b.x, b.y, b.z & 0xffff, b.z >> 16); }

template <typename T, typename Tid, int U, bool PZ = false>
__global__ void __launch_bounds__(kMaxTileThreads, InteriorBounds<T, U, PZ>::kMinBlocksBatch)
e_interior_batch(const StepArgs<T, Tid> *__restrict__ args, int q, const int4 *__restrict__ items) {
    const int4 b = items[blockIdx.x];
    e_interior_body<T, Tid, U, PZ>(args[b.w], q, batch_item(b));
}
template <typename T, typename Tid, int U, bool PZ = false>
__global__ void __launch_bounds__(kMaxTileThreads, InteriorBounds<T, U, PZ>::kMinBlocksBatch)
h_interior_batch(const StepArgs<T, Tid> *__restrict__ args, int q, const int4 *__restrict__ items) {
    const int4 b = items[blockIdx.x];
    h_interior_body<T, Tid, U, PZ>(args[b.w], q, batch_item(b));
}
template <typename T, typename Tid, unsigned F>
__global__ void __launch_bounds__(kMaxTileThreads)
e_boundary_batch(const StepArgs<T, Tid> *__restrict__ args, int q, const int4 *__restrict__ items) {
    const int4 b = items[blockIdx.x];
    e_boundary_body<T, Tid, F>(args[b.w], q, batch_item(b));
}
template <typename T, typename Tid, unsigned F>
__global__ void __launch_bounds__(kMaxTileThreads)
h_boundary_batch(const StepArgs<T, Tid> *__restrict__ args, int q, const int4 *__restrict__ items) {
    const int4 b = items[blockIdx.x];
    h_boundary_body<T, Tid, F>(args[b.w], q, batch_item(b));
}

}  // namespace aefdtd

#include "interior_tma.cuh"

namespace aefdtd {

// ---- launchers: group g of a half-step's WorkSplit ------------------------
template <typename T, typename Tid>
void launch_e_group_impl(const StepArgs<T, Tid> &a, const int4 *items, const WorkSplit &w, int g, cudaStream_t s) {
    const int n = w.n[g];
    if (n <= 0) return;
    const int4 *p = items + w.off[g];
    const dim3 blk(kTileX, w.tile_y);
    switch (g) {
        case kGroupInterior:
            if (w.tma) launch_tma_impl<T, Tid, false>(a, *w.tma, s);
            else if (w.pair_mask & (1u << kGroupInterior)) e_interior_v2<T, Tid, false><<<n, blk, 0, s>>>(a, p);
            else if (w.unroll >= 2) e_interior<T, Tid, 2><<<n, blk, 0, s>>>(a, p);
            else e_interior<T, Tid, 1><<<n, blk, 0, s>>>(a, p);
            break;
        case kGroupPmlZ:
            if (w.pair_mask & (1u << kGroupPmlZ)) e_interior_v2<T, Tid, true><<<n, blk, 0, s>>>(a, p);
            else if (w.unroll >= 2) e_interior<T, Tid, 2, true><<<n, blk, 0, s>>>(a, p);
            else e_interior<T, Tid, 1, true><<<n, blk, 0, s>>>(a, p);
            break;
        case kGroupDisp: e_boundary<T, Tid, kFDisp><<<n, blk, 0, s>>>(a, p); break;
        case kGroupPmlXY:
            // items with x-CPML cells first (one cell per thread), then the y-only pairs
            if (n > w.n_py) e_boundary<T, Tid, kFPmlXY | kFPmlZ><<<n - w.n_py, blk, 0, s>>>(a, p);
            if (w.n_py > 0) e_pmly_v2<T, Tid><<<w.n_py, blk, 0, s>>>(a, p + (n - w.n_py));
            break;
        default: e_boundary<T, Tid, kFAll><<<n, blk, 0, s>>>(a, p); break;
    }
}

template <typename T, typename Tid>
void launch_h_group_impl(const StepArgs<T, Tid> &a, const int4 *items, const WorkSplit &w, int g, cudaStream_t s) {
    const int n = w.n[g];
    if (n <= 0) return;
    const int4 *p = items + w.off[g];
    const dim3 blk(kTileX, w.tile_y);
    switch (g) {
        case kGroupInterior:
            if (w.tma) launch_tma_impl<T, Tid, true>(a, *w.tma, s);
            else if (w.pair_mask & (1u << kGroupInterior)) h_interior_v2<T, Tid, false><<<n, blk, 0, s>>>(a, p);
            else if (w.unroll >= 2) h_interior<T, Tid, 2><<<n, blk, 0, s>>>(a, p);
            else h_interior<T, Tid, 1><<<n, blk, 0, s>>>(a, p);
            break;
        case kGroupPmlZ:
            if (w.pair_mask & (1u << kGroupPmlZ)) h_interior_v2<T, Tid, true><<<n, blk, 0, s>>>(a, p);
            else if (w.unroll >= 2) h_interior<T, Tid, 2, true><<<n, blk, 0, s>>>(a, p);
            else h_interior<T, Tid, 1, true><<<n, blk, 0, s>>>(a, p);
            break;
        case kGroupPmlXY:
            if (n > w.n_py) h_boundary<T, Tid, kFPmlXY | kFPmlZ><<<n - w.n_py, blk, 0, s>>>(a, p);
            if (w.n_py > 0) h_pmly_v2<T, Tid><<<w.n_py, blk, 0, s>>>(a, p + (n - w.n_py));
            break;
        default: h_boundary<T, Tid, kFAll><<<n, blk, 0, s>>>(a, p); break;
    }
}

template <typename T, typename Tid>
void launch_e_group_batch_impl(const StepArgs<T, Tid> *args, int q, const int4 *items, const WorkSplit &w, int g,
                               cudaStream_t s) {
    const int n = w.n[g];
    if (n <= 0) return;
    const int4 *p = items + w.off[g];
    const dim3 blk(kTileX, w.tile_y);
    switch (g) {
        case kGroupInterior:
            if (w.unroll >= 2) e_interior_batch<T, Tid, 2><<<n, blk, 0, s>>>(args, q, p);
            else e_interior_batch<T, Tid, 1><<<n, blk, 0, s>>>(args, q, p);
            break;
        case kGroupPmlZ:
            if (w.unroll >= 2) e_interior_batch<T, Tid, 2, true><<<n, blk, 0, s>>>(args, q, p);
            else e_interior_batch<T, Tid, 1, true><<<n, blk, 0, s>>>(args, q, p);
            break;
        case kGroupDisp: e_boundary_batch<T, Tid, kFDisp><<<n, blk, 0, s>>>(args, q, p); break;
        default: e_boundary_batch<T, Tid, kFAll><<<n, blk, 0, s>>>(args, q, p); break;
    }
}

template <typename T, typename Tid>
void launch_h_group_batch_impl(const StepArgs<T, Tid> *args, int q, const int4 *items, const WorkSplit &w, int g,
                               cudaStream_t s) {
    const int n = w.n[g];
    if (n <= 0) return;
    const int4 *p = items + w.off[g];
    const dim3 blk(kTileX, w.tile_y);
    switch (g) {
        case kGroupInterior:
            if (w.unroll >= 2) h_interior_batch<T, Tid, 2><<<n, blk, 0, s>>>(args, q, p);
            else h_interior_batch<T, Tid, 1><<<n, blk, 0, s>>>(args, q, p);
            break;
        case kGroupPmlZ:
            if (w.unroll >= 2) h_interior_batch<T, Tid, 2, true><<<n, blk, 0, s>>>(args, q, p);
            else h_interior_batch<T, Tid, 1, true><<<n, blk, 0, s>>>(args, q, p);
            break;
        default: h_boundary_batch<T, Tid, kFAll><<<n, blk, 0, s>>>(args, q, p); break;
    }
}

}  // namespace aefdtd
