// leapfrog.cuh — one launch per time step: the E and the H half-step fused in
// one pass over the grid (FDTD::update_E then FDTD::update_H,
// fdtd_core.cpp:1163-1335, with every phase that the split kernels of
// yee.cuh fuse per cell).
//
// Why: the split half-steps each read all six field arrays, 18 values per
// cell-update (145 B in FP64, 73 B in FP32). Here a CTA marches a tile's
// columns along z and, at each plane k, updates E(k) and then H(k-1): the new
// E of a plane is still in registers (own column) or in shared memory
// (neighbour rows) when the H update of the plane below needs it, so each
// field value is read once and written once per step.
//
// Buffers. The pass reads the old fields (E^n, H^{n-1/2}) and writes new
// ones into a second set (ping-pong), and likewise the E-side CPML psi and the
// recursive-convolution psi: tiles and z-chunks then never see each other's
// new values, whatever order the CTAs run in. H-side psi is updated in place
// (each H cell is updated by exactly one CTA and read by no other).
//
// Tile. A CTA of 32 x (TY + 1) threads owns 64 x TY columns (x0, y0) and a
// z-chunk [k0, k1). Warp w < TY owns row y0 + w; lane L its columns
// x0 + 2L, x0 + 2L + 1 (8/16-byte pair loads; per-cell loads when Nx is odd). The H update
// of the tile's last column and last row needs the new E one cell beyond the
// tile, so that E is computed again here (the owner computes the same value
// from the same old state): the extra warp TY computes E of row y0 + TY (mod
// Ny), the lane holding the last owned column computes E of the next column
// (mod Nx) as a third cell, and the chunk's last iteration computes E of plane
// k1 (mod Nz). Such cells write neither fields nor state.
//
// Per plane, one __syncthreads: each warp publishes Hz, Hx of its row at
// plane k (read by the row above for the y-1 differences of E) before it, and
// Ez, Ex of its new E row (read by the row below for the y+1 differences of
// H(k-1) in the next iteration) after it; both arrays are double-buffered by
// plane parity. x neighbours come through lane shuffles, z neighbours stay in
// registers.
//
// Arithmetic per cell: the operations and their order are those of
// e_boundary_body / h_boundary_body (yee.cuh), so the FP64 instantiation is
// bit-identical to the split kernels and to the reference core.
#pragma once

#include "yee.cuh"

namespace aefdtd {


// E update of cell (i, j, k) from its old value and the H values around it, in
// the phase order of e_boundary_body. own: write the cell's new state (RC psi,
// CPML psi); a recomputed cell only returns its value.
template <typename T, typename Tid, unsigned F>
__device__ __forceinline__ void e_cell(const FusedArgs<T, Tid> &A, int q, int i, int j, int k, bool own, int m,
                                       T ex, T ey, T ez, T hx, T hy, T hz, T hx_km, T hy_km, T hz_jm, T hx_jm,
                                       T hz_im, T hy_im, T &nex, T &ney, T &nez) {
    const StepArgs<T, Tid> &a = A.e;
    const MatCoef<T> c = a.coef[m];
    const T ikx = __ldg(a.ikx + i);
    const T iky = __ldg(a.iky + j);
    const T ikz = __ldg(a.ikz + k);
    const long long col = i + (long long)j * a.Nx;
    T s0 = 0, s1 = 0, s2 = 0;
    int np_m = 0;
    if constexpr ((F & kFDisp) != 0) {
        np_m = a.disp ? __ldg(&a.disp[m].np) : 0;
        if (np_m > 0) {
            const DispInfo d = a.disp[m];
            const long long qq = (i - d.x1) + (long long)(j - d.y1) * d.xs + (long long)(k - d.z1) * d.xs * d.ys;
            const Cplx<T> *__restrict__ P = a.psi + d.psi_off + qq;
            Cplx<T> *__restrict__ Pn = A.npsi + d.psi_off + qq;
            const T ev[3] = {ex, ey, ez};
            // two poles at a time (loads before stores); sums in pole order
            for (int p0 = 0; p0 < d.np; p0 += 2) {
                const int pn = min(2, d.np - p0);
                Cplx<T> v[2][3], cr[2], dc[2];
#pragma unroll
                for (int p = 0; p < 2; ++p)
                    if (p < pn) {
                        cr[p] = a.crec[d.pole_off + p0 + p];
                        dc[p] = a.dchi[d.pole_off + p0 + p];
#pragma unroll
                        for (int dd = 0; dd < 3; ++dd) v[p][dd] = P[(long long)(3 * (p0 + p) + dd) * d.box];
                    }
#pragma unroll
                for (int p = 0; p < 2; ++p)
                    if (p < pn) {
#pragma unroll
                        for (int dd = 0; dd < 3; ++dd) {
                            Cplx<T> r;
                            if constexpr (Exact<T>::value) {
                                r.re = (cr[p].re * v[p][dd].re - cr[p].im * v[p][dd].im) + dc[p].re * ev[dd];
                                r.im = (cr[p].re * v[p][dd].im + cr[p].im * v[p][dd].re) + dc[p].im * ev[dd];
                            } else {
                                r.re = v[p][dd].re + ((cr[p].re * v[p][dd].re - cr[p].im * v[p][dd].im) + dc[p].re * ev[dd]);
                                r.im = v[p][dd].im + ((cr[p].re * v[p][dd].im + cr[p].im * v[p][dd].re) + dc[p].im * ev[dd]);
                            }
                            if (own) Pn[(long long)(3 * (p0 + p) + dd) * d.box] = r;
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
    nex = (c.C1 * ex + (c.C2y * iky) * dHz_y) - (c.C2z * ikz) * dHy_z;
    ney = (c.C1 * ey + (c.C2z * ikz) * dHx_z) - (c.C2x * ikx) * dHz_x;
    nez = (c.C1 * ez + (c.C2x * ikx) * dHy_x) - (c.C2y * iky) * dHx_y;
    if constexpr ((F & kFDisp) != 0) {
        if (np_m > 0) {
            nex += c.C3 * s0;
            ney += c.C3 * s1;
            nez += c.C3 * s2;
        }
    }
    // CPML and PEC planes in app_pml_Ex / Ey / Ez order (E-side ranges
    // [1, pml_m) and [N - pml_p + 1, N), fdtd_pml.cpp:518,527,547,559)
    bool xe = false, ye = false, ze = false;
    int xn = 0, yn = 0, zn = 0;
    const int nxs = a.pml_xm + a.pml_xp, nys = a.pml_ym + a.pml_yp;
    if constexpr ((F & kFPmlXY) != 0) {
        xe = a.px && ((i >= 1 && i < a.pml_xm) || (i >= a.Nx - a.pml_xp + 1));
        ye = a.py && ((j >= 1 && j < a.pml_ym) || (j >= a.Ny - a.pml_yp + 1));
        xn = (i < a.pml_xm) ? i : i - (a.Nx - a.pml_xp) + a.pml_xm;
        yn = (j < a.pml_ym) ? j : j - (a.Ny - a.pml_yp) + a.pml_ym;
    }
    if constexpr ((F & kFPmlZ) != 0) {
        ze = a.pz && ((k >= 1 && k < a.pml_zm) || (k >= a.Nz - a.pml_zp + 1));
        zn = (k < a.pml_zm) ? k : k - (a.Nz - a.pml_zp) + a.pml_zm;
    }
    // Ex: y block, then z block
    if constexpr ((F & kFPmlXY) != 0) {
        if (ye) {
            const long long o = i + (long long)yn * a.Nx + (long long)k * a.Nx * nys;
            const T ps = cpml_rec(__ldg(a.by + j), a.psi_y0[o], __ldg(a.cy + j), dHz_y);
            if (own) A.npy0[o] = ps;
            nex += c.C4 * ps;
        }
        if (a.py && j == 0) nex = 0;
    }
    if constexpr ((F & kFPmlZ) != 0) {
        if (ze) {
            const long long o = col + (long long)zn * a.NxNy;
            const T ps = cpml_rec(__ldg(a.bz + k), a.psi_z0[o], __ldg(a.cz + k), dHy_z);
            if (own) A.npz0[o] = ps;
            nex -= c.C4 * ps;
        }
        if (a.pz && k == 0) nex = 0;
    }
    // Ey: x block, then z block
    if constexpr ((F & kFPmlXY) != 0) {
        if (xe) {
            const long long o = xn + (long long)j * nxs + (long long)k * nxs * a.Ny;
            const T ps = cpml_rec(__ldg(a.bx + i), a.psi_x0[o], __ldg(a.cx + i), dHz_x);
            if (own) A.npx0[o] = ps;
            ney -= c.C4 * ps;
        }
        if (a.px && i == 0) ney = 0;
    }
    if constexpr ((F & kFPmlZ) != 0) {
        if (ze) {
            const long long o = col + (long long)zn * a.NxNy;
            const T ps = cpml_rec(__ldg(a.bz + k), a.psi_z1[o], __ldg(a.cz + k), dHx_z);
            if (own) A.npz1[o] = ps;
            ney += c.C4 * ps;
        }
        if (a.pz && k == 0) ney = 0;
    }
    // Ez: x block, then y block
    if constexpr ((F & kFPmlXY) != 0) {
        if (xe) {
            const long long o = xn + (long long)j * nxs + (long long)k * nxs * a.Ny;
            const T ps = cpml_rec(__ldg(a.bx + i), a.psi_x1[o], __ldg(a.cx + i), dHy_x);
            if (own) A.npx1[o] = ps;
            nez += c.C4 * ps;
        }
        if (a.px && i == 0) nez = 0;
        if (ye) {
            const long long o = i + (long long)yn * a.Nx + (long long)k * a.Nx * nys;
            const T ps = cpml_rec(__ldg(a.by + j), a.psi_y1[o], __ldg(a.cy + j), dHx_y);
            if (own) A.npy1[o] = ps;
            nez -= c.C4 * ps;
        }
        if (a.py && j == 0) nez = 0;
    }
    if constexpr ((F & kFMisc) != 0) {
        // normal-incidence plane injection after update_E (normal_incidence.cpp:338-342)
        if (k == a.kinj) {
            nex = nex - (T)a.sc[q].inj_eA;
            ney = ney + (T)a.sc[q].inj_eB;
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
}

// H update of cell (i, j, k) (always owned), in the phase order of
// h_boundary_body. e*: new E at the cell, e*_kp at k+1, e*_jp at j+1, e*_ip at i+1.
template <typename T, typename Tid, unsigned F>
__device__ __forceinline__ void h_cell(const FusedArgs<T, Tid> &A, int q, int i, int j, int k, T hx, T hy, T hz,
                                       T ex, T ey, T ez, T ex_kp, T ey_kp, T ez_jp, T ex_jp, T ez_ip, T ey_ip,
                                       T &nhx, T &nhy, T &nhz) {
    const StepArgs<T, Tid> &a = A.h;
    const T ax = a.dtdmx * __ldg(a.ikx + i);
    const T ay = a.dtdmy * __ldg(a.iky + j);
    const T az = a.dtdmz * __ldg(a.ikz + k);
    const long long col = i + (long long)j * a.Nx;
    const T dEy_z = ey_kp - ey, dEz_y = ez_jp - ez;
    const T dEz_x = ez_ip - ez, dEx_z = ex_kp - ex;
    const T dEx_y = ex_jp - ex, dEy_x = ey_ip - ey;
    nhx = hx + (az * dEy_z - ay * dEz_y);
    nhy = hy + (ax * dEz_x - az * dEx_z);
    nhz = hz + (ay * dEx_y - ax * dEy_x);
    // H-side CPML ranges [0, pml_m) and [N - pml_p, N - 1) (fdtd_pml.cpp:750,756,775,784)
    bool xh = false, yh = false, zh = false;
    int xn = 0, yn = 0, zn = 0;
    const int nxs = a.pml_xm + a.pml_xp, nys = a.pml_ym + a.pml_yp;
    if constexpr ((F & kFPmlXY) != 0) {
        xh = a.px && ((i < a.pml_xm) || (i >= a.Nx - a.pml_xp && i < a.Nx - 1));
        yh = a.py && ((j < a.pml_ym) || (j >= a.Ny - a.pml_yp && j < a.Ny - 1));
        xn = (i < a.pml_xm) ? i : i - (a.Nx - a.pml_xp) + a.pml_xm;
        yn = (j < a.pml_ym) ? j : j - (a.Ny - a.pml_yp) + a.pml_ym;
    }
    if constexpr ((F & kFPmlZ) != 0) {
        zh = a.pz && ((k < a.pml_zm) || (k >= a.Nz - a.pml_zp && k < a.Nz - 1));
        zn = (k < a.pml_zm) ? k : k - (a.Nz - a.pml_zp) + a.pml_zm;
    }
    // Hx: y block, then z block
    if constexpr ((F & kFPmlXY) != 0) {
        if (yh) {
            T *pp = a.psi_y0 + i + (long long)yn * a.Nx + (long long)k * a.Nx * nys;
            const T ps = cpml_rec(__ldg(a.by + j), *pp, __ldg(a.cy + j), dEz_y);
            *pp = ps;
            nhx -= a.dtm * ps;
        }
        if (a.py && j == a.Ny - 1) nhx = 0;
    }
    if constexpr ((F & kFPmlZ) != 0) {
        if (zh) {
            T *pp = a.psi_z0 + col + (long long)zn * a.NxNy;
            const T ps = cpml_rec(__ldg(a.bz + k), *pp, __ldg(a.cz + k), dEy_z);
            *pp = ps;
            nhx += a.dtm * ps;
        }
        if (a.pz && k == a.Nz - 1) nhx = 0;
    }
    // Hy: x block, then z block
    if constexpr ((F & kFPmlXY) != 0) {
        if (xh) {
            T *pp = a.psi_x0 + xn + (long long)j * nxs + (long long)k * nxs * a.Ny;
            const T ps = cpml_rec(__ldg(a.bx + i), *pp, __ldg(a.cx + i), dEz_x);
            *pp = ps;
            nhy += a.dtm * ps;
        }
        if (a.px && i == a.Nx - 1) nhy = 0;
    }
    if constexpr ((F & kFPmlZ) != 0) {
        if (zh) {
            T *pp = a.psi_z1 + col + (long long)zn * a.NxNy;
            const T ps = cpml_rec(__ldg(a.bz + k), *pp, __ldg(a.cz + k), dEx_z);
            *pp = ps;
            nhy -= a.dtm * ps;
        }
        if (a.pz && k == a.Nz - 1) nhy = 0;
    }
    // Hz: x block, then y block
    if constexpr ((F & kFPmlXY) != 0) {
        if (xh) {
            T *pp = a.psi_x1 + xn + (long long)j * nxs + (long long)k * nxs * a.Ny;
            const T ps = cpml_rec(__ldg(a.bx + i), *pp, __ldg(a.cx + i), dEy_x);
            *pp = ps;
            nhz -= a.dtm * ps;
        }
        if (a.px && i == a.Nx - 1) nhz = 0;
        if (yh) {
            T *pp = a.psi_y1 + i + (long long)yn * a.Nx + (long long)k * a.Nx * nys;
            const T ps = cpml_rec(__ldg(a.by + j), *pp, __ldg(a.cy + j), dEx_y);
            *pp = ps;
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
    }
}

constexpr int kFusedPrefetch = 6;   // planes of L2 prefetch ahead of the march

template <typename T> struct FusedSmem {
    using T2 = typename Vec2<T>::type;
    T2 hz[2][kFusedMaxTY][32], hx[2][kFusedMaxTY][32];       // H(k) of the owned rows, by plane parity
    T2 ez[2][kFusedMaxTY + 1][32], ex[2][kFusedMaxTY + 1][32]; // new E(k) rows 1 .. TY (TY: the extra row)
    T hzl[2][kFusedMaxTY], hyl[2][kFusedMaxTY];                // H(k) of each row's last owned column
    T eze[2][kFusedMaxTY], eye[2][kFusedMaxTY];                // new E(k) of the column after it
};

// Load staging: each thread copies the values it reads at a plane (its pair of
// the six fields, plus lane 0's x-1 neighbours, warp 0's row y-1, the column
// warp's cell) into its own slot of a ring of stages with cp.async, planes
// ahead of the march; it then waits only for its own copies (no barrier).
template <typename T> struct alignas(16) FusedStage {
    using T2 = typename Vec2<T>::type;
    static constexpr int kRowThreads = 32 * (kFusedMaxTY + 1);
    T2 f[6][kRowThreads];        // Hx Hy Hz Ex Ey Ez of each row thread's pair
    T2 y[2][32];                 // Hz, Hx of row y0 - 1 (warp 0)
    T c[6][32];                  // the column warp's cell: Hx Hy Hz Ex Ey Ez
    T e[2][kFusedMaxTY + 1];     // Hz, Hy at x0 - 1 (lane 0 of each row warp)
    T cy[2];                     // Hz, Hx of row y0 - 1 at the column after the tile
};
// stages in the ring: FP64 two (two CTAs fit an SM), FP32 three
template <typename T> constexpr int fused_stages() { return sizeof(T) == 8 ? 2 : 3; }
template <typename T> constexpr size_t fused_stage_bytes() { return fused_stages<T>() * sizeof(FusedStage<T>); }

template <int BYTES> __device__ __forceinline__ void cp_async(void *smem, const void *gmem) {
    const uint32_t s = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
    if constexpr (BYTES == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(s), "l"(gmem), "n"(BYTES) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// One step over item (x0, y0, k0, k1): blockDim (32, TY + 2), TY <= kFusedMaxTY.
// Warps 0 .. TY-1 own the rows, warp TY recomputes E of the row after them,
// warp TY+1 (lane r for row r) recomputes E of the column after them.
// ODD: Nx is odd. Each cell is then loaded and stored on its own (rows are not
// pair-aligned), and on a tile of odd width the last lane's second cell is the
// column after the tile (mod Nx): its E is recomputed there, not stored, and
// serves as the x+1 neighbour of the tile's last column.
template <typename T, typename Tid, unsigned F, bool ODD>
__device__ __forceinline__ void fused_body(const FusedArgs<T, Tid> &A, int q, int4 it) {
    using T2 = typename Vec2<T>::type;
    using I2 = typename IdPair<Tid>::type;
    __shared__ FusedSmem<T> sm;
    const StepArgs<T, Tid> &a = A.e;
    const int Nx = a.Nx, Ny = a.Ny, Nz = a.Nz;
    const long long NxNy = a.NxNy;
    const int TY = blockDim.y - 2;
    const int w = threadIdx.y, lane = threadIdx.x;
    const int x0 = it.x, y0 = it.y, k0 = it.z, k1 = it.w;
    const int hrows = min(TY, Ny - y0);
    const int wcols = min(kFusedTileX, Nx - x0);         // even unless ODD on the last tile
    const int llast = wcols / 2 - 1;                     // lane of the last owned pair (even width)
    const int ie = (x0 + wcols) % Nx;                    // the column after the tile (mod Nx)
    const long long mNxNy = (long long)a.mpitch * Ny;
    const T *__restrict__ Ex = a.Ex;
    const T *__restrict__ Ey = a.Ey;
    const T *__restrict__ Ez = a.Ez;
    const T *__restrict__ Hx = a.Hx;
    const T *__restrict__ Hy = a.Hy;
    const T *__restrict__ Hz = a.Hz;
    const Tid *__restrict__ mat = a.mat;

    extern __shared__ __align__(16) unsigned char fused_dyn[];
    FusedStage<T> *stage = reinterpret_cast<FusedStage<T> *>(fused_dyn);
    constexpr int S = fused_stages<T>();
    constexpr int TB = (int)sizeof(T);

    if (w == TY + 1) {
        // ---- the column warp: E of (ie, y0 + r) for r < hrows, lane r
        const bool on = lane < hrows;
        const int j = (y0 + min(lane, hrows - 1)) % Ny;
        const int jm0 = (y0 == 0) ? Ny - 1 : y0 - 1;
        const long long c = ie + (long long)j * Nx, cm = ie + (long long)j * a.mpitch;
        const long long cy = ie + (long long)jm0 * Nx;
        const T *src[6] = {Hx, Hy, Hz, Ex, Ey, Ez};
        auto issue = [&](int kq, int st) {
            if (kq <= k1 && on) {
                const long long o = (long long)(kq % Nz) * NxNy;
#pragma unroll
                for (int f = 0; f < 6; ++f) cp_async<TB>(&stage[st].c[f][lane], src[f] + c + o);
                if (lane == 0) {
                    cp_async<TB>(&stage[st].cy[0], Hz + cy + o);
                    cp_async<TB>(&stage[st].cy[1], Hx + cy + o);
                }
            }
            cp_async_commit();
        };
        for (int s0 = 0; s0 < S - 1; ++s0) issue(k0 + s0, s0);
        const int kb = (k0 == 0) ? Nz - 1 : k0 - 1;
        T hxp = __ldg(Hx + c + kb * NxNy), hyp = __ldg(Hy + c + kb * NxNy);
        int m = __ldg(mat + cm + (long long)(k0 % Nz) * mNxNy);
        for (int kq = k0; kq <= k1; ++kq) {
            const int k = kq % Nz;
            const int buf = kq & 1;
            const int st = (kq - k0) % S;
            issue(kq + S - 1, (kq - k0 + S - 1) % S);
            const int m_next = (kq < k1) ? __ldg(mat + cm + (long long)((kq + 1) % Nz) * mNxNy) : 0;
            cp_async_wait<S - 1>();
            const FusedStage<T> &g = stage[st];
            const T hx = g.c[0][lane], hy = g.c[1][lane], hz = g.c[2][lane];
            const T ex = g.c[3][lane], ey = g.c[4][lane], ez = g.c[5][lane];
            T hzy = 0, hxy = 0;
            if (lane == 0) { hzy = g.cy[0]; hxy = g.cy[1]; }
            const T hz_up = __shfl_up_sync(kFullMask, hz, 1), hx_up = __shfl_up_sync(kFullMask, hx, 1);
            if (lane > 0) { hzy = hz_up; hxy = hx_up; }
            __syncthreads();
            if (on) {
                const T hz_im = sm.hzl[buf][lane], hy_im = sm.hyl[buf][lane];
                T nex, ney, nez;
                e_cell<T, Tid, F>(A, q, ie, j, k, false, m, ex, ey, ez, hx, hy, hz, hxp, hyp, hzy, hxy, hz_im, hy_im,
                                  nex, ney, nez);
                sm.eze[buf][lane] = nez;
                sm.eye[buf][lane] = ney;
            }
            hxp = hx;
            hyp = hy;
            m = m_next;
        }
        cp_async_wait<0>();
        return;   // no barrier follows the loop
    }

    // ---- row warps: r = w (owned rows) or r = hrows (warp TY, the row after them)
    const bool xw = (w == TY);
    const bool active = xw || w < hrows;
    const int r = xw ? hrows : w;
    const int j = (y0 + r) % Ny;
    const int jm = (j == 0) ? Ny - 1 : j - 1;            // row y-1 (loaded by r == 0)
    const bool lown = 2 * lane < wcols;                  // the pair's first column is owned
    const bool lown1 = 2 * lane + 1 < wcols;             // ... and its second
    const int ic = lown ? x0 + 2 * lane : (ODD ? x0 : x0 + wcols - 2);
    // the pair's second column: ic + 1, or the column after the tile (mod Nx)
    // when it lies past the grid (ODD)
    const int ic1 = ODD ? ((ic + 1 < Nx) ? ic + 1 : ic + 1 - Nx) : ic + 1;
    const int im0 = (x0 == 0) ? Nx - 1 : x0 - 1;         // x-1 of lane 0's first cell
    const bool hrow = !xw && w < hrows;                  // owns H (and E) of its row
    // the lane whose second cell is the tile's last column takes the x+1
    // neighbour of H from the column warp (an odd-width tile recomputes it itself)
    const bool xl = hrow && (wcols % 2 == 0) && lane == llast;
    const long long col = ic + (long long)j * Nx;
    const long long colb = ic1 + (long long)j * Nx;      // ODD: the second cell's offset
    const long long colm = ic + (long long)j * a.mpitch;
    const long long colmb = ic1 + (long long)j * a.mpitch;
    const long long colym = ic + (long long)jm * Nx;
    const long long colymb = ic1 + (long long)jm * Nx;
    auto ld = [&](const T *p, long long a0, long long b0) {
        if constexpr (ODD) {
            T2 v;
            v.x = __ldg(p + a0);
            v.y = __ldg(p + b0);
            return v;
        } else {
            return ldg2<T2>(p + a0);
        }
    };
    auto st = [&](T *p, long long a0, long long b0, T2 v, bool s0, bool s1) {
        if constexpr (ODD) {
            if (s0) p[a0] = v.x;
            if (s1) p[b0] = v.y;
        } else {
            st2<T2>(p + a0, v);
        }
    };

    // L2 prefetch kFusedPrefetch planes ahead of the march (the first ones up front)
    const bool pf = active && (a.prefetch & 1);
    auto prefetch_plane = [&](int kq) {
        const int kk = kq % Nz;
        const long long o = (long long)kk * NxNy;
        prefetch_l2(Hx + col + o); prefetch_l2(Hy + col + o); prefetch_l2(Hz + col + o);
        prefetch_l2(Ex + col + o); prefetch_l2(Ey + col + o); prefetch_l2(Ez + col + o);
        prefetch_l2(mat + colm + (long long)kk * mNxNy);
        if (r == 0) { prefetch_l2(Hz + colym + o); prefetch_l2(Hx + colym + o); }
    };
    if (pf)
        for (int kq = k0; kq <= min(k1, k0 + kFusedPrefetch - 1); ++kq) prefetch_plane(kq);
    // staged copies of plane kq into stage st (every thread commits one group per plane)
    const int tr = w * 32 + lane;
    const T *src[6] = {Hx, Hy, Hz, Ex, Ey, Ez};
    auto issue = [&](int kq, int st) {
        if (kq <= k1 && active) {
            const int kk = kq % Nz;
            const long long o = (long long)kk * NxNy;
            FusedStage<T> &g = stage[st];
#pragma unroll
            for (int f = 0; f < 6; ++f) {
                if constexpr (ODD) {
                    cp_async<TB>(&g.f[f][tr].x, src[f] + col + o);
                    cp_async<TB>(&g.f[f][tr].y, src[f] + colb + o);
                } else {
                    cp_async<2 * TB>(&g.f[f][tr], src[f] + col + o);
                }
            }
            if (lane == 0) {
                cp_async<TB>(&g.e[0][w], Hz + im0 + (long long)j * Nx + o);
                cp_async<TB>(&g.e[1][w], Hy + im0 + (long long)j * Nx + o);
            }
            if (r == 0) {
                if constexpr (ODD) {
                    cp_async<TB>(&g.y[0][lane].x, Hz + colym + o);
                    cp_async<TB>(&g.y[0][lane].y, Hz + colymb + o);
                    cp_async<TB>(&g.y[1][lane].x, Hx + colym + o);
                    cp_async<TB>(&g.y[1][lane].y, Hx + colymb + o);
                } else {
                    cp_async<2 * TB>(&g.y[0][lane], Hz + colym + o);
                    cp_async<2 * TB>(&g.y[1][lane], Hx + colym + o);
                }
            }
        }
        cp_async_commit();
    };
    auto load_ids = [&](int kq) {
        I2 v;
        v.x = 0;
        v.y = 0;
        if (active && kq <= k1) {
            const long long om = (long long)(kq % Nz) * mNxNy;
            if constexpr (ODD) {
                v.x = __ldg(mat + colm + om);
                v.y = __ldg(mat + colmb + om);
            } else {
                v = ldg2<I2>(mat + colm + om);
            }
        }
        return v;
    };
    for (int s0 = 0; s0 < S - 1; ++s0) issue(k0 + s0, s0);
    I2 mm = load_ids(k0);
    // H(k0 - 1): the z-1 neighbours of E(k0)
    const int kb = (k0 == 0) ? Nz - 1 : k0 - 1;
    T2 hxp, hyp, hzp;
    hxp.x = hxp.y = hyp.x = hyp.y = hzp.x = hzp.y = 0;
    if (active) {
        hxp = ld(Hx, col + kb * NxNy, colb + kb * NxNy);
        hyp = ld(Hy, col + kb * NxNy, colb + kb * NxNy);
    }
    T2 exp_, eyp, ezp;                                   // new E(k - 1), own pair
    exp_.x = exp_.y = eyp.x = eyp.y = ezp.x = ezp.y = 0;

    for (int kq = k0; kq <= k1; ++kq) {
        const int k = kq % Nz;                           // plane k1 may wrap to 0
        const int buf = kq & 1;
        const long long o = (long long)k * NxNy;
        T2 hx, hy, hz, ex, ey, ez, hzy, hxy;
        T hz_e = 0, hy_e = 0;                            // x-1 of lane 0
        if (pf && kq + kFusedPrefetch <= k1) prefetch_plane(kq + kFusedPrefetch);
        issue(kq + S - 1, (kq - k0 + S - 1) % S);
        const I2 mm_next = load_ids(kq + 1);
        cp_async_wait<S - 1>();                          // this thread's copies of plane kq have landed
        if (active) {
            const FusedStage<T> &g = stage[(kq - k0) % S];
            hx = g.f[0][tr]; hy = g.f[1][tr]; hz = g.f[2][tr];
            ex = g.f[3][tr]; ey = g.f[4][tr]; ez = g.f[5][tr];
            if (lane == 0) { hz_e = g.e[0][w]; hy_e = g.e[1][w]; }
            if (r == 0) { hzy = g.y[0][lane]; hxy = g.y[1][lane]; }
            if (hrow) {   // rows read by the row above, and the column warp's x-1
                sm.hz[buf][r][lane] = hz;
                sm.hx[buf][r][lane] = hx;
                if (xl) { sm.hzl[buf][r] = hz.y; sm.hyl[buf][r] = hy.y; }
            }
        }
        __syncthreads();
        T2 nex, ney, nez;
        if (active) {
            if (r > 0) { hzy = sm.hz[buf][r - 1][lane]; hxy = sm.hx[buf][r - 1][lane]; }
            const T hz_up = __shfl_up_sync(kFullMask, hz.y, 1), hy_up = __shfl_up_sync(kFullMask, hy.y, 1);
            const T hz_im0 = lane == 0 ? hz_e : hz_up, hy_im0 = lane == 0 ? hy_e : hy_up;
            const bool sx = hrow && lown && kq < k1;     // owned cells of owned planes
            const bool sy = ODD ? (hrow && lown1 && kq < k1) : sx;
            e_cell<T, Tid, F>(A, q, ic, j, k, sx, mm.x, ex.x, ey.x, ez.x, hx.x, hy.x, hz.x, hxp.x, hyp.x, hzy.x, hxy.x,
                              hz_im0, hy_im0, nex.x, ney.x, nez.x);
            e_cell<T, Tid, F>(A, q, ic1, j, k, sy, mm.y, ex.y, ey.y, ez.y, hx.y, hy.y, hz.y, hxp.y, hyp.y, hzy.y,
                              hxy.y, hz.x, hy.x, nex.y, ney.y, nez.y);
            if (sx) {
                st(A.nEx, col + o, colb + o, nex, true, sy);
                st(A.nEy, col + o, colb + o, ney, true, sy);
                st(A.nEz, col + o, colb + o, nez, true, sy);
            }
            if (r > 0) {   // rows read by the row below
                sm.ez[buf][r][lane] = nez;
                sm.ex[buf][r][lane] = nex;
            }
        }
        // H(k - 1) of the owned rows from new E of plane k - 1 (registers,
        // shuffles, shared memory of the previous iteration) and of plane k
        const T ez_dn = __shfl_down_sync(kFullMask, ezp.x, 1), ey_dn = __shfl_down_sync(kFullMask, eyp.x, 1);
        if (hrow && lown && kq > k0) {
            const int kh = (kq - 1) % Nz;
            const int pb = buf ^ 1;
            const T2 ezj = sm.ez[pb][r + 1][lane], exj = sm.ex[pb][r + 1][lane];
            const T ez_ip1 = xl ? sm.eze[pb][r] : ez_dn, ey_ip1 = xl ? sm.eye[pb][r] : ey_dn;
            T2 nhx, nhy, nhz;
            h_cell<T, Tid, F>(A, q, ic, j, kh, hxp.x, hyp.x, hzp.x, exp_.x, eyp.x, ezp.x, nex.x, ney.x, ezj.x, exj.x,
                              ezp.y, eyp.y, nhx.x, nhy.x, nhz.x);
            const bool sy = ODD ? lown1 : true;
            if (sy)
                h_cell<T, Tid, F>(A, q, ic1, j, kh, hxp.y, hyp.y, hzp.y, exp_.y, eyp.y, ezp.y, nex.y, ney.y, ezj.y,
                                  exj.y, ez_ip1, ey_ip1, nhx.y, nhy.y, nhz.y);
            const long long oh = (long long)kh * NxNy;
            st(A.nHx, col + oh, colb + oh, nhx, true, sy);
            st(A.nHy, col + oh, colb + oh, nhy, true, sy);
            st(A.nHz, col + oh, colb + oh, nhz, true, sy);
        }
        if (active) {
            hxp = hx; hyp = hy; hzp = hz;
            exp_ = nex; eyp = ney; ezp = nez;
        }
        mm = mm_next;
    }
    cp_async_wait<0>();
}

template <typename T, typename Tid, unsigned F> struct FusedBounds {
    static constexpr int kThreads = 32 * (kFusedMaxTY + 2);
    // one (FP64) or two (FP32) CTAs per SM: registers for a march without
    // spills (the staging ring keeps loads in flight at this occupancy)
    static constexpr int kMinBlocks = sizeof(T) == 8 ? 1 : 2;
};

template <typename T, typename Tid, unsigned F, bool ODD>
__global__ void __launch_bounds__(FusedBounds<T, Tid, F>::kThreads, FusedBounds<T, Tid, F>::kMinBlocks)
yee_fused(const __grid_constant__ FusedArgs<T, Tid> A, const int4 *__restrict__ items) {
    fused_body<T, Tid, F, ODD>(A, A.e.q, items[blockIdx.x]);
}

// One launch of one instantiation; its staging ring (dynamic shared memory,
// above the 48 KiB default) is allowed once per instantiation.
template <typename T, typename Tid, unsigned F, bool O>
void launch_fused_one(const FusedArgs<T, Tid> &A, const int4 *p, int n, dim3 blk, cudaStream_t s) {
    constexpr size_t dyn = fused_stage_bytes<T>();
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(yee_fused<T, Tid, F, O>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
        attr = true;
    }
    yee_fused<T, Tid, F, O><<<n, blk, dyn, s>>>(A, p);
}

template <typename T, typename Tid>
void launch_fused_group_impl(const FusedArgs<T, Tid> &A, const int4 *items, int off, int n, int g, int ty,
                             cudaStream_t s) {
    if (n <= 0) return;
    const dim3 blk(32, ty + 2);
    const int4 *p = items + off;
    auto go = [&](auto odd) {
        constexpr bool O = decltype(odd)::value;
        switch (g) {
            case kFusedInterior: launch_fused_one<T, Tid, 0, O>(A, p, n, blk, s); break;
            case kFusedPmlZ: launch_fused_one<T, Tid, kFPmlZ, O>(A, p, n, blk, s); break;
            case kFusedDisp: launch_fused_one<T, Tid, kFDisp, O>(A, p, n, blk, s); break;
            case kFusedPmlXY: launch_fused_one<T, Tid, kFPmlXY | kFPmlZ, O>(A, p, n, blk, s); break;
            default: launch_fused_one<T, Tid, kFPmlXY | kFPmlZ | kFDisp | kFMisc, O>(A, p, n, blk, s); break;
        }
    };
    if (A.e.Nx % 2) go(std::true_type{});
    else go(std::false_type{});
}

}  // namespace aefdtd
