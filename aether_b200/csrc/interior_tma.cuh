// interior_tma.cuh — curl-only half-steps over 64 x 8 column tiles whose
// planes stream through a shared-memory ring filled by tensor copies.
//
// The cells are those of e_interior_body / h_interior_body (yee.cuh): the
// curl update of FDTD::advEx..advHz (fdtd_core.cpp:363-663, 715-969) with
// the same per-cell operations in the same order, so FP64 results are bit
// for bit those of the one-cell kernels. The difference is how the data
// arrive:
//   * one producer thread takes units (tile, z-run) from a device counter
//     and, for each plane of a unit, issues cp.async.bulk.tensor copies of
//     every value the plane's cells read into one stage of an S-stage ring,
//     S - 1 planes ahead of the consumers; an extra stage at the start of a
//     unit carries the z-neighbour plane (E: k0 - 1, H: k1, periodic);
//   * eight consumer warps (one per tile row, two x-adjacent cells per lane)
//     wait on the stage's mbarrier, read the values from shared memory,
//     write the new fields straight to global memory and release the stage;
//   * E marches up, H marches down, each keeping the z-neighbour of the
//     previous stage in registers.
// Staged per plane (E side; the H side mirrors it with E and H swapped and
// the halos on the +1 side): Hz and Hy with one 16-byte step of x halo, the
// Hz and Hx rows at y - 1, the own blocks of Hx, Ex, Ey, Ez and the material
// ids. Tiles at the x edge also copy the periodic-wrap column. Copies are
// tile-mode loads without multicast from this GPU's own arrays.
//
// Every wait is bounded; a wait that runs out raises the CTA's abort flag
// and the device error flag (AEFDTD_TIMEOUT on the host), and the producer
// waits for its copies in flight before the CTA exits.
#pragma once

#include "mbar.cuh"

namespace aefdtd {

constexpr int kTmaConsumers = kTmaTileY;                // one warp per tile row
constexpr int kTmaThreads = 32 * (kTmaConsumers + 1);   // plus the producer warp
constexpr int kTmaHalo = 1, kTmaWrapX = 2, kTmaStop = 4; // stage header flags

// Byte layout of one ring stage.
template <typename T, typename Tid> struct TmaStage {
    static constexpr int hx = 16 / (int)sizeof(T);      // x halo: one 16-byte step
    static constexpr int WX = kTmaTileX + hx;           // row length of the x-halo blocks
    static constexpr int kW = WX * kTmaTileY * (int)sizeof(T);
    static constexpr int kC = hx * kTmaTileY * (int)sizeof(T);
    static constexpr int kR = kTmaTileX * (int)sizeof(T);
    static constexpr int kB = kTmaTileX * kTmaTileY * (int)sizeof(T);
    static constexpr int kM = kTmaTileX * kTmaTileY * (int)sizeof(Tid);
    static constexpr int oW0 = 0, oW1 = kW, oC0 = 2 * kW, oC1 = oC0 + kC, oR0 = oC1 + kC, oR1 = oR0 + kR,
                         oB = oR1 + kR, oM = oB + 4 * kB, oHdr = oM + kM;
    static constexpr int kBytes = (oHdr + 16 + 127) / 128 * 128;
    static_assert(kW % 128 == 0 && kC % 128 == 0 && kR % 128 == 0 && kB % 128 == 0 && kM % 128 == 0,
                  "tensor-copy destinations stay 128-byte aligned");
};

// z-CPML planes of a half-step: E [1, pml_zm) and [Nz - pml_zp + 1, Nz); H
// [0, pml_zm) and [Nz - pml_zp, Nz - 1) (fdtd_pml.cpp:547,559,775,784).
template <typename T, typename Tid>
__device__ __forceinline__ bool zpsi_range(const StepArgs<T, Tid> &a, bool hs, int k) {
    if (!a.pz) return false;
    return hs ? (k < a.pml_zm || (k >= a.Nz - a.pml_zp && k < a.Nz - 1))
              : ((k >= 1 && k < a.pml_zm) || k >= a.Nz - a.pml_zp + 1);
}
// The z psi pair (PsiE/Hxz, PsiE/Hyz) of one lane's two cells at one plane,
// loaded ahead of the plane that uses it.
template <typename T> struct ZPsi {
    using V = typename Vec2<T>::type;
    V p0, p1;
    int i = -1, j = -1, k = -1;
    __device__ __forceinline__ bool has(int ii, int jj, int kk) const { return i == ii && j == jj && k == kk; }
    template <typename Tid> __device__ __forceinline__ long long index(const StepArgs<T, Tid> &a, int ii, int jj, int kk) const {
        const int zn = (kk < a.pml_zm) ? kk : kk - (a.Nz - a.pml_zp) + a.pml_zm;
        return ii + (long long)jj * a.Nx + (long long)zn * a.NxNy;
    }
    template <typename Tid> __device__ __forceinline__ void fetch(const StepArgs<T, Tid> &a, bool hs, int ii, int jj, int kk) {
        if (!zpsi_range(a, hs, kk)) return;
        const long long o = index(a, ii, jj, kk);
        p0 = *reinterpret_cast<const V *>(a.psi_z0 + o);
        p1 = *reinterpret_cast<const V *>(a.psi_z1 + o);
        i = ii; j = jj; k = kk;
    }
};

// Producer: one thread. HS: the H half-step.
// limit: bound of each wait (SM cycles); withhold (test hook): no copy and
// no arrive on any data stage, so the consumers' waits run out.
template <typename T, typename Tid, int S, bool HS>
__device__ __forceinline__ void tma_produce(const StepArgs<T, Tid> &a, const TmaMaps &m, const int4 *units,
                                            int nunits, int *ctr, unsigned char *sm, uint64_t *full,
                                            uint64_t *empty, volatile int *abort, long long limit, int withhold) {
    using L = TmaStage<T, Tid>;
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        mbar::prefetch_tmap(&m.w[q]); mbar::prefetch_tmap(&m.c[q]); mbar::prefetch_tmap(&m.r[q]);
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) mbar::prefetch_tmap(&m.b[q]);
    if (!HS) mbar::prefetch_tmap(&m.mat);
    int st = 0, issued = 0;
    uint32_t ph = 0;
    bool ok = true;
    // one unit per CTA (grid = units: CTAs come and go like any other
    // kernel's), or units taken in turn from the counter
    const bool one = (int)gridDim.x == nunits;
    int u = one ? (int)blockIdx.x : atomicAdd(ctr, 1);
    for (;;) {
        if (!mbar::wait_or_abort(&empty[st], ph ^ 1, limit, abort)) { ok = false; break; }
        int4 *hdr = reinterpret_cast<int4 *>(sm + st * L::kBytes + L::oHdr);
        if (u >= nunits) {   // no unit left: a stop stage without copies
            *hdr = make_int4(0, 0, 0, kTmaStop);
            mbar::arrive(&full[st]);
            break;
        }
        const int4 it = units[u];
        const int nxt = one ? nunits : atomicAdd(ctr, 1);   // the next unit, fetched while this one is issued
        const int x0 = it.x, y0 = it.y, k0 = it.z, k1 = it.w;
        const bool wrapx = HS ? (x0 + kTmaTileX == a.Nx) : (x0 == 0);
        const int xw = HS ? x0 : x0 - L::hx;                                // x-halo block start
        const int xc = HS ? 0 : a.Nx - L::hx;                               // periodic-wrap column
        const int yr = HS ? (y0 + kTmaTileY == a.Ny ? 0 : y0 + kTmaTileY)   // y-halo row
                          : (y0 == 0 ? a.Ny - 1 : y0 - 1);
        const int flags = wrapx ? kTmaWrapX : 0;
        for (int p = -1; p < k1 - k0; ++p) {
            if (p >= 0 && !mbar::wait_or_abort(&empty[st], ph ^ 1, limit, abort)) { ok = false; break; }
            unsigned char *b = sm + st * L::kBytes;
            uint64_t *f = &full[st];
            if (withhold) {
                // test hook: the stage's header only
                *reinterpret_cast<int4 *>(b + L::oHdr) = make_int4(x0, y0, 0, flags | (p < 0 ? kTmaHalo : 0));
            } else if (p < 0) {
                // the z-neighbour plane: own columns of Hx and Hy (E) or Ex and Ey (H)
                const int k = HS ? (k1 == a.Nz ? 0 : k1) : (k0 == 0 ? a.Nz - 1 : k0 - 1);
                *reinterpret_cast<int4 *>(b + L::oHdr) = make_int4(x0, y0, k, flags | kTmaHalo);
                mbar::expect_tx(f, L::kB + L::kW);
                mbar::tensor_g2s_3d(b + L::oB, &m.b[0], x0, y0, k, f);
                mbar::tensor_g2s_3d(b + L::oW1, &m.w[1], xw, y0, k, f);
            } else {
                const int k = HS ? k1 - 1 - p : k0 + p;
                *reinterpret_cast<int4 *>(b + L::oHdr) = make_int4(x0, y0, k, flags);
                mbar::expect_tx(f, 2 * L::kW + 2 * L::kR + 4 * L::kB + (HS ? 0 : L::kM) + (wrapx ? 2 * L::kC : 0));
                mbar::tensor_g2s_3d(b + L::oW0, &m.w[0], xw, y0, k, f);
                mbar::tensor_g2s_3d(b + L::oW1, &m.w[1], xw, y0, k, f);
                mbar::tensor_g2s_3d(b + L::oR0, &m.r[0], x0, yr, k, f);
                mbar::tensor_g2s_3d(b + L::oR1, &m.r[1], x0, yr, k, f);
#pragma unroll
                for (int q = 0; q < 4; ++q) mbar::tensor_g2s_3d(b + L::oB + q * L::kB, &m.b[q], x0, y0, k, f);
                if (!HS) mbar::tensor_g2s_3d(b + L::oM, &m.mat, x0, y0, k, f);
                if (wrapx) {
                    mbar::tensor_g2s_3d(b + L::oC0, &m.c[0], xc, y0, k, f);
                    mbar::tensor_g2s_3d(b + L::oC1, &m.c[1], xc, y0, k, f);
                }
            }
            ++issued;
            if (++st == S) { st = 0; ph ^= 1; }
        }
        if (!ok) break;
        u = nxt;
    }
    if (!ok) {
        // a wait ran out: stop the consumers, then wait for the copies of the
        // last S stages so that none lands after the CTA has exited
        *abort = 1;
        atomicExch(a.err, 1);
        for (int d = 1; d <= min(issued, S); ++d) {
            const int s = (st - d + S) % S;
            if (!withhold) mbar::wait(&full[s], s < st ? ph : ph ^ 1, limit);
        }
    }
    // the last CTA to finish resets the counters for the next launch
    if (one) return;
    __threadfence();
    if (atomicAdd(ctr + 1, 1) == (int)gridDim.x - 1) {
        ctr[0] = 0;
        ctr[1] = 0;
        __threadfence();
    }
}

template <typename T, typename Tid, int S>
__device__ __forceinline__ void e_tma_consume(const StepArgs<T, Tid> &a, unsigned char *sm, uint64_t *full,
                                              uint64_t *empty, volatile int *abort, long long limit) {
    using L = TmaStage<T, Tid>;
    using V = typename Vec2<T>::type;
    using P = typename IdPair<Tid>::type;
    constexpr int X = kTmaTileX, B1 = kTmaTileX * kTmaTileY;
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31, c = 2 * l;
    int st = 0;
    uint32_t ph = 0;
    T hxm0 = 0, hxm1 = 0, hym0 = 0, hym1 = 0, ikx0 = 0, ikx1 = 0, iky = 0;
    // z-CPML psi of the lane's pair, loaded one plane ahead (tagged by tile and plane)
    ZPsi<T> zp;
    for (;;) {
        if (!mbar::wait_or_abort(&full[st], ph, limit, abort)) {
            *abort = 1;
            atomicExch(a.err, 1);
            return;
        }
        const unsigned char *b = sm + st * L::kBytes;
        const int4 hdr = *reinterpret_cast<const int4 *>(b + L::oHdr);
        if (hdr.w & kTmaStop) return;
        const T *W0 = reinterpret_cast<const T *>(b + L::oW0);   // Hz, x halo
        const T *W1 = reinterpret_cast<const T *>(b + L::oW1);   // Hy, x halo
        const T *Bk = reinterpret_cast<const T *>(b + L::oB);    // Hx, Ex, Ey, Ez
        const int x0 = hdr.x, y0 = hdr.y, k = hdr.z;
        if (hdr.w & kTmaHalo) {
            const V hx = *reinterpret_cast<const V *>(Bk + w * X + c);
            const V hy = *reinterpret_cast<const V *>(W1 + w * L::WX + L::hx + c);
            hxm0 = hx.x; hxm1 = hx.y; hym0 = hy.x; hym1 = hy.y;
            ikx0 = __ldg(a.ikx + x0 + c); ikx1 = __ldg(a.ikx + x0 + c + 1); iky = __ldg(a.iky + y0 + w);
            zp.fetch(a, false, x0 + c, y0 + w, k == a.Nz - 1 ? 0 : k + 1);   // the unit's first plane
        } else {
            const T *R0 = reinterpret_cast<const T *>(b + L::oR0);   // Hz row y - 1
            const T *R1 = reinterpret_cast<const T *>(b + L::oR1);   // Hx row y - 1
            const V hz = *reinterpret_cast<const V *>(W0 + w * L::WX + L::hx + c);
            const V hy = *reinterpret_cast<const V *>(W1 + w * L::WX + L::hx + c);
            T hz_im = W0[w * L::WX + L::hx + c - 1];
            T hy_im = W1[w * L::WX + L::hx + c - 1];
            if ((hdr.w & kTmaWrapX) && l == 0) {
                hz_im = reinterpret_cast<const T *>(b + L::oC0)[w * L::hx + L::hx - 1];
                hy_im = reinterpret_cast<const T *>(b + L::oC1)[w * L::hx + L::hx - 1];
            }
            const V hz_jm = w ? *reinterpret_cast<const V *>(W0 + (w - 1) * L::WX + L::hx + c)
                              : *reinterpret_cast<const V *>(R0 + c);
            const V hx = *reinterpret_cast<const V *>(Bk + w * X + c);
            const V hx_jm = w ? *reinterpret_cast<const V *>(Bk + (w - 1) * X + c) : *reinterpret_cast<const V *>(R1 + c);
            const V ex = *reinterpret_cast<const V *>(Bk + B1 + w * X + c);
            const V ey = *reinterpret_cast<const V *>(Bk + 2 * B1 + w * X + c);
            const V ez = *reinterpret_cast<const V *>(Bk + 3 * B1 + w * X + c);
            const P mp = *reinterpret_cast<const P *>(reinterpret_cast<const Tid *>(b + L::oM) + w * X + c);
            const T ikz = __ldg(a.ikz + k);
            T nex[2], ney[2], nez[2];
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const MatCoef<T> *cp = a.coef + (q ? mp.y : mp.x);
                const T C1 = __ldg(&cp->C1), C2x = __ldg(&cp->C2x), C2y = __ldg(&cp->C2y), C2z = __ldg(&cp->C2z);
                const T ikx = q ? ikx1 : ikx0;
                const T exq = q ? ex.y : ex.x, eyq = q ? ey.y : ey.x, ezq = q ? ez.y : ez.x;
                const T hxq = q ? hx.y : hx.x, hyq = q ? hy.y : hy.x, hzq = q ? hz.y : hz.x;
                const T hzjm = q ? hz_jm.y : hz_jm.x, hxjm = q ? hx_jm.y : hx_jm.x;
                const T hzim = q ? hz.x : hz_im, hyim = q ? hy.x : hy_im;
                const T hxm = q ? hxm1 : hxm0, hym = q ? hym1 : hym0;
                nex[q] = (C1 * exq + (C2y * iky) * (hzq - hzjm)) - (C2z * ikz) * (hyq - hym);
                ney[q] = (C1 * eyq + (C2z * ikz) * (hxq - hxm)) - (C2x * ikx) * (hzq - hzim);
                nez[q] = (C1 * ezq + (C2x * ikx) * (hyq - hyim)) - (C2y * iky) * (hxq - hxjm);
            }
            if (zpsi_range(a, false, k)) {
                // z-CPML planes: PsiExz, PsiEyz in app_pml_Ex / Ey order (after the curl update)
                if (!zp.has(x0 + c, y0 + w, k)) zp.fetch(a, false, x0 + c, y0 + w, k);
                const T bzk = __ldg(a.bz + k), czk = __ldg(a.cz + k);
                V ps0, ps1;
#pragma unroll
                for (int q = 0; q < 2; ++q) {
                    const T C4 = __ldg(&(a.coef + (q ? mp.y : mp.x))->C4);
                    const T hxq = q ? hx.y : hx.x, hyq = q ? hy.y : hy.x;
                    const T hxm = q ? hxm1 : hxm0, hym = q ? hym1 : hym0;
                    const T p0 = cpml_rec(bzk, q ? zp.p0.y : zp.p0.x, czk, hyq - hym);
                    const T p1 = cpml_rec(bzk, q ? zp.p1.y : zp.p1.x, czk, hxq - hxm);
                    nex[q] -= C4 * p0;
                    ney[q] += C4 * p1;
                    if (q) { ps0.y = p0; ps1.y = p1; } else { ps0.x = p0; ps1.x = p1; }
                }
                const long long pz = zp.index(a, x0 + c, y0 + w, k);
                *reinterpret_cast<V *>(a.psi_z0 + pz) = ps0;
                *reinterpret_cast<V *>(a.psi_z1 + pz) = ps1;
            }
            if (a.pz && k == 0) { nex[0] = 0; nex[1] = 0; ney[0] = 0; ney[1] = 0; }
            const long long id = (x0 + c) + (long long)(y0 + w) * a.Nx + (long long)k * a.NxNy;
            V o;
            o.x = nex[0]; o.y = nex[1]; *reinterpret_cast<V *>(a.Ex + id) = o;
            o.x = ney[0]; o.y = ney[1]; *reinterpret_cast<V *>(a.Ey + id) = o;
            o.x = nez[0]; o.y = nez[1]; *reinterpret_cast<V *>(a.Ez + id) = o;
            hxm0 = hx.x; hxm1 = hx.y; hym0 = hy.x; hym1 = hy.y;
            if (k + 1 < a.Nz) zp.fetch(a, false, x0 + c, y0 + w, k + 1);   // the next plane, while this stage is released
        }
        __syncwarp();
        if (l == 0) mbar::arrive(&empty[st]);
        if (++st == S) { st = 0; ph ^= 1; }
    }
}

template <typename T, typename Tid, int S>
__device__ __forceinline__ void h_tma_consume(const StepArgs<T, Tid> &a, unsigned char *sm, uint64_t *full,
                                              uint64_t *empty, volatile int *abort, long long limit) {
    using L = TmaStage<T, Tid>;
    using V = typename Vec2<T>::type;
    constexpr int X = kTmaTileX, B1 = kTmaTileX * kTmaTileY;
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31, c = 2 * l;
    int st = 0;
    uint32_t ph = 0;
    T exp0 = 0, exp1 = 0, eyp0 = 0, eyp1 = 0, ax0 = 0, ax1 = 0, ay = 0;
    ZPsi<T> zp;
    for (;;) {
        if (!mbar::wait_or_abort(&full[st], ph, limit, abort)) {
            *abort = 1;
            atomicExch(a.err, 1);
            return;
        }
        const unsigned char *b = sm + st * L::kBytes;
        const int4 hdr = *reinterpret_cast<const int4 *>(b + L::oHdr);
        if (hdr.w & kTmaStop) return;
        const T *W0 = reinterpret_cast<const T *>(b + L::oW0);   // Ez, x halo
        const T *W1 = reinterpret_cast<const T *>(b + L::oW1);   // Ey, x halo
        const T *Bk = reinterpret_cast<const T *>(b + L::oB);    // Ex, Hx, Hy, Hz
        const int x0 = hdr.x, y0 = hdr.y, k = hdr.z;
        if (hdr.w & kTmaHalo) {
            const V ex = *reinterpret_cast<const V *>(Bk + w * X + c);
            const V ey = *reinterpret_cast<const V *>(W1 + w * L::WX + c);
            exp0 = ex.x; exp1 = ex.y; eyp0 = ey.x; eyp1 = ey.y;
            ax0 = a.dtdmx * __ldg(a.ikx + x0 + c);
            ax1 = a.dtdmx * __ldg(a.ikx + x0 + c + 1);
            ay = a.dtdmy * __ldg(a.iky + y0 + w);
            zp.fetch(a, true, x0 + c, y0 + w, k == 0 ? a.Nz - 1 : k - 1);   // the unit's first (top) plane
        } else {
            const T *R0 = reinterpret_cast<const T *>(b + L::oR0);   // Ez row y + 1
            const T *R1 = reinterpret_cast<const T *>(b + L::oR1);   // Ex row y + 1
            const V ez = *reinterpret_cast<const V *>(W0 + w * L::WX + c);
            const V ey = *reinterpret_cast<const V *>(W1 + w * L::WX + c);
            T ez_ip = W0[w * L::WX + c + 2];
            T ey_ip = W1[w * L::WX + c + 2];
            if ((hdr.w & kTmaWrapX) && l == 31) {
                ez_ip = reinterpret_cast<const T *>(b + L::oC0)[w * L::hx];
                ey_ip = reinterpret_cast<const T *>(b + L::oC1)[w * L::hx];
            }
            const V ez_jp = w < kTmaTileY - 1 ? *reinterpret_cast<const V *>(W0 + (w + 1) * L::WX + c)
                                              : *reinterpret_cast<const V *>(R0 + c);
            const V ex = *reinterpret_cast<const V *>(Bk + w * X + c);
            const V ex_jp = w < kTmaTileY - 1 ? *reinterpret_cast<const V *>(Bk + (w + 1) * X + c)
                                              : *reinterpret_cast<const V *>(R1 + c);
            const V hx = *reinterpret_cast<const V *>(Bk + B1 + w * X + c);
            const V hy = *reinterpret_cast<const V *>(Bk + 2 * B1 + w * X + c);
            const V hz = *reinterpret_cast<const V *>(Bk + 3 * B1 + w * X + c);
            const T az = a.dtdmz * __ldg(a.ikz + k);
            T nhx[2], nhy[2], nhz[2];
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const T ax = q ? ax1 : ax0;
                const T exq = q ? ex.y : ex.x, eyq = q ? ey.y : ey.x, ezq = q ? ez.y : ez.x;
                const T exkp = q ? exp1 : exp0, eykp = q ? eyp1 : eyp0;
                const T ezjp = q ? ez_jp.y : ez_jp.x, exjp = q ? ex_jp.y : ex_jp.x;
                const T ezip = q ? ez_ip : ez.y, eyip = q ? ey_ip : ey.y;
                const T hxq = q ? hx.y : hx.x, hyq = q ? hy.y : hy.x, hzq = q ? hz.y : hz.x;
                nhx[q] = hxq + (az * (eykp - eyq) - ay * (ezjp - ezq));
                nhy[q] = hyq + (ax * (ezip - ezq) - az * (exkp - exq));
                nhz[q] = hzq + (ay * (exjp - exq) - ax * (eyip - eyq));
            }
            if (zpsi_range(a, true, k)) {
                // z-CPML planes: PsiHxz, PsiHyz in app_pml_Hx / Hy order (after the curl update)
                if (!zp.has(x0 + c, y0 + w, k)) zp.fetch(a, true, x0 + c, y0 + w, k);
                const T bzk = __ldg(a.bz + k), czk = __ldg(a.cz + k);
                V ps0, ps1;
#pragma unroll
                for (int q = 0; q < 2; ++q) {
                    const T exq = q ? ex.y : ex.x, eyq = q ? ey.y : ey.x;
                    const T exkp = q ? exp1 : exp0, eykp = q ? eyp1 : eyp0;
                    const T p0 = cpml_rec(bzk, q ? zp.p0.y : zp.p0.x, czk, eykp - eyq);
                    const T p1 = cpml_rec(bzk, q ? zp.p1.y : zp.p1.x, czk, exkp - exq);
                    nhx[q] += a.dtm * p0;
                    nhy[q] -= a.dtm * p1;
                    if (q) { ps0.y = p0; ps1.y = p1; } else { ps0.x = p0; ps1.x = p1; }
                }
                const long long pz = zp.index(a, x0 + c, y0 + w, k);
                *reinterpret_cast<V *>(a.psi_z0 + pz) = ps0;
                *reinterpret_cast<V *>(a.psi_z1 + pz) = ps1;
            }
            if (a.pz && k == a.Nz - 1) { nhx[0] = 0; nhx[1] = 0; nhy[0] = 0; nhy[1] = 0; }
            const long long id = (x0 + c) + (long long)(y0 + w) * a.Nx + (long long)k * a.NxNy;
            V o;
            o.x = nhx[0]; o.y = nhx[1]; *reinterpret_cast<V *>(a.Hx + id) = o;
            o.x = nhy[0]; o.y = nhy[1]; *reinterpret_cast<V *>(a.Hy + id) = o;
            o.x = nhz[0]; o.y = nhz[1]; *reinterpret_cast<V *>(a.Hz + id) = o;
            exp0 = ex.x; exp1 = ex.y; eyp0 = ey.x; eyp1 = ey.y;
            if (k > 0) zp.fetch(a, true, x0 + c, y0 + w, k - 1);   // the next plane down
        }
        __syncwarp();
        if (l == 0) mbar::arrive(&empty[st]);
        if (++st == S) { st = 0; ph ^= 1; }
    }
}

// S: ring stages (4 or 6)
template <typename T, typename Tid, bool HS, int S>
__global__ void __launch_bounds__(kTmaThreads, 2)
interior_tma(const __grid_constant__ StepArgs<T, Tid> a, const __grid_constant__ TmaMaps m,
             const int4 *__restrict__ units, int nunits, int *ctr, long long limit, int withhold) {
    __shared__ __align__(8) uint64_t full[S], empty[S];
    __shared__ int abort_flag;
    extern __shared__ __align__(128) unsigned char tma_dsm[];
    unsigned char *sm = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(tma_dsm) + 127) & ~uintptr_t(127));
    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) {
            mbar::init(&full[s], 1);
            mbar::init(&empty[s], kTmaConsumers);
        }
        abort_flag = 0;
        mbar::fence_init();
    }
    __syncthreads();
    if (threadIdx.x >= 32 * kTmaConsumers) {
        if (threadIdx.x == 32 * kTmaConsumers)
            tma_produce<T, Tid, S, HS>(a, m, units, nunits, ctr, sm, full, empty, &abort_flag, limit, withhold);
        return;
    }
    if constexpr (HS) h_tma_consume<T, Tid, S>(a, sm, full, empty, &abort_flag, limit);
    else e_tma_consume<T, Tid, S>(a, sm, full, empty, &abort_flag, limit);
}

template <typename T, typename Tid, bool HS, int S> void launch_tma_one(const StepArgs<T, Tid> &a, const TmaPlan &p, cudaStream_t s) {
    constexpr int smem = S * TmaStage<T, Tid>::kBytes + 128;
    static bool attr = false;   // one instantiation per (T, Tid, HS, S)
    if (!attr) {
        cudaFuncSetAttribute(interior_tma<T, Tid, HS, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        attr = true;
    }
    interior_tma<T, Tid, HS, S><<<p.grid, kTmaThreads, smem, s>>>(a, p.maps, p.units, p.nunits, p.ctr, p.wait_cycles,
                                                                  p.withhold);
}
template <typename T, typename Tid, bool HS> void launch_tma_impl(const StepArgs<T, Tid> &a, const TmaPlan &p, cudaStream_t s) {
    if (p.stages >= 6) launch_tma_one<T, Tid, HS, 6>(a, p, s);
    else launch_tma_one<T, Tid, HS, 4>(a, p, s);
}

}  // namespace aefdtd
