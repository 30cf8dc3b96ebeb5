// dft_tc.cu — the buffered DFT of the planar sensors on the tensor cores
// (FP32 path).
//
// For one sensor and a block of K buffered steps the DFT update of
// SensorFieldHolder::FT_comp (src/finite_differences/FDTD/sensors/
// sensors.cpp:456-479) is the product
//     acc[c][l][p] += sum_k S[k][c][p] * W_c[k][l]
// of the samples (P points x K steps, per field component c) with the phasor
// matrix (K x nl complex; W_E for E components, W_H for H components). It runs
// as a real GEMM D[128 x N] = A[128 x K] * B[K x N] per CTA, with N = 2 nl
// columns (Re, Im of each wavelength) in tiles of at most 256:
//   * A: 128 points of one component, split into TF32 hi + lo parts in shared
//     memory (K-major, 8-row x 16-byte core matrices, no swizzle);
//   * B: phasors split into TF32 hi + lo by the phasor kernel, already in the
//     shared-memory image layout, brought in with one bulk copy per part;
//   * three tcgen05.mma kind::tf32 per K step (hi*hi + hi*lo + lo*hi) issued by
//     one thread into a TMEM accumulator of 128 lanes x N columns, completion
//     through tcgen05.commit on an mbarrier;
//   * epilogue: tcgen05.ld of the warp's 32 lanes, added to the FP64
//     accumulators (split precision: FP32 tensor products per block, FP64
//     across blocks).
// All mbarrier waits are bounded; on timeout the CTA flags an error, frees its
// TMEM and returns.
#include <cuda_runtime.h>
#include <cstdint>

#include "aefdtd_dev.hpp"
#include "kernels.hpp"
#include "mbar.cuh"

namespace aefdtd {

namespace {

using mbar::saddr;
__device__ __forceinline__ void bar_init(uint64_t *b, uint32_t n) { mbar::init(b, n); }
__device__ __forceinline__ void bar_expect_tx(uint64_t *b, uint32_t bytes) { mbar::expect_tx(b, bytes); }
// gives up after `limit` SM cycles (2^32 by default, about 2 s)
__device__ __forceinline__ bool bar_wait(uint64_t *b, uint32_t parity, long long limit) {
    return mbar::wait(b, parity, limit);
}
using mbar::bulk_g2s;
__device__ __forceinline__ uint32_t to_tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}
// K-major, no-swizzle shared-memory matrix descriptor (tcgen05 format, version 1)
__device__ __forceinline__ uint64_t smem_desc(const void *start, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr(start) >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;   // descriptor version for tcgen05
    return d;                 // base offset 0, layout type 0 (no swizzle)
}
// instruction descriptor: D f32, A/B tf32, both K-major, M = 128, N
__device__ __forceinline__ uint32_t instr_desc(int N) {
    return (1u << 4)            // D format F32
         | (2u << 7)            // A format TF32
         | (2u << 10)           // B format TF32
         | ((uint32_t)(N >> 3) << 17)
         | ((uint32_t)(128 >> 4) << 24);
}
__device__ __forceinline__ void mma_tf32(uint32_t tmem, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        ::"r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
}
__device__ __forceinline__ void mma_commit(uint64_t *b) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(saddr(b))
                 : "memory");
}
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int q = 0; q < 16; ++q) v[q] = __uint_as_float(r[q]);
}

// byte offset of element (r, k) in a K-major core-matrix image of R rows
__host__ __device__ __forceinline__ uint32_t km_off(int r, int k, int R) {
    return (uint32_t)(((k >> 2) * (R >> 3) + (r >> 3)) * 128 + (r & 7) * 16 + (k & 3) * 4);
}

}  // namespace

// Phasors of the block in the B image layout: for tile t (columns
// [256 t, 256 t + Nt)), hi and lo parts, E and H families. Columns 2l and
// 2l+1 hold Re and Im of wavelength l; rows k >= nk and columns >= 2 nl are 0.
__global__ void dft_phasors_tc(DftTcPhasorArgs a) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    const int ncol = a.N0 + a.N1;
    if (idx >= a.K * ncol) return;
    const int k = idx / ncol, n = idx % ncol;
    const int t = n >= a.N0 ? 1 : 0;
    const int nn = t ? n - a.N0 : n;
    const int R = t ? a.N1 : a.N0;
    const int gn = t ? 256 + nn : nn;   // global column
    float vE = 0.f, vH = 0.f;
    if (k < a.nk && gn < 2 * a.nl) {
        const int l = gn >> 1, im = gn & 1;
        const int step = (a.step_ptr ? *a.step_ptr : 0) + a.step_add + k;
        double tE = 1.0, tH = 1.0;
        if (step - 1 >= a.Nt - a.Ntap && step >= 1) {
            // Sensor::feed tapering (sensors.cpp:236-240) with s_curve (mathUT.cpp:1186-1193)
            auto sc = [](double x, double xmin, double xmax) {
                const double u = (x - xmin) / (xmax - xmin);
                return u <= 0 ? 0.0 : (u >= 1.0 ? 1.0 : u * u * (3.0 - 2.0 * u));
            };
            tE = sc(step - 1, a.Nt - 1.0, a.Nt - a.Ntap);
            tH = sc(step - 1 + 0.5, a.Nt - 1.0, a.Nt - a.Ntap);
        }
        const double w = a.w[l];
        double s, c;
        sincos(w * step * a.Dt, &s, &c);
        vE = (float)(tE * (im ? s : c));
        sincos(w * (step + 0.5) * a.Dt, &s, &c);
        vH = (float)(tH * (im ? s : c));
    }
    const uint32_t off = km_off(nn, k, R) / 4;
    float *base = a.B + (size_t)t * a.tile_stride;   // [tile][E hi, E lo, H hi, H lo][R*K]
    const size_t part = (size_t)R * a.K;
    const uint32_t eh = to_tf32(vE), hh = to_tf32(vH);
    base[0 * part + off] = __uint_as_float(eh);
    base[1 * part + off] = __uint_as_float(to_tf32(vE - __uint_as_float(eh)));
    base[2 * part + off] = __uint_as_float(hh);
    base[3 * part + off] = __uint_as_float(to_tf32(vH - __uint_as_float(hh)));
}

// grid: (ceil(P / 128), 6); block kDftTcThreads (16 warps); dynamic smem
// kDftTcSmem. Warp w reads TMEM lanes 32 (w % 4) .. 32 (w % 4) + 31 (the
// lane quarter a warp may access) and the 16-column chunks w / 4, w / 4 + 4,
// ... of the tile, so four warps share each lane quarter and the FP64
// accumulator read-modify-write has 16 warps of loads in flight per SM.
__global__ void __launch_bounds__(kDftTcThreads, 1) dft_accumulate_tc(const __grid_constant__ DftTcArgs a) {
    extern __shared__ __align__(1024) unsigned char sm[];
    const int K = a.K;
    float *Ahi = reinterpret_cast<float *>(sm);
    float *Alo = Ahi + 128 * K;
    float *Bhi = Alo + 128 * K;
    float *Blo = Bhi + 256 * K;
    uint64_t *bars = reinterpret_cast<uint64_t *>(Blo + 256 * K);   // [0]: B copies, [1]: MMA done
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 2);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int c = blockIdx.y;
    const int p0 = blockIdx.x * 128;
    const int fam = c < 3 ? 0 : 2;   // E or H phasors

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(tmem_slot)),
                     "r"(256));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        bar_init(&bars[0], 1);
        bar_init(&bars[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    // A: this CTA's 128 points of component c, TF32 hi / lo; thread (m, kq)
    // converts steps kq, kq + 4, ... of point m
    {
        const int m = tid & 127, kq = tid >> 7;
        const int p = p0 + m;
        for (int k = kq; k < K; k += kDftTcThreads / 128) {
            const float v = (p < a.P && k < a.nk) ? a.S[((size_t)k * 6 + c) * a.P + p] : 0.f;
            const uint32_t h = to_tf32(v);
            const uint32_t o = km_off(m, k, 128) / 4;
            Ahi[o] = __uint_as_float(h);
            Alo[o] = __uint_as_float(to_tf32(v - __uint_as_float(h)));
        }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();

    const int lq = warp & 3, cg = warp >> 2;
    const int p = p0 + lq * 32 + lane;
    const uint32_t tlane = (uint32_t)(lq * 32) << 16;
    bool ok = true;
    const int ntiles = a.N1 > 0 ? 2 : 1;
    for (int t = 0; t < ntiles && ok; ++t) {
        const int Nt = t ? a.N1 : a.N0;
        const uint32_t part = (uint32_t)(Nt * K * 4);
        if (tid == 0 && !a.withhold_copy) {
            const float *src = a.B + (size_t)t * a.tile_stride + (size_t)fam * Nt * K;
            bar_expect_tx(&bars[0], 2 * part);
            bulk_g2s(Bhi, src, part, &bars[0]);
            bulk_g2s(Blo, src + (size_t)Nt * K, part, &bars[0]);
        }
        // withheld (test hook): no arrive and no copy in flight, so this wait
        // runs out and the CTA takes the error path below
        if (!bar_wait(&bars[0], t & 1, a.wait_cycles)) ok = false;
        if (tid == 0 && ok) {
            tc_fence_after();
            const uint32_t idesc = instr_desc(Nt);
            const uint32_t lboA = 16 * 128, lboB = (uint32_t)(Nt / 8) * 128;   // between the two K chunks
            for (int s = 0; s < K / 8; ++s) {
                const uint64_t ah = smem_desc(Ahi + km_off(0, 8 * s, 128) / 4, lboA, 128);
                const uint64_t al = smem_desc(Alo + km_off(0, 8 * s, 128) / 4, lboA, 128);
                const uint64_t bh = smem_desc(Bhi + km_off(0, 8 * s, Nt) / 4, lboB, 128);
                const uint64_t bl = smem_desc(Blo + km_off(0, 8 * s, Nt) / 4, lboB, 128);
                mma_tf32(tmem, al, bh, idesc, s > 0 ? 1u : 0u);
                mma_tf32(tmem, ah, bl, idesc, 1u);
                mma_tf32(tmem, ah, bh, idesc, 1u);
            }
            mma_commit(&bars[1]);
        }
        // FP64 accumulators of this warp's 16-column chunks, one chunk ahead:
        // the first chunk's loads go out before the MMA wait, each later one
        // while the previous chunk is added and stored
        auto load_chunk = [&](int col, double2 (&o)[8]) {
            const int gn0 = 256 * t + col;
            if (p < a.P && col < Nt) {
#pragma unroll
                for (int q = 0; q < 8; ++q)
                    if (gn0 + 2 * q < 2 * a.nl)
                        o[q] = __ldcs(a.acc + ((size_t)c * a.nl + ((gn0 >> 1) + q)) * a.P + p);
            }
        };
        double2 cur[8], nxt[8];
        load_chunk(16 * cg, cur);
        if (ok && !bar_wait(&bars[1], t & 1, a.wait_cycles)) ok = false;
        // every thread leaves the tile loop together: a failed wait on any
        // thread stops all of them before the next tile's copies
        ok = __syncthreads_and(ok);
        if (!ok) break;
        tc_fence_after();
        for (int col = 16 * cg; col < Nt; col += 64) {
            const int gn0 = 256 * t + col;
            load_chunk(col + 64, nxt);
            float v[16];
            ld16(tmem + tlane + (uint32_t)col, v);
            if (p < a.P) {
#pragma unroll
                for (int q = 0; q < 8; ++q)
                    if (gn0 + 2 * q < 2 * a.nl) {
                        cur[q].x += (double)v[2 * q];
                        cur[q].y += (double)v[2 * q + 1];
                        __stcs(a.acc + ((size_t)c * a.nl + ((gn0 >> 1) + q)) * a.P + p, cur[q]);
                    }
            }
#pragma unroll
            for (int q = 0; q < 8; ++q) cur[q] = nxt[q];
        }
        tc_fence_before();
        __syncthreads();   // TMEM and B read; next tile may overwrite both
    }
    if (!ok && tid == 0) atomicExch(a.err, 3);
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(256));
    }
}

void launch_phasors_tc(const DftTcPhasorArgs &a, cudaStream_t s) {
    const int n = a.K * (a.N0 + a.N1);
    dft_phasors_tc<<<(n + 255) / 256, 256, 0, s>>>(a);
}

void launch_accumulate_tc(const DftTcArgs &a, cudaStream_t s) {
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(dft_accumulate_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, kDftTcSmem);
        attr = true;
    }
    dim3 g((a.P + 127) / 128, 6);
    dft_accumulate_tc<<<g, kDftTcThreads, kDftTcSmem, s>>>(a);
}

}  // namespace aefdtd
