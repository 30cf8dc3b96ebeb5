// voxel.cu — structure discretisation on the device.
//
// Structure::discretize (src/structure/structure.cpp:94-113) tags every cell
// corner (i*Dx, j*Dy, k*Dz) with Structure::index (structure.cpp:228-258): the
// last operation whose primitive contains the point (or one of its periodic
// images) wins, else the default material. Primitive tests follow
// Add_Block::index (structure_primitives.cpp:34-39), Add_Layer::index
// (:323-339), Add_Sphere::index (:490-499) and Add_Cylinder (:255-285), in
// FP64 with the reference's operation order. Built with --fmad=false, so the
// tags are bit-identical to the CPU tagging.
#include <cuda_runtime.h>
#include <cstdint>

#include "../../include/aefdtd.h"

namespace aefdtd {

struct VoxOp {
    int kind, mat;
    double p[8];
    // cylinder precompute: unit axis and length (Add_Cylinder ctor)
    double bx, by, bz, length;
};

__device__ __forceinline__ int op_index(const VoxOp &o, double x, double y, double z) {
    switch (o.kind) {
        case AEFDTD_OP_BLOCK:
            if (x < o.p[0] || x >= o.p[1] || y < o.p[2] || y >= o.p[3] || z < o.p[4] || z >= o.p[5]) return -1;
            return o.mat;
        case AEFDTD_OP_LAYER: {
            int t = (int)o.p[0];
            double v = t == 0 ? x : (t == 1 ? y : z);
            if (v >= o.p[1] && v < o.p[2]) return o.mat;
            return -1;
        }
        case AEFDTD_OP_SPHERE: {
            double dx = x - o.p[0], dy = y - o.p[1], dz = z - o.p[2];
            if (dx * dx + dy * dy + dz * dz <= o.p[3] * o.p[3]) return o.mat;
            return -1;
        }
        case AEFDTD_OP_CYLINDER: {
            const double x1 = o.p[0], y1 = o.p[1], z1 = o.p[2], x2 = o.p[3], y2 = o.p[4], z2 = o.p[5], r = o.p[6];
            if (x < fmin(x1, x2) - r || x > fmax(x1, x2) + r || y < fmin(y1, y2) - r || y > fmax(y1, y2) + r ||
                z < fmin(z1, z2) - r || z > fmax(z1, z2) + r)
                return -1;
            double dx = x - x1, dy = y - y1, dz = z - z1;
            double proj = o.bx * dx + o.by * dy + o.bz * dz;
            if (proj >= 0 && proj <= o.length) {
                dx = dx - proj * o.bx;
                dy = dy - proj * o.by;
                dz = dz - proj * o.bz;
                double rt = dx * dx + dy * dy + dz * dz;
                if (rt <= r * r) return o.mat;
            }
            return -1;
        }
    }
    return -1;
}

struct VoxArgs {
    int nx, ny, nz, nops, def, per[3];
    double dx, dy, dz, l[3];
    const VoxOp *ops;
    uint32_t *out;
};

__global__ void voxelize_kernel(VoxArgs a) {
    const long long n = (long long)a.nx * a.ny * a.nz;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(q % a.nx);
        const int j = (int)((q / a.nx) % a.ny);
        const int k = (int)(q / ((long long)a.nx * a.ny));
        double x = i * a.dx, y = j * a.dy, z = k * a.dz;
        // modulus (src/common/mathUT.h:606-612)
        if (a.per[0]) { while (x < 0) x += a.l[0]; while (x >= a.l[0]) x -= a.l[0]; }
        if (a.per[1]) { while (y < 0) y += a.l[1]; while (y >= a.l[1]) y -= a.l[1]; }
        if (a.per[2]) { while (z < 0) z += a.l[2]; while (z >= a.l[2]) z -= a.l[2]; }
        int res = a.def;
        for (int l = a.nops - 1; l >= 0; --l) {
            int hit = -1;
            for (int ii = -a.per[0]; ii <= a.per[0] && hit < 0; ++ii)
                for (int jj = -a.per[1]; jj <= a.per[1] && hit < 0; ++jj)
                    for (int kk = -a.per[2]; kk <= a.per[2] && hit < 0; ++kk)
                        hit = op_index(a.ops[l], x + ii * a.l[0], y + jj * a.l[1], z + kk * a.l[2]);
            if (hit != -1) { res = hit; break; }
        }
        a.out[q] = (uint32_t)res;
    }
}

cudaError_t launch_voxelize(int nx, int ny, int nz, double dx, double dy, double dz, const aefdtd_structure_op *ops,
                            int nops, int def, const int per[3], const double l[3], uint32_t *d_out, cudaStream_t s) {
    VoxOp *d_ops = nullptr;
    VoxOp h[256];
    if (nops > 256) return cudaErrorInvalidValue;
    for (int q = 0; q < nops; q++) {
        h[q].kind = ops[q].kind;
        h[q].mat = ops[q].mat_index;
        for (int t = 0; t < 8; t++) h[q].p[t] = ops[q].p[t];
        h[q].bx = h[q].by = h[q].bz = h[q].length = 0;
        if (ops[q].kind == AEFDTD_OP_BLOCK) {
            // Add_Block ctor swaps reversed bounds (structure_primitives.cpp:24-32)
            for (int a = 0; a < 3; a++)
                if (h[q].p[2 * a] > h[q].p[2 * a + 1]) { double t = h[q].p[2 * a]; h[q].p[2 * a] = h[q].p[2 * a + 1]; h[q].p[2 * a + 1] = t; }
        }
        if (ops[q].kind == AEFDTD_OP_CYLINDER) {
            // Add_Cylinder ctor: base_vec = p2 - p1, length = |base_vec|, normalised (vector23.cpp:266-282)
            double vx = h[q].p[3] - h[q].p[0], vy = h[q].p[4] - h[q].p[1], vz = h[q].p[5] - h[q].p[2];
            double nrm = sqrt(vx * vx + vy * vy + vz * vz);
            h[q].length = nrm;
            h[q].bx = vx / nrm; h[q].by = vy / nrm; h[q].bz = vz / nrm;
        }
    }
    cudaError_t e = cudaSuccess;
    if (nops > 0) {
        e = cudaMallocAsync((void **)&d_ops, sizeof(VoxOp) * nops, s);
        if (e != cudaSuccess) return e;
        e = cudaMemcpyAsync(d_ops, h, sizeof(VoxOp) * nops, cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess) { cudaFreeAsync(d_ops, s); return e; }
    }
    VoxArgs a{nx, ny, nz, nops, def, {per[0], per[1], per[2]}, dx, dy, dz, {l[0], l[1], l[2]}, d_ops, d_out};
    long long n = (long long)nx * ny * nz;
    int blocks = (int)((n + 255) / 256 < 148 * 64 ? (n + 255) / 256 : 148 * 64);
    if (blocks < 1) blocks = 1;
    voxelize_kernel<<<blocks, 256, 0, s>>>(a);
    e = cudaGetLastError();
    if (d_ops) cudaFreeAsync(d_ops, s);
    return e;
}

}  // namespace aefdtd
