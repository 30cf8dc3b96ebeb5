// voxel.cu — structure discretisation on the device.
//
// Structure::discretize (src/structure/structure.cpp:94-113) tags every cell
// corner (i*Dx, j*Dy, k*Dz) with Structure::index (structure.cpp:223-258):
// mirror flips, then the periodic modulus, then the last operation whose
// primitive contains the point (or one of its periodic images) wins, else the
// default material. The primitive tests follow structure_primitives.cpp in
// FP64 with the reference's operation order; this file is built with
// --fmad=false, so the tags are bit-identical to the reference's CPU tagging.
//
// Coatings query the structure below themselves (Structure::index with a
// restricted operation count), so struct_index/op_index are templates over
// the remaining nesting depth: a coating at depth D evaluates the lower stack
// at depth D-1. The host checks the nesting before launch.
//
// Values the device cannot reproduce bit for bit are prepared on the host
// with the reference's own expressions: the sine terms of Add_Sin_Layer at the
// grid corners (std::sin), the coating direction (std::cos/std::sin of the
// angles), the unit axis of cylinders and cones, and the pivoted LU factors of
// the vector-block edge matrix.
//
// A mesh point counts ray crossings over all triangles with the reference's
// Moller-Trumbore test. The reference draws the ray direction at random for
// every point; here it is a hash of the point. The crossing parity agrees
// except for rays through a triangle's edge or vertex.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include "../../include/aefdtd.h"

namespace aefdtd {

namespace {

constexpr int kVoxDepth = 3;                 // coatings nest at most this deep
constexpr int kMaxMarch = 1 << 22;           // bound on every device loop that walks space
constexpr double kPi = 3.141592653589793;    // std::numbers::pi_v<double>

struct VoxOp {
    int kind, mat, stack, origin;
    double p[16];
    double bx, by, bz, length;               // cylinder, cone: unit axis and length
    double vmin[3], vmax[3];                 // vector block / triangle: bounding box
    double lu[3][3];                         // vector block: pivoted LU of the edge matrix
    int pidx[3], qidx[3], rank;
    double dir[3];                           // directional coating
    double inv_px, inv_py;                   // sine layer
    long long sin_off;                       // sine layer: offset of its x then y tables
    int nl[3];                               // conformal coating: seed lattice size
    long long lat_off;                       // conformal coating: offset of its lattice masks
    long long tri_off;                       // mesh: offset of its triangles (V1, E1, E2: 9 doubles each)
    int n_tri;
};

struct VoxArgs {
    int nx, ny, nz, nops, def, per[3], flip[3];
    double dx, dy, dz, l[3];
    const VoxOp *ops;
    const uint8_t *lattice;
    const double *sintab;
    const double *tris;
    uint32_t *out;
    int *err;
};

struct Ctx {
    int i, j;  // grid corner of a top-level query, -1 inside coating queries
};

__device__ __forceinline__ double vmod(double v, double m, const VoxArgs &a) {
    // modulus (src/common/mathUT.h:606-612), with a bound on the walk
    int n = 0;
    while (v < 0) { v += m; if (++n > kMaxMarch) { atomicExch(a.err, 1); return 0; } }
    while (v >= m) { v -= m; if (++n > kMaxMarch) { atomicExch(a.err, 1); return 0; } }
    return v;
}

template <int D>
__device__ int struct_index(const VoxArgs &a, double x, double y, double z, int restrict_level, Ctx c);

// Solves the edge-matrix system with the stored factors: P, unit-lower L
// column by column, upper U column by column from the last pivot, then Q.
__device__ __forceinline__ void solve3(const VoxOp &o, double x, double y, double z, double &ra, double &rb,
                                       double &rc) {
    double b[3] = {x, y, z}, c[3] = {0, 0, 0}, r[3] = {0, 0, 0};
    if (o.rank > 0) {
        for (int i = 0; i < 3; i++) c[o.pidx[i]] = b[i];
        for (int i = 0; i < 3; i++)
            for (int s = i + 1; s < 3; s++) c[s] = c[s] - c[i] * o.lu[s][i];
        for (int i = o.rank - 1; i >= 0; i--) {
            c[i] = c[i] / o.lu[i][i];
            for (int s = 0; s < i; s++) c[s] = c[s] - c[i] * o.lu[s][i];
        }
        for (int i = 0; i < 3; i++) r[o.qidx[i]] = i < o.rank ? c[i] : 0.0;
    }
    ra = r[0];
    rb = r[1];
    rc = r[2];
}

template <int D>
__device__ int op_index(const VoxArgs &a, const VoxOp &o, double x, double y, double z, Ctx c, int ii, int jj) {
    const double *p = o.p;
    switch (o.kind) {
        case AEFDTD_OP_BLOCK:  // Add_Block::index (structure_primitives.cpp:34-39)
            if (x < p[0] || x >= p[1] || y < p[2] || y >= p[3] || z < p[4] || z >= p[5]) return -1;
            return o.mat;
        case AEFDTD_OP_LAYER: {  // Add_Layer::index (:323-339)
            int t = (int)p[0];
            double v = t == 0 ? x : (t == 1 ? y : z);
            if (v >= p[1] && v < p[2]) return o.mat;
            return -1;
        }
        case AEFDTD_OP_SPHERE: {  // Add_Sphere::index (:490-499)
            double ex = x - p[0], ey = y - p[1], ez = z - p[2];
            if (ex * ex + ey * ey + ez * ez <= p[3] * p[3]) return o.mat;
            return -1;
        }
        case AEFDTD_OP_CYLINDER:
        case AEFDTD_OP_CONE: {  // Add_Cylinder::index (:266-284), Add_Cone::index (:112-134)
            const double x1 = p[0], y1 = p[1], z1 = p[2], x2 = p[3], y2 = p[4], z2 = p[5], r = p[6];
            if (x < fmin(x1, x2) - r || x > fmax(x1, x2) + r || y < fmin(y1, y2) - r || y > fmax(y1, y2) + r ||
                z < fmin(z1, z2) - r || z > fmax(z1, z2) + r)
                return -1;
            double ex = x - x1, ey = y - y1, ez = z - z1;
            double proj = o.bx * ex + o.by * ey + o.bz * ez;
            if (proj >= 0 && proj <= o.length) {
                ex = ex - proj * o.bx;
                ey = ey - proj * o.by;
                ez = ez - proj * o.bz;
                double rt = ex * ex + ey * ey + ez * ez;
                double r2 = r * r;
                if (o.kind == AEFDTD_OP_CONE) {
                    r2 = r * (1.0 - proj / o.length);
                    r2 = r2 * r2;
                }
                if (rt <= r2) return o.mat;
            }
            return -1;
        }
        case AEFDTD_OP_ELLIPSOID: {  // Add_Ellipsoid::index (:298-312)
            if (x < p[0] - p[3] || x > p[0] + p[3] || y < p[1] - p[4] || y > p[1] + p[4] || z < p[2] - p[5] ||
                z > p[2] + p[5])
                return -1;
            double ex = (x - p[0]) / p[3], ey = (y - p[1]) / p[4], ez = (z - p[2]) / p[5];
            if (ex * ex + ey * ey + ez * ez <= 1.0) return o.mat;
            return -1;
        }
        case AEFDTD_OP_SIN_LAYER: {  // Add_Sin_Layer::index (:459-478)
            double sx, sy;
            if (c.i >= 0) {
                sx = a.sintab[o.sin_off + (long long)(ii + 1) * a.nx + c.i];
                sy = a.sintab[o.sin_off + 3LL * a.nx + (long long)(jj + 1) * a.ny + c.j];
            } else {
                sx = sin((2.0 * kPi) * (x * o.inv_px + p[5]));
                sy = sin((2.0 * kPi) * (y * o.inv_py + p[7]));
            }
            double t = 0.5 * (sx + sy);
            double h1 = p[0] + p[1] * t, h2 = p[2] + p[3] * t;
            if (h1 <= z && h2 >= z) return o.mat;
            return -1;
        }
        case AEFDTD_OP_VECT_BLOCK:
        case AEFDTD_OP_VECT_TRI: {  // Add_Vect_Block::index (:552-566), Add_Vect_Tri::index (:586-601)
            if (x < o.vmin[0] || x > o.vmax[0] || y < o.vmin[1] || y > o.vmax[1] || z < o.vmin[2] || z > o.vmax[2])
                return -1;
            double ca, cb, cc;
            solve3(o, x - p[0], y - p[1], z - p[2], ca, cb, cc);
            if (o.kind == AEFDTD_OP_VECT_BLOCK) {
                if (ca >= 0 && ca <= 1.0 && cb >= 0 && cb <= 1.0 && cc >= 0 && cc <= 1.0) return o.mat;
                return -1;
            }
            const double alp = p[12];
            if (cb >= 0 && cb <= 1.0 && cc >= 0 && cc <= 1.0) {
                if (ca >= cc * alp && ca <= 1.0 - cc * (1.0 - alp)) return o.mat;
            }
            return -1;
        }
        case AEFDTD_OP_COATING: {  // Add_Coating::index (:55-95)
            if constexpr (D == 0) {
                atomicExch(a.err, 2);
                return -1;
            } else {
                const Ctx none{-1, -1};
                if (struct_index<D - 1>(a, x, y, z, o.stack, none) != o.origin) return -1;
                const double t2 = p[2] * p[2], delta = p[3];
                double px = x, py = y, pz = z;
                bool support = false;
                for (int i = 0;; ++i) {
                    double ex = px - x, ey = py - y, ez = pz - z;
                    if (!(ex * ex + ey * ey + ez * ez <= t2 && pz > 0)) break;
                    if (i > kMaxMarch) { atomicExch(a.err, 1); return -1; }
                    double s = i * delta;
                    px = x + s * o.dir[0];
                    py = y + s * o.dir[1];
                    pz = z + s * o.dir[2];
                    if (struct_index<D - 1>(a, px, py, pz, o.stack, none) != o.origin) {
                        support = true;
                        break;
                    }
                }
                if (!support) return -1;
                px = x; py = y; pz = z;
                for (int i = 0; pz <= a.l[2]; ++i) {
                    if (i > kMaxMarch) { atomicExch(a.err, 1); return -1; }
                    double s = i * delta;
                    px = x - s * o.dir[0];
                    py = y - s * o.dir[1];
                    pz = z - s * o.dir[2];
                    if (struct_index<D - 1>(a, px, py, pz, o.stack, none) != o.origin) return -1;
                }
                return o.mat;
            }
        }
        case AEFDTD_OP_CONF_COATING: {  // Add_Conf_Coating::index (:156-178)
            if constexpr (D == 0) {
                atomicExch(a.err, 2);
                return -1;
            } else {
                if (struct_index<D - 1>(a, x, y, z, o.stack, Ctx{-1, -1}) != o.origin) return -1;
                // the seed octree spans [0, lx] x [0, ly] x [0, lz]; outside it finds nothing
                if (!(x >= 0 && x <= a.l[0] && y >= 0 && y <= a.l[1] && z >= 0 && z <= a.l[2])) return -1;
                const double th = p[0], delta = p[1], t2 = th * th;
                // seeds of lattice point i lie at i*delta and one delta either side
                const int i0 = max(0, (int)floor((x - th) / delta) - 2), i1 = min(o.nl[0] - 1, (int)floor((x + th) / delta) + 2);
                const int j0 = max(0, (int)floor((y - th) / delta) - 2), j1 = min(o.nl[1] - 1, (int)floor((y + th) / delta) + 2);
                const int k0 = max(0, (int)floor((z - th) / delta) - 2), k1 = min(o.nl[2] - 1, (int)floor((z + th) / delta) + 2);
                for (int k = k0; k <= k1; k++)
                    for (int j = j0; j <= j1; j++)
                        for (int i = i0; i <= i1; i++) {
                            const unsigned m = a.lattice[o.lat_off + i + (long long)o.nl[0] * (j + (long long)o.nl[1] * k)];
                            if (!m) continue;
                            const double sx = i * delta, sy = j * delta, sz = k * delta;
                            for (int b = 0; b < 6; b++) {
                                if (!((m >> b) & 1u)) continue;
                                double qx = sx, qy = sy, qz = sz;
                                switch (b) {
                                    case 0: qx = sx - delta; break;
                                    case 1: qx = sx + delta; break;
                                    case 2: qy = sy - delta; break;
                                    case 3: qy = sy + delta; break;
                                    case 4: qz = sz - delta; break;
                                    default: qz = sz + delta; break;
                                }
                                double ex = x - qx, ey = y - qy, ez = z - qz;
                                if (ex * ex + ey * ey + ez * ez < t2) return o.mat;
                            }
                        }
                return -1;
            }
        }
        case AEFDTD_OP_MESH: {  // Add_Mesh::index (:428-440)
            if (x < o.vmin[0] || x > o.vmax[0] || y < o.vmin[1] || y > o.vmax[1] || z < o.vmin[2] || z > o.vmax[2])
                return -1;
            // The reference casts one ray in a random direction (Vector3::rand_sph); the crossing
            // parity does not depend on it away from rays through edges and vertices. Here the
            // direction is a hash of the point, uniform on the sphere.
            unsigned long long h = __double_as_longlong(x) * 0x9E3779B97F4A7C15ull;
            h ^= __double_as_longlong(y) + 0x632BE59BD9B4E019ull + (h << 6) + (h >> 2);
            h ^= __double_as_longlong(z) + 0x85EBCA77C2B2AE63ull + (h << 6) + (h >> 2);
            h ^= h >> 33; h *= 0xFF51AFD7ED558CCDull; h ^= h >> 33; h *= 0xC4CEB9FE1A85EC53ull; h ^= h >> 33;
            const double u1 = (double)(h >> 11) * (1.0 / 9007199254740992.0);
            const double u2 = (double)((h * 0x2545F4914F6CDD1Dull) >> 11) * (1.0 / 9007199254740992.0);
            const double dz = 1.0 - 2.0 * u1, rr = sqrt(fmax(0.0, 1.0 - dz * dz));
            double sphi, cphi;
            sincos(2.0 * kPi * u2, &sphi, &cphi);
            const double dxr = rr * cphi, dyr = rr * sphi;
            int n = 0;
            const double *t = a.tris + o.tri_off;
            for (int f = 0; f < o.n_tri; f++, t += 9) {
                // ray_N_inter (ray_intersect.h:121-166): T = O - V1, P = D x E2, Q = T x E1
                const double e1x = t[3], e1y = t[4], e1z = t[5], e2x = t[6], e2y = t[7], e2z = t[8];
                const double tx = x - t[0], ty = y - t[1], tz = z - t[2];
                const double px = dyr * e2z - dz * e2y, py = dz * e2x - dxr * e2z, pz = dxr * e2y - dyr * e2x;
                const double qx = ty * e1z - tz * e1y, qy = tz * e1x - tx * e1z, qz = tx * e1y - ty * e1x;
                const double det = px * e1x + py * e1y + pz * e1z;
                const double invdet = 1.0 / det;
                const double u = (px * tx + py * ty + pz * tz) * invdet;
                if (u >= 0 && u <= 1.0) {
                    const double v = (qx * dxr + qy * dyr + qz * dz) * invdet;
                    if (v >= 0 && u + v <= 1.0) {
                        if ((qx * e2x + qy * e2y + qz * e2z) * invdet >= 0) n += 1;
                    }
                }
            }
            return (n % 2 != 0) ? o.mat : -1;
        }
    }
    return -1;
}

template <int D>
__device__ __noinline__ int struct_index(const VoxArgs &a, double x, double y, double z, int restrict_level, Ctx c) {
    if (a.flip[0]) x = a.l[0] - x;
    if (a.flip[1]) y = a.l[1] - y;
    if (a.flip[2]) z = a.l[2] - z;
    if (a.per[0]) x = vmod(x, a.l[0], a);
    if (a.per[1]) y = vmod(y, a.l[1], a);
    if (a.per[2]) z = vmod(z, a.l[2], a);
    for (int l = restrict_level - 1; l >= 0; --l) {
        const VoxOp &o = a.ops[l];
        for (int ii = -a.per[0]; ii <= a.per[0]; ++ii)
            for (int jj = -a.per[1]; jj <= a.per[1]; ++jj)
                for (int kk = -a.per[2]; kk <= a.per[2]; ++kk) {
                    int hit = op_index<D>(a, o, x + ii * a.l[0], y + jj * a.l[1], z + kk * a.l[2], c, ii, jj);
                    if (hit != -1) return hit;
                }
    }
    return a.def;
}

__global__ void voxelize_kernel(VoxArgs a) {
    const long long n = (long long)a.nx * a.ny * a.nz;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(q % a.nx);
        const int j = (int)((q / a.nx) % a.ny);
        const int k = (int)(q / ((long long)a.nx * a.ny));
        a.out[q] = (uint32_t)struct_index<kVoxDepth>(a, i * a.dx, j * a.dy, k * a.dz, a.nops, Ctx{i, j});
    }
}

// Add_Conf_Coating::precompute (:181-248): lattice point (i, j, k) at
// (i*delta, j*delta, k*delta) of the origin material marks, one bit each, the
// six neighbours one delta away that are not of it (the seeds).
__global__ void conf_lattice_kernel(VoxArgs a, int q) {
    const VoxOp &o = a.ops[q];
    const double delta = o.p[1];
    const long long n = (long long)o.nl[0] * o.nl[1] * o.nl[2];
    uint8_t *lat = const_cast<uint8_t *>(a.lattice) + o.lat_off;
    const Ctx none{-1, -1};
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t % o.nl[0]);
        const int j = (int)((t / o.nl[0]) % o.nl[1]);
        const int k = (int)(t / ((long long)o.nl[0] * o.nl[1]));
        const double x = i * delta, y = j * delta, z = k * delta;
        unsigned m = 0;
        if (struct_index<kVoxDepth - 1>(a, x, y, z, q, none) == o.origin) {
            if (struct_index<kVoxDepth - 1>(a, x - delta, y, z, q, none) != o.origin) m |= 1u;
            if (struct_index<kVoxDepth - 1>(a, x + delta, y, z, q, none) != o.origin) m |= 2u;
            if (struct_index<kVoxDepth - 1>(a, x, y - delta, z, q, none) != o.origin) m |= 4u;
            if (struct_index<kVoxDepth - 1>(a, x, y + delta, z, q, none) != o.origin) m |= 8u;
            if (struct_index<kVoxDepth - 1>(a, x, y, z - delta, q, none) != o.origin) m |= 16u;
            if (struct_index<kVoxDepth - 1>(a, x, y, z + delta, q, none) != o.origin) m |= 32u;
        }
        lat[t] = (uint8_t)m;
    }
}

// Full-pivoting LU of a 3x3 matrix as Eigen's FullPivLU computes it (the first
// largest |a| of the remaining corner in column-major order is the pivot;
// multipliers stored below the diagonal), with its permutation index arrays
// and the rank that its solve uses (pivots above max|pivot| * 3 * DBL_EPSILON).
void full_piv_lu(VoxOp &o, const double m[3][3]) {
    double (&lu)[3][3] = o.lu;
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) lu[r][c] = m[r][c];
    int rowt[3] = {0, 1, 2}, colt[3] = {0, 1, 2}, nonzero = 3;
    double maxpivot = 0;
    for (int k = 0; k < 3; k++) {
        int br = k, bc = k;
        double big = std::fabs(lu[k][k]);
        for (int c = k; c < 3; c++)
            for (int r = k; r < 3; r++)
                if (std::fabs(lu[r][c]) > big) {
                    big = std::fabs(lu[r][c]);
                    br = r;
                    bc = c;
                }
        if (big == 0) {
            nonzero = k;
            break;
        }
        maxpivot = std::max(maxpivot, big);
        rowt[k] = br;
        colt[k] = bc;
        if (br != k)
            for (int c = 0; c < 3; c++) std::swap(lu[k][c], lu[br][c]);
        if (bc != k)
            for (int r = 0; r < 3; r++) std::swap(lu[r][k], lu[r][bc]);
        for (int r = k + 1; r < 3; r++) lu[r][k] = lu[r][k] / lu[k][k];
        for (int c = k + 1; c < 3; c++)
            for (int r = k + 1; r < 3; r++) lu[r][c] = lu[r][c] - lu[r][k] * lu[k][c];
    }
    const double thr = maxpivot * (2.220446049250313e-16 * 3.0);
    o.rank = 0;
    for (int i = 0; i < nonzero; i++) o.rank += std::fabs(lu[i][i]) > thr;
    for (int i = 0; i < 3; i++) o.pidx[i] = o.qidx[i] = i;
    for (int k = 2; k >= 0; k--) std::swap(o.pidx[k], o.pidx[rowt[k]]);
    for (int k = 0; k < 3; k++) std::swap(o.qidx[k], o.qidx[colt[k]]);
}

}  // namespace

cudaError_t launch_discretize(int nx, int ny, int nz, double dx, double dy, double dz, const aefdtd_structure_op *ops,
                              int nops, const aefdtd_structure_desc &d, uint32_t *d_out, int *d_err, cudaStream_t s) {
    if (nops > 256) return cudaErrorInvalidValue;
    std::vector<VoxOp> h(nops);
    std::vector<double> sintab, tris;
    long long lat_total = 0;
    const double L[3] = {d.lengths[0], d.lengths[1], d.lengths[2]};
    const int per[3] = {d.periodic[0] ? 1 : 0, d.periodic[1] ? 1 : 0, d.periodic[2] ? 1 : 0};
    const int flip[3] = {d.flip[0] ? 1 : 0, d.flip[1] ? 1 : 0, d.flip[2] ? 1 : 0};
    // top-level corner coordinates after flip and modulus, as struct_index computes them
    auto corner = [&](int axis, int i, double D) {
        double v = i * D;
        if (flip[axis]) v = L[axis] - v;
        if (per[axis]) {
            while (v < 0) v += L[axis];
            while (v >= L[axis]) v -= L[axis];
        }
        return v;
    };
    for (int q = 0; q < nops; q++) {
        VoxOp &o = h[q];
        o = VoxOp{};
        o.kind = ops[q].kind;
        o.mat = ops[q].mat_index;
        o.stack = q;
        for (int t = 0; t < 16; t++) o.p[t] = ops[q].p[t];
        if (o.kind == AEFDTD_OP_BLOCK) {
            // Add_Block ctor swaps reversed bounds (structure_primitives.cpp:24-32)
            for (int a = 0; a < 3; a++)
                if (o.p[2 * a] > o.p[2 * a + 1]) std::swap(o.p[2 * a], o.p[2 * a + 1]);
        }
        if (o.kind == AEFDTD_OP_CYLINDER || o.kind == AEFDTD_OP_CONE) {
            // base_vec = p2 - p1, length = |base_vec|, normalised (vector23.cpp:266-282)
            double vx = o.p[3] - o.p[0], vy = o.p[4] - o.p[1], vz = o.p[5] - o.p[2];
            double nrm = std::sqrt(vx * vx + vy * vy + vz * vz);
            o.length = nrm;
            o.bx = vx / nrm;
            o.by = vy / nrm;
            o.bz = vz / nrm;
        }
        if (o.kind == AEFDTD_OP_SIN_LAYER) {
            const double px = o.p[4], py = o.p[6];
            o.inv_px = px == 0 ? 0.0 : 1.0 / px;
            o.inv_py = py == 0 ? 0.0 : 1.0 / py;
            o.sin_off = (long long)sintab.size();
            for (int ii = -1; ii <= 1; ii++)
                for (int i = 0; i < nx; i++) {
                    double x = corner(0, i, dx) + ii * L[0];
                    sintab.push_back(std::sin(2.0 * kPi * (x * o.inv_px + o.p[5])));
                }
            for (int jj = -1; jj <= 1; jj++)
                for (int j = 0; j < ny; j++) {
                    double y = corner(1, j, dy) + jj * L[1];
                    sintab.push_back(std::sin(2.0 * kPi * (y * o.inv_py + o.p[7])));
                }
        }
        if (o.kind == AEFDTD_OP_VECT_BLOCK || o.kind == AEFDTD_OP_VECT_TRI) {
            // Add_Vect_Block ctor (:505-540): edge matrix columns A, B, C; box of the eight corners
            const double *p = o.p;
            double m[3][3] = {{p[3], p[6], p[9]}, {p[4], p[7], p[10]}, {p[5], p[8], p[11]}};
            full_piv_lu(o, m);
            for (int a = 0; a < 3; a++) {
                const double O = p[a], A = p[3 + a], B = p[6 + a], C = p[9 + a];
                const double v[8] = {O, A + O, B + O, C + O, (O + A) + B, (O + A) + C, (O + B) + C, ((O + A) + B) + C};
                o.vmin[a] = *std::min_element(v, v + 8);
                o.vmax[a] = *std::max_element(v, v + 8);
            }
        }
        if (o.kind == AEFDTD_OP_COATING) {
            // Add_Coating ctor (:45-53): angles in degrees through AngleRad (val * (Pi/180))
            const double theta = o.p[0] * (kPi / 180.0), phi = o.p[1] * (kPi / 180.0);
            o.dir[0] = std::cos(phi) * std::sin(theta);
            o.dir[1] = std::sin(phi) * std::sin(theta);
            o.dir[2] = -std::cos(theta);
            o.origin = (int)o.p[4];
        }
        if (o.kind == AEFDTD_OP_CONF_COATING) {
            if (o.p[1] <= 0) o.p[1] = 5e-9;  // Add_Conf_Coating ctor
            o.origin = (int)o.p[2];
            for (int a = 0; a < 3; a++) o.nl[a] = std::max(0, static_cast<int>(L[a] / o.p[1]));
            o.lat_off = lat_total;
            lat_total += (long long)o.nl[0] * o.nl[1] * o.nl[2];
        }
        if (o.kind == AEFDTD_OP_MESH) {
            // Add_Mesh ctor (:396-425): vertices scaled in place; the box starts from the first
            // vertex before scaling, as the reference's does
            const aefdtd_mesh &m = d.meshes[(int)o.p[4]];
            const double sc = o.p[3];
            for (int a = 0; a < 3; a++) o.vmin[a] = o.vmax[a] = m.vertices[a];
            std::vector<double> v(3 * (size_t)m.n_vertices);
            for (int i = 0; i < m.n_vertices; i++)
                for (int a = 0; a < 3; a++) {
                    v[3 * i + a] = m.vertices[3 * i + a] * sc;
                    o.vmin[a] = std::min(o.vmin[a], v[3 * i + a]);
                    o.vmax[a] = std::max(o.vmax[a], v[3 * i + a]);
                }
            o.tri_off = (long long)tris.size();
            o.n_tri = m.n_faces;
            for (int f = 0; f < m.n_faces; f++) {
                const double *v1 = &v[3 * (size_t)m.faces[3 * f]], *v2 = &v[3 * (size_t)m.faces[3 * f + 1]],
                             *v3 = &v[3 * (size_t)m.faces[3 * f + 2]];
                for (int a = 0; a < 3; a++) tris.push_back(v1[a]);
                for (int a = 0; a < 3; a++) tris.push_back(v2[a] - v1[a]);
                for (int a = 0; a < 3; a++) tris.push_back(v3[a] - v1[a]);
            }
        }
    }
    VoxOp *d_ops = nullptr;
    double *d_sin = nullptr, *d_tri = nullptr;
    uint8_t *d_lat = nullptr;
    cudaError_t e = cudaSuccess;
    auto release = [&] {
        if (d_ops) cudaFreeAsync(d_ops, s);
        if (d_sin) cudaFreeAsync(d_sin, s);
        if (d_tri) cudaFreeAsync(d_tri, s);
        if (d_lat) cudaFreeAsync(d_lat, s);
    };
    if (nops > 0) {
        e = cudaMallocAsync((void **)&d_ops, sizeof(VoxOp) * nops, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(d_ops, h.data(), sizeof(VoxOp) * nops, cudaMemcpyHostToDevice, s);
    }
    if (e == cudaSuccess && !sintab.empty()) {
        e = cudaMallocAsync((void **)&d_sin, sizeof(double) * sintab.size(), s);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(d_sin, sintab.data(), sizeof(double) * sintab.size(), cudaMemcpyHostToDevice, s);
    }
    if (e == cudaSuccess && !tris.empty()) {
        e = cudaMallocAsync((void **)&d_tri, sizeof(double) * tris.size(), s);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(d_tri, tris.data(), sizeof(double) * tris.size(), cudaMemcpyHostToDevice, s);
    }
    if (e == cudaSuccess && lat_total > 0) e = cudaMallocAsync((void **)&d_lat, (size_t)lat_total, s);
    if (e != cudaSuccess) {
        release();
        return e;
    }
    VoxArgs a{};
    a.nx = nx; a.ny = ny; a.nz = nz; a.nops = nops; a.def = d.default_material;
    for (int t = 0; t < 3; t++) {
        a.per[t] = per[t];
        a.flip[t] = flip[t];
        a.l[t] = L[t];
    }
    a.dx = dx; a.dy = dy; a.dz = dz;
    a.ops = d_ops;
    a.lattice = d_lat;
    a.sintab = d_sin;
    a.tris = d_tri;
    a.out = d_out;
    a.err = d_err;
    // conformal-coating seed lattices, lowest operation first: each depends on the ones below it
    for (int q = 0; q < nops && e == cudaSuccess; q++) {
        if (h[q].kind != AEFDTD_OP_CONF_COATING) continue;
        long long n = (long long)h[q].nl[0] * h[q].nl[1] * h[q].nl[2];
        if (n == 0) continue;
        int blocks = (int)std::min<long long>((n + 127) / 128, 148LL * 16);
        conf_lattice_kernel<<<blocks, 128, 0, s>>>(a, q);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        long long n = (long long)nx * ny * nz;
        int blocks = (int)std::min<long long>((n + 127) / 128, 148LL * 32);
        if (blocks < 1) blocks = 1;
        voxelize_kernel<<<blocks, 128, 0, s>>>(a);
        e = cudaGetLastError();
    }
    release();
    return e;
}

}  // namespace aefdtd
