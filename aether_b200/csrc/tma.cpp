// tma.cpp — tensor maps of the staged interior half-steps (interior_tma.cuh).
//
// One 3-D map (x, y, z in elements) per array and box shape, over this
// simulation's own field and material-id arrays. The encoder is the driver's
// cuTensorMapEncodeTiled, reached through the runtime's entry-point query so
// that the library needs no link against the driver library. Maps use no
// swizzle, no interleave and zero fill outside the array; no map is ever used
// with a multicast copy.
#include <cudaTypedefs.h>

#include <cstring>

#include "sim.hpp"

using namespace aefdtd;

namespace {

PFN_cuTensorMapEncodeTiled_v12000 encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        else
            cudaGetLastError();
    }
    return fn;
}

// map over an (nx x ny x nz) array with row pitch `pitch` elements, box (bx, by, 1)
bool encode(CUtensorMap *m, CUtensorMapDataType dt, int esize, const void *base, int nx, int ny, int nz, int pitch,
            int bx, int by) {
    PFN_cuTensorMapEncodeTiled_v12000 fn = encoder();
    if (!fn) return false;
    const cuuint64_t dims[3] = {(cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)nz};
    const cuuint64_t strides[2] = {(cuuint64_t)pitch * esize, (cuuint64_t)pitch * esize * ny};
    const cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, 1};
    const cuuint32_t es[3] = {1, 1, 1};
    std::memset(m, 0, sizeof(*m));
    return fn(m, dt, 3, const_cast<void *>(base), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
              CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace

bool aefdtd_sim::tma_possible() const {
    const int es = fp64 ? 8 : 4;
    return use_tma && tma_allowed && !obl && Nx >= kTmaTileX && Ny >= kTmaTileY && (size_t(Nx) * es) % 16 == 0 &&
           kTmaTileY % tile_y == 0 && kTmaTileX == 2 * kTileXHost;
}

bool aefdtd_sim::tma_maps_current() const {
    for (int c = 0; c < 6; c++)
        if (tma_ptrs[c] != F[c].p) return false;
    return tma_ptrs[6] == mat.p;
}

bool aefdtd_sim::build_tma_maps() {
    const int es = fp64 ? 8 : 4, hx = 16 / es;
    const CUtensorMapDataType dt = fp64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    const CUtensorMapDataType di = id_bytes == 1 ? CU_TENSOR_MAP_DATA_TYPE_UINT8 : CU_TENSOR_MAP_DATA_TYPE_UINT16;
    for (int c = 0; c < 6; c++)
        if (!F[c].p || (reinterpret_cast<uintptr_t>(F[c].p) & 15)) return false;
    if (!mat.p || (reinterpret_cast<uintptr_t>(mat.p) & 15) || (size_t(mpitch) * id_bytes) % 16) return false;
    const int X = kTmaTileX, Y = kTmaTileY;
    auto fld = [&](CUtensorMap *m, int c, int bx, int by) { return encode(m, dt, es, F[c].p, Nx, Ny, Nz, Nx, bx, by); };
    bool ok = true;
    // E side: w = Hz, Hy; c = Hz, Hy; r = Hz, Hx; b = Hx, Ex, Ey, Ez; mat
    TmaMaps &e = tma_plan[0].maps;
    ok = ok && fld(&e.w[0], 5, X + hx, Y) && fld(&e.w[1], 4, X + hx, Y);
    ok = ok && fld(&e.c[0], 5, hx, Y) && fld(&e.c[1], 4, hx, Y);
    ok = ok && fld(&e.r[0], 5, X, 1) && fld(&e.r[1], 3, X, 1);
    ok = ok && fld(&e.b[0], 3, X, Y) && fld(&e.b[1], 0, X, Y) && fld(&e.b[2], 1, X, Y) && fld(&e.b[3], 2, X, Y);
    ok = ok && encode(&e.mat, di, id_bytes, mat.p, Nx, Ny, Nz, mpitch, X, Y);
    // H side: w = Ez, Ey; c = Ez, Ey; r = Ez, Ex; b = Ex, Hx, Hy, Hz (no ids)
    TmaMaps &h = tma_plan[1].maps;
    ok = ok && fld(&h.w[0], 2, X + hx, Y) && fld(&h.w[1], 1, X + hx, Y);
    ok = ok && fld(&h.c[0], 2, hx, Y) && fld(&h.c[1], 1, hx, Y);
    ok = ok && fld(&h.r[0], 2, X, 1) && fld(&h.r[1], 0, X, 1);
    ok = ok && fld(&h.b[0], 0, X, Y) && fld(&h.b[1], 3, X, Y) && fld(&h.b[2], 4, X, Y) && fld(&h.b[3], 5, X, Y);
    h.mat = e.mat;
    if (!ok) return false;
    for (int c = 0; c < 6; c++) tma_ptrs[c] = F[c].p;
    tma_ptrs[6] = mat.p;
    return true;
}
