// aefdtd_dev.hpp — data layouts shared by the host runtime and the kernels.
//
// HBM layout of one simulation (total grid Nx x Ny x Nz, x fastest, the
// reference Grid3 order, src/common/grid.h:862-868):
//   Ex Ey Ez Hx Hy Hz    : Nx*Ny*Nz reals each (FP64 or FP32)
//   mat                  : Nx*Ny*Nz material ids (uint8, or uint16 above 256 materials)
//   CPML psi             : slab-compact arrays as in FDTD::allocate_pml
//                          (src/finite_differences/FDTD/core/fdtd_pml.cpp:26-86):
//                          x: (pml_xm+pml_xp) x Ny x Nz, y: Nx x (pml_ym+pml_yp) x Nz,
//                          z: Nx x Ny x (pml_zm+pml_zp); 4 arrays per axis
//   dispersive psi       : per dispersive material, its bounding box x 3*Np complex
//                          values, component-major (like FDTD_Material::m_Psi_c,
//                          src/finite_differences/FDTD/core/mats.cpp:394-496)
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda.h>
#include <vector_types.h>

namespace aefdtd {

constexpr int kMaxPoles = 16;  // 4 terms x 4 model families

template <typename T> struct Cplx { T re, im; };

// Per-material update coefficients: FDTD_Material C1, C2x, C2y, C2z, C3, C4
// (src/finite_differences/FDTD/core/fdtd_material.h:46).
template <typename T> struct MatCoef {
    T C1, C2x, C2y, C2z, C3, C4;
};

// Dispersive (recursive-convolution) material record, one per material id.
// np == 0 for constant materials.
struct DispInfo {
    int np;
    int pole_off;            // first pole in the pole tables
    int x1, y1, z1, xs, ys, zs;
    long long psi_off;       // complex-element offset of this material's psi block
    long long box;           // xs*ys*zs
};

// Per-step scalars of the excitation and sensors, computed on the host in
// FP64 and read by the kernels from a device table, so that a captured
// sequence of steps replays with new values.
struct StepScalars {
    double inj_eA, inj_eB;   // E plane injection: subtracted from Ex / added to Ey
    double inj_hA, inj_hB;   // H plane injection: added to Hx / subtracted from Hy
    double src[4];           // oscillator values
    double tb, taper;        // plane-sum sample time (t + 1/2) Dt and tapering
    int step;                // global step index
    int snap;                // FT-mode completion: ring snapshot slot after this step (-1: none)
};

// Parameters of one fused half-step launch. Pointers are device pointers.
template <typename T, typename Tid> struct StepArgs {
    int Nx, Ny, Nz;
    long long NxNy;
    T *Ex, *Ey, *Ez, *Hx, *Hy, *Hz;
    const Tid *mat;                 // pitched: (mpitch x Ny x Nz)
    int mpitch;                     // material-id row pitch, elements (multiple of 16 bytes)
    const MatCoef<T> *coef;
    int nmat;                       // entries in coef / disp
    const DispInfo *disp;           // nullptr when no material is dispersive
    const Cplx<T> *crec;            // FP64: Crec; FP32: Crec - 1
    const Cplx<T> *dchi;
    Cplx<T> *psi;
    // CPML (fdtd_pml.cpp): thicknesses and per-index coefficient tables
    int pml_xm, pml_xp, pml_ym, pml_yp, pml_zm, pml_zp;
    bool px, py, pz;                // axis has any PML
    const T *ikx, *iky, *ikz;       // 1/kappa for the Yee update (reference selection rules)
    const T *bx, *by, *bz;          // FP64: b; FP32: b - 1
    const T *cx, *cy, *cz;          // c / D
    T *psi_x0, *psi_x1;             // E: PsiEyx, PsiEzx  H: PsiHyx, PsiHzx
    T *psi_y0, *psi_y1;             // E: PsiExy, PsiEzy  H: PsiHxy, PsiHzy
    T *psi_z0, *psi_z1;             // E: PsiExz, PsiEyz  H: PsiHxz, PsiHyz
    // H-side constants
    T dtdmx, dtdmy, dtdmz, dtm;
    // plane injection (normal mode): subtract/add on plane kinj, or kinj < 0
    int kinj;
    // box sources (custom mode, E only): up to 4 boxes
    int nsrc;
    int src_box[4][6];
    int src_comp[4];
    // this step's scalars: sc[q] (injection values, oscillator values)
    const StepScalars *sc;
    int q;
    int kchunk;                     // z planes per thread
    int prefetch;                   // prefetch the item's planes into L2 at start: bit 0 interior, bit 1 CPML kernels
    int *err;                       // device error flag (bounded waits)
    // oblique driver: two grids hold the real and imaginary parts of a
    // Bloch-periodic field; their wrap cells run in the general kernels
    int bloch;                      // 0: periodic wraps; 1: this is the real grid; 2: the imaginary grid
    const T *oEx, *oEy, *oEz, *oHx, *oHy, *oHz;   // the other grid's fields
    double bxr, bxi, byr, byi;      // Bloch phase of the x and y wraps (E side e^{-ikL}, H side e^{+ikL})
    int kobl;                       // Bloch_Wideband injection plane (-1: none)
    double obl_coef;                // E side: C2z of the injection plane's material; H side: dtdmz
    const double2 *obl_px, *obl_py; // per-column phases at the x- and y-staggered points
    const double *obl_inc;          // per-step incident sums [step][14] (E side 0..3, H side 4..7)
};

// One fused time step (leapfrog.cuh): the E and the H half-step in one pass,
// reading the old fields and E-side state and writing new ones (ping-pong).
template <typename T, typename Tid> struct FusedArgs {
    StepArgs<T, Tid> e;      // E side: old fields (all six), E tables, old E-side CPML psi, old RC psi
    StepArgs<T, Tid> h;      // H side: H tables and H-side CPML psi (updated in place)
    T *nEx, *nEy, *nEz, *nHx, *nHy, *nHz;          // new fields
    T *npx0, *npx1, *npy0, *npy1, *npz0, *npz1;    // new E-side CPML psi
    Cplx<T> *npsi;                                 // new RC psi
};
constexpr int kFusedTileX = 64;   // columns per fused tile (32 lanes x 2)
constexpr int kFusedMaxTY = 8;    // owned rows per fused tile (warps), plus one recomputed row
// Fused item groups, numbered like the split groups below (the timing slots
// are shared): curl only, z-CPML planes, dispersive cells only, every phase,
// x/y (and z) CPML.
enum { kFusedInterior = 0, kFusedPmlZ = 1, kFusedDisp = 2, kFusedAll = 3, kFusedPmlXY = 4, kFusedGroups = 5 };

// Item groups of one half-step: a device array of int4 items (x0, y0, k0,
// k1) sorted by group; group g is items [off[g], off[g] + n[g]).
enum { kGroupInterior = 0, kGroupPmlZ = 1, kGroupDisp = 2, kGroupAll = 3, kGroupPmlXY = 4, kGroups = 5 };
// Staged interior half-steps (interior_tma.cuh): tiles of 64 x 8 columns
// whose planes are brought into a shared-memory ring by tensor copies.
constexpr int kTmaTileX = 64;
constexpr int kTmaTileY = 8;
// Tensor maps of one half-step's staged kernel over this simulation's own
// field arrays (3-D, x y z in elements; s = element size).
struct TmaMaps {
    CUtensorMap w[2];   // x-halo blocks {64 + 16/s, 8, 1}: E side Hz, Hy; H side Ez, Ey
    CUtensorMap c[2];   // periodic-wrap columns {16/s, 8, 1} of the same two arrays
    CUtensorMap r[2];   // y-halo rows {64, 1, 1}: E side Hz, Hx; H side Ez, Ex
    CUtensorMap b[4];   // own blocks {64, 8, 1}: E side Hx, Ex, Ey, Ez; H side Ex, Hx, Hy, Hz
    CUtensorMap mat;    // own block of material ids (E side)
};
// One half-step's staged launch: units (x0, y0, k0, k1) taken by the CTAs
// in turn through a device counter.
struct TmaPlan {
    TmaMaps maps;
    const int4 *units;
    int nunits;
    int *ctr;           // [0] next unit, [1] CTAs done (the last CTA resets both)
    int grid;           // CTAs per launch
    int stages;         // ring stages (4 or 6)
    long long cells;    // cells per launch
    long long wait_cycles;   // bound of each mbarrier wait
    int withhold;            // test hook: the producer issues no copy and arrives on no stage
};
struct WorkSplit {
    int off[kGroups];
    int n[kGroups];
    int unroll;                     // z-planes per iteration of the interior kernels (1 or 2)
    int tile_y;                     // tile height: CTAs of 32 x tile_y threads (2, 4 or 8)
    unsigned pair_mask;             // bit g: group g runs the two-cells-per-thread kernels on 64-column items
                                    // (x/y-CPML group: its y-only items, n_py of them at the group's end)
    int n_py = 0;                   // x/y-CPML group: trailing items without x-CPML cells, on the pair kernel
    const TmaPlan *tma = nullptr;   // set: the interior group is the staged kernel over these units
};
// Kernel launches of one half-step's groups (the x/y-CPML group launches
// two kernels when it holds both kinds of item).
inline int group_kernels(const WorkSplit &w) {
    int c = 0;
    for (int g = 0; g < kGroups; g++) c += w.n[g] > 0;
    return c + (w.n_py > 0 && w.n[kGroupPmlXY] > w.n_py);
}
// x0 flag of a 32-column item in a group of 64-column (pair) items
constexpr int kHalfItem = 1 << 30;

// ---- persistent batch kernel (batch_persist.cuh)
// A unit: a band of tile rows (every x tile) of one member times one z-chunk
// of its work items. Its items for each half-step, the units it waits on,
// and the plane-sum planes it holds.
struct PsUnit {
    int m;              // member (index into the argument arrays)
    int e_off, e_n;     // E items [e_off, e_off + e_n)
    int h_off, h_n;     // H items
    int nb[4];          // waited on: before E the y-1 and z-1 units, before H the y+1 and z+1 units
    int band, j0, j1;   // plane-sum band: rows [j0, j1)
    int planes;         // bit 0: the band's reflection plane kr is in this unit; bit 1: the transmission plane kt
};
template <typename T> struct SensorStepArgs;
template <typename T, typename Tid> struct PersistArgs {
    const StepArgs<T, Tid> *ea, *ha;   // per member
    const SensorStepArgs<T> *sa;       // per member: nbp = bands, partial [steps][bands][12]
    const PsUnit *units;
    const int4 *items;                 // (x0, y0, k0 | k1 << 16, group)
    int nunits, steps;
    int *prog;                         // per unit: half-steps finished in this launch (zero at launch)
    int *flags;                        // [0]: device error flag (1: a wait ran out), [1]: abort
    long long wait_cycles;             // bound of each wait
    int withhold;                      // test hook: unit 0 never reports its progress
};

// ---- sensor-path launch arguments (kernels in sensors.cuh)

struct PulseDev {
    double k, omega, kx, ky, kz, n_ind, dz, C1;
    double Ex0, Ey0, Ez0;
};

struct GatherDesc {
    int type;                // 0/1: x-normal, 2/3: y-normal, 4/5: z-normal
    int x1, y1, z1, span1, span2, P;
    int block0, nblocks;     // blocks of the fused launch serving this sensor
    void *S;                 // sample slot of this step: [6][P] of T
};

constexpr int kMaxGather = 8;

// One launch per step: normal-incidence plane-sum partials (blocks
// [0, nbp)) and the interpolated samples of every DFT plane (the rest).
template <typename T> struct SensorStepArgs {
    int Nx, Ny, Nz;
    long long NxNy;
    const T *Ex, *Ey, *Ez, *Hx, *Hy, *Hz;
    int nbp;                 // plane-sum blocks (0 outside normal mode)
    int kr, kt;              // zs_e-2, zs_s
    double Dx, Dy, Dz;
    PulseDev P;
    const StepScalars *sc;
    int q;
    double *partial;         // [nbp][12] of this step
    int ng;
    GatherDesc g[kMaxGather];
    int part;                // 0: plane sums + E gathers (reads E only); 1: H gathers (reads H only)
    double *out;             // batch: plane-sum history [Nt][12]
};

// Single-wavelength field sensors (s_fieldmap.cpp): one launch per sensor
// part of a step over every map of that part. Part 0 reads E (E plane maps,
// the E half of blocks, points) beside H; part 1 reads H (H plane maps, the
// H half of blocks) beside the next E.
struct MapDesc {
    int kind;                // AEFDTD_MAP_PLANE / BLOCK / POINT
    int type;                // plane maps: 0 x-, 1 y-, 2 z-normal
    int x1, y1, z1;          // first cell, total grid
    int span1, span2, span3; // plane: map span1 x span2, span3 planes summed (1 unless cumulative); block: x, y, z
    int mag;                 // plane maps: H components
    int P;                   // threads' cells: span1*span2 (plane), span1*span2*span3 (block), 1 (point)
    int block0, nblocks;     // blocks of the launch serving this map
    int slot;                // this map's entry in the coefficient table rows
    int cap, step0;          // points: history rows, and the step of row 0
    double *acc;             // plane/block: complex [components][span3 x span2 x span1]; point: [cap][3]
};

constexpr int kMaxMaps = 8;
enum { kMapPlane = 0, kMapBlock = 1, kMapPoint = 2 };   // AEFDTD_MAP_* of aefdtd.h

template <typename T> struct MapStepArgs {
    int Nx, Ny, Nz;
    long long NxNy;
    const T *Ex, *Ey, *Ez, *Hx, *Hy, *Hz;
    const double *coef;      // this segment's phases: [step q][kMaxMaps][E re, E im, H re, H im]
    const StepScalars *sc;   // per-step scalars (global step index)
    int q, part, nm;
    MapDesc m[kMaxMaps];
};

// R/T sums of the oblique driver (oblique_biphase.cpp:300-327): per step, the
// complex sums over the plane of incident (BR), reflected-plane (R, z =
// zs_e+2) and transmitted-plane (T, z = zs_s) E times e^{-i k.r}.
template <typename T> struct OblSumArgs {
    int Nx, Ny;
    long long NxNy;
    const T *Ex, *Ey, *Ez;          // the real grid
    int kr, kt;                     // zs_e + 2, zs_s
    const double2 *mk;              // [3][Nx*Ny] mk_x, mk_y, mk_z
    const double2 *ph;              // [3][Nx*Ny] phases of the incident field at the Ex, Ey, Ez points
    const double *inc;              // per-step incident sums [step][14] (8..13: E at zs_s)
    const StepScalars *sc;
    int q;
    double *partial;                // [blocks][18] of this step
};

// Per-step sums of the wideband Bloch source (Bloch_Wideband::inject_E,
// inject_H and get_E, sc_bloch.cpp:43-83, 216-285) for steps t0 .. t0+n-1:
// out[t][0..3] H_x, H_y at (z2 - 1/2, t - 1/2), [4..7] E_x, E_y at (z2, t),
// [8..13] E_x, E_y, E_z at zs_s, time (t + 1/2) Dt, as complex (re, im).
struct OblIncArgs {
    int nl;                  // spectral lines
    const double *w, *kz;    // [nl]
    const double *eb;        // [nl][3] E_base
    const double *hb;        // [nl][2] H_base x, y
    double Dt, Dz;
    int z2, zs_s, t_offset;
    int t0, n;
    double *out;             // [t0 + n][14]
};

// Completion sensor, FT mode (CompletionSensor::deep_feed, s_completion.cpp:
// 137-160): per probe, acc += local E x e^{i w step Dt}, then the running sums
// into slot step % n_avg of the ring [Ex re, Ey re, Ez re, Ex im, Ey im, Ez im][np][n_avg].
template <typename T> struct CcFtArgs {
    int Nx, Ny, Nz;
    long long NxNy;
    const T *Ex, *Ey, *Ez;
    int np, n_avg, step0;
    const int *pts;                 // [np][3] probe cells
    const double2 *coef;            // this segment's phases [q][np]
    const StepScalars *sc;
    int q;
    double2 *acc;                   // [np][3]
    double *ring;
    double *snap;                   // ring snapshots [slot][6][np][n_avg] (batch members), or null
};

struct PhasorArgs {
    int nk, nl, Nt, Ntap;
    const int *step_ptr;     // step of buffer slot 0 = (*step_ptr if set) + step_add
    int step_add;
    double Dt;
    const double *w;         // angular frequencies, nl
    double2 *WE, *WH;        // [nk][nl]
};

template <typename T> struct AccumArgs {
    int P, nl, nk;
    const T *S;              // [K][6][P]
    const double2 *WE, *WH;  // [nk][nl]
    double2 *acc;            // [6][nl][P]
    int mma;                 // 1: the FP64 tensor-path kernel (dft_accumulate_mma), 0: FMA kernel
};

struct FluxArgs {
    int P, nl, type;
    double area_factor;      // Dy*Dz, Dx*Dz or Dx*Dy
    const double2 *acc;      // [6][nl][P]
    double *out;             // nl
};

// Tensor-core DFT (dft_tc.cu). B image: per tile [E hi, E lo, H hi, H lo] of
// R x K floats in the K-major core-matrix layout, tiles tile_stride apart.
struct DftTcPhasorArgs {
    int K, nk, nl, N0, N1, Nt, Ntap;
    const int *step_ptr;
    int step_add;
    double Dt;
    const double *w;
    float *B;
    size_t tile_stride;
};
struct DftTcArgs {
    int K, nk, nl, P, N0, N1;
    const float *S;          // [K][6][P]
    const float *B;
    size_t tile_stride;
    double2 *acc;            // [6][nl][P]
    int *err;
    long long wait_cycles;   // bound of each mbarrier wait (SM cycles)
    int withhold_copy;       // test hook: 1 = issue no phasor copy, so the first wait runs out
};
constexpr int kDftTcMaxK = 64;
constexpr int kDftTcThreads = 512;   // 16 warps: 4 per TMEM lane quarter
constexpr int kDftTcSmem = (128 * kDftTcMaxK * 2 + 256 * kDftTcMaxK * 2) * 4 + 64;

constexpr int kPlaneBlocks = 64;    // plane-sum stage-1 blocks
constexpr int kPlaneThreads = 256;

}  // namespace aefdtd
