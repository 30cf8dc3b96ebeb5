// sim.hpp — private: the host-side state of one simulation (struct
// aefdtd_sim) and the runtime helpers shared by runtime.cpp (single
// simulations and the C ABI) and batch.cpp (batched stepping).
#pragma once

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numbers>
#include <string>
#include <array>
#include <map>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/aefdtd.h"
#include "kernels.hpp"

namespace aefdtd {
constexpr int kTileXHost = 32, kTileYHost = 4;   // kTileX, kTileY of yee.cuh
// whether simulations take the fused time step unless AEFDTD_FUSED says otherwise
constexpr bool kFusedDefault = false;
}

namespace aefdtd {

// f(0) .. f(n-1) on up to hardware_concurrency host threads (static blocks);
// f must only write state of its own index.
template <typename F> void parallel_for(int n, F &&f) {
    const int nt = std::max(1, std::min<int>(n, std::min(32u, std::max(1u, std::thread::hardware_concurrency()))));
    if (nt <= 1 || n < 8) {
        for (int i = 0; i < n; i++) f(i);
        return;
    }
    std::vector<std::thread> th;
    for (int w = 0; w < nt; w++)
        th.emplace_back([&, w] {
            for (int i = w * n / nt; i < (w + 1) * n / nt; i++) f(i);
        });
    for (auto &x : th) x.join();
}

// Hands a graph executable to a background thread that destroys it: with a
// few thousand nodes each destroy takes ~20 ms, which would otherwise land in
// aefdtd_destroy and in work-list rebuilds. In-flight graphs are freed by the
// driver on completion, as for a direct destroy.
void reap_graph(cudaGraphExec_t g, int device);

cudaError_t launch_discretize(int nx, int ny, int nz, double dx, double dy, double dz, const aefdtd_structure_op *ops,
                              int nops, const aefdtd_structure_desc &d, uint32_t *d_out, int *d_err, cudaStream_t s);

namespace phys {
// src/common/phys_constants.h:18-20
constexpr double e0 = 8.854187817e-12;
constexpr double mu0 = 12.566370614e-7;
constexpr double c_light = 299792458.0;
constexpr double Pi = std::numbers::pi_v<double>;
}  // namespace phys
using namespace phys;
typedef std::complex<double> cplx;

struct Error {
    aefdtd_status st;
    std::string msg;
};

#define AE_CUDA(call)                                                                        \
    do {                                                                                     \
        cudaError_t e__ = (call);                                                            \
        if (e__ != cudaSuccess)                                                              \
            throw Error{e__ == cudaErrorMemoryAllocation ? AEFDTD_OOM : AEFDTD_CUDA_ERROR,   \
                        std::string(#call) + ": " + cudaGetErrorString(e__)};                 \
    } while (0)

inline void fail(aefdtd_status st, const std::string &m) { throw Error{st, m}; }

// Device buffer with byte size bookkeeping.
struct DBuf {
    void *p = nullptr;
    size_t n = 0;
    void alloc(size_t bytes, size_t &total) {
        release(total);
        if (bytes == 0) return;
        AE_CUDA(cudaMalloc(&p, bytes));
        n = bytes;
        total += bytes;
    }
    void release(size_t &total) {
        if (p) { cudaFree(p); total -= n; }
        p = nullptr;
        n = 0;
    }
    template <typename T> T *as() const { return static_cast<T *>(p); }
};

// Per-material coefficients (FDTD_Material, fdtd_material.h:38-268).
struct HostMat {
    bool set = false, rc = false;
    int np = 0;
    double C1 = 1, C2x = 0, C2y = 0, C2z = 0, C3 = 0, C4 = 0, ei = 1, sig = 0;
    std::vector<cplx> crec, dchi, chi;
    int x1 = 0, x2 = -1, y1 = 0, y2 = -1, z1 = 0, z2 = -1;   // bounding box in the total grid
};

struct Pulse {
    // ChpIn (chpin.cpp:44-90, 479-545) at incidence 0, direction 0.
    double k, omega, kx, ky, kz, n_ind, dz, C1, Ex0, Ey0, Ez0, Hx0, Hy0, Hz0;
    void init(double li, double lf, double poli, double startz, double n_ind_i) {
        double wi = 2.0 * Pi * c_light / li, wf = 2.0 * Pi * c_light / lf;
        double w0 = (wi + wf) / 2.0;
        double lambda = 2.0 * Pi * c_light / w0;
        double dw = std::abs(0.5 * (wi - w0));
        n_ind = n_ind_i;
        double inc = 0 * Pi / 180.0, pol = poli * Pi / 180.0, dir = 0 * Pi / 180.0;
        dz = 2.0 * c_light / dw / n_ind;
        k = 2.0 * Pi / lambda * n_ind;
        omega = 2.0 * Pi * c_light / lambda;
        double incr = Pi / 2.0 - inc;
        double Ca = std::cos(incr), Sa = std::sin(incr), Cb = std::cos(dir), Sb = std::sin(dir);
        double Cc = std::cos(pol), Sc = std::sin(pol);
        kx = k * (Ca * Cb); ky = k * (Ca * Sb); kz = k * (-Sa);
        Ex0 = (Sa * Cb * Sc - Sb * Cc) * 1.0; Ey0 = (Sa * Sb * Sc + Cb * Cc) * 1.0; Ez0 = Ca * Sc * 1.0;
        double tmp = 1.0 / (c_light * mu0) * 1.0 * n_ind;
        Hx0 = tmp * (Sa * Cb * Cc + Sb * Sc); Hy0 = tmp * (Sa * Sb * Cc - Cb * Sc); Hz0 = tmp * (Ca * Cc);
        C1 = -1.0 / k * (kx * 0 + ky * 0 + kz * startz) + dz * std::sqrt(-std::log(1e-4));
    }
    double f(double A0, double x, double y, double z, double t) const {
        double p = kx * x + ky * y + kz * z;
        double a = p - omega * t;
        double b = (1.0 / k * p - c_light * t / n_ind + C1) / dz;
        return A0 * std::exp(-b * b) * std::cos(a);
    }
};

struct Osc {
    int comp, box[6], step = 0, tshift;
    double w0, dw;
};

struct PlaneSensor {
    aefdtd_sensor_desc d;
    int type, x1, x2, y1, y2, z1, z2, span1, span2, P, nl;
    std::vector<double> lambda, w;
    int step = 0;          // steps fed
    int nbuf = 0;          // filled slots of the sample buffer half being written
    int buf_step0 = 0;     // step of slot 0
    int half = 0;          // sample-buffer half the gathers write (S holds two halves of K steps)
    // a filled half whose DFT block is still to be accumulated: launched at the
    // start of the next segment beside its steps, or when results are read
    bool pending = false;
    int pend_half = 0, pend_n = 0, pend_step0 = 0;
    const StepScalars *pend_tbl = nullptr;   // step of slot 0 read from this table, else pend_step0
    DBuf S, acc, wdev, WE, WH, flux;
    DBuf Btc;              // tensor-core phasor image (FP32 path)
    int N0 = 0, N1 = 0;
};

// Completion sensor in FT mode (CompletionSensor, s_completion.cpp): probe
// cells and wavelengths, the transform ring on the device and its host copy.
struct CompletionFT {
    double lmin = 0, lmax = 0;
    int np = 0, n_avg = 1, step0 = 0;
    std::string layout;
    std::vector<int> pts;          // [np][3]
    std::vector<double> w;         // [np] angular frequencies
    std::vector<double> ring_host, rows;
    DBuf dpts, acc, ring, ctab;    // ctab: [2 slots][seg_len][np] complex phases
    DBuf snap;                     // batch members: ring snapshots at check steps
    int nsnap = 0;
    double open_ratio = 0;         // fraction of probes not settled at the last check
};

// Single-wavelength field sensor (FieldMap, FieldBlock, FieldPoint of
// s_fieldmap.cpp); dev.acc holds the device accumulators or point history.
struct FieldMapHost {
    aefdtd_fieldmap_desc d;
    MapDesc dev{};           // block0/nblocks/slot set per launch
    int ncomp = 3;
    double w = 0;            // 2 pi c / lambda
    int step0 = 0;           // tstep when added (points: step of history row 0)
    DBuf acc;
};

// Oblique driver state (FDTD_oblique_biphase_comp, oblique_biphase.cpp:29-330):
// the imaginary grid's fields and CPML / dispersive state, the wideband Bloch
// source (Bloch_Wideband, sc_bloch.cpp), phases and the R/T sum history.
struct Oblique {
    aefdtd_oblique_desc d{};
    double kx = 0, ky = 0, kxy = 0;     // k_in * n_sup
    double eps_sup = 1, eps_sub = 1, index_sup = 1, index_sub = 1;
    cplx dE_x, dE_y, dH_x, dH_y;        // Bloch phases of the wraps: e^{+-i k N D}
    // Bloch_Wideband (sc_bloch.cpp:85-214)
    int z2 = 0, t_offset = 0, nlines = 0;
    double eps_inf = 1, c2z = 0;
    std::vector<double> w, kz, eb, hb;  // eb: [l][3], hb: [l][2]
    DBuf dw, dkz, deb, dhb;
    DBuf Fi[6], psiEi[6], psiHi[6], psi_i;   // imaginary grid
    DBuf ph;                            // [3][Nx*Ny] complex e^{+i k.r} at the Ex, Ey, Ez points
    DBuf mk;                            // [3][Nx*Ny] complex mk_x, mk_y, mk_z = e^{-i k.r}
    DBuf inc;                           // [cap][14] per-step incident sums
    DBuf part, hist;                    // R/T sums: per-step block partials, [cap][18] history
    int cap = 0, nb = 0;
};

static inline double s_curve(double x, double xmin, double xmax) {
    // src/common/mathUT.cpp:1186-1193
    double u = (x - xmin) / (xmax - xmin);
    if (u <= 0) return 0;
    else if (u >= 1.0) return 1.0;
    else return u * u * (3.0 - 2.0 * u);
}

}  // namespace aefdtd

using namespace aefdtd;

struct aefdtd_sim {
    aefdtd_grid_desc g{};
    std::string last_error;
    bool fp64 = true;
    int device = 0;
    cudaStream_t stream = nullptr;
    // side streams for the boundary groups of a half-step, forked from and
    // joined back into `stream` by events (parallel branches in the graphs)
    cudaStream_t side[kGroups - 1] = {};
    cudaEvent_t ev_fork = nullptr, ev_join[kGroups - 1] = {};
    // side streams of the two sensor parts (part 0 beside H, part 1 beside the next E)
    cudaStream_t side_s[2] = {};
    cudaEvent_t ev_s_fork[2] = {}, ev_s_join[2] = {};
    bool concurrent_groups = true;
    template <typename Launch> void run_groups(const WorkSplit &w, Launch &&launch);
    size_t dev_bytes = 0;
    uint64_t launches = 0;

    // geometry (FDTD members)
    int Nx = 0, Ny = 0, Nz = 0, Nx_s = 0, Ny_s = 0, Nz_s = 0;
    int xs_s = 0, xs_e = 0, ys_s = 0, ys_e = 0, zs_s = 0, zs_e = 0;
    int pml[6] = {0}, pad[6] = {0};
    double Dx = 0, Dy = 0, Dz = 0, Dt = 0, dtm = 0, dtdez = 0, dtdmx = 0, dtdmy = 0, dtdmz = 0;
    double pml_kappa[6], pml_sigma[6], pml_alpha[6];
    double pml_m = 4, pml_ma = 2;
    int Nt = 0, Ntap = 0, dft_k = 64;
    int tstep = 0;

    // fields and state
    DBuf F[6], mat;
    int id_bytes = 1;
    int mpitch = 0;
    std::vector<uint32_t> map;      // total-grid material ids
    bool map_set = false;
    unsigned Nmat = 1;
    std::vector<HostMat> mats;
    bool tables_dirty = true;
    DBuf coef, disp, crec, dchi, psi;
    bool any_disp = false;
    // CPML
    DBuf ik[6], bE[3], cE[3], bH[3], cH[3];
    DBuf psiE[6], psiH[6];          // x0,x1,y0,y1,z0,z1
    // normal mode
    bool normal = false;
    aefdtd_normal_desc nd{};
    Pulse pulse{};
    double eps_sup = 1, eps_sub = 1, index_sup = 1, index_sub = 1;
    DBuf psums, psum_partial;
    int psums_cap = 0;
    std::vector<double> psums_host;
    // custom mode
    std::vector<Osc> oscs;
    std::vector<PlaneSensor *> sensors;
    std::vector<std::array<int, 6>> boxes;   // box sensors: planar sensor per face (-1: disabled)
    Oblique *obl = nullptr;                  // mode OBLIQUE after aefdtd_setup_oblique
    void obl_ensure(int steps);              // incident table and history for `steps` steps
    template <typename T> int launch_obl_sums(int q, const StepScalars *tbl, cudaStream_t st);
    void find_slab(int sub_ref, int sup_ref, double &hsub, double &hstruc, double &hsup) const;
    DBuf *grid_fields(int grid) { return grid && obl ? obl->Fi : F; }
    std::vector<FieldMapHost *> fmaps;       // single-wavelength field sensors
    DBuf fm_tbl;                             // their phases: [slot][seg_len][kMaxMaps][4] doubles
    std::vector<double> map_rows;            // host staging of one segment's phase rows
    void fill_map_phases(int t0, int L, double *rows) const;
    template <typename T> int launch_maps(int part, int q, const double *coef, const StepScalars *tbl, cudaStream_t st);
    // half-step work lists: (x0, y0, k0, k1) items of 32 x 4 columns x a
    // z-chunk, in one device array: the E groups, then the H groups
    bool work_dirty = true;
    int kchunk = 0;
    WorkSplit wsE{}, wsH{};
    DBuf items;
    std::vector<int> items_host;    // host copy of `items` (merged into batch work lists)
    void build_work();
    DBuf err;
    void check_err();
    // timing: one event quadruple per step of the last aefdtd_step call
    // (before E, after E, after H, after sensors), summed on query
    bool timing = false;
    int timing_mode = 1;            // 1: per phase (concurrent branches); 2: per work-item group, in order
    std::vector<cudaEvent_t> tge;   // group mode: [step][half][group][start, end]
    double t_grp[2][kGroups] = {};  // group mode: summed ms per half-step group
    long long grp_cells[2][kGroups] = {};   // cells each group updates per half-step
    std::vector<cudaEvent_t> tev;
    int tev_steps = 0;
    double t_e = 0, t_h = 0, t_s = 0;

    ~aefdtd_sim();
    void construct(const aefdtd_grid_desc *d);
    void set_device() const { cudaSetDevice(device); }
    void build_pml_tables();
    void set_map(const uint32_t *m, size_t count);
    void set_material(uint32_t idx, const aefdtd_material_desc *md);
    void finalize_tables();
    template <typename T, typename Tid> void fill_args(StepArgs<T, Tid> &a, bool e_side, int grid = 0);
    template <typename T, typename Tid> void run_steps(int n);
    template <typename T>
    void flush_block(PlaneSensor &s, int half, int n, const StepScalars *step0_ptr, int step0, cudaStream_t st);
    template <typename T> void launch_pending(PlaneSensor &s, cudaStream_t st);
    void drain_sensors();
    cudaStream_t side_f = nullptr;
    cudaEvent_t ev_f_fork = nullptr, ev_f_join = nullptr;
    template <typename T, typename Tid> void enqueue_segment(int L, StepScalars *tbl, bool record);
    template <typename T, typename Tid>
    void make_step_args(StepArgs<T, Tid> &ea, StepArgs<T, Tid> &ha, const StepScalars *tbl, int grid = 0);
    template <typename T> void make_sensor_args(SensorStepArgs<T> &sa, const StepScalars *tbl);
    void *batch = nullptr;          // the batch this simulation is a member of (it steps it)
    void fill_scalars(int t, int osc_offset, StepScalars &s) const;
    void drop_graphs();
    void accumulate_timing(int L);
    int plane_blocks() const {
        const int n = Nx * Ny;
        return n >= kPlaneBlocks * kPlaneThreads ? kPlaneBlocks : (n + kPlaneThreads - 1) / kPlaneThreads;
    }
    // step segments: device tables of per-step scalars (two slots) and the
    // CUDA graphs of full segments, one per slot
    int seg_len = 64;
    int seg_slot = 0;
    DBuf tables;
    bool use_graphs = true;
    bool graphs_dirty = true;
    // FP64-sample DFT blocks on the FP64 tensor path (mma.sync f64) rather than
    // the FMA kernel (AEFDTD_DFT_MMA=0/1; the FP32 path uses dft_tc unless AEFDTD_NO_TC)
    bool dft_mma = true;
    // tensor-core DFT wait bound and the withheld-copy test hook (aefdtd_test_hook)
    long long tc_wait_cycles = 1LL << 32;
    int tc_withhold_copy = 0;
    // persistent batch launch: wait bound and withheld-progress test hook (aefdtd_test_hook)
    long long ps_wait_cycles = 1LL << 31;
    int ps_withhold = 0;
    // captured segments, keyed by table slot, pending-flush state and the
    // sensors' buffer halves (the pointers a segment's launches bake in)
    std::map<uint64_t, cudaGraphExec_t> graph_exec;
    uint64_t graph_launches = 0;
    void step(int n);
    void zero_state();
    int kchunk_override = 0;
    int zunroll = 2;
    int tile_y = kTileYHost;        // tile height of the work items (2, 4 or 8)
    unsigned pair_mask = 0;         // groups run two cells per thread (WorkSplit::pair_mask; even Nx only)
    int prefetch_l2 = 3;            // L2 prefetch of each item's planes: bit 0 interior kernels, bit 1 CPML kernels
    unsigned pair_mask0 = 0;        // the simulation's own choices (restored when it runs alone)
    int h_reverse0 = -1;
    int h_reverse = -1;             // H work lists top plane first (L2 reuse between half-steps); -1: by size
    // fused time steps (leapfrog.cuh): one launch per step and feature group,
    // reading the current field / E-side state set and writing the other one
    bool use_fused = true;           // when the simulation allows it (fused_eligible)
    int fused_ty = kFusedMaxTY;      // owned rows per fused tile
    int fused_kchunk = 0;            // planes per fused item (0: chosen by build_fused_work)
    int fused_chunk = 0;             // the chunk depth in use
    DBuf F2[6], psiE2[6], psi2;      // the other set: fields, E-side CPML psi, RC psi
    bool set_b = false;              // the current set sits in the buffers allocated second
    bool fwork_dirty = true;
    DBuf fitems;
    int foff[kFusedGroups] = {}, fnum[kFusedGroups] = {};
    long long fcells[kFusedGroups] = {};   // owned cells per group (all chunks)
    bool timed_fused = false;        // the timed segments ran fused (group timings in fused slots)
    bool fused_eligible() const;
    void build_fused_work();
    void ensure_other_set();
    void swap_sets();
    template <typename T, typename Tid> void make_fused_args(FusedArgs<T, Tid> &A, const StepScalars *tbl, bool other);
    template <typename T, typename Tid> void enqueue_segment_fused(int L, StepScalars *tbl, bool record);
    // staged interior half-steps (interior_tma.cuh): curl-only 64 x 8 tiles
    // whose planes arrive through tensor copies. Not for batch members (their
    // merged lists take every interior item) or the oblique driver (whose
    // second grid runs on the same lists).
    bool use_tma = false;            // AEFDTD_TMA
    bool tma_allowed = true;         // cleared while the simulation is in a batch
    int tma_unit = 8;                // planes per unit (AEFDTD_TMA_UNIT)
    int tma_ctas = 2;                // AEFDTD_TMA_CTAS: 0 one unit per CTA; 1 or 2 CTAs per SM taking
                                     // units in turn (persistent)
    int tma_stages = 4;              // ring stages (AEFDTD_TMA_STAGES, 4 or 6)
    int tma_reserve = 0;             // SMs left to the concurrent boundary groups (AEFDTD_TMA_RESERVE)
    bool tma_pz = true;              // staged tiles may hold z-CPML planes (AEFDTD_TMA_PZ)
    long long tma_wait_cycles = 1LL << 32;   // wait bound and withheld-copy test hook (aefdtd_test_hook)
    int tma_withhold = 0;
    TmaPlan tma_plan[2] = {};        // E, H half-step
    DBuf tma_units, tma_ctr;
    const void *tma_ptrs[7] = {};    // the arrays the maps were encoded over (fields, ids)
    bool tma_possible() const;       // the grid and the mode allow the staged kernels
    bool build_tma_maps();           // false when the driver refuses a map
    bool tma_maps_current() const;
    // completion sensor, energy mode (CompletionSensor(coeff), s_completion.cpp)
    double cc_coeff = 0;            // > 0: enabled
    int cc_step = 500;              // checked after steps t with t % cc_step == 0
    bool cc_done = false;
    int cc_stop = -1;               // completion step t: the driver's Nt = t
    int cc_read = 0;                // energies read back so far
    double cc_last = 0, cc_max = 0;
    int cc_nb = 0, cc_cap = 0;      // energy blocks per step; history capacity
    DBuf cc_partial, cc_hist;
    CompletionFT *ccft = nullptr;   // FT mode (else energy mode)
    void completion_check();
    bool ft_check();
    bool ft_eval(const double *ring, int step);
};

inline aefdtd_sim::~aefdtd_sim() {
    set_device();
    if (stream) cudaStreamSynchronize(stream);
    size_t t = 0;
    for (auto &b : F) b.release(t);
    for (auto &b : F2) b.release(t);
    for (auto &b : psiE2) b.release(t);
    psi2.release(t);
    fitems.release(t);
    mat.release(t); coef.release(t); disp.release(t); crec.release(t); dchi.release(t); psi.release(t);
    for (auto &b : ik) b.release(t);
    for (int a = 0; a < 3; a++) { bE[a].release(t); cE[a].release(t); bH[a].release(t); cH[a].release(t); }
    for (auto &b : psiE) b.release(t);
    for (auto &b : psiH) b.release(t);
    psums.release(t);
    psum_partial.release(t);
    cc_partial.release(t);
    cc_hist.release(t);
    err.release(t);
    tables.release(t);
    for (auto &gx : graph_exec) if (gx.second) reap_graph(gx.second, device);
    items.release(t);
    tma_units.release(t);
    tma_ctr.release(t);
    fm_tbl.release(t);
    if (obl) {
        for (int c = 0; c < 6; c++) { obl->Fi[c].release(t); obl->psiEi[c].release(t); obl->psiHi[c].release(t); }
        DBuf *b[] = {&obl->psi_i, &obl->ph, &obl->mk, &obl->inc, &obl->part, &obl->hist,
                     &obl->dw, &obl->dkz, &obl->deb, &obl->dhb};
        for (DBuf *x : b) x->release(t);
        delete obl;
    }
    for (auto *m : fmaps) { m->acc.release(t); delete m; }
    if (ccft) {
        ccft->dpts.release(t); ccft->acc.release(t); ccft->ring.release(t); ccft->ctab.release(t); ccft->snap.release(t);
        delete ccft;
    }
    for (auto *s : sensors) {
        s->S.release(t); s->acc.release(t); s->wdev.release(t); s->WE.release(t); s->WH.release(t); s->flux.release(t);
        s->Btc.release(t);
        delete s;
    }
    for (auto &e : tev) if (e) cudaEventDestroy(e);
    for (auto &e : tge) if (e) cudaEventDestroy(e);
    for (auto &e : ev_join) if (e) cudaEventDestroy(e);
    if (ev_fork) cudaEventDestroy(ev_fork);
    for (auto &x : side) if (x) cudaStreamDestroy(x);
    for (int k = 0; k < 2; k++) {
        if (ev_s_fork[k]) cudaEventDestroy(ev_s_fork[k]);
        if (ev_s_join[k]) cudaEventDestroy(ev_s_join[k]);
        if (side_s[k]) cudaStreamDestroy(side_s[k]);
    }
    if (ev_f_fork) cudaEventDestroy(ev_f_fork);
    if (ev_f_join) cudaEventDestroy(ev_f_join);
    if (side_f) cudaStreamDestroy(side_f);
    if (stream) cudaStreamDestroy(stream);
}


// Removes a simulation from its batch (batch.cpp); called when it is destroyed.
namespace aefdtd {
void batch_detach(void *batch, aefdtd_sim *s);
}

// Runs f, turning exceptions into a status and the handle's last error.
template <typename F> inline aefdtd_status guarded(aefdtd_sim *s, F &&f) {
    try {
        f();
        if (s) s->last_error.clear();
        return AEFDTD_OK;
    } catch (Error &e) {
        if (s) s->last_error = e.msg;
        return e.st;
    } catch (std::bad_alloc &) {
        if (s) s->last_error = "host allocation failed";
        return AEFDTD_OOM;
    } catch (std::exception &e) {
        if (s) s->last_error = e.what();
        return AEFDTD_BAD_ARG;
    }
}

