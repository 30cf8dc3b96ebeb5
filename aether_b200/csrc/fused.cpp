// fused.cpp — host side of the fused time step (leapfrog.cuh): the second
// state set, the work list of fused items and the enqueueing of a segment of
// steps with its sensor work.
//
// The reference's time loop (normal_incidence.cpp:325-436, default_fdtd.cpp:
// 156-204) does update_E, injection, update_H, injection and the sensor feed
// per step. Here one launch per feature group advances both half-steps of a
// step from the current set into the other set; the sensors of step q read
// step q's output set beside step q + 1 (which only reads that set) and are
// joined before step q + 2 writes it again.
#include "sim.hpp"

namespace {

// Swaps the current and the other field set in a scope: the sensor-argument
// builders read F, and the output of an even step of a segment is the other set.
struct FieldSwap {
    aefdtd_sim &s;
    bool on;
    FieldSwap(aefdtd_sim &sim, bool o) : s(sim), on(o) {
        if (on) for (int c = 0; c < 6; c++) std::swap(s.F[c], s.F2[c]);
    }
    ~FieldSwap() {
        if (on) for (int c = 0; c < 6; c++) std::swap(s.F[c], s.F2[c]);
    }
};

}  // namespace

bool aefdtd_sim::fused_eligible() const {
    // the oblique driver's Bloch-coupled grids run on the split kernels
    return use_fused && !obl && Nx >= 1;
}

void aefdtd_sim::ensure_other_set() {
    auto same = [&](DBuf &o, const DBuf &c) {
        if (o.n == c.n) return;
        o.alloc(c.n, dev_bytes);
        if (o.p) AE_CUDA(cudaMemsetAsync(o.p, 0, o.n, stream));
        graphs_dirty = true;
    };
    for (int c = 0; c < 6; c++) same(F2[c], F[c]);
    for (int c = 0; c < 6; c++) same(psiE2[c], psiE[c]);
    same(psi2, psi);
}

void aefdtd_sim::swap_sets() {
    for (int c = 0; c < 6; c++) {
        std::swap(F[c], F2[c]);
        std::swap(psiE[c], psiE2[c]);
    }
    std::swap(psi, psi2);
    set_b = !set_b;
}

// Items (x0, y0, k0, k1) of 64 x fused_ty columns by a z-run of at most
// fused_chunk planes. An item's group covers the features of every cell it
// updates or recomputes: its columns plus the column after them (mod Nx), its
// rows plus the row after them (mod Ny), its planes plus the plane after them
// (mod Nz). Features: CPML or PEC on x/y (either half-step's ranges), on z,
// dispersive cells, the injection plane and oscillator boxes.
void aefdtd_sim::build_fused_work() {
    const int TX = kFusedTileX, TY = std::max(1, std::min(fused_ty, kFusedMaxTY));
    const int ntx = (Nx + TX - 1) / TX, nty = (Ny + TY - 1) / TY;
    const long long tiles = (long long)ntx * nty;
    constexpr unsigned kPXY = 1, kPZ = 2, kDISP = 4, kOTHER = 8;
    std::vector<unsigned char> feat(size_t(tiles) * Nz, 0);
    // tiles whose updated or recomputed columns include column c (rows: likewise)
    auto tiles_x = [&](int c, int out[2]) {
        int n = 0;
        out[n++] = c / TX;
        if (c % TX == 0) out[n++] = (c == 0) ? ntx - 1 : c / TX - 1;   // the column after tile c/TX - 1
        if (n == 2 && out[1] == out[0]) n = 1;
        return n;
    };
    auto tiles_y = [&](int r, int out[2]) {
        int n = 0;
        out[n++] = r / TY;
        if (r % TY == 0) out[n++] = (r == 0) ? nty - 1 : r / TY - 1;
        if (n == 2 && out[1] == out[0]) n = 1;
        return n;
    };
    auto mark = [&](int x0, int x1, int y0, int y1, int z0, int z1, unsigned f) {   // half-open cell ranges
        if (x0 >= x1 || y0 >= y1 || z0 >= z1) return;
        std::vector<char> tx(ntx, 0), ty(nty, 0);
        int o[2];
        for (int c = x0; c < x1; c++) for (int n = tiles_x(c, o), m = 0; m < n; m++) tx[o[m]] = 1;
        for (int r = y0; r < y1; r++) for (int n = tiles_y(r, o), m = 0; m < n; m++) ty[o[m]] = 1;
        for (int k = z0; k < z1; k++)
            for (int b = 0; b < nty; b++) {
                if (!ty[b]) continue;
                for (int a = 0; a < ntx; a++)
                    if (tx[a]) feat[(size_t(k) * nty + b) * ntx + a] |= f;
            }
    };
    const bool px = pml[0] || pml[1], py = pml[2] || pml[3], pz = pml[4] || pml[5];
    if (px) {
        mark(0, std::max(pml[0], 1), 0, Ny, 0, Nz, kPXY);
        mark(Nx - std::max(pml[1], 1), Nx, 0, Ny, 0, Nz, kPXY);
    }
    if (py) {
        mark(0, Nx, 0, std::max(pml[2], 1), 0, Nz, kPXY);
        mark(0, Nx, Ny - std::max(pml[3], 1), Ny, 0, Nz, kPXY);
    }
    if (pz) {
        mark(0, Nx, 0, Ny, 0, std::max(pml[4], 1), kPZ);
        mark(0, Nx, 0, Ny, Nz - std::max(pml[5], 1), Nz, kPZ);
    }
    if (normal) mark(0, Nx, 0, Ny, zs_e - 1, zs_e, kOTHER);
    for (auto &o : oscs) mark(o.box[0], o.box[1], o.box[2], o.box[3], o.box[4], o.box[5], kOTHER);
    for (unsigned m = 0; m < Nmat; m++) {
        HostMat &h = mats[m];
        if (!(h.rc && h.np > 0)) continue;
        for (int k = h.z1; k <= h.z2; k++)
            for (int j = h.y1; j <= h.y2; j++) {
                const uint32_t *row = &map[size_t(j) * Nx + size_t(k) * Nx * Ny];
                int o[2], p[2];
                for (int i = h.x1; i <= h.x2; i++)
                    if (row[i] == m)
                        for (int n = tiles_x(i, o), a = 0; a < n; a++)
                            for (int nn = tiles_y(j, p), b = 0; b < nn; b++)
                                feat[(size_t(k) * nty + p[b]) * ntx + o[a]] |= kDISP;
            }
    }
    // a plane's group also covers the plane after it (recomputed by the item ending there)
    // AEFDTD_ALL_BOUNDARY=1 routes every item through the kernel with every phase (same results)
    const bool all_features = std::getenv("AEFDTD_ALL_BOUNDARY") != nullptr;
    auto group_of = [&](unsigned f) {
        if (all_features) return (int)kFusedAll;
        if (f == 0) return (int)kFusedInterior;
        if (f == kPZ) return (int)kFusedPmlZ;
        if (f == kDISP) return (int)kFusedDisp;
        if ((f & ~(kPXY | kPZ)) == 0) return (int)kFusedPmlXY;
        return (int)kFusedAll;
    };
    // chunk depth: fewest waves of resident CTAs (1 per SM in FP64, 2 in FP32), times the planes an item walks
    const int slots = 148 * (fp64 ? 1 : 2);
    fused_chunk = fused_kchunk;
    if (fused_chunk <= 0) {
        double best = 1e300;
        for (int D : {8, 12, 16, 24, 32, 48, 64}) {
            const long long items = tiles * ((Nz + D - 1) / D);
            const double cost = double((items + slots - 1) / slots) * (std::min(D, Nz) + 1);
            if (cost < best - 1e-9 || (cost <= best + 1e-9 && D > fused_chunk)) { best = cost; fused_chunk = D; }
        }
    }
    std::vector<int> v[kFusedGroups];
    for (int g = 0; g < kFusedGroups; g++) fcells[g] = 0;
    for (int b = 0; b < nty; b++)
        for (int a = 0; a < ntx; a++) {
            const int x0 = a * TX, y0 = b * TY;
            const long long cols = (long long)std::min(TX, Nx - x0) * std::min(TY, Ny - y0);
            auto pg = [&](int k) {
                const unsigned f = feat[(size_t(k) * nty + b) * ntx + a] | feat[(size_t((k + 1) % Nz) * nty + b) * ntx + a];
                return group_of(f);
            };
            int z = 0;
            while (z < Nz) {
                const int g = pg(z);
                int ze = z + 1;
                while (ze < Nz && ze - z < fused_chunk && pg(ze) == g) ze++;
                v[g].push_back(x0);
                v[g].push_back(y0);
                v[g].push_back(z);
                v[g].push_back(ze);
                fcells[g] += cols * (ze - z);
                z = ze;
            }
        }
    std::vector<int> all;
    for (int g = 0; g < kFusedGroups; g++) {
        foff[g] = (int)(all.size() / 4);
        fnum[g] = (int)(v[g].size() / 4);
        all.insert(all.end(), v[g].begin(), v[g].end());
    }
    fitems.alloc(std::max<size_t>(all.size(), 4) * sizeof(int), dev_bytes);
    if (!all.empty()) AE_CUDA(cudaMemcpy(fitems.p, all.data(), all.size() * sizeof(int), cudaMemcpyHostToDevice));
    fwork_dirty = false;
    graphs_dirty = true;
}

// Arguments of one fused step: from the current set into the other one
// (other = false) or back (other = true).
template <typename T, typename Tid>
void aefdtd_sim::make_fused_args(FusedArgs<T, Tid> &A, const StepScalars *tbl, bool other) {
    A = FusedArgs<T, Tid>{};
    make_step_args(A.e, A.h, tbl);
    DBuf *Fo = other ? F2 : F, *Fn = other ? F : F2;
    DBuf *Po = other ? psiE2 : psiE, *Pn = other ? psiE : psiE2;
    DBuf &Ro = other ? psi2 : psi, &Rn = other ? psi : psi2;
    StepArgs<T, Tid> &a = A.e;
    a.Ex = Fo[0].as<T>(); a.Ey = Fo[1].as<T>(); a.Ez = Fo[2].as<T>();
    a.Hx = Fo[3].as<T>(); a.Hy = Fo[4].as<T>(); a.Hz = Fo[5].as<T>();
    a.psi_x0 = Po[0].as<T>(); a.psi_x1 = Po[1].as<T>();
    a.psi_y0 = Po[2].as<T>(); a.psi_y1 = Po[3].as<T>();
    a.psi_z0 = Po[4].as<T>(); a.psi_z1 = Po[5].as<T>();
    a.psi = Ro.as<Cplx<T>>();
    A.nEx = Fn[0].as<T>(); A.nEy = Fn[1].as<T>(); A.nEz = Fn[2].as<T>();
    A.nHx = Fn[3].as<T>(); A.nHy = Fn[4].as<T>(); A.nHz = Fn[5].as<T>();
    A.npx0 = Pn[0].as<T>(); A.npx1 = Pn[1].as<T>();
    A.npy0 = Pn[2].as<T>(); A.npy1 = Pn[3].as<T>();
    A.npz0 = Pn[4].as<T>(); A.npz1 = Pn[5].as<T>();
    A.npsi = Rn.as<Cplx<T>>();
}

// The kernels of L consecutive fused steps (see the file comment), then the
// plane-sum reduction of the L steps. With record = true per-step timing
// events are recorded and everything runs in order on the main stream. Step
// 0 reads the current set; with L odd the caller calls swap_sets() after
// enqueueing (or after launching the captured graph).
template <typename T, typename Tid>
void aefdtd_sim::enqueue_segment_fused(int L, StepScalars *tbl, bool record) {
    FusedArgs<T, Tid> A[2];
    make_fused_args(A[0], tbl, false);
    make_fused_args(A[1], tbl, true);
    const int4 *fi = fitems.as<int4>();
    const int ty = std::max(1, std::min(fused_ty, kFusedMaxTY));
    int groups = 0;
    for (int g = 0; g < kFusedGroups; g++) groups += fnum[g] > 0;
    // sensor arguments for each output set: step q's output is the other set when q is even
    SensorStepArgs<T> sa_set[2];
    {
        FieldSwap sw(*this, true);
        make_sensor_args(sa_set[0], tbl);
    }
    make_sensor_args(sa_set[1], tbl);
    bool maps_any = !fmaps.empty();
    const double *fm_coef =
        fmaps.empty() ? nullptr
                      : fm_tbl.as<double>() + size_t(tbl - tables.as<StepScalars>()) * kMaxMaps * 4;
    const bool conc = concurrent_groups && !record;
    // DFT blocks filled in the previous segment accumulate beside this one's steps
    bool f_pending = false;
    bool any_pending = false;
    for (PlaneSensor *ps : sensors) any_pending |= ps->pending;
    if (any_pending) {
        if (conc) {
            AE_CUDA(cudaEventRecord(ev_f_fork, stream));
            AE_CUDA(cudaStreamWaitEvent(side_f, ev_f_fork, 0));
            for (PlaneSensor *ps : sensors) launch_pending<T>(*ps, side_f);
            AE_CUDA(cudaEventRecord(ev_f_join, side_f));
            f_pending = true;
        } else {
            for (PlaneSensor *ps : sensors) launch_pending<T>(*ps, stream);
        }
    }
    // the fused groups of one step, concurrent on the side streams (disjoint cells, old set read only)
    auto launch_step = [&](FusedArgs<T, Tid> &a, int q) {
        a.e.q = a.h.q = q;
        if (record && timing_mode == 2) {
            for (int g = 0; g < kFusedGroups; g++) {
                if (fnum[g] <= 0) continue;
                const int slot = g;   // fused groups are reported in the E-side group slots of the same number
                const size_t i = ((size_t(q) * 2 + 0) * kGroups + slot) * 2;
                AE_CUDA(cudaEventRecord(tge[i], stream));
                launch_fused_group(a, fi, foff[g], fnum[g], g, ty, stream);
                AE_CUDA(cudaEventRecord(tge[i + 1], stream));
            }
            return;
        }
        int nside = 0;
        for (int g = 1; g < kFusedGroups; g++) nside += fnum[g] > 0;
        if (!conc || nside == 0) {
            for (int g = 0; g < kFusedGroups; g++) launch_fused_group(a, fi, foff[g], fnum[g], g, ty, stream);
            return;
        }
        AE_CUDA(cudaEventRecord(ev_fork, stream));
        int si = 0;
        for (int g = 1; g < kFusedGroups; g++) {
            if (fnum[g] <= 0) continue;
            AE_CUDA(cudaStreamWaitEvent(side[si], ev_fork, 0));
            launch_fused_group(a, fi, foff[g], fnum[g], g, ty, side[si]);
            AE_CUDA(cudaEventRecord(ev_join[si], side[si]));
            si++;
        }
        launch_fused_group(a, fi, foff[kFusedInterior], fnum[kFusedInterior], kFusedInterior, ty, stream);
        for (int k = 0; k < si; k++) AE_CUDA(cudaStreamWaitEvent(stream, ev_join[k], 0));
    };
    bool spend[2] = {false, false};   // sensor work of the last step of each parity still in flight
    const bool cc = cc_coeff > 0;
    for (int q = 0; q < L; q++) {
        const bool out_other = (q % 2) == 0;
        // step q writes the set the sensors of step q - 2 read
        if (spend[q & 1]) {
            AE_CUDA(cudaStreamWaitEvent(stream, ev_s_join[q & 1], 0));
            spend[q & 1] = false;
        }
        if (record) AE_CUDA(cudaEventRecord(tev[4 * q + 0], stream));
        launch_step(A[q & 1], q);
        launches += groups;
        if (record) {
            AE_CUDA(cudaEventRecord(tev[4 * q + 1], stream));
            AE_CUDA(cudaEventRecord(tev[4 * q + 2], stream));
        }
        // sensors of step q: plane sums and E samples, H samples, completion, field maps
        SensorStepArgs<T> sa = sa_set[out_other ? 0 : 1];
        sa.q = q;
        sa.partial = psum_partial.as<double>() + size_t(q) * std::max(sa.nbp, 1) * 12;
        sa.ng = 0;
        int blk = sa.nbp;
        for (PlaneSensor *ps : sensors) {
            if (sa.ng >= kMaxGather) break;
            PlaneSensor &s = *ps;
            if (s.nbuf == 0) s.buf_step0 = s.step;
            GatherDesc &g = sa.g[sa.ng++];
            g.type = s.type; g.x1 = s.x1; g.y1 = s.y1; g.z1 = s.z1; g.span1 = s.span1; g.span2 = s.span2; g.P = s.P;
            g.block0 = blk;
            g.nblocks = (s.P + kPlaneThreads - 1) / kPlaneThreads;
            blk += g.nblocks;
            g.S = s.S.as<T>() + ((size_t)s.half * dft_k + s.nbuf) * 6 * s.P;
        }
        const bool work = sa.nbp > 0 || sa.ng > 0 || cc || maps_any;
        if (work) {
            cudaStream_t st = stream;
            if (conc) {
                AE_CUDA(cudaEventRecord(ev_s_fork[q & 1], stream));
                AE_CUDA(cudaStreamWaitEvent(side_s[0], ev_s_fork[q & 1], 0));
                st = side_s[0];
            }
            FieldSwap sw(*this, out_other);
            sa.part = 0;
            launches += launch_sensor_step(sa, st);
            if (sa.ng > 0) {
                sa.part = 1;
                launches += launch_sensor_step(sa, st);
            }
            if (cc) {
                if (ccft) {
                    // FT mode: the probes' running transforms (CompletionSensor::deep_feed)
                    CcFtArgs<T> fa{};
                    fa.Nx = Nx; fa.Ny = Ny; fa.Nz = Nz; fa.NxNy = (long long)Nx * Ny;
                    fa.Ex = F[0].as<T>(); fa.Ey = F[1].as<T>(); fa.Ez = F[2].as<T>();
                    fa.np = ccft->np; fa.n_avg = ccft->n_avg; fa.step0 = ccft->step0;
                    fa.pts = ccft->dpts.as<int>();
                    fa.coef = ccft->ctab.as<double2>() + size_t(tbl - tables.as<StepScalars>()) * ccft->np;
                    fa.sc = tbl; fa.q = q;
                    fa.acc = ccft->acc.as<double2>();
                    fa.ring = ccft->ring.as<double>();
                    launch_completion_ft(fa, st);
                } else {
                    launch_energy_partial(F[0].as<T>(), F[1].as<T>(), F[2].as<T>(), (long long)Nx * Ny * Nz, cc_nb,
                                          cc_partial.as<double>() + size_t(q) * cc_nb, st);
                }
                launches++;
            }
            if (maps_any) {
                launches += launch_maps<T>(0, q, fm_coef, tbl, st);
                launches += launch_maps<T>(1, q, fm_coef, tbl, st);
            }
            if (conc) {
                AE_CUDA(cudaEventRecord(ev_s_join[q & 1], side_s[0]));
                spend[q & 1] = true;
            }
        }
        for (PlaneSensor *ps : sensors) {
            ps->nbuf++;
            ps->step++;
            if (ps->nbuf == dft_k) {
                // a filled half: accumulated at the next segment's start (or on a read)
                PlaneSensor &s = *ps;
                if (s.pending) {
                    // its sample half is rewritten from now on: the older block goes first
                    for (int k = 0; k < 2; k++)
                        if (spend[k]) { AE_CUDA(cudaStreamWaitEvent(stream, ev_s_join[k], 0)); spend[k] = false; }
                    launch_pending<T>(s, stream);
                }
                s.pending = true;
                s.pend_half = s.half;
                s.pend_n = s.nbuf;
                s.pend_step0 = s.buf_step0;
                s.pend_tbl = (s.buf_step0 == tstep + q + 1 - dft_k && q + 1 == dft_k) ? tbl : nullptr;
                s.half ^= 1;
                s.nbuf = 0;
            }
        }
        if (record) AE_CUDA(cudaEventRecord(tev[4 * q + 3], stream));
    }
    for (int k = 0; k < 2; k++)
        if (spend[k]) AE_CUDA(cudaStreamWaitEvent(stream, ev_s_join[k], 0));
    if (f_pending) AE_CUDA(cudaStreamWaitEvent(stream, ev_f_join, 0));
    if (normal) {
        launch_plane_reduce(psum_partial.as<double>(), sa_set[0].nbp, tbl, psums.as<double>(), L, stream);
        launches++;
    }
    if (cc_coeff > 0 && !ccft) {
        launch_energy_reduce(cc_partial.as<double>(), cc_nb, tbl, cc_hist.as<double>(), L, stream);
        launches++;
    }
    // after an odd L the current set is the other one: the caller swaps the
    // sets once these launches are enqueued (or their captured graph is)
}

template void aefdtd_sim::enqueue_segment_fused<double, uint8_t>(int, StepScalars *, bool);
template void aefdtd_sim::enqueue_segment_fused<double, uint16_t>(int, StepScalars *, bool);
template void aefdtd_sim::enqueue_segment_fused<float, uint8_t>(int, StepScalars *, bool);
template void aefdtd_sim::enqueue_segment_fused<float, uint16_t>(int, StepScalars *, bool);
