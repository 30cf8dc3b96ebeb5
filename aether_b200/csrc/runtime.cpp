// runtime.cpp — host runtime of the FDTD core behind the C ABI (include/aefdtd.h).
//
// Owns the device state of one simulation, generates every coefficient in
// FP64 on the host with the reference's formulas and operation order, and
// issues the fused kernels on the handle's stream in the mode driver's order.
// There is no CPU compute path: without a CUDA device every call that would
// touch the device returns AEFDTD_NO_DEVICE.
#include "sim.hpp"

#include <condition_variable>
#include <deque>
#include <mutex>
#include <random>
#include <thread>



// FDTD::FDTD (fdtd_core.cpp:158-285) for modes NORM and CUSTOM, with the
// normal-incidence driver's own argument choice (normal_incidence.cpp:188-200).
void aefdtd_sim::construct(const aefdtd_grid_desc *d) {
    g = *d;
    if (g.abi_version != AEFDTD_ABI_VERSION) fail(AEFDTD_BAD_ARG, "abi_version mismatch");
    if (g.mode != AEFDTD_MODE_NORMAL && g.mode != AEFDTD_MODE_CUSTOM && g.mode != AEFDTD_MODE_OBLIQUE)
        fail(AEFDTD_BAD_ARG, "unknown mode");
    if (g.precision != AEFDTD_FP64 && g.precision != AEFDTD_FP32) fail(AEFDTD_BAD_ARG, "unknown precision");
    if (g.nx < 1 || g.ny < 1 || g.nz < 1) fail(AEFDTD_BAD_ARG, "grid sizes must be positive");
    if (!(g.dx > 0 && g.dy > 0 && g.dz > 0)) fail(AEFDTD_BAD_ARG, "cell sizes must be positive");
    fp64 = g.precision == AEFDTD_FP64;
    device = g.device;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) fail(AEFDTD_NO_DEVICE, "no CUDA device visible");
    if (device < 0 || device >= ndev) fail(AEFDTD_BAD_ARG, "device ordinal out of range");
    AE_CUDA(cudaSetDevice(device));
    // Stream priorities: the half-steps and sensors on the highest, the DFT
    // blocks (which run beside the next segment's steps) on the lowest, so
    // that free SM slots go to the step's kernels first. Captured kernels
    // keep their stream's priority (graphs instantiate with node priorities).
    // AEFDTD_PRIO=0: every stream at the default priority.
    int lo = 0, hi = 0;
    if (!(std::getenv("AEFDTD_PRIO") && atoi(std::getenv("AEFDTD_PRIO")) == 0))
        AE_CUDA(cudaDeviceGetStreamPriorityRange(&lo, &hi));
    AE_CUDA(cudaStreamCreateWithPriority(&stream, cudaStreamNonBlocking, hi));
    for (auto &x : side) AE_CUDA(cudaStreamCreateWithPriority(&x, cudaStreamNonBlocking, hi));
    AE_CUDA(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
    for (auto &e : ev_join) AE_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    AE_CUDA(cudaStreamCreateWithPriority(&side_f, cudaStreamNonBlocking, lo));
    AE_CUDA(cudaEventCreateWithFlags(&ev_f_fork, cudaEventDisableTiming));
    AE_CUDA(cudaEventCreateWithFlags(&ev_f_join, cudaEventDisableTiming));
    for (int k = 0; k < 2; k++) {
        AE_CUDA(cudaStreamCreateWithPriority(&side_s[k], cudaStreamNonBlocking, hi));
        AE_CUDA(cudaEventCreateWithFlags(&ev_s_fork[k], cudaEventDisableTiming));
        AE_CUDA(cudaEventCreateWithFlags(&ev_s_join[k], cudaEventDisableTiming));
    }
    concurrent_groups = std::getenv("AEFDTD_SERIAL_GROUPS") == nullptr;

    Dx = g.dx; Dy = g.dy; Dz = g.dz;
    Dt = g.dt > 0 ? g.dt : std::min(std::min(Dx, Dy), Dz) / (std::sqrt(3.0) * c_light) * 0.99 * g.time_mod;
    if (!(Dt > 0)) fail(AEFDTD_BAD_ARG, "time step must be positive (dt or time_mod)");
    Nt = g.nt;
    Ntap = g.tapering;
    dft_k = g.dft_block > 0 ? g.dft_block : 64;
    if (g.pml_m > 0) pml_m = g.pml_m;
    if (g.pml_ma > 0) pml_ma = g.pml_ma;
    for (int f = 0; f < 6; f++) { pml[f] = g.pml[f]; pad[f] = g.pad[f]; }
    for (int f = 0; f < 6; f++) if (pml[f] < 0 || pad[f] < 0) fail(AEFDTD_BAD_ARG, "negative PML or pad");
    if (g.mode == AEFDTD_MODE_NORMAL || g.mode == AEFDTD_MODE_OBLIQUE) {
        // normal_incidence.cpp:195-200 (FDTD ctor pad rule) and oblique_biphase.cpp:55-60
        for (int f = 0; f < 4; f++) { pml[f] = 0; pad[f] = 0; }
        pad[4] = std::max(5, pad[4]);
        pad[5] = std::max(5, pad[5]);
    } else {
        for (int a = 0; a < 3; a++)
            if (pml[2 * a] || pml[2 * a + 1]) {
                pad[2 * a] = std::max(5, pad[2 * a]);
                pad[2 * a + 1] = std::max(5, pad[2 * a + 1]);
            }
    }
    Nx_s = g.nx; Ny_s = g.ny; Nz_s = g.nz;
    Nx = Nx_s + pml[0] + pad[0] + pad[1] + pml[1];
    Ny = Ny_s + pml[2] + pad[2] + pad[3] + pml[3];
    Nz = Nz_s + pml[4] + pad[4] + pad[5] + pml[5];
    xs_s = pml[0] + pad[0]; xs_e = xs_s + Nx_s;
    ys_s = pml[2] + pad[2]; ys_e = ys_s + Ny_s;
    zs_s = pml[4] + pad[4]; zs_e = zs_s + Nz_s;
    if ((long long)Nx * Ny * Nz > (1LL << 40)) fail(AEFDTD_BAD_ARG, "grid too large");
    // basic_differentials_compute (fdtd_core.cpp:1137-1148)
    dtm = Dt / mu0;
    dtdez = Dt / (Dz * e0);
    dtdmx = Dt / (Dx * mu0); dtdmy = Dt / (Dy * mu0); dtdmz = Dt / (Dz * mu0);
    // set_pml_* (fdtd_pml.cpp:445-497): sigma_max = 0.8(m+1)/(eta0 D) * scale
    for (int f = 0; f < 6; f++) {
        double D = f < 2 ? Dx : (f < 4 ? Dy : Dz);
        pml_kappa[f] = g.pml_kappa[f];
        pml_sigma[f] = 0.8 * (pml_m + 1.0) / (std::sqrt(mu0 / e0) * D) * g.pml_sigma[f];
        pml_alpha[f] = g.pml_alpha[f];
    }
    size_t es = fp64 ? 8 : 4;
    size_t N = size_t(Nx) * Ny * Nz;
    for (auto &b : F) { b.alloc(N * es, dev_bytes); AE_CUDA(cudaMemsetAsync(b.p, 0, b.n, stream)); }
    // CPML psi, slab-compact (allocate_pml, fdtd_pml.cpp:26-86)
    size_t nxs = pml[0] + pml[1], nys = pml[2] + pml[3], nzs = pml[4] + pml[5];
    for (int s = 0; s < 2; s++) {
        DBuf *P = s == 0 ? psiE : psiH;
        for (int q = 0; q < 2; q++) {
            P[q].alloc(nxs * Ny * Nz * es, dev_bytes);
            P[2 + q].alloc(Nx * nys * Nz * es, dev_bytes);
            P[4 + q].alloc(size_t(Nx) * Ny * nzs * es, dev_bytes);
        }
        for (int q = 0; q < 6; q++) if (P[q].p) AE_CUDA(cudaMemsetAsync(P[q].p, 0, P[q].n, stream));
    }
    build_pml_tables();
    seg_len = dft_k;
    tables.alloc(sizeof(StepScalars) * 2 * seg_len, dev_bytes);
    if (std::getenv("AEFDTD_NO_GRAPHS")) use_graphs = false;
    err.alloc(sizeof(int), dev_bytes);
    AE_CUDA(cudaMemsetAsync(err.p, 0, sizeof(int), stream));
    map.assign(N, 0);
    Nmat = 1;
    mats.assign(1, HostMat());
    if (const char *kc = std::getenv("AEFDTD_KCHUNK")) kchunk_override = std::max(0, atoi(kc));
    if (const char *zu = std::getenv("AEFDTD_ZUNROLL")) zunroll = atoi(zu) >= 2 ? 2 : 1;
    if (const char *pf = std::getenv("AEFDTD_PREFETCH")) prefetch_l2 = std::clamp(atoi(pf), 0, 3);
    if (const char *hr = std::getenv("AEFDTD_HREV")) h_reverse = atoi(hr) != 0 ? 1 : 0;
    // two cells per thread: FP32 interior and z-CPML items, FP64 z-CPML items
    // and the y-only items of the x/y-CPML group
    pair_mask = (fp64 ? (1u << kGroupPmlZ) : (1u << kGroupInterior) | (1u << kGroupPmlZ)) | (1u << kGroupPmlXY);
    if (const char *pm = std::getenv("AEFDTD_PAIR")) pair_mask = unsigned(atoi(pm)) & 0x13u;
    pair_mask0 = pair_mask;
    h_reverse0 = h_reverse;
    // fused time steps: on by default where they measure faster (kFusedDefault),
    // AEFDTD_FUSED=1 / 0 forces them on / off (same results in FP64 either way)
    use_fused = kFusedDefault;
    if (const char *fz = std::getenv("AEFDTD_FUSED")) use_fused = atoi(fz) != 0;
    if (const char *fy = std::getenv("AEFDTD_FUSED_TY")) fused_ty = std::clamp(atoi(fy), 1, kFusedMaxTY);
    if (const char *fk = std::getenv("AEFDTD_FUSED_KCHUNK")) fused_kchunk = std::max(0, atoi(fk));
    if (const char *dm = std::getenv("AEFDTD_DFT_MMA")) dft_mma = atoi(dm) != 0;
    if (const char *tm = std::getenv("AEFDTD_TMA")) use_tma = atoi(tm) != 0;
    if (const char *tu = std::getenv("AEFDTD_TMA_UNIT")) tma_unit = std::clamp(atoi(tu), 1, 4096);
    if (const char *tc = std::getenv("AEFDTD_TMA_CTAS")) tma_ctas = std::clamp(atoi(tc), 0, 2);
    if (const char *tg = std::getenv("AEFDTD_TMA_STAGES")) tma_stages = atoi(tg) >= 6 ? 6 : 4;
    if (const char *tr = std::getenv("AEFDTD_TMA_RESERVE")) tma_reserve = std::clamp(atoi(tr), 0, 128);
    if (const char *tz = std::getenv("AEFDTD_TMA_PZ")) tma_pz = atoi(tz) != 0;
    if (const char *ty = std::getenv("AEFDTD_TILE_Y")) {
        const int v = atoi(ty);
        tile_y = (v == 2 || v == 8) ? v : 4;
    }
    AE_CUDA(cudaStreamSynchronize(stream));
}

// pml_coeff_calc and pml_{x,y,z}_coeffs (fdtd_pml.cpp:305-433) evaluated once
// with the final set_pml_* parameters; 1/kappa follows the selection rules of
// advE*/advH* (x: pml_xm||pml_xp, y: pml_ym||pml_xp, z: pml_zm||pml_zp;
// fdtd_core.cpp:378,397,457,504,523,561,580,631,669,688).
void aefdtd_sim::build_pml_tables() {
    auto coeffs = [&](double ind, int N, int pm, int pp, int f, double &kappa, double &b, double &c) {
        kappa = 1.0;
        if (ind < pm) {
            double x = (pm - ind) / static_cast<double>(pm);
            kappa = 1.0 + (pml_kappa[f] - 1.0) * std::pow(x, pml_m);
            double sig = pml_sigma[f] * std::pow(x, pml_m);
            double alp = pml_alpha[f] * std::pow(1.0 - x, pml_ma);
            b = std::exp(-(sig / kappa + alp) * Dt / e0);
            c = sig / (sig * kappa + kappa * kappa * alp) * (b - 1.0);
        }
        if (ind > N - pp) {
            double x = (ind - (N - pp)) / static_cast<double>(pp);
            kappa = 1.0 + (pml_kappa[f + 1] - 1.0) * std::pow(x, pml_m);
            double sig = pml_sigma[f + 1] * std::pow(x, pml_m);
            double alp = pml_alpha[f + 1] * std::pow(1.0 - x, pml_ma);
            b = std::exp(-(sig / kappa + alp) * Dt / e0);
            c = sig / (sig * kappa + kappa * kappa * alp) * (b - 1.0);
        }
    };
    int Ns[3] = {Nx, Ny, Nz};
    double invD[3] = {1.0 / Dx, 1.0 / Dy, 1.0 / Dz};
    bool kappa_sel[3] = {pml[0] || pml[1], pml[2] || pml[1], pml[4] || pml[5]};
    for (int ax = 0; ax < 3; ax++) {
        int N = Ns[ax], pm = pml[2 * ax], pp = pml[2 * ax + 1];
        std::vector<double> kE(N, 1.0), kH(N, 1.0), be(N, 0.0), bh(N, 0.0), ce(N, 0.0), ch(N, 0.0);
        if (pm || pp)
            for (int i = 0; i < N; i++) {
                coeffs(i, N, pm, pp, 2 * ax, kE[i], be[i], ce[i]);
                coeffs(i + 0.5, N, pm, pp, 2 * ax, kH[i], bh[i], ch[i]);
            }
        std::vector<double> ikE(N), ikH(N), bE64(N), bH64(N), cE64(N), cH64(N);
        for (int i = 0; i < N; i++) {
            ikE[i] = 1.0 / (kappa_sel[ax] ? kE[i] : 1.0);
            ikH[i] = 1.0 / (kappa_sel[ax] ? kH[i] : 1.0);
            // the reference multiplies c by 1/D inside the psi update: c*inv_D*(diff)
            cE64[i] = ce[i] * invD[ax];
            cH64[i] = ch[i] * invD[ax];
            bE64[i] = fp64 ? be[i] : be[i] - 1.0;
            bH64[i] = fp64 ? bh[i] : bh[i] - 1.0;
        }
        auto up = [&](DBuf &b, const std::vector<double> &v) {
            size_t es = fp64 ? 8 : 4;
            b.alloc(v.size() * es, dev_bytes);
            if (fp64) AE_CUDA(cudaMemcpy(b.p, v.data(), v.size() * 8, cudaMemcpyHostToDevice));
            else {
                std::vector<float> f(v.begin(), v.end());
                AE_CUDA(cudaMemcpy(b.p, f.data(), f.size() * 4, cudaMemcpyHostToDevice));
            }
        };
        up(ik[ax], ikE); up(ik[3 + ax], ikH);
        up(bE[ax], bE64); up(cE[ax], cE64); up(bH[ax], bH64); up(cH[ax], cH64);
    }
}

// FDTD::set_matsgrid (fdtd_utils.cpp:572-766): structure map into the grid,
// edge slices replicated into pads and PML.
void aefdtd_sim::set_map(const uint32_t *m, size_t count) {
    if (!m) fail(AEFDTD_BAD_ARG, "null map");
    if (count != size_t(Nx_s) * Ny_s * Nz_s) fail(AEFDTD_BAD_ARG, "map size must be nx*ny*nz of the structure grid");
    auto M = [&](int i, int j, int k) -> uint32_t & { return map[i + size_t(j) * Nx + size_t(k) * Nx * Ny]; };
    for (int k = zs_s; k < zs_e; k++)
        for (int j = ys_s; j < ys_e; j++) {
            const uint32_t *src = m + size_t(j - ys_s) * Nx_s + size_t(k - zs_s) * Nx_s * Ny_s;
            std::memcpy(&M(xs_s, j, k), src, Nx_s * sizeof(uint32_t));
            for (int i = 0; i < xs_s; i++) M(i, j, k) = M(xs_s, j, k);
            for (int i = xs_e; i < Nx; i++) M(i, j, k) = M(xs_e - 1, j, k);
        }
    for (int k = zs_s; k < zs_e; k++) {
        for (int j = 0; j < ys_s; j++) std::memcpy(&M(0, j, k), &M(0, ys_s, k), Nx * sizeof(uint32_t));
        for (int j = ys_e; j < Ny; j++) std::memcpy(&M(0, j, k), &M(0, ys_e - 1, k), Nx * sizeof(uint32_t));
    }
    for (int k = 0; k < zs_s; k++) std::memcpy(&M(0, 0, k), &M(0, 0, zs_s), size_t(Nx) * Ny * sizeof(uint32_t));
    for (int k = zs_e; k < Nz; k++) std::memcpy(&M(0, 0, k), &M(0, 0, zs_e - 1), size_t(Nx) * Ny * sizeof(uint32_t));
    uint32_t mx = 0;
    for (uint32_t v : map) mx = std::max(mx, v);
    if (mx >= 65535u) fail(AEFDTD_BAD_ARG, "at most 65535 material indices");
    Nmat = mx + 1;
    mats.assign(Nmat, HostMat());
    // bounding boxes for every index in one pass (FDTD_Material::link_grid,
    // mats.cpp:394-443), one update per run of equal indices along x
    for (int k = 0; k < Nz; k++)
        for (int j = 0; j < Ny; j++) {
            const uint32_t *row = &M(0, j, k);
            for (int i = 0; i < Nx;) {
                const uint32_t v = row[i];
                const int i0 = i;
                while (i < Nx && row[i] == v) i++;
                HostMat &h = mats[v];
                if (h.x2 < h.x1) { h.x1 = i0; h.x2 = i - 1; h.y1 = h.y2 = j; h.z1 = h.z2 = k; continue; }
                h.x1 = std::min(h.x1, i0); h.x2 = std::max(h.x2, i - 1);
                h.y1 = std::min(h.y1, j); h.y2 = std::max(h.y2, j);
                h.z1 = std::min(h.z1, k); h.z2 = std::max(h.z2, k);
            }
        }
    id_bytes = Nmat <= 256 ? 1 : 2;
    // device copy with a 16-byte row pitch (TMA strides), padding columns = 0
    mpitch = (Nx + (16 / id_bytes) - 1) / (16 / id_bytes) * (16 / id_bytes);
    size_t NP = size_t(mpitch) * Ny * Nz;
    mat.alloc(NP * id_bytes, dev_bytes);
    if (id_bytes == 1) {
        std::vector<uint8_t> v(NP, 0);
        for (size_t r = 0; r < size_t(Ny) * Nz; r++)
            for (int i = 0; i < Nx; i++) v[r * mpitch + i] = (uint8_t)map[r * Nx + i];
        AE_CUDA(cudaMemcpy(mat.p, v.data(), NP, cudaMemcpyHostToDevice));
    } else {
        std::vector<uint16_t> v(NP, 0);
        for (size_t r = 0; r < size_t(Ny) * Nz; r++)
            for (int i = 0; i < Nx; i++) v[r * mpitch + i] = (uint16_t)map[r * Nx + i];
        AE_CUDA(cudaMemcpy(mat.p, v.data(), NP * 2, cudaMemcpyHostToDevice));
    }
    work_dirty = true;
    map_set = true;
    tables_dirty = true;
}

// FDTD::set_material (fdtd_utils.cpp:810-820): FDTD_Material::set_base_mat
// (mats.cpp:445-464), const_recalc (mats_const.cpp:71-80), RC_dielec_treat and
// RC_recalc (mats_RC.cpp:126-184), pole pairs of Dielec_model::get_time_exp
// (dielec_models.cpp:71-107) and DrudeModel::get_sigma (dielec_models.cpp:287-290).
void aefdtd_sim::set_material(uint32_t idx, const aefdtd_material_desc *md) {
    if (!map_set) fail(AEFDTD_NOT_READY, "set the material map first");
    if (!md) fail(AEFDTD_BAD_ARG, "null material");
    if (md->n_debye < 0 || md->n_drude < 0 || md->n_lorentz < 0 || md->n_critpoint < 0 ||
        md->n_debye > AEFDTD_MAX_TERMS || md->n_drude > AEFDTD_MAX_TERMS ||
        md->n_lorentz > AEFDTD_MAX_TERMS || md->n_critpoint > AEFDTD_MAX_TERMS)
        fail(AEFDTD_BAD_ARG, "term counts out of range");
    if (idx >= Nmat || mats[idx].x2 < mats[idx].x1) return;   // not in the grid: ignored, as mats_in_grid
    HostMat &h = mats[idx];
    h.set = true;
    const cplx Im(0, 1);
    int nmod = md->n_debye + md->n_drude + md->n_lorentz + md->n_critpoint;
    h.ei = md->eps_inf;
    if (nmod == 0) {
        h.rc = false; h.np = 0; h.sig = 0;
        h.C1 = 1;
        h.C2x = Dt / (Dx * e0 * h.ei);
        h.C2y = Dt / (Dy * e0 * h.ei);
        h.C2z = Dt / (Dz * e0 * h.ei);
        h.C3 = 0;
        h.C4 = Dt / (e0 * h.ei);
        tables_dirty = true;
        return;
    }
    std::vector<cplx> pa, pb;
    for (int n = 0; n < md->n_debye; n++) {
        double ds = md->debye[n][0], t0 = md->debye[n][1];
        pa.push_back(ds / t0);
        pb.push_back(-1.0 / t0);
    }
    for (int n = 0; n < md->n_drude; n++) {
        double wd = md->drude[n][0], gm = md->drude[n][1];
        double wd2 = wd * wd;
        pa.push_back(-wd2 / gm);
        pb.push_back(-gm);
    }
    for (int n = 0; n < md->n_lorentz; n++) {
        double A = md->lorentz[n][0], O = md->lorentz[n][1], G = md->lorentz[n][2];
        double alp = G / 2.0;
        cplx bet = std::sqrt(O * O - alp * alp);
        cplx eta = A * O * O / bet;
        pa.push_back(-eta * Im);
        pb.push_back(-alp + bet * Im);
    }
    for (int n = 0; n < md->n_critpoint; n++) {
        double A = md->critpoint[n][0], O = md->critpoint[n][1], P = md->critpoint[n][2], G = md->critpoint[n][3];
        pa.push_back(-2.0 * A * O * std::exp(-P * Im) * Im);
        pb.push_back(-G + O * Im);
    }
    double sig = 0;
    for (int n = 0; n < md->n_drude; n++) {
        double wd = md->drude[n][0], gm = md->drude[n][1];
        sig += e0 * (wd * wd) / gm;
    }
    h.rc = true; h.np = nmod; h.sig = sig;
    h.crec.resize(nmod); h.chi.resize(nmod); h.dchi.resize(nmod);
    for (int n = 0; n < nmod; n++) {
        h.crec[n] = std::exp(pb[n] * Dt);
        h.chi[n] = pa[n] / pb[n] * (std::exp(pb[n] * Dt) - 1.0);
        h.dchi[n] = -pa[n] / pb[n] * std::pow(1.0 - std::exp(pb[n] * Dt), 2.0);
    }
    double chitmp = 0;
    for (int n = 0; n < nmod; n++) chitmp += std::real(h.chi[n]);
    double e_eff = h.ei + chitmp + h.sig * Dt / e0;
    h.C1 = h.ei / e_eff;
    h.C2x = Dt / (Dx * e0 * e_eff);
    h.C2y = Dt / (Dy * e0 * e_eff);
    h.C2z = Dt / (Dz * e0 * e_eff);
    h.C3 = 1.0 / e_eff;
    h.C4 = Dt / (e0 * e_eff);
    tables_dirty = true;
    work_dirty = true;
    graphs_dirty = true;
}

// Device tables of material coefficients and the dispersive-state layout.
void aefdtd_sim::finalize_tables() {
    if (!tables_dirty) return;
    if (!map_set) fail(AEFDTD_NOT_READY, "no material map");
    std::vector<double> cf(size_t(Nmat) * 6);
    std::vector<DispInfo> di(Nmat);
    std::vector<double> cr, dc;
    long long off = 0;
    int poles = 0;
    any_disp = false;
    for (unsigned m = 0; m < Nmat; m++) {
        HostMat &h = mats[m];
        double v[6] = {h.C1, h.C2x, h.C2y, h.C2z, h.C3, h.C4};
        for (int q = 0; q < 6; q++) cf[m * 6 + q] = v[q];
        DispInfo d{};
        if (h.rc && h.np > 0) {
            any_disp = true;
            d.np = h.np;
            d.pole_off = poles;
            d.x1 = h.x1; d.y1 = h.y1; d.z1 = h.z1;
            d.xs = h.x2 + 1 - h.x1; d.ys = h.y2 + 1 - h.y1; d.zs = h.z2 + 1 - h.z1;
            d.box = (long long)d.xs * d.ys * d.zs;
            d.psi_off = off;
            off += d.box * 3 * h.np;
            for (int p = 0; p < h.np; p++) {
                cplx c = h.crec[p];
                // FP32 stores Crec-1: the decrement is small next to 1 for weakly damped poles
                cr.push_back(fp64 ? c.real() : c.real() - 1.0);
                cr.push_back(c.imag());
                dc.push_back(h.dchi[p].real());
                dc.push_back(h.dchi[p].imag());
            }
            poles += h.np;
        }
        di[m] = d;
    }
    auto up = [&](DBuf &b, const std::vector<double> &v) {
        size_t es = fp64 ? 8 : 4;
        b.alloc(std::max<size_t>(v.size(), 1) * es, dev_bytes);
        if (v.empty()) return;
        if (fp64) AE_CUDA(cudaMemcpy(b.p, v.data(), v.size() * 8, cudaMemcpyHostToDevice));
        else {
            std::vector<float> f(v.begin(), v.end());
            AE_CUDA(cudaMemcpy(b.p, f.data(), f.size() * 4, cudaMemcpyHostToDevice));
        }
    };
    up(coef, cf);
    up(crec, cr);
    up(dchi, dc);
    disp.alloc(sizeof(DispInfo) * Nmat, dev_bytes);
    AE_CUDA(cudaMemcpy(disp.p, di.data(), sizeof(DispInfo) * Nmat, cudaMemcpyHostToDevice));
    size_t es = fp64 ? 16 : 8;
    if ((size_t)off * es != psi.n) {
        psi.alloc(size_t(off) * es, dev_bytes);
        if (psi.p) AE_CUDA(cudaMemsetAsync(psi.p, 0, psi.n, stream));
    }
    if (obl && obl->psi_i.n != psi.n) {
        obl->psi_i.alloc(psi.n, dev_bytes);
        if (obl->psi_i.p) AE_CUDA(cudaMemsetAsync(obl->psi_i.p, 0, obl->psi_i.n, stream));
    }
    AE_CUDA(cudaStreamSynchronize(stream));
    tables_dirty = false;
}

template <typename T, typename Tid>
void aefdtd_sim::fill_args(StepArgs<T, Tid> &a, bool e_side, int grid) {
    std::memset(&a, 0, sizeof(a));
    a.Nx = Nx; a.Ny = Ny; a.Nz = Nz;
    a.NxNy = (long long)Nx * Ny;
    DBuf *G = grid_fields(grid);
    a.Ex = G[0].as<T>(); a.Ey = G[1].as<T>(); a.Ez = G[2].as<T>();
    a.Hx = G[3].as<T>(); a.Hy = G[4].as<T>(); a.Hz = G[5].as<T>();
    a.mat = mat.as<Tid>();
    a.mpitch = mpitch;
    a.coef = coef.as<MatCoef<T>>();
    a.nmat = (int)Nmat;
    a.disp = any_disp ? disp.as<DispInfo>() : nullptr;
    a.crec = crec.as<Cplx<T>>();
    a.dchi = dchi.as<Cplx<T>>();
    a.psi = (grid && obl ? obl->psi_i : psi).as<Cplx<T>>();
    a.pml_xm = pml[0]; a.pml_xp = pml[1]; a.pml_ym = pml[2]; a.pml_yp = pml[3]; a.pml_zm = pml[4]; a.pml_zp = pml[5];
    a.px = pml[0] || pml[1]; a.py = pml[2] || pml[3]; a.pz = pml[4] || pml[5];
    int o = e_side ? 0 : 3;
    a.ikx = ik[o + 0].as<T>(); a.iky = ik[o + 1].as<T>(); a.ikz = ik[o + 2].as<T>();
    DBuf *B = e_side ? bE : bH, *Cc = e_side ? cE : cH, *P = e_side ? psiE : psiH;
    if (grid && obl) P = e_side ? obl->psiEi : obl->psiHi;
    a.bx = B[0].as<T>(); a.by = B[1].as<T>(); a.bz = B[2].as<T>();
    a.cx = Cc[0].as<T>(); a.cy = Cc[1].as<T>(); a.cz = Cc[2].as<T>();
    a.psi_x0 = P[0].as<T>(); a.psi_x1 = P[1].as<T>();
    a.psi_y0 = P[2].as<T>(); a.psi_y1 = P[3].as<T>();
    a.psi_z0 = P[4].as<T>(); a.psi_z1 = P[5].as<T>();
    a.dtdmx = (T)dtdmx; a.dtdmy = (T)dtdmy; a.dtdmz = (T)dtdmz; a.dtm = (T)dtm;
    a.kinj = -1;
    a.kobl = -1;
    a.err = err.as<int>();
    if (obl) {
        // the other grid's fields and the Bloch phases of this half-step's wraps
        DBuf *O = grid_fields(grid ^ 1);
        a.oEx = O[0].as<T>(); a.oEy = O[1].as<T>(); a.oEz = O[2].as<T>();
        a.oHx = O[3].as<T>(); a.oHy = O[4].as<T>(); a.oHz = O[5].as<T>();
        a.bloch = grid + 1;
        const cplx bx = e_side ? obl->dH_x : obl->dE_x, by = e_side ? obl->dH_y : obl->dE_y;
        a.bxr = bx.real(); a.bxi = bx.imag(); a.byr = by.real(); a.byi = by.imag();
        a.kobl = e_side ? obl->z2 : obl->z2 - 1;
        a.obl_coef = e_side ? obl->c2z : dtdmz;
        a.obl_px = obl->ph.as<double2>();
        a.obl_py = obl->ph.as<double2>() + size_t(Nx) * Ny;
        a.obl_inc = obl->inc.as<double>();
    }
}

// Accumulates one DFT block of a sensor: n buffered steps in sample-buffer
// half `half`, slot 0 being step *step0_ptr (a step table entry) or step0.
template <typename T>
void aefdtd_sim::flush_block(PlaneSensor &s, int half, int n, const StepScalars *step0_ptr, int step0, cudaStream_t st) {
    if (n == 0) return;
    const size_t hoff = size_t(half) * dft_k * 6 * s.P;
    if (!fp64 && s.Btc.p) {
        // tensor-core DFT: phasors split into TF32 hi/lo in the B image, then the GEMM
        DftTcPhasorArgs pa{dft_k, n, s.nl, s.N0, s.N1, Nt, Ntap, step0_ptr ? &step0_ptr->step : nullptr,
                           step0_ptr ? 0 : step0, Dt, s.wdev.as<double>(), s.Btc.as<float>(),
                           size_t(4) * 256 * dft_k};
        launch_phasors_tc(pa, st);
        DftTcArgs aa{dft_k, n, s.nl, s.P, s.N0, s.N1, s.S.as<float>() + hoff, s.Btc.as<float>(),
                     size_t(4) * 256 * dft_k, s.acc.as<double2>(), err.as<int>(), tc_wait_cycles,
                     tc_withhold_copy};
        launch_accumulate_tc(aa, st);
        launches += 2;
        return;
    }
    PhasorArgs pa{n, s.nl, Nt, Ntap, step0_ptr ? &step0_ptr->step : nullptr, step0_ptr ? 0 : step0, Dt,
                  s.wdev.as<double>(), s.WE.as<double2>(), s.WH.as<double2>()};
    launch_phasors(pa, st);
    AccumArgs<T> aa{s.P, s.nl, n, s.S.as<T>() + hoff, s.WE.as<double2>(), s.WH.as<double2>(), s.acc.as<double2>(),
                    dft_mma ? 1 : 0};
    launch_accumulate(aa, st);
    launches += 2;
}

template <typename T> void aefdtd_sim::launch_pending(PlaneSensor &s, cudaStream_t st) {
    if (!s.pending) return;
    flush_block<T>(s, s.pend_half, s.pend_n, s.pend_tbl, s.pend_step0, st);
    s.pending = false;
}

// Accumulates every buffered sample of every sensor on the main stream:
// pending blocks first, then the partly filled halves (all sensors stay
// aligned on block boundaries).
void aefdtd_sim::drain_sensors() {
    for (auto *p : sensors) { if (fp64) launch_pending<double>(*p, stream); else launch_pending<float>(*p, stream); }
    for (auto *p : sensors) {
        if (p->nbuf == 0) continue;
        if (fp64) flush_block<double>(*p, p->half, p->nbuf, nullptr, p->buf_step0, stream);
        else flush_block<float>(*p, p->half, p->nbuf, nullptr, p->buf_step0, stream);
        p->nbuf = 0;
    }
}

// Host values of one step's scalars (excitation, sensors), FP64.
void aefdtd_sim::fill_scalars(int t, int osc_offset, StepScalars &s) const {
    std::memset(&s, 0, sizeof(s));
    s.step = t;
    s.snap = -1;
    if (normal) {
        // normal_incidence.cpp:334-357
        double tb = t * Dt;
        double inj_Hx = pulse.f(pulse.Hx0, 0, 0, (zs_e - 1 + 0.5) * Dz, tb);
        double inj_Hy = pulse.f(pulse.Hy0, 0, 0, (zs_e - 1 + 0.5) * Dz, tb);
        s.inj_eA = dtdez * inj_Hy / eps_sup;
        s.inj_eB = dtdez * inj_Hx / eps_sup;
        tb = (t + 0.5) * Dt;
        double inj_Ex = pulse.f(pulse.Ex0, 0, 0, (zs_e - 1) * Dz, tb);
        double inj_Ey = pulse.f(pulse.Ey0, 0, 0, (zs_e - 1) * Dz, tb);
        s.inj_hA = dtdmz * inj_Ey;
        s.inj_hB = dtdmz * inj_Ex;
        // plane sums (normal_incidence.cpp:378-386)
        s.tb = (t + 0.5) * Dt;
        double tapering = 1.0;
        if (t >= Nt - Ntap) tapering = s_curve(t, Nt - 1.0, Nt - Ntap);
        s.taper = tapering;
    }
    for (size_t k = 0; k < oscs.size() && k < 4; k++) {
        // Oscillator::deep_inject_E (sc_oscillator.cpp:38-39)
        const Osc &o = oscs[k];
        const int st = o.step + osc_offset;
        const cplx Im(0, 1);
        cplx im_val = std::exp(-o.w0 * st * Dt * Im) * std::exp(-std::pow(o.dw / 2.0 * ((st - o.tshift) * Dt), 2.0));
        s.src[k] = std::real(im_val) * 50;
    }
}

static_assert(kMapPlane == AEFDTD_MAP_PLANE && kMapBlock == AEFDTD_MAP_BLOCK && kMapPoint == AEFDTD_MAP_POINT,
              "field-sensor kinds");

// Phases of the field sensors for steps t0 .. t0+L-1, row q = step t0+q:
// per map E then H phase as (re, im). The expressions are those of
// FieldMap::FT_compute (s_fieldmap.cpp:356-358) and
// FieldBlock::threaded_computation (:197-202), evaluated on the host in FP64.
void aefdtd_sim::fill_map_phases(int t0, int L, double *rows) const {
    const cplx Im(0, 1);
    for (int q = 0; q < L; q++) {
        const int step = t0 + q;
        for (size_t m = 0; m < fmaps.size(); m++) {
            const double w = fmaps[m]->w;
            const cplx ce = std::exp(w * step * Dt * Im);
            const cplx ch = std::exp(w * (step + 0.5) * Dt * Im);
            double *r = rows + (size_t(q) * kMaxMaps + m) * 4;
            r[0] = ce.real(); r[1] = ce.imag(); r[2] = ch.real(); r[3] = ch.imag();
        }
    }
}

// One part of step q's field sensors in one launch: part 0 the maps that read
// E (E plane maps, blocks' E half, points), part 1 those that read H.
template <typename T>
int aefdtd_sim::launch_maps(int part, int q, const double *coef, const StepScalars *tbl, cudaStream_t st) {
    MapStepArgs<T> a{};
    a.Nx = Nx; a.Ny = Ny; a.Nz = Nz; a.NxNy = (long long)Nx * Ny;
    a.Ex = F[0].as<T>(); a.Ey = F[1].as<T>(); a.Ez = F[2].as<T>();
    a.Hx = F[3].as<T>(); a.Hy = F[4].as<T>(); a.Hz = F[5].as<T>();
    a.coef = coef;
    a.sc = tbl;
    a.q = q;
    a.part = part;
    int blk = 0;
    for (size_t m = 0; m < fmaps.size(); m++) {
        const MapDesc &d = fmaps[m]->dev;
        const bool reads_h = d.kind == kMapBlock || (d.kind == kMapPlane && d.mag);
        const bool reads_e = d.kind != kMapPlane || !d.mag;
        if (!(part ? reads_h : reads_e)) continue;
        MapDesc &o = a.m[a.nm++];
        o = d;
        o.slot = (int)m;
        o.block0 = blk;
        o.nblocks = (d.P + kPlaneThreads - 1) / kPlaneThreads;
        blk += o.nblocks;
    }
    return a.nm ? launch_fieldmap_step(a, st) : 0;
}

// Launches the groups of one half-step. The groups update disjoint cells and
// read only the other field family, so the boundary groups run on side
// streams forked from the main stream, concurrently with the interior group,
// and are joined back before the next half-step. Under stream capture this
// records parallel graph branches.
template <typename Launch> void aefdtd_sim::run_groups(const WorkSplit &w, Launch &&launch) {
    int nside = 0;
    for (int g = 1; g < kGroups; g++) nside += w.n[g] > 0;
    if (!concurrent_groups || nside == 0) {
        for (int g = 0; g < kGroups; g++) launch(g, stream);
        return;
    }
    AE_CUDA(cudaEventRecord(ev_fork, stream));
    int si = 0;
    for (int g = 1; g < kGroups; g++) {
        if (w.n[g] <= 0) continue;
        AE_CUDA(cudaStreamWaitEvent(side[si], ev_fork, 0));
        launch(g, side[si]);
        AE_CUDA(cudaEventRecord(ev_join[si], side[si]));
        si++;
    }
    launch(kGroupInterior, stream);
    for (int k = 0; k < si; k++) AE_CUDA(cudaStreamWaitEvent(stream, ev_join[k], 0));
}

// Arguments of the E and H half-step kernels for steps whose scalars are in
// the table `tbl` (shared by single-simulation segments and batches).
template <typename T, typename Tid>
void aefdtd_sim::make_step_args(StepArgs<T, Tid> &ea, StepArgs<T, Tid> &ha, const StepScalars *tbl, int grid) {
    fill_args(ea, true, grid);
    fill_args(ha, false, grid);
    ea.kchunk = ha.kchunk = kchunk;
    ea.prefetch = ha.prefetch = prefetch_l2;
    ea.sc = ha.sc = tbl;
    if (normal) ea.kinj = ha.kinj = zs_e - 1;
    ea.nsrc = 0;
    for (size_t s = 0; s < oscs.size() && s < 4; s++) {
        std::memcpy(ea.src_box[s], oscs[s].box, sizeof(oscs[s].box));
        ea.src_comp[s] = oscs[s].comp;
        ea.nsrc++;
    }
}

// Sensor-launch arguments without gathers: fields, plane-sum geometry and pulse.
template <typename T> void aefdtd_sim::make_sensor_args(SensorStepArgs<T> &sa, const StepScalars *tbl) {
    sa = SensorStepArgs<T>{};
    sa.Nx = Nx; sa.Ny = Ny; sa.Nz = Nz; sa.NxNy = (long long)Nx * Ny;
    sa.Ex = F[0].as<T>(); sa.Ey = F[1].as<T>(); sa.Ez = F[2].as<T>();
    sa.Hx = F[3].as<T>(); sa.Hy = F[4].as<T>(); sa.Hz = F[5].as<T>();
    sa.sc = tbl;
    if (normal) {
        sa.nbp = plane_blocks();
        sa.kr = zs_e - 2; sa.kt = zs_s;
        sa.Dx = Dx; sa.Dy = Dy; sa.Dz = Dz;
        sa.P = PulseDev{pulse.k, pulse.omega, pulse.kx, pulse.ky, pulse.kz, pulse.n_ind, pulse.dz, pulse.C1,
                        pulse.Ex0, pulse.Ey0, pulse.Ez0};
        sa.partial = psum_partial.as<double>();
        sa.out = psums.as<double>();
    }
}

template void aefdtd_sim::make_step_args<double, uint8_t>(StepArgs<double, uint8_t> &, StepArgs<double, uint8_t> &,
                                                           const StepScalars *, int);
template void aefdtd_sim::make_step_args<double, uint16_t>(StepArgs<double, uint16_t> &, StepArgs<double, uint16_t> &,
                                                            const StepScalars *, int);
template void aefdtd_sim::make_step_args<float, uint8_t>(StepArgs<float, uint8_t> &, StepArgs<float, uint8_t> &,
                                                          const StepScalars *, int);
template void aefdtd_sim::make_step_args<float, uint16_t>(StepArgs<float, uint16_t> &, StepArgs<float, uint16_t> &,
                                                           const StepScalars *, int);
template void aefdtd_sim::make_sensor_args<double>(SensorStepArgs<double> &, const StepScalars *);
template void aefdtd_sim::make_sensor_args<float>(SensorStepArgs<float> &, const StepScalars *);
// used by the fused segments (fused.cpp)
template void aefdtd_sim::launch_pending<double>(PlaneSensor &, cudaStream_t);
template void aefdtd_sim::launch_pending<float>(PlaneSensor &, cudaStream_t);
template int aefdtd_sim::launch_maps<double>(int, int, const double *, const StepScalars *, cudaStream_t);
template int aefdtd_sim::launch_maps<float>(int, int, const double *, const StepScalars *, cudaStream_t);

// Enqueues the kernels of L consecutive steps on the stream: for each step
// the E half-step (interior + boundary items), the H half-step, and the fused
// sensor launch; then the plane-sum reduction of the L steps and, when a DFT
// buffer fills, its accumulation. `tbl` is the device table of the L steps'
// scalars. With record = true per-step timing events are recorded.
template <typename T, typename Tid>
void aefdtd_sim::enqueue_segment(int L, StepScalars *tbl, bool record) {
    StepArgs<T, Tid> ea, ha, ea_i, ha_i;
    make_step_args(ea, ha, tbl);
    if (obl) make_step_args(ea_i, ha_i, tbl, 1);   // the oblique driver's imaginary grid
    const int4 *wi = items.as<int4>();
    int groups = group_kernels(wsE) + group_kernels(wsH);
    if (obl) groups *= 2;
    SensorStepArgs<T> sa;
    make_sensor_args(sa, tbl);
    // field sensors: this segment's phase rows (same table slot as tbl)
    bool maps_e = false, maps_h = false;
    for (auto *m : fmaps) {
        maps_e |= m->dev.kind != kMapPlane || !m->dev.mag;
        maps_h |= m->dev.kind == kMapBlock || (m->dev.kind == kMapPlane && m->dev.mag);
    }
    const double *fm_coef =
        fmaps.empty() ? nullptr
                      : fm_tbl.as<double>() + size_t(tbl - tables.as<StepScalars>()) * kMaxMaps * 4;
    // Sensor work of step q runs in two parts (sensors.cuh, sensor_step): part 0
    // (plane sums, E samples) reads E only and runs beside H(q); part 1 (H
    // samples) reads H only and runs beside E(q+1). H(q+1) and any DFT flush
    // wait for part 1. Timing events sit on `stream` between the joins, so a
    // phase's time covers the branches that run beside it.
    const bool conc = concurrent_groups && !(record && timing_mode == 2);
    // group timing: each group of a half-step alone on the main stream between two events
    auto timed_groups = [&](int q, int half, const WorkSplit &w, auto &&launch) {
        for (int g = 0; g < kGroups; g++) {
            if (w.n[g] <= 0) continue;
            const size_t i = ((size_t(q) * 2 + half) * kGroups + g) * 2;
            AE_CUDA(cudaEventRecord(tge[i], stream));
            launch(g, stream);
            AE_CUDA(cudaEventRecord(tge[i + 1], stream));
        }
    };
    bool h_pending = false;
    // DFT blocks filled in the previous segment accumulate beside this one's
    // steps: they read the other sample-buffer half and only touch acc
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
    auto join_h = [&] {
        if (h_pending) AE_CUDA(cudaStreamWaitEvent(stream, ev_s_join[1], 0));
        h_pending = false;
    };
    auto fork = [&](int k, auto &&launch) {
        AE_CUDA(cudaEventRecord(ev_s_fork[k], stream));
        AE_CUDA(cudaStreamWaitEvent(side_s[k], ev_s_fork[k], 0));
        launch(side_s[k]);
        AE_CUDA(cudaEventRecord(ev_s_join[k], side_s[k]));
    };
    for (int q = 0; q < L; q++) {
        if (record) AE_CUDA(cudaEventRecord(tev[4 * q + 0], stream));
        ea.q = ha.q = ea_i.q = ha_i.q = q;
        if (record && timing_mode == 2) timed_groups(q, 0, wsE, [&](int g, cudaStream_t st) { launch_e_group(ea, wi, wsE, g, st); });
        else run_groups(wsE, [&](int g, cudaStream_t st) { launch_e_group(ea, wi, wsE, g, st); });
        // both grids' E read only H: the imaginary grid follows on the same phase
        if (obl) run_groups(wsE, [&](int g, cudaStream_t st) { launch_e_group(ea_i, wi, wsE, g, st); });
        if (record) AE_CUDA(cudaEventRecord(tev[4 * q + 1], stream));
        // sensors: fed after H in both drivers; plane sums read E of this step
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
        const bool cc = cc_coeff > 0;
        const bool part0 = sa.nbp > 0 || sa.ng > 0 || cc || maps_e || obl;
        sa.part = 0;
        // completion energy of this step reads E only: with part 0, beside H
        auto energy = [&](cudaStream_t st) {
            if (!cc) return;
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
        };
        auto maps = [&](int part, cudaStream_t st) {
            if (part ? maps_h : maps_e) launches += launch_maps<T>(part, q, fm_coef, tbl, st);
        };
        if (part0 && conc)
            fork(0, [&](cudaStream_t st) {
                launches += launch_sensor_step(sa, st);
                energy(st);
                maps(0, st);
                if (obl) launches += launch_obl_sums<T>(q, tbl, st);
            });
        join_h();
        if (record && timing_mode == 2) timed_groups(q, 1, wsH, [&](int g, cudaStream_t st) { launch_h_group(ha, wi, wsH, g, st); });
        else run_groups(wsH, [&](int g, cudaStream_t st) { launch_h_group(ha, wi, wsH, g, st); });
        if (obl) run_groups(wsH, [&](int g, cudaStream_t st) { launch_h_group(ha_i, wi, wsH, g, st); });
        launches += groups;
        if (record) AE_CUDA(cudaEventRecord(tev[4 * q + 2], stream));
        if (part0) {
            if (conc) {
                AE_CUDA(cudaStreamWaitEvent(stream, ev_s_join[0], 0));
            } else {
                launches += launch_sensor_step(sa, stream);
                energy(stream);
                maps(0, stream);
                if (obl) launches += launch_obl_sums<T>(q, tbl, stream);
            }
        }
        if (sa.ng > 0 || maps_h) {
            sa.part = 1;
            if (conc) {
                fork(1, [&](cudaStream_t st) {
                    launches += launch_sensor_step(sa, st);
                    maps(1, st);
                });
                h_pending = true;
            } else {
                launches += launch_sensor_step(sa, stream);
                maps(1, stream);
            }
        }
        for (PlaneSensor *ps : sensors) {
            ps->nbuf++;
            ps->step++;
            if (ps->nbuf == dft_k) {
                // a filled half: accumulated at the next segment's start (or on a read)
                PlaneSensor &s = *ps;
                if (s.pending) launch_pending<T>(s, stream);
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
    join_h();
    if (f_pending) AE_CUDA(cudaStreamWaitEvent(stream, ev_f_join, 0));
    if (normal) {
        launch_plane_reduce(psum_partial.as<double>(), sa.nbp, tbl, psums.as<double>(), L, stream);
        launches++;
    }
    if (cc_coeff > 0 && !ccft) {
        launch_energy_reduce(cc_partial.as<double>(), cc_nb, tbl, cc_hist.as<double>(), L, stream);
        launches++;
    }
    if (obl) {
        launch_obl_reduce(obl->part.as<double>(), obl->nb, tbl, obl->hist.as<double>(), L, stream);
        launches++;
    }
}

// CompletionSensor::completion_check in energy mode (s_completion.cpp:39-43,
// 121-130) after check step t = tstep - 1: the energies since the last check
// update the running maximum; the run completes when the last energy is below
// coeff times the maximum, once tstep >= 2 max(Nx, Ny, Nz).
// CompletionSensor::completion_check in FT mode (s_completion.cpp:45-121),
// FP64 on the host over the device ring, in the reference's order (its six
// averages carry over from one probe to the next, as there).
bool aefdtd_sim::ft_check() {
    CompletionFT &c = *ccft;
    const int step = tstep - c.step0;   // the sensor's step after this step's feed
    if (step < 2 * std::max(Nx, std::max(Ny, Nz))) return false;
    const size_t n = size_t(6) * c.np * c.n_avg;
    c.ring_host.resize(n);
    AE_CUDA(cudaMemcpyAsync(c.ring_host.data(), c.ring.p, n * 8, cudaMemcpyDeviceToHost, stream));
    AE_CUDA(cudaStreamSynchronize(stream));
    return ft_eval(c.ring_host.data(), step);
}

// The FT-mode decision over a host copy of the ring (layout [6][np][n_avg]),
// `step` the sensor's step after the checked step's feed.
bool aefdtd_sim::ft_eval(const double *ring, int step) {
    CompletionFT &c = *ccft;
    if (step < 2 * std::max(Nx, std::max(Ny, Nz))) return false;
    auto R = [&](int comp, int i, int j) { return ring[(size_t(comp) * c.np + i) * c.n_avg + j]; };
    double av[6] = {0, 0, 0, 0, 0, 0};
    int N_ok = 0;
    for (int i = 0; i < c.np; i++) {
        for (int j = 0; j < c.n_avg; j++)
            for (int d = 0; d < 6; d++) av[d] += R(d, i, j);
        for (int d = 0; d < 6; d++) av[d] = std::abs(av[d] / (c.n_avg + 0.0));
        // var_max(Ex_r, Ey_r, Ez_r, Ex_i, Ey_i, Ez_i): max(a, max(b, ...))
        double avg_max = av[5];
        for (int d = 4; d >= 0; d--) avg_max = std::max(av[d], avg_max);
        int g = 0;
        for (int d = 0; d < 6; d++)
            if (avg_max == av[d]) { g = d; break; }
        double t_min = R(g, i, 0), t_max = R(g, i, 0);
        for (int k = 0; k < c.n_avg; k++) {
            t_min = std::min(t_min, R(g, i, k));
            t_max = std::max(t_max, R(g, i, k));
        }
        const double span = std::abs(t_max - t_min);
        if (span <= avg_max * cc_coeff) N_ok++;
    }
    const double ok_rat = N_ok / (c.np + 0.0);
    c.open_ratio = 1.0 - ok_rat;
    return ok_rat >= 0.9;
}

void aefdtd_sim::completion_check() {
    if (ccft) {
        if (ft_check()) {
            cc_done = true;
            cc_stop = tstep - 1;
        }
        return;
    }
    const int n = tstep - cc_read;
    if (n > 0) {
        std::vector<double> e(n);
        AE_CUDA(cudaMemcpyAsync(e.data(), cc_hist.as<double>() + cc_read, n * sizeof(double), cudaMemcpyDeviceToHost,
                                stream));
        AE_CUDA(cudaStreamSynchronize(stream));
        for (double x : e) cc_max = std::max(cc_max, x);
        cc_last = e.back();
        cc_read = tstep;
    }
    if (tstep < 2 * std::max(Nx, std::max(Ny, Nz))) return;
    if (cc_last / cc_max < cc_coeff) {
        cc_done = true;
        cc_stop = tstep - 1;
    }
}

template <typename T, typename Tid>
void aefdtd_sim::run_steps(int n) {
    // the staged kernels' tensor maps bake in the field and id arrays
    if (!work_dirty && (wsE.tma || wsH.tma) && !tma_maps_current()) work_dirty = true;
    if (work_dirty) { build_work(); graphs_dirty = true; fwork_dirty = true; }
    const bool fused = fused_eligible();
    if (fused) {
        if (fwork_dirty) build_fused_work();
        ensure_other_set();
    }
    if (graphs_dirty) drop_graphs();
    // capacity of the plane-sum history
    if (normal && tstep + n > psums_cap) {
        // sized to the run length Nt (the reference's 12 Grid1(Nt) histories), grown past it
        int cap = std::max(tstep + n, std::max(2 * psums_cap, std::max(Nt, 1024)));
        DBuf nb;
        nb.alloc(size_t(cap) * 12 * 8, dev_bytes);
        if (psums.p) AE_CUDA(cudaMemcpyAsync(nb.p, psums.p, size_t(psums_cap) * 12 * 8, cudaMemcpyDeviceToDevice, stream));
        AE_CUDA(cudaStreamSynchronize(stream));
        psums.release(dev_bytes);
        psums = nb;
        psums_cap = cap;
        graphs_dirty = true;
        drop_graphs();
    }
    if (obl && tstep + n > obl->cap) {
        obl_ensure(tstep + n);   // incident sums and R/T history (pointers the graphs bake in)
        graphs_dirty = true;
        drop_graphs();
    }
    if (cc_coeff > 0) {
        if (cc_done) return;   // completed: the driver's loop has ended
        if (!ccft && tstep + n > cc_cap) {
            const int cap = std::max(tstep + n, std::max(2 * cc_cap, std::max(Nt, 1024)));
            DBuf nb;
            nb.alloc(size_t(cap) * 8, dev_bytes);
            if (cc_hist.p) AE_CUDA(cudaMemcpyAsync(nb.p, cc_hist.p, size_t(cc_cap) * 8, cudaMemcpyDeviceToDevice, stream));
            AE_CUDA(cudaStreamSynchronize(stream));
            cc_hist.release(dev_bytes);
            cc_hist = nb;
            cc_cap = cap;
            graphs_dirty = true;
            drop_graphs();
        }
        if (!ccft && !cc_partial.p) {
            cc_nb = std::max(1, std::min(2 * 148, (int)(((long long)Nx * Ny * Nz + 4095) / 4096)));
            cc_partial.alloc(size_t(seg_len) * cc_nb * 8, dev_bytes);
        }
    }
    if (timing) {
        while ((int)tev.size() < 4 * seg_len) {
            cudaEvent_t e;
            AE_CUDA(cudaEventCreate(&e));
            tev.push_back(e);
        }
        while (timing_mode == 2 && (int)tge.size() < seg_len * 2 * kGroups * 2) {
            cudaEvent_t e;
            AE_CUDA(cudaEventCreate(&e));
            tge.push_back(e);
        }
        t_e = t_h = t_s = 0;
        for (auto &r : t_grp) for (auto &x : r) x = 0;
        tev_steps = 0;
    }
    std::vector<StepScalars> host(seg_len);
    int done = 0;
    while (done < n) {
        // a segment ends where a DFT buffer half fills, so captured segments start empty
        int L = std::min(n - done, seg_len);
        bool empty = true;
        for (auto *s : sensors) { L = std::min(L, dft_k - s->nbuf); empty &= s->nbuf == 0; }
        if (cc_coeff > 0) {
            // a segment ends right after each check step t (t % cc_step == 0)
            const int tchk = (tstep + cc_step - 1) / cc_step * cc_step;
            L = std::min(L, tchk + 1 - tstep);
        }
        const int slot = seg_slot;
        seg_slot ^= 1;
        StepScalars *tbl = tables.as<StepScalars>() + size_t(slot) * seg_len;
        const StepScalars *other = tables.as<StepScalars>() + size_t(slot ^ 1) * seg_len;
        // pending blocks a graph may carry: each one filled by the previous
        // (full, other-slot) segment; any other pending block is accumulated now
        bool canon = true, anyp = false;
        for (auto *s : sensors)
            if (s->pending) {
                anyp = true;
                canon &= s->pend_tbl == other && s->pend_n == dft_k && s->pend_half == (s->half ^ 1);
            }
        // with DFT sensors only the first segment after a drain has no pending
        // block: it runs as direct launches instead of a graph used once
        const bool full = (L == seg_len) && empty && !timing && use_graphs && !(sensors.size() && !anyp);
        if (full && anyp && !canon) {
            for (auto *s : sensors) launch_pending<T>(*s, stream);
            anyp = false;
        }
        for (int q = 0; q < L; q++) fill_scalars(tstep + q, q, host[q]);
        AE_CUDA(cudaMemcpyAsync(tbl, host.data(), sizeof(StepScalars) * L, cudaMemcpyHostToDevice, stream));
        if (ccft && cc_coeff > 0) {
            // CompletionSensor::deep_feed's phases e^{i w step Dt} (s_completion.cpp:149)
            CompletionFT &c = *ccft;
            c.rows.resize(size_t(L) * c.np * 2);
            const cplx Im(0, 1);
            for (int q = 0; q < L; q++) {
                const int step = tstep + q - c.step0;
                for (int p = 0; p < c.np; p++) {
                    const cplx coeff = std::exp(c.w[p] * step * Dt * Im);
                    c.rows[(size_t(q) * c.np + p) * 2] = coeff.real();
                    c.rows[(size_t(q) * c.np + p) * 2 + 1] = coeff.imag();
                }
            }
            AE_CUDA(cudaMemcpyAsync(c.ctab.as<double>() + size_t(slot) * seg_len * c.np * 2, c.rows.data(),
                                    c.rows.size() * sizeof(double), cudaMemcpyHostToDevice, stream));
        }
        if (!fmaps.empty()) {
            map_rows.assign(size_t(L) * kMaxMaps * 4, 0.0);
            fill_map_phases(tstep, L, map_rows.data());
            AE_CUDA(cudaMemcpyAsync(fm_tbl.as<double>() + size_t(slot) * seg_len * kMaxMaps * 4, map_rows.data(),
                                    map_rows.size() * sizeof(double), cudaMemcpyHostToDevice, stream));
        }
        auto enqueue = [&](bool record) {
            if (fused) enqueue_segment_fused<T, Tid>(L, tbl, record);
            else enqueue_segment<T, Tid>(L, tbl, record);
        };
        // an odd fused segment leaves the current state in the other set (graphs hold even segments)
        auto settle = [&] {
            if (fused && L % 2) swap_sets();
        };
        if (timing) {
            enqueue(true);
            settle();
            timed_fused = fused;
            if (fused) {
                // cells per fused group, in the slots the timings use
                for (auto &r : grp_cells) for (auto &x : r) x = 0;
                for (int g = 0; g < kFusedGroups; g++) grp_cells[0][g] = fcells[g];
            }
            accumulate_timing(L);
        } else if (full) {
            uint64_t key = uint64_t(slot) | (uint64_t(anyp) << 1);
            // fused segments bake in which buffers hold the current set
            key |= (uint64_t(fused) << 62) | (uint64_t(fused && set_b) << 61);
            for (size_t k = 0; k < sensors.size(); k++) key |= uint64_t(sensors[k]->half) << (2 + k);
            // host-side effect of a full segment on the sensors (what enqueue_segment does)
            auto advance = [&] {
                for (auto *s : sensors) {
                    s->pending = true;
                    s->pend_half = s->half;
                    s->pend_n = dft_k;
                    s->pend_step0 = s->step;
                    s->pend_tbl = tbl;
                    s->half ^= 1;
                    s->step += L;
                    s->buf_step0 = s->step;
                    s->nbuf = 0;
                }
            };
            cudaGraphExec_t &gx = graph_exec[key];
            if (!gx) {
                // capture once; the sequence reads every per-step value from the table
                std::vector<PlaneSensor> snap;
                for (auto *s : sensors) snap.push_back(*s);
                uint64_t l0 = launches;
                AE_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
                enqueue(false);
                cudaGraph_t gr = nullptr;
                AE_CUDA(cudaStreamEndCapture(stream, &gr));
                AE_CUDA(cudaGraphInstantiate(&gx, gr, cudaGraphInstantiateFlagUseNodePriority));
                cudaGraphDestroy(gr);
                graph_launches = launches - l0;
                launches = l0;
                for (size_t k = 0; k < sensors.size(); k++) {
                    PlaneSensor &d = *sensors[k];
                    const PlaneSensor &o = snap[k];
                    d.step = o.step; d.nbuf = o.nbuf; d.buf_step0 = o.buf_step0; d.half = o.half;
                    d.pending = o.pending; d.pend_half = o.pend_half; d.pend_n = o.pend_n;
                    d.pend_step0 = o.pend_step0; d.pend_tbl = o.pend_tbl;
                }
            }
            AE_CUDA(cudaGraphLaunch(gx, stream));
            launches += graph_launches;
            advance();
            settle();
        } else {
            enqueue(false);
            settle();
        }
        for (auto &o : oscs) o.step += L;
        tstep += L;
        done += L;
        if (cc_coeff > 0 && (tstep - 1) % cc_step == 0) {
            completion_check();
            if (cc_done) break;
        }
    }
    AE_CUDA(cudaGetLastError());
}

void aefdtd_sim::drop_graphs() {
    for (auto &g : graph_exec)
        if (g.second) reap_graph(g.second, device);
    graph_exec.clear();
    graphs_dirty = false;
}

namespace aefdtd {
namespace {
// The reaper: one detached thread and a queue. At process exit (an atexit
// handler registered after the CUDA runtime's, so it runs first) it stops
// between two destroys and leaves the rest to the driver's teardown.
struct Reaper {
    std::mutex mu;
    std::condition_variable cv;
    std::deque<std::pair<cudaGraphExec_t, int>> q;
    bool exiting = false;
};
Reaper &reaper() {
    static Reaper *r = [] {
        auto *x = new Reaper();   // never deleted: outlives static destruction
        std::atexit([] {
            Reaper &R = reaper();
            std::lock_guard<std::mutex> lock(R.mu);
            R.exiting = true;
            R.q.clear();
            R.cv.notify_all();
        });
        std::thread([x] {
            std::unique_lock<std::mutex> lock(x->mu);
            for (;;) {
                x->cv.wait(lock, [x] { return x->exiting || !x->q.empty(); });
                if (x->exiting) return;
                const auto item = x->q.front();
                x->q.pop_front();
                cudaSetDevice(item.second);
                cudaGraphExecDestroy(item.first);
            }
        }).detach();
        return x;
    }();
    return *r;
}
}  // namespace

void reap_graph(cudaGraphExec_t g, int device) {
    Reaper &R = reaper();
    std::lock_guard<std::mutex> lock(R.mu);
    if (R.exiting) return;
    R.q.emplace_back(g, device);
    R.cv.notify_one();
}
}  // namespace aefdtd

void aefdtd_sim::accumulate_timing(int L) {
    AE_CUDA(cudaEventSynchronize(tev[4 * L - 1]));
    for (int q = 0; q < L; q++) {
        float a = 0, b = 0, c = 0;
        AE_CUDA(cudaEventElapsedTime(&a, tev[4 * q + 0], tev[4 * q + 1]));
        AE_CUDA(cudaEventElapsedTime(&b, tev[4 * q + 1], tev[4 * q + 2]));
        AE_CUDA(cudaEventElapsedTime(&c, tev[4 * q + 2], tev[4 * q + 3]));
        t_e += a; t_h += b; t_s += c;
        if (timing_mode == 2)
            for (int half = 0; half < 2; half++)
                for (int g = 0; g < kGroups; g++) {
                    const WorkSplit &w = half == 0 ? wsE : wsH;
                    if (timed_fused) {
                        // fused group g is reported in E-side slot g
                        if (half == 1 || fnum[g] <= 0) continue;
                    } else if (w.n[g] <= 0) {
                        continue;
                    }
                    const size_t i = ((size_t(q) * 2 + half) * kGroups + g) * 2;
                    float d = 0;
                    AE_CUDA(cudaEventElapsedTime(&d, tge[i], tge[i + 1]));
                    t_grp[half][g] += d;
                }
    }
    tev_steps += L;
}

// Work lists of the half-step kernels. The grid is cut into items of 32 x 4
// columns by kchunk planes; an item is "boundary" when any of its cells is in
// a CPML range or PEC plane of either half-step, on the injection plane, in
// an oscillator box, or of a dispersive material; all others are "interior"
// and run the curl-only kernels. Groups in pair_mask (two cells per thread,
// even Nx only) take 64-column items where both 32-column tiles of a pair
// fall in the group, and 32-column items flagged kHalfItem elsewhere.
void aefdtd_sim::build_work() {
    // host-only list index of the x/y-CPML group's y-only tiles (two cells per
    // thread); appended to the x/y-CPML group's items, counted in WorkSplit::n_py
    constexpr int kGroupPY = kGroups;
    unsigned pmask = (Nx % 2 == 0) ? pair_mask & ((1u << kGroupInterior) | (1u << kGroupPmlZ)) : 0u;
    if (Nx % 2 == 0 && (pair_mask & (1u << kGroupPmlXY))) pmask |= 1u << kGroupPY;
    const int tx = kTileXHost, ty = tile_y;
    const int ntx = (Nx + tx - 1) / tx, nty = (Ny + ty - 1) / ty;
    const long long tiles = (long long)ntx * nty;
    if (kchunk_override > 0) kchunk = kchunk_override;
    else {
        // 8 planes per item unless that leaves fewer than three waves of
        // 148 SMs x 12 resident items; never fewer than 4 planes
        long long want = 148LL * 12 * 3;
        kchunk = 8;
        while (kchunk > 4 && tiles * ((Nz + kchunk - 1) / kchunk) < want) kchunk /= 2;
    }
    const int nch = (Nz + kchunk - 1) / kchunk;
    // feature mask per (tile, plane) (kF* of yee.cuh); oscillator boxes matter to E only
    // kPXY: an x-CPML cell or PEC plane; kPY: a y-CPML cell or PEC plane (both
    // take the x/y-CPML group; tiles with kPY alone may take the pair kernel)
    constexpr unsigned kPXY = 1, kPZ = 2, kDISP = 4, kMISC = 8, kOSC = 16, kPY = 32;
    std::vector<unsigned char> feat(size_t(tiles) * Nz, 0);
    auto mark_range = [&](int x0, int x1, int y0, int y1, int z0, int z1, unsigned f) {   // half-open cell ranges
        if (x0 >= x1 || y0 >= y1 || z0 >= z1) return;
        for (int k = z0; k < z1; k++)
            for (int b = y0 / ty; b <= (y1 - 1) / ty; b++)
                for (int a = x0 / tx; a <= (x1 - 1) / tx; a++) feat[(size_t(k) * nty + b) * ntx + a] |= f;
    };
    const bool px = pml[0] || pml[1], py = pml[2] || pml[3], pz = pml[4] || pml[5];
    if (px) {
        mark_range(0, std::max(pml[0], 1), 0, Ny, 0, Nz, kPXY);
        mark_range(Nx - std::max(pml[1], 1), Nx, 0, Ny, 0, Nz, kPXY);
    }
    if (py) {
        mark_range(0, Nx, 0, std::max(pml[2], 1), 0, Nz, kPY);
        mark_range(0, Nx, Ny - std::max(pml[3], 1), Ny, 0, Nz, kPY);
    }
    if (pz) {
        mark_range(0, Nx, 0, Ny, 0, std::max(pml[4], 1), kPZ);
        mark_range(0, Nx, 0, Ny, Nz - std::max(pml[5], 1), Nz, kPZ);
    }
    if (normal) mark_range(0, Nx, 0, Ny, zs_e - 1, zs_e, kMISC);
    if (obl) {
        // oblique driver: Bloch wrap columns and rows (both half-steps) and the
        // Bloch_Wideband planes z2 - 1 (H) and z2 (E)
        mark_range(0, 1, 0, Ny, 0, Nz, kMISC);
        mark_range(Nx - 1, Nx, 0, Ny, 0, Nz, kMISC);
        mark_range(0, Nx, 0, 1, 0, Nz, kMISC);
        mark_range(0, Nx, Ny - 1, Ny, 0, Nz, kMISC);
        mark_range(0, Nx, 0, Ny, obl->z2 - 1, obl->z2 + 1, kMISC);
    }
    for (auto &o : oscs) mark_range(o.box[0], o.box[1], o.box[2], o.box[3], o.box[4], o.box[5], kOSC);
    for (unsigned m = 0; m < Nmat; m++) {
        HostMat &h = mats[m];
        if (!(h.rc && h.np > 0)) continue;
        for (int k = h.z1; k <= h.z2; k++)
            for (int j = h.y1; j <= h.y2; j++) {
                const uint32_t *row = &map[size_t(j) * Nx + size_t(k) * Nx * Ny];
                for (int i = h.x1; i <= h.x2; i++)
                    if (row[i] == m) feat[(size_t(k) * nty + j / ty) * ntx + i / tx] |= kDISP;
            }
    }
    // AEFDTD_ALL_BOUNDARY=1 routes every item through the general kernels (same results)
    const bool all_boundary = std::getenv("AEFDTD_ALL_BOUNDARY") != nullptr;
    // group of a (tile, plane) for the E and the H half-step
    // AEFDTD_MERGE_PZ=1: curl-only items run with the z-CPML items' kernels (one launch for both)
    const bool merge_pz = std::getenv("AEFDTD_MERGE_PZ") != nullptr;
    // AEFDTD_MERGE_DISP=1: dispersive-only items run with the general kernels (one launch for both)
    const bool merge_disp = std::getenv("AEFDTD_MERGE_DISP") != nullptr;
    auto group_e = [&](unsigned f) {
        if (all_boundary) return (int)kGroupAll;
        f = (f & ~kOSC) | ((f & kOSC) ? kMISC : 0);
        f = (f & ~kPY) | ((f & kPY) ? kPXY : 0);
        if (f == 0) return merge_pz ? (int)kGroupPmlZ : (int)kGroupInterior;
        if (f == kPZ) return (int)kGroupPmlZ;
        if (f == kDISP) return merge_disp ? (int)kGroupAll : (int)kGroupDisp;
        if (f == kPXY || f == (kPXY | kPZ)) return (int)kGroupPmlXY;
        return (int)kGroupAll;
    };
    auto group_h = [&](unsigned f) {
        if (all_boundary) return (int)kGroupAll;
        f = (f & ~kPY) | ((f & kPY) ? kPXY : 0);
        f &= (kPXY | kPZ | kMISC);
        if (f == 0) return merge_pz ? (int)kGroupPmlZ : (int)kGroupInterior;
        if (f == kPZ) return (int)kGroupPmlZ;
        if (f == kPXY || f == (kPXY | kPZ)) return (int)kGroupPmlXY;
        return (int)kGroupAll;
    };
    // Staged interior units: 64 x 8 tiles (two 32-column tiles by 8 / ty
    // rows) inside the grid, runs of planes where every covered tile is
    // curl-only for the half-step, cut into units of at most tma_unit
    // planes. Their tiles are taken out of the lists below; the other
    // curl-only tiles run with the z-CPML group's kernels (which leave cells
    // outside the z-CPML ranges at the curl update).
    bool tma = tma_possible();
    std::vector<unsigned char> taken[2];
    std::vector<int> tunits[2];
    long long tcells[2] = {0, 0};
    if (tma) {
        const int rb = kTmaTileY / ty, nA = Nx / kTmaTileX, nB = Ny / kTmaTileY;
        for (int half = 0; half < 2; half++) {
            taken[half].assign(size_t(tiles) * Nz, 0);
            // curl-only or z-CPML-only planes of every covered tile
            auto interior = [&](int A, int B, int k) {
                for (int bb = 0; bb < rb; bb++)
                    for (int aa = 0; aa < 2; aa++) {
                        const unsigned f = feat[(size_t(k) * nty + B * rb + bb) * ntx + 2 * A + aa];
                        const int g = half == 0 ? group_e(f) : group_h(f);
                        if (g != kGroupInterior && !(g == kGroupPmlZ && tma_pz)) return false;
                    }
                return true;
            };
            std::vector<int4> runs;   // (x0, y0, k0, k1) of every curl-only run
            long long planes = 0;
            for (int B = 0; B < nB; B++)
                for (int A = 0; A < nA; A++)
                    for (int k = 0; k < Nz;) {
                        if (!interior(A, B, k)) { k++; continue; }
                        int ke = k + 1;
                        while (ke < Nz && interior(A, B, ke)) ke++;
                        runs.push_back(make_int4(A * kTmaTileX, B * kTmaTileY, k, ke));
                        for (int kk = k; kk < ke; kk++)
                            for (int bb = 0; bb < rb; bb++)
                                for (int aa = 0; aa < 2; aa++) taken[half][(size_t(kk) * nty + B * rb + bb) * ntx + 2 * A + aa] = 1;
                        tcells[half] += (long long)(ke - k) * kTmaTileX * kTmaTileY;
                        planes += ke - k;
                        k = ke;
                    }
            // Guided sizes: CTAs take units in list order, so a unit's length
            // follows the planes still unassigned, R / (2 x CTAs) capped at
            // tma_unit: long units first, single planes at the end, and the
            // CTAs finish within about one plane of each other.
            int nsm = 148;
            AE_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
            const long long ctas = (long long)std::max(1, tma_ctas) * std::max(1, nsm - tma_reserve);
            // The H list runs top plane first (the planes E touched last), its
            // runs cut from the top down.
            if (half == 1) std::reverse(runs.begin(), runs.end());
            long long rem = planes;
            for (const int4 &r : runs)
                for (int k = r.z, ke = r.w; k < ke;) {
                    const int len = (int)std::clamp<long long>(rem / (2 * ctas), 1, tma_unit);
                    if (half == 0) {
                        const int zb = std::min(ke, k + len);
                        tunits[half].insert(tunits[half].end(), {r.x, r.y, k, zb});
                        rem -= zb - k;
                        k = zb;
                    } else {
                        const int za = std::max(k, ke - len);
                        tunits[half].insert(tunits[half].end(), {r.x, r.y, za, ke});
                        rem -= ke - za;
                        ke = za;
                    }
                }
        }
        tma = !tunits[0].empty() || !tunits[1].empty();
        if (tma && !build_tma_maps()) tma = false;
        if (!tma) {
            taken[0].clear(); taken[1].clear();
            tunits[0].clear(); tunits[1].clear();
            tcells[0] = tcells[1] = 0;
        }
    }
    // items: within each tile (or pair of tiles) and z-chunk, runs of planes
    // of one group; dispersive E planes one plane per item (their cells carry
    // the pole state)
    std::vector<int> v[2][kGroups + 1];
    const int step_a = pmask ? 2 : 1;
    for (int c = 0; c < nch; c++)
        for (int b = 0; b < nty; b++)
            for (int a = 0; a < ntx; a += step_a) {
                const int z0 = c * kchunk, z1 = std::min(Nz, (c + 1) * kchunk);
                for (int half = 0; half < 2; half++) {
                    // -1: the tile's plane runs in a staged unit
                    auto grp = [&](int t, int k) {
                        const size_t fi = (size_t(k) * nty + b) * ntx + t;
                        if (tma && taken[half][fi]) return -1;
                        const int g = half == 0 ? group_e(feat[fi]) : group_h(feat[fi]);
                        if (g == kGroupPmlXY && ((pmask >> kGroupPY) & 1u) && !(feat[fi] & kPXY)) return kGroupPY;
                        return (tma && g == kGroupInterior) ? (int)kGroupPmlZ : g;
                    };
                    auto emit = [&](int g, int x0, int za, int zb) {
                        std::vector<int> &dst = v[half][g];
                        dst.push_back(x0);
                        dst.push_back(b * ty);
                        dst.push_back(za);
                        dst.push_back(zb);
                    };
                    // runs of one group within [za, zb) of tile t
                    auto runs = [&](int t, int za, int zb) {
                        int z = za;
                        while (z < zb) {
                            const int g = grp(t, z);
                            int ze = z + 1;
                            if (!(half == 0 && g == kGroupDisp))
                                while (ze < zb && grp(t, ze) == g) ze++;
                            if (g >= 0) emit(g, t * tx | ((pmask >> g) & 1u ? kHalfItem : 0), z, ze);
                            z = ze;
                        }
                    };
                    if (!pmask) {
                        runs(a, z0, z1);
                        continue;
                    }
                    const bool right = a + 1 < ntx;
                    // plane k pairs when both tiles (or the last, lone tile) are in one pair group
                    auto paired = [&](int k) {
                        const int g = grp(a, k);
                        return g >= 0 && ((pmask >> g) & 1u) && (!right || grp(a + 1, k) == g);
                    };
                    int z = z0;
                    while (z < z1) {
                        int ze = z + 1;
                        if (paired(z)) {
                            const int g = grp(a, z);
                            while (ze < z1 && paired(ze) && grp(a, ze) == g) ze++;
                            emit(g, a * tx, z, ze);
                        } else {
                            while (ze < z1 && !paired(ze)) ze++;
                            runs(a, z, ze);
                            if (right) runs(a + 1, z, ze);
                        }
                        z = ze;
                    }
                }
            }
    // The H lists run in reverse (top plane first): each half-step starts on
    // the planes the previous one touched last, which are still in L2. Pays
    // when the fields are about the size of L2 (126 MB) or smaller.
    const size_t field_bytes = size_t(6) * Nx * Ny * Nz * (fp64 ? 8 : 4);
    if (h_reverse > 0 || (h_reverse < 0 && field_bytes <= (size_t(128) << 20)))
        for (int g = 0; g <= kGroups; g++) {
            std::vector<int> &h = v[1][g];
            const size_t n = h.size() / 4;
            for (size_t a = 0, b = n ? n - 1 : 0; a < b; a++, b--)
                for (int c = 0; c < 4; c++) std::swap(h[4 * a + c], h[4 * b + c]);
        }
    std::vector<int> all;
    for (int half = 0; half < 2; half++) {
        WorkSplit &w = half == 0 ? wsE : wsH;
        w.unroll = zunroll;
        w.tile_y = tile_y;
        w.pair_mask = pmask;
        auto cells_of = [&](int g) {
            long long c = 0;
            for (size_t k = 0; k < v[half][g].size(); k += 4) {
                const int *it = &v[half][g][k];
                const int x0 = it[0] & ~kHalfItem, gw = ((pmask >> g) & 1u) && !(it[0] & kHalfItem) ? 2 * tx : tx;
                c += (long long)(std::min(x0 + gw, Nx) - x0) * (std::min(it[1] + ty, Ny) - it[1]) * (it[3] - it[2]);
            }
            return c;
        };
        for (int g = 0; g < kGroups; g++) {
            w.off[g] = (int)(all.size() / 4);
            w.n[g] = (int)(v[half][g].size() / 4);
            all.insert(all.end(), v[half][g].begin(), v[half][g].end());
            grp_cells[half][g] = cells_of(g);
            if (g == kGroupPmlXY) {
                // the y-only pair items follow the group's one-cell items
                w.n_py = (int)(v[half][kGroupPY].size() / 4);
                w.n[g] += w.n_py;
                all.insert(all.end(), v[half][kGroupPY].begin(), v[half][kGroupPY].end());
                grp_cells[half][g] += cells_of(kGroupPY);
            }
        }
    }
    // staged units: E then H
    for (int half = 0; half < 2; half++) {
        WorkSplit &w = half == 0 ? wsE : wsH;
        w.tma = nullptr;
        tma_plan[half].nunits = 0;
    }
    if (tma) {
        std::vector<int> tu = tunits[0];
        tu.insert(tu.end(), tunits[1].begin(), tunits[1].end());
        tma_units.alloc(tu.size() * sizeof(int), dev_bytes);
        AE_CUDA(cudaMemcpy(tma_units.p, tu.data(), tu.size() * sizeof(int), cudaMemcpyHostToDevice));
        if (!tma_ctr.p) tma_ctr.alloc(4 * sizeof(int), dev_bytes);
        AE_CUDA(cudaMemsetAsync(tma_ctr.p, 0, 4 * sizeof(int), stream));
        int nsm = 148;
        AE_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
        for (int half = 0; half < 2; half++) {
            TmaPlan &p = tma_plan[half];
            p.nunits = (int)(tunits[half].size() / 4);
            p.units = tma_units.as<int4>() + (half ? tunits[0].size() / 4 : 0);
            p.ctr = tma_ctr.as<int>() + 2 * half;
            // tma_ctas 0: one unit per CTA; else units taken in turn by tma_ctas CTAs per SM
            p.grid = tma_ctas == 0 ? p.nunits : std::min(p.nunits, tma_ctas * std::max(1, nsm - tma_reserve));
            p.stages = tma_stages;
            p.wait_cycles = tma_wait_cycles;
            p.withhold = tma_withhold;
            p.cells = tcells[half];
            if (p.nunits == 0) continue;
            WorkSplit &w = half == 0 ? wsE : wsH;
            w.tma = &p;
            w.n[kGroupInterior] = p.grid;
            grp_cells[half][kGroupInterior] = p.cells;
        }
    }
    items_host = all;
    items.alloc(std::max<size_t>(all.size(), 4) * sizeof(int), dev_bytes);
    graphs_dirty = true;   // captured segments point at the old lists
    if (!all.empty()) AE_CUDA(cudaMemcpy(items.p, all.data(), all.size() * sizeof(int), cudaMemcpyHostToDevice));
    work_dirty = false;
}

// Reads the device error flag set by a bounded wait that ran out.
void aefdtd_sim::check_err() {
    int h = 0;
    AE_CUDA(cudaMemcpyAsync(&h, err.p, sizeof(int), cudaMemcpyDeviceToHost, stream));
    AE_CUDA(cudaStreamSynchronize(stream));
    if (h) {
        AE_CUDA(cudaMemsetAsync(err.p, 0, sizeof(int), stream));
        // a staged launch that gave up may have left its unit counters set
        if (tma_ctr.p) AE_CUDA(cudaMemsetAsync(tma_ctr.p, 0, tma_ctr.n, stream));
        fail(AEFDTD_TIMEOUT, "a bounded device wait ran out");
    }
}

void aefdtd_sim::step(int n) {
    if (n < 0) fail(AEFDTD_BAD_ARG, "negative step count");
    if (!map_set) fail(AEFDTD_NOT_READY, "no material map");
    if (g.mode == AEFDTD_MODE_NORMAL && !normal) fail(AEFDTD_NOT_READY, "normal mode needs aefdtd_setup_normal");
    if (g.mode == AEFDTD_MODE_OBLIQUE && !obl) fail(AEFDTD_NOT_READY, "oblique mode needs aefdtd_setup_oblique");
    set_device();
    finalize_tables();
    if (fp64) {
        if (id_bytes == 1) run_steps<double, uint8_t>(n); else run_steps<double, uint16_t>(n);
    } else {
        if (id_bytes == 1) run_steps<float, uint8_t>(n); else run_steps<float, uint16_t>(n);
    }
}

void aefdtd_sim::zero_state() {
    set_device();
    cc_done = false;
    cc_stop = -1;
    cc_read = 0;
    cc_last = cc_max = 0;
    for (auto &b : F) if (b.p) AE_CUDA(cudaMemsetAsync(b.p, 0, b.n, stream));
    for (auto &b : psiE) if (b.p) AE_CUDA(cudaMemsetAsync(b.p, 0, b.n, stream));
    for (auto &b : psiH) if (b.p) AE_CUDA(cudaMemsetAsync(b.p, 0, b.n, stream));
    if (psi.p) AE_CUDA(cudaMemsetAsync(psi.p, 0, psi.n, stream));
    if (tma_ctr.p) AE_CUDA(cudaMemsetAsync(tma_ctr.p, 0, tma_ctr.n, stream));
    if (obl) {
        for (int c = 0; c < 6; c++) {
            DBuf *b[3] = {&obl->Fi[c], &obl->psiEi[c], &obl->psiHi[c]};
            for (DBuf *x : b) if (x->p) AE_CUDA(cudaMemsetAsync(x->p, 0, x->n, stream));
        }
        if (obl->psi_i.p) AE_CUDA(cudaMemsetAsync(obl->psi_i.p, 0, obl->psi_i.n, stream));
    }
    for (auto *s : sensors) {
        if (s->acc.p) AE_CUDA(cudaMemsetAsync(s->acc.p, 0, s->acc.n, stream));
        s->step = 0; s->nbuf = 0; s->half = 0; s->pending = false;
    }
    for (auto &o : oscs) o.step = 0;
    if (ccft) {
        AE_CUDA(cudaMemsetAsync(ccft->acc.p, 0, ccft->acc.n, stream));
        AE_CUDA(cudaMemsetAsync(ccft->ring.p, 0, ccft->ring.n, stream));
        ccft->step0 = 0;
    }
    for (auto *m : fmaps) {
        if (m->acc.p) AE_CUDA(cudaMemsetAsync(m->acc.p, 0, m->acc.n, stream));
        m->step0 = 0;
        m->dev.step0 = 0;
    }
    tstep = 0;
    AE_CUDA(cudaStreamSynchronize(stream));
}

// ------------------------------------------------------------------------
// C ABI
// ------------------------------------------------------------------------

static thread_local std::string g_create_error;

extern "C" {

aefdtd_status aefdtd_create(const aefdtd_grid_desc *desc, aefdtd_sim **out) {
    if (!desc || !out) return AEFDTD_BAD_ARG;
    *out = nullptr;
    aefdtd_sim *s = new (std::nothrow) aefdtd_sim();
    if (!s) return AEFDTD_OOM;
    aefdtd_status st = guarded(s, [&] { s->construct(desc); });
    if (st != AEFDTD_OK) {
        g_create_error = s->last_error;
        delete s;
        return st;
    }
    *out = s;
    return AEFDTD_OK;
}

aefdtd_status aefdtd_destroy(aefdtd_sim *s) {
    if (!s) return AEFDTD_BAD_ARG;
    if (s->batch) aefdtd::batch_detach(s->batch, s);
    delete s;
    return AEFDTD_OK;
}

const char *aefdtd_last_error(const aefdtd_sim *s) {
    return s ? s->last_error.c_str() : g_create_error.c_str();
}

const char *aefdtd_status_string(aefdtd_status st) {
    switch (st) {
        case AEFDTD_OK: return "ok";
        case AEFDTD_BAD_ARG: return "bad argument";
        case AEFDTD_OOM: return "out of device memory";
        case AEFDTD_TIMEOUT: return "timeout";
        case AEFDTD_CUDA_ERROR: return "CUDA error";
        case AEFDTD_NOT_READY: return "not ready";
        case AEFDTD_NO_DEVICE: return "no CUDA device";
    }
    return "unknown status";
}

aefdtd_status aefdtd_get_dims(const aefdtd_sim *s, aefdtd_dims *o) {
    if (!s || !o) return AEFDTD_BAD_ARG;
    o->nx = s->Nx; o->ny = s->Ny; o->nz = s->Nz;
    o->xs_s = s->xs_s; o->xs_e = s->xs_e; o->ys_s = s->ys_s; o->ys_e = s->ys_e; o->zs_s = s->zs_s; o->zs_e = s->zs_e;
    o->n_materials = (int32_t)s->Nmat;
    o->step = s->tstep;
    o->dt = s->Dt;
    o->device_bytes = s->dev_bytes;
    return AEFDTD_OK;
}

aefdtd_status aefdtd_set_material_map(aefdtd_sim *s, const uint32_t *map, size_t count) {
    if (!s) return AEFDTD_BAD_ARG;
    return guarded(s, [&] { s->set_device(); s->set_map(map, count); });
}

aefdtd_status aefdtd_set_material(aefdtd_sim *s, uint32_t index, const aefdtd_material_desc *m) {
    if (!s) return AEFDTD_BAD_ARG;
    return guarded(s, [&] { s->set_material(index, m); });
}

aefdtd_status aefdtd_setup_normal(aefdtd_sim *s, const aefdtd_normal_desc *nd) {
    if (!s || !nd) return AEFDTD_BAD_ARG;
    return guarded(s, [&] {
        if (s->g.mode != AEFDTD_MODE_NORMAL) fail(AEFDTD_BAD_ARG, "setup_normal needs mode NORMAL");
        if (!s->map_set) fail(AEFDTD_NOT_READY, "set the material map first");
        if (nd->nl < 2 || !(nd->lambda_min > 0) || !(nd->lambda_max > 0)) fail(AEFDTD_BAD_ARG, "bad spectrum");
        s->nd = *nd;
        // normal_incidence.cpp:238-249: superstrate/substrate from the map at
        // (0,0,zs_e) and (0,0,zs_s); ei is eps_inf of the material.
        auto M = [&](int i, int j, int k) { return s->map[i + size_t(j) * s->Nx + size_t(k) * s->Nx * s->Ny]; };
        s->eps_sub = s->mats[M(0, 0, s->zs_s)].ei;
        s->eps_sup = s->mats[M(0, 0, s->zs_e)].ei;
        s->index_sub = std::sqrt(s->eps_sub);
        s->index_sup = std::sqrt(s->eps_sup);
        double pol = nd->polarization == 1 ? 90 : 0;
        s->pulse.init(nd->lambda_min, nd->lambda_max, pol, (s->zs_e - 1) * s->Dz, s->index_sup);
        if (!s->psum_partial.p) s->psum_partial.alloc(size_t(s->seg_len) * kPlaneBlocks * 12 * 8, s->dev_bytes);
        s->graphs_dirty = true;
        s->normal = true;
        s->work_dirty = true;
    });
}

aefdtd_status aefdtd_add_oscillator(aefdtd_sim *s, const aefdtd_source_desc *d, int32_t *id) {
    if (!s || !d) return AEFDTD_BAD_ARG;
    return guarded(s, [&] {
        if (s->g.mode != AEFDTD_MODE_CUSTOM) fail(AEFDTD_BAD_ARG, "oscillators need mode CUSTOM");
        if (s->oscs.size() >= 4) fail(AEFDTD_BAD_ARG, "at most 4 oscillators");
        if (d->orientation < 0 || d->orientation > 5) fail(AEFDTD_BAD_ARG, "bad orientation");
        if (!(d->lambda_min > 0 && d->lambda_max > 0)) fail(AEFDTD_BAD_ARG, "bad spectrum");
        Osc o;
        o.comp = d->orientation <= 1 ? 0 : (d->orientation <= 3 ? 1 : 2);
        // Source::link (sources.cpp:252-283)
        o.box[0] = std::clamp(d->box[0] + s->xs_s, 0, s->Nx); o.box[1] = std::clamp(d->box[1] + s->xs_s, 0, s->Nx);
        o.box[2] = std::clamp(d->box[2] + s->ys_s, 0, s->Ny); o.box[3] = std::clamp(d->box[3] + s->ys_s, 0, s->Ny);
        o.box[4] = std::clamp(d->box[4] + s->zs_s, 0, s->Nz); o.box[5] = std::clamp(d->box[5] + s->zs_s, 0, s->Nz);
        // Oscillator::initialize (sc_oscillator.cpp:69-84)
        double alp = std::sqrt(0.1), bet = 1e-7;
        double w1 = 2.0 * Pi * c_light / d->lambda_max, w2 = 2.0 * Pi * c_light / d->lambda_min;
        o.w0 = (w1 + w2) / 2.0;
        o.dw = std::abs(w2 - w1) / (2.0 * std::sqrt(-std::log(alp)));
        o.tshift = (int)(std::sqrt(-4.0 / (o.dw * o.dw) * std::log(bet)) / s->Dt);
        o.step = s->tstep;
        s->oscs.push_back(o);
        s->work_dirty = true;
        s->graphs_dirty = true;
        if (id) *id = (int32_t)s->oscs.size() - 1;
    });
}

aefdtd_status aefdtd_add_planar_sensor(aefdtd_sim *s, const aefdtd_sensor_desc *d, int32_t *id) {
    if (!s || !d) return AEFDTD_BAD_ARG;
    return guarded(s, [&] {
        if (d->orientation < 0 || d->orientation > 5) fail(AEFDTD_BAD_ARG, "bad orientation");
        if (d->nl < 1) fail(AEFDTD_BAD_ARG, "nl must be positive");
        if (!(d->lambda_min > 0 && d->lambda_max > 0)) fail(AEFDTD_BAD_ARG, "bad spectrum");
        s->set_device();
        PlaneSensor *p = new PlaneSensor();
        p->d = *d;
        p->type = d->orientation;
        // Sensor::link (sensors.cpp:196-230) and SensorFieldHolder::initialize (sensors.cpp:496-527)
        p->x1 = std::clamp(d->box[0] + s->xs_s, 0, s->Nx); p->x2 = std::clamp(d->box[1] + s->xs_s, 0, s->Nx);
        p->y1 = std::clamp(d->box[2] + s->ys_s, 0, s->Ny); p->y2 = std::clamp(d->box[3] + s->ys_s, 0, s->Ny);
        p->z1 = std::clamp(d->box[4] + s->zs_s, 0, s->Nz); p->z2 = std::clamp(d->box[5] + s->zs_s, 0, s->Nz);
        if (p->type <= 1) { p->span1 = p->y2 - p->y1; p->span2 = p->z2 - p->z1; }
        else if (p->type <= 3) { p->span1 = p->x2 - p->x1; p->span2 = p->z2 - p->z1; }
        else { p->span1 = p->x2 - p->x1; p->span2 = p->y2 - p->y1; }
        if (p->span1 <= 0 || p->span2 <= 0) { delete p; fail(AEFDTD_BAD_ARG, "sensor plane is empty"); }
        int plane_i = p->type <= 1 ? p->x1 : (p->type <= 3 ? p->y1 : p->z1);
        int plane_n = p->type <= 1 ? s->Nx : (p->type <= 3 ? s->Ny : s->Nz);
        if (plane_i >= plane_n) { delete p; fail(AEFDTD_BAD_ARG, "sensor plane outside the grid"); }
        p->P = p->span1 * p->span2;
        p->nl = d->nl;
        p->lambda.resize(p->nl);
        p->w.resize(p->nl);
        for (int l = 0; l < p->nl; l++) {
            p->lambda[l] = d->nl > 1 ? d->lambda_min + (d->lambda_max - d->lambda_min) * l / (d->nl - 1.0) : d->lambda_min;
            p->w[l] = 2.0 * Pi * c_light / p->lambda[l];
        }
        size_t es = s->fp64 ? 8 : 4;
        try {
            p->S.alloc(size_t(2) * s->dft_k * 6 * p->P * es, s->dev_bytes);
            p->acc.alloc(size_t(6) * p->nl * p->P * 16, s->dev_bytes);
            p->wdev.alloc(size_t(p->nl) * 8, s->dev_bytes);
            p->WE.alloc(size_t(s->dft_k) * p->nl * 16, s->dev_bytes);
            p->WH.alloc(size_t(s->dft_k) * p->nl * 16, s->dev_bytes);
            p->flux.alloc(size_t(p->nl) * 8, s->dev_bytes);
            AE_CUDA(cudaMemsetAsync(p->acc.p, 0, p->acc.n, s->stream));
            AE_CUDA(cudaMemsetAsync(p->S.p, 0, p->S.n, s->stream));
            // FP32 path: DFT blocks on the tensor cores when K is a multiple of 8
            // (at most 64) and 2 nl columns fit two 256-wide tiles
            if (!s->fp64 && s->dft_k % 8 == 0 && s->dft_k <= kDftTcMaxK && p->nl <= 256 &&
                !std::getenv("AEFDTD_NO_TC")) {
                int n2 = 2 * p->nl;
                p->N0 = std::min(256, (n2 + 15) / 16 * 16);
                p->N1 = n2 > 256 ? (n2 - 256 + 15) / 16 * 16 : 0;
                p->Btc.alloc(size_t(2) * 4 * 256 * s->dft_k * sizeof(float), s->dev_bytes);
                AE_CUDA(cudaMemsetAsync(p->Btc.p, 0, p->Btc.n, s->stream));
            }
            AE_CUDA(cudaMemcpyAsync(p->wdev.p, p->w.data(), p->nl * 8, cudaMemcpyHostToDevice, s->stream));
            AE_CUDA(cudaStreamSynchronize(s->stream));
        } catch (...) {
            p->S.release(s->dev_bytes); p->acc.release(s->dev_bytes); p->wdev.release(s->dev_bytes);
            p->WE.release(s->dev_bytes); p->WH.release(s->dev_bytes); p->flux.release(s->dev_bytes);
            p->Btc.release(s->dev_bytes);
            delete p;
            throw;
        }
        p->step = s->tstep;
        if (s->sensors.size() >= (size_t)kMaxGather) {
            p->S.release(s->dev_bytes); p->acc.release(s->dev_bytes); p->wdev.release(s->dev_bytes);
            p->WE.release(s->dev_bytes); p->WH.release(s->dev_bytes); p->flux.release(s->dev_bytes);
            delete p;
            fail(AEFDTD_BAD_ARG, "at most 8 planar sensors per simulation");
        }
        s->drain_sensors();
        s->sensors.push_back(p);
        s->graphs_dirty = true;
        if (id) *id = (int32_t)s->sensors.size() - 1;
    });
}

aefdtd_status aefdtd_step(aefdtd_sim *s, int32_t n) {
    if (!s) return AEFDTD_BAD_ARG;
    return guarded(s, [&] {
        if (s->batch) fail(AEFDTD_NOT_READY, "the simulation is stepped by its batch (aefdtd_batch_advance)");
        s->step(n);
    });
}

aefdtd_status aefdtd_synchronize(aefdtd_sim *s) {
    if (!s) return AEFDTD_BAD_ARG;
    return guarded(s, [&] {
        s->set_device();
        AE_CUDA(cudaStreamSynchronize(s->stream));
        s->check_err();
    });
}

aefdtd_status aefdtd_reset(aefdtd_sim *s) {
    if (!s) return AEFDTD_BAD_ARG;
    return guarded(s, [&] { s->zero_state(); });
}

aefdtd_status aefdtd_get_field(aefdtd_sim *s, int32_t c, double *out, size_t count) {
    if (!s || !out) return AEFDTD_BAD_ARG;
    return guarded(s, [&] {
        if (c < 0 || c > (s->obl ? 11 : 5)) fail(AEFDTD_BAD_ARG, "component out of range");
        size_t N = size_t(s->Nx) * s->Ny * s->Nz;
        if (count != N) fail(AEFDTD_BAD_ARG, "count must be Nx*Ny*Nz of the total grid");
        s->set_device();
        const void *src = s->grid_fields(c / 6)[c % 6].p;
        if (s->fp64) {
            AE_CUDA(cudaMemcpyAsync(out, src, N * 8, cudaMemcpyDeviceToHost, s->stream));
            AE_CUDA(cudaStreamSynchronize(s->stream));
        } else {
            std::vector<float> tmp(N);
            AE_CUDA(cudaMemcpyAsync(tmp.data(), src, N * 4, cudaMemcpyDeviceToHost, s->stream));
            AE_CUDA(cudaStreamSynchronize(s->stream));
            for (size_t q = 0; q < N; q++) out[q] = tmp[q];
        }
    });
}

aefdtd_status aefdtd_set_field(aefdtd_sim *s, int32_t c, const double *in, size_t count) {
    if (!s || !in) return AEFDTD_BAD_ARG;
    return guarded(s, [&] {
        if (c < 0 || c > (s->obl ? 11 : 5)) fail(AEFDTD_BAD_ARG, "component out of range");
        size_t N = size_t(s->Nx) * s->Ny * s->Nz;
        if (count != N) fail(AEFDTD_BAD_ARG, "count must be Nx*Ny*Nz of the total grid");
        s->set_device();
        void *dst = s->grid_fields(c / 6)[c % 6].p;
        if (s->fp64) {
            AE_CUDA(cudaMemcpyAsync(dst, in, N * 8, cudaMemcpyHostToDevice, s->stream));
        } else {
            std::vector<float> tmp(in, in + N);
            AE_CUDA(cudaMemcpyAsync(dst, tmp.data(), N * 4, cudaMemcpyHostToDevice, s->stream));
        }
        AE_CUDA(cudaStreamSynchronize(s->stream));
    });
}

aefdtd_status aefdtd_field_device_ptr(aefdtd_sim *s, int32_t c, void **ptr) {
    if (!s || !ptr || c < 0 || c > (s->obl ? 11 : 5)) return AEFDTD_BAD_ARG;
    *ptr = s->grid_fields(c / 6)[c % 6].p;
    return AEFDTD_OK;
}

aefdtd_status aefdtd_get_plane_sums(aefdtd_sim *s, double *out, int32_t steps) {
    if (!s || !out) return AEFDTD_BAD_ARG;
    return guarded(s, [&] {
        if (!s->normal) fail(AEFDTD_NOT_READY, "plane sums exist in normal mode only");
        if (steps != s->tstep) fail(AEFDTD_BAD_ARG, "steps must equal the number of completed steps");
        s->set_device();
        std::vector<double> tmp(size_t(steps) * 12);
        if (steps > 0) {
            AE_CUDA(cudaMemcpyAsync(tmp.data(), s->psums.p, tmp.size() * 8, cudaMemcpyDeviceToHost, s->stream));
            AE_CUDA(cudaStreamSynchronize(s->stream));
        }
        for (int c = 0; c < 12; c++)
            for (int t = 0; t < steps; t++) out[size_t(c) * steps + t] = tmp[size_t(t) * 12 + c];
    });
}

// Post-processing of FDTD_normal_incidence (normal_incidence.cpp:442-570),
// FP64 on the host over the completed steps.
aefdtd_status aefdtd_get_normal_spectra(aefdtd_sim *s, double *out, int32_t nl) {
    if (!s || !out) return AEFDTD_BAD_ARG;
    return guarded(s, [&] {
        if (!s->normal) fail(AEFDTD_NOT_READY, "spectra exist in normal mode only");
        if (nl != s->nd.nl) fail(AEFDTD_BAD_ARG, "nl must equal the normal-mode spectrum size");
        const int Ntot = s->tstep;
        // after a completion at step t the driver analyses Nt = t steps (normal_incidence.cpp:417-427)
        const int NtP = s->cc_done ? s->cc_stop : Ntot;
        if (NtP < 2) fail(AEFDTD_NOT_READY, "run at least two steps");
        std::vector<double> S(size_t(Ntot) * 12);
        aefdtd_status st = aefdtd_get_plane_sums(s, S.data(), Ntot);
        if (st != AEFDTD_OK) fail(st, s->last_error);
        auto M = [&](int i, int j, int k) { return s->map[i + size_t(j) * s->Nx + size_t(k) * s->Nx * s->Ny]; };
        // FDTD::find_slab (fdtd_utils.cpp:347-392)
        int sub_ref = s->zs_s, sup_ref = s->zs_e - 1;
        int Nsub = 0, Nsup = 0, IDmoy = 0, IDsup = 0, IDsub = 0, k;
        for (int i = s->xs_s; i < s->xs_e; i++)
            for (int j = s->ys_s; j < s->ys_e; j++) { IDsup += M(i, j, s->zs_e); IDsub += M(i, j, s->zs_s); }
        IDmoy = IDsub; k = sub_ref;
        while (IDmoy == IDsub && k < sup_ref) {
            IDmoy = 0;
            for (int i = s->xs_s; i < s->xs_e; i++) for (int j = s->ys_s; j < s->ys_e; j++) IDmoy += M(i, j, k + 1);
            Nsub++; k++;
        }
        IDmoy = IDsup; k = sup_ref;
        while (IDmoy == IDsup && k >= sub_ref) {
            IDmoy = 0;
            for (int i = s->xs_s; i < s->xs_e; i++) for (int j = s->ys_s; j < s->ys_e; j++) IDmoy += M(i, j, k - 1);
            Nsup++; k--;
        }
        double Dz = s->Dz, Dt = s->Dt;
        double hsup = (Nsup - 1) * Dz, hsub = Nsub * Dz, hstruc = (s->Nz_s - Nsup - Nsub) * Dz;
        hsup -= Dz / 2.0;
        hsub -= Dz / 2.0;
        const cplx Im(0, 1);
        const double *SS[12];
        for (int c = 0; c < 12; c++) SS[c] = S.data() + size_t(c) * Ntot;
        // wavelengths are independent; each one's sums run in the driver's order
        auto one = [&](int l) {
            double lam = s->nd.lambda_min + (s->nd.lambda_max - s->nd.lambda_min) * l / (nl - 1.0);
            double w = 2.0 * Pi * c_light / lam;
            cplx r1x = 0, r1y = 0, r1z = 0, r2x = 0, r2y = 0, r2z = 0, t1x = 0, t1y = 0, t1z = 0, t2x = 0, t2y = 0, t2z = 0;
            double k0 = -w / c_light, k1 = k0 * s->index_sup, k3 = k0 * s->index_sub;
            cplx tmp_sup = std::exp(2.0 * k1 * hsup * Im);
            cplx tmp_sub = std::exp((k3 * hsub - k0 * (hstruc + hsub)) * Im);
            for (int t = 0; t < NtP; t++) {
                cplx tmp1 = std::exp(t * Dt * w * Im) / (NtP - 1.0);
                cplx tmp2 = tmp1 * tmp_sup, tmp3 = tmp1 * tmp_sub;
                r1x += SS[0][t] * tmp1; r1y += SS[1][t] * tmp1; r1z += SS[2][t] * tmp1;
                r2x += SS[3][t] * tmp2; r2y += SS[4][t] * tmp2; r2z += SS[5][t] * tmp2;
                t1x += SS[6][t] * tmp1; t1y += SS[7][t] * tmp1; t1z += SS[8][t] * tmp1;
                t2x += SS[9][t] * tmp3; t2y += SS[10][t] * tmp3; t2z += SS[11][t] * tmp3;
            }
            double *o = out + size_t(l) * 15;
            o[0] = lam;
            double a = std::sqrt(std::norm(r2x) + std::norm(r2y) + std::norm(r2z));
            double b = std::sqrt(std::norm(r1x) + std::norm(r1y) + std::norm(r1z));
            o[1] = a / b;
            a = std::sqrt(std::norm(t2x) + std::norm(t2y) + std::norm(t2z));
            b = std::sqrt(std::norm(t1x) + std::norm(t1y) + std::norm(t1z));
            o[2] = a / b;
            cplx ref0 = r1y, trans0 = t1y;
            if (s->nd.polarization == 1) { ref0 = r1x; trans0 = t1x; }
            cplx refx = r2x / ref0, refy = r2y / ref0, transx = t2x / trans0, transy = t2y / trans0;
            o[3] = std::abs(refx); o[4] = std::arg(refx); o[5] = std::norm(refx);
            o[6] = std::abs(refy); o[7] = std::arg(refy); o[8] = std::norm(refy);
            o[9] = std::abs(transx); o[10] = std::arg(transx); o[11] = std::norm(transx) * s->index_sub / s->index_sup;
            o[12] = std::abs(transy); o[13] = std::arg(transy); o[14] = std::norm(transy) * s->index_sub / s->index_sup;
        };
        parallel_for(nl, one);
    });
}

// Box_Spect_Poynting (s_spec_power.cpp:124-232): six planar spectral Poynting
// faces, xm, xp, ym, yp, zm, zp, on the faces of the box; flux = their sum in
// that order.
aefdtd_status aefdtd_add_box_sensor(aefdtd_sim *s, const aefdtd_box_sensor_desc *d, int32_t *id) {
    if (!s || !d) return AEFDTD_BAD_ARG;
    const int x1 = d->box[0], x2 = d->box[1], y1 = d->box[2], y2 = d->box[3], z1 = d->box[4], z2 = d->box[5];
    const int fb[6][7] = {{AEFDTD_NORMAL_XM, x1, x1 + 1, y1, y2, z1, z2}, {AEFDTD_NORMAL_X, x2 - 1, x2, y1, y2, z1, z2},
                          {AEFDTD_NORMAL_YM, x1, x2, y1, y1 + 1, z1, z2}, {AEFDTD_NORMAL_Y, x1, x2, y2 - 1, y2, z1, z2},
                          {AEFDTD_NORMAL_ZM, x1, x2, y1, y2, z1, z1 + 1}, {AEFDTD_NORMAL_Z, x1, x2, y1, y2, z2 - 1, z2}};
    int n = 0;
    for (int f = 0; f < 6; f++) n += !(d->disabled & (1 << f));
    if (n == 0 || x2 <= x1 || y2 <= y1 || z2 <= z1 || d->nl < 1) {
        s->last_error = "a box needs positive extents, nl >= 1 and at least one face";
        return AEFDTD_BAD_ARG;
    }
    if (s->sensors.size() + n > (size_t)kMaxGather) {
        s->last_error = "a box takes one planar sensor per face; at most 8 per simulation";
        return AEFDTD_BAD_ARG;
    }
    std::array<int, 6> ids;
    ids.fill(-1);
    for (int f = 0; f < 6; f++) {
        if (d->disabled & (1 << f)) continue;
        aefdtd_sensor_desc sd{};
        sd.orientation = fb[f][0];
        for (int k = 0; k < 6; k++) sd.box[k] = fb[f][1 + k];
        sd.nl = d->nl;
        sd.lambda_min = d->lambda_min;
        sd.lambda_max = d->lambda_max;
        int32_t sid = -1;
        const aefdtd_status st = aefdtd_add_planar_sensor(s, &sd, &sid);
        if (st != AEFDTD_OK) return st;
        ids[f] = sid;
    }
    s->boxes.push_back(ids);
    if (id) *id = (int32_t)s->boxes.size() - 1;
    return AEFDTD_OK;
}

aefdtd_status aefdtd_get_box_flux(aefdtd_sim *s, int32_t id, double *out, int32_t nl) {
    if (!s || !out) return AEFDTD_BAD_ARG;
    if (id < 0 || id >= (int)s->boxes.size()) {
        s->last_error = "unknown box sensor";
        return AEFDTD_BAD_ARG;
    }
    std::vector<double> face(std::max(nl, 1));
    for (int l = 0; l < nl; l++) out[l] = 0;
    for (int f = 0; f < 6; f++) {
        const int sid = s->boxes[id][f];
        if (sid < 0) continue;
        const aefdtd_status st = aefdtd_get_sensor_flux(s, sid, face.data(), nl);
        if (st != AEFDTD_OK) return st;
        for (int l = 0; l < nl; l++) out[l] += face[l];
    }
    return AEFDTD_OK;
}

aefdtd_status aefdtd_add_fieldmap(aefdtd_sim *s, const aefdtd_fieldmap_desc *d, int32_t *id) {
    if (!s || !d) return AEFDTD_BAD_ARG;
    return guarded(s, [&] {
        if (s->batch) fail(AEFDTD_NOT_READY, "batch members carry no field sensors");
        if (d->kind < AEFDTD_MAP_PLANE || d->kind > AEFDTD_MAP_POINT) fail(AEFDTD_BAD_ARG, "bad field-sensor kind");
        if (d->kind == AEFDTD_MAP_PLANE && (d->orientation < 0 || d->orientation > 5))
            fail(AEFDTD_BAD_ARG, "bad orientation");
        if (d->kind != AEFDTD_MAP_POINT && !(d->lambda > 0)) fail(AEFDTD_BAD_ARG, "lambda must be positive");
        if (s->fmaps.size() >= (size_t)kMaxMaps) fail(AEFDTD_BAD_ARG, "at most 8 field sensors per simulation");
        s->set_device();
        // Sensor::link (sensors.cpp:196-230): structure cells -> total grid, clamped
        int b[6] = {d->box[0], d->box[1], d->box[2], d->box[3], d->box[4], d->box[5]};
        if (d->kind == AEFDTD_MAP_POINT) { b[1] = b[0] + 1; b[3] = b[2] + 1; b[5] = b[4] + 1; }   // FieldPoint ctor
        const int x1 = std::clamp(b[0] + s->xs_s, 0, s->Nx), x2 = std::clamp(b[1] + s->xs_s, 0, s->Nx);
        const int y1 = std::clamp(b[2] + s->ys_s, 0, s->Ny), y2 = std::clamp(b[3] + s->ys_s, 0, s->Ny);
        const int z1 = std::clamp(b[4] + s->zs_s, 0, s->Nz), z2 = std::clamp(b[5] + s->zs_s, 0, s->Nz);
        if (x2 <= x1 || y2 <= y1 || z2 <= z1 || x1 >= s->Nx || y1 >= s->Ny || z1 >= s->Nz)
            fail(AEFDTD_BAD_ARG, "field-sensor box is empty or outside the grid");
        auto *m = new FieldMapHost();
        m->d = *d;
        MapDesc &v = m->dev;
        v.kind = d->kind;
        v.x1 = x1; v.y1 = y1; v.z1 = z1;
        size_t n = 0;
        if (d->kind == AEFDTD_MAP_PLANE) {
            // FieldMap::initialize (s_fieldmap.cpp:425-440): -M orientations map to the plus ones
            v.type = d->orientation / 2;
            v.mag = d->magnetic != 0;
            if (v.type == 0) { v.span1 = y2 - y1; v.span2 = z2 - z1; v.span3 = x2 - x1; }
            else if (v.type == 1) { v.span1 = x2 - x1; v.span2 = z2 - z1; v.span3 = y2 - y1; }
            else { v.span1 = x2 - x1; v.span2 = y2 - y1; v.span3 = z2 - z1; }
            if (!d->cumulative) v.span3 = 1;
            v.P = v.span1 * v.span2;
            m->ncomp = 3;
            n = size_t(3) * v.P * 16;
        } else if (d->kind == AEFDTD_MAP_BLOCK) {
            // FieldBlock::initialize (s_fieldmap.cpp:177-190)
            v.span1 = x2 - x1; v.span2 = y2 - y1; v.span3 = z2 - z1;
            v.P = v.span1 * v.span2 * v.span3;
            m->ncomp = 6;
            n = size_t(6) * v.P * 16;
        } else {
            v.span1 = v.span2 = v.span3 = 1;
            v.P = 1;
            v.cap = std::max(1, s->Nt);
            m->ncomp = 3;
            n = size_t(v.cap) * 3 * 8;
        }
        if (d->kind != AEFDTD_MAP_POINT) m->w = 2.0 * Pi * c_light / d->lambda;
        m->step0 = s->tstep;
        v.step0 = s->tstep;
        try {
            m->acc.alloc(n, s->dev_bytes);
            AE_CUDA(cudaMemsetAsync(m->acc.p, 0, m->acc.n, s->stream));
            if (!s->fm_tbl.p) s->fm_tbl.alloc(size_t(2) * s->seg_len * kMaxMaps * 4 * sizeof(double), s->dev_bytes);
            AE_CUDA(cudaStreamSynchronize(s->stream));
        } catch (...) {
            m->acc.release(s->dev_bytes);
            delete m;
            throw;
        }
        v.acc = m->acc.as<double>();
        s->fmaps.push_back(m);
        s->graphs_dirty = true;
        if (id) *id = (int32_t)s->fmaps.size() - 1;
    });
}

aefdtd_status aefdtd_get_fieldmap_shape(aefdtd_sim *s, int32_t id, int32_t shape[4]) {
    if (!s || !shape) return AEFDTD_BAD_ARG;
    if (id < 0 || id >= (int)s->fmaps.size()) {
        s->last_error = "unknown field sensor";
        return AEFDTD_BAD_ARG;
    }
    const FieldMapHost &m = *s->fmaps[id];
    if (m.dev.kind == kMapPoint) {
        shape[0] = std::clamp(s->tstep - m.step0, 0, m.dev.cap);
        shape[1] = shape[2] = 1;
    } else {
        shape[0] = m.dev.span1;
        shape[1] = m.dev.span2;
        shape[2] = m.dev.kind == kMapBlock ? m.dev.span3 : 1;
    }
    shape[3] = m.ncomp;
    return AEFDTD_OK;
}

aefdtd_status aefdtd_get_fieldmap(aefdtd_sim *s, int32_t id, double *out, size_t count) {
    if (!s || !out) return AEFDTD_BAD_ARG;
    return guarded(s, [&] {
        if (id < 0 || id >= (int)s->fmaps.size()) fail(AEFDTD_BAD_ARG, "unknown field sensor");
        const FieldMapHost &m = *s->fmaps[id];
        size_t want;
        if (m.dev.kind == kMapPoint) want = size_t(std::clamp(s->tstep - m.step0, 0, m.dev.cap)) * 3;
        else want = size_t(m.ncomp) * m.dev.P * 2;
        if (count != want) fail(AEFDTD_BAD_ARG, "count must be " + std::to_string(want));
        s->set_device();
        AE_CUDA(cudaStreamSynchronize(s->stream));
        if (want) AE_CUDA(cudaMemcpy(out, m.acc.p, want * sizeof(double), cudaMemcpyDeviceToHost));
    });
}

aefdtd_status aefdtd_get_sensor_shape(aefdtd_sim *s, int32_t id, int32_t *span1, int32_t *span2, int32_t *nl) {
    if (!s || id < 0 || id >= (int)s->sensors.size()) return AEFDTD_BAD_ARG;
    if (span1) *span1 = s->sensors[id]->span1;
    if (span2) *span2 = s->sensors[id]->span2;
    if (nl) *nl = s->sensors[id]->nl;
    return AEFDTD_OK;
}

aefdtd_status aefdtd_get_sensor_flux(aefdtd_sim *s, int32_t id, double *out, int32_t nl) {
    if (!s || !out) return AEFDTD_BAD_ARG;
    return guarded(s, [&] {
        if (id < 0 || id >= (int)s->sensors.size()) fail(AEFDTD_BAD_ARG, "unknown sensor");
        PlaneSensor &p = *s->sensors[id];
        if (nl != p.nl) fail(AEFDTD_BAD_ARG, "nl must equal the sensor's spectrum size");
        s->set_device();
        s->drain_sensors();
        double af = p.type <= 1 ? s->Dy * s->Dz : (p.type <= 3 ? s->Dx * s->Dz : s->Dx * s->Dy);
        FluxArgs fa{p.P, p.nl, p.type, af, p.acc.as<double2>(), p.flux.as<double>()};
        launch_flux(fa, s->stream);
        s->launches++;
        AE_CUDA(cudaMemcpyAsync(out, p.flux.p, size_t(nl) * 8, cudaMemcpyDeviceToHost, s->stream));
        AE_CUDA(cudaStreamSynchronize(s->stream));
        AE_CUDA(cudaGetLastError());
    });
}

aefdtd_status aefdtd_get_sensor_dft(aefdtd_sim *s, int32_t id, double *out, size_t count) {
    if (!s || !out) return AEFDTD_BAD_ARG;
    return guarded(s, [&] {
        if (id < 0 || id >= (int)s->sensors.size()) fail(AEFDTD_BAD_ARG, "unknown sensor");
        PlaneSensor &p = *s->sensors[id];
        if (count != size_t(6) * p.P * p.nl * 2) fail(AEFDTD_BAD_ARG, "count must be 6*span1*span2*nl*2");
        s->set_device();
        s->drain_sensors();
        AE_CUDA(cudaMemcpyAsync(out, p.acc.p, count * 8, cudaMemcpyDeviceToHost, s->stream));
        AE_CUDA(cudaStreamSynchronize(s->stream));
    });
}

aefdtd_status aefdtd_discretize(aefdtd_sim *sim, int32_t nx, int32_t ny, int32_t nz, double dx, double dy, double dz,
                                const aefdtd_structure_op *ops, int32_t n_ops, const aefdtd_structure_desc *desc,
                                uint32_t *out_map, int32_t device) {
    if (nx < 1 || ny < 1 || nz < 1 || n_ops < 0 || n_ops > 256 || (n_ops > 0 && !ops) || !out_map || !desc)
        return AEFDTD_BAD_ARG;
    return guarded(sim, [&] {
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) fail(AEFDTD_NO_DEVICE, "no CUDA device visible");
        int dev = sim ? sim->device : device;
        AE_CUDA(cudaSetDevice(dev));
        aefdtd_structure_desc d = *desc;
        for (int a = 0; a < 3; a++) {
            if (d.periodic[a] && !(d.lengths[a] > 0)) fail(AEFDTD_BAD_ARG, "periodic axis needs a positive length");
            if (!std::isfinite(d.lengths[a])) fail(AEFDTD_BAD_ARG, "structure lengths must be finite");
        }
        // coatings evaluate the structure below them; the device follows at most 3 nested coatings
        std::vector<int> depth(n_ops, 0);
        long long lattice = 0;
        for (int q = 0; q < n_ops; q++) {
            const aefdtd_structure_op &o = ops[q];
            if (o.kind < AEFDTD_OP_BLOCK || o.kind > AEFDTD_OP_MESH || o.mat_index < 0)
                fail(AEFDTD_BAD_ARG, "bad structure operation " + std::to_string(q));
            if (o.kind == AEFDTD_OP_MESH) {
                const int mi = (int)o.p[4];
                if (o.p[4] != mi || mi < 0 || mi >= d.n_meshes || !d.meshes) fail(AEFDTD_BAD_ARG, "mesh number out of range");
                const aefdtd_mesh &m = d.meshes[mi];
                if (m.n_vertices < 1 || m.n_faces < 0 || !m.vertices || (m.n_faces > 0 && !m.faces))
                    fail(AEFDTD_BAD_ARG, "empty mesh");
                for (long long t = 0; t < 3LL * m.n_faces; t++)
                    if (m.faces[t] < 0 || m.faces[t] >= m.n_vertices) fail(AEFDTD_BAD_ARG, "mesh face refers to a missing vertex");
                for (long long t = 0; t < 3LL * m.n_vertices; t++)
                    if (!std::isfinite(m.vertices[t])) fail(AEFDTD_BAD_ARG, "mesh vertices must be finite");
            }
            for (int t = 0; t < 16; t++)
                if (!std::isfinite(o.p[t])) fail(AEFDTD_BAD_ARG, "structure operation parameters must be finite");
            if (o.kind == AEFDTD_OP_COATING || o.kind == AEFDTD_OP_CONF_COATING) {
                int below = 0;
                for (int p = 0; p < q; p++) below = std::max(below, depth[p]);
                depth[q] = below + 1;
                if (depth[q] > 3) fail(AEFDTD_BAD_ARG, "coatings nest more than 3 deep");
            }
            if (o.kind == AEFDTD_OP_COATING) {
                const double delta = o.p[3], cz = std::cos(o.p[0] * (3.141592653589793 / 180.0));
                if (!(delta > 0)) fail(AEFDTD_BAD_ARG, "a coating needs delta > 0");
                if (!(cz > 0) || !(d.lengths[2] > 0) || 3.0 * d.lengths[2] / (delta * cz) > 1e6)
                    fail(AEFDTD_BAD_ARG, "coating direction too shallow for its delta (the march through z would not end)");
                if (!(o.p[2] >= 0)) fail(AEFDTD_BAD_ARG, "coating thickness must be >= 0");
            }
            if (o.kind == AEFDTD_OP_CONF_COATING) {
                const double delta = o.p[1] > 0 ? o.p[1] : 5e-9;
                long long n = 1;
                for (int a = 0; a < 3; a++) n *= std::max(0LL, (long long)(d.lengths[a] / delta));
                lattice += n;
                if (lattice > (1LL << 31)) fail(AEFDTD_BAD_ARG, "conformal-coating seed lattice too large");
            }
            if ((o.kind == AEFDTD_OP_ELLIPSOID) && !(o.p[3] > 0 && o.p[4] > 0 && o.p[5] > 0))
                fail(AEFDTD_BAD_ARG, "ellipsoid radii must be positive");
        }
        size_t n = size_t(nx) * ny * nz;
        cudaStream_t st = sim ? sim->stream : nullptr;
        uint32_t *dmap = nullptr;
        int *derr = nullptr;
        AE_CUDA(cudaMallocAsync((void **)&dmap, n * 4 + 16, st));
        derr = reinterpret_cast<int *>(reinterpret_cast<char *>(dmap) + (n * 4 + 15) / 16 * 16);
        cudaError_t e = cudaMemsetAsync(derr, 0, sizeof(int), st);
        if (e == cudaSuccess) e = launch_discretize(nx, ny, nz, dx, dy, dz, ops, n_ops, d, dmap, derr, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(out_map, dmap, n * 4, cudaMemcpyDeviceToHost, st);
        int herr = 0;
        if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost, st);
        cudaFreeAsync(dmap, st);
        cudaError_t e2 = cudaStreamSynchronize(st);
        if (e != cudaSuccess) fail(AEFDTD_CUDA_ERROR, std::string("discretize: ") + cudaGetErrorString(e));
        if (e2 != cudaSuccess) fail(AEFDTD_CUDA_ERROR, std::string("discretize: ") + cudaGetErrorString(e2));
        if (herr == 1) fail(AEFDTD_TIMEOUT, "discretize: a walk through the structure exceeded its bound");
        if (herr) fail(AEFDTD_BAD_ARG, "discretize: coatings nest too deep");
        if (sim) {
            sim->launches++;
            if (nx != sim->Nx_s || ny != sim->Ny_s || nz != sim->Nz_s) fail(AEFDTD_BAD_ARG, "map size differs from the structure grid");
            sim->set_map(out_map, n);
        }
    });
}

aefdtd_status aefdtd_voxelize(aefdtd_sim *sim, int32_t nx, int32_t ny, int32_t nz, double dx, double dy, double dz,
                              const aefdtd_structure_op *ops, int32_t n_ops, int32_t default_material,
                              const int32_t periodic[3], const double lengths[3], uint32_t *out_map, int32_t device) {
    aefdtd_structure_desc d{};
    d.default_material = default_material;
    for (int a = 0; a < 3; a++) {
        d.periodic[a] = periodic ? (periodic[a] ? 1 : 0) : 0;
        d.lengths[a] = lengths ? lengths[a] : 0;
    }
    return aefdtd_discretize(sim, nx, ny, nz, dx, dy, dz, ops, n_ops, &d, out_map, device);
}

aefdtd_status aefdtd_get_timings(aefdtd_sim *s, double *e_ms, double *h_ms, double *sensor_ms) {
    if (!s) return AEFDTD_BAD_ARG;
    if (e_ms) *e_ms = s->t_e;
    if (h_ms) *h_ms = s->t_h;
    if (sensor_ms) *sensor_ms = s->t_s;
    return AEFDTD_OK;
}

aefdtd_status aefdtd_enable_timing(aefdtd_sim *s, int32_t enable) {
    if (!s) return AEFDTD_BAD_ARG;
    if (enable < 0 || enable > 2) return AEFDTD_BAD_ARG;
    s->timing = enable != 0;
    if (enable) s->timing_mode = enable;
    return AEFDTD_OK;
}

aefdtd_status aefdtd_set_completion(aefdtd_sim *s, double coeff, int32_t check_every) {
    if (!s) return AEFDTD_BAD_ARG;
    return guarded(s, [&] {
        if (check_every < 0) fail(AEFDTD_BAD_ARG, "negative check interval");
        if (s->batch) fail(AEFDTD_NOT_READY, "set the completion sensor before the simulation joins a batch");
        if (s->ccft) {
            size_t t = 0;
            s->ccft->dpts.release(t); s->ccft->acc.release(t); s->ccft->ring.release(t); s->ccft->ctab.release(t); s->ccft->snap.release(t);
            s->dev_bytes -= std::min(s->dev_bytes, t);
            delete s->ccft;
            s->ccft = nullptr;
        }
        s->cc_coeff = coeff > 0 ? coeff : 0;
        s->cc_step = check_every > 0 ? check_every : 500;
        s->cc_done = false;
        s->cc_stop = -1;
        s->cc_read = s->tstep;
        s->cc_last = s->cc_max = 0;
        s->graphs_dirty = true;
    });
}

// CompletionSensor(lmin, lmax, coeff, Np, layout) and its initialize()
// (s_completion.cpp:26-37, 246-361): probe cells on the named faces and their
// wavelengths, drawn with randp (mathUT.cpp:65-68) from a std::mt19937.
aefdtd_status aefdtd_set_completion_ft(aefdtd_sim *s, double lambda_min, double lambda_max, double coeff,
                                       int32_t n_points, const char *layout, uint32_t seed, int32_t check_every) {
    if (!s) return AEFDTD_BAD_ARG;
    aefdtd_status st = aefdtd_set_completion(s, coeff, check_every);   // clears either mode
    if (st != AEFDTD_OK || !(coeff > 0)) return st;
    return guarded(s, [&] {
        if (n_points < 1) fail(AEFDTD_BAD_ARG, "n_points must be positive");
        if (!(lambda_min > 0) || !(lambda_max > 0)) fail(AEFDTD_BAD_ARG, "bad probe wavelengths");
        s->set_device();
        auto *c = new CompletionFT();
        c->lmin = lambda_min; c->lmax = lambda_max; c->np = n_points;
        std::string lay = layout ? layout : "";
        bool known = lay == "v";
        const char combi[4] = {'n', 'd', 'u', 'b'};
        for (int a = 0; a < 4; a++) for (int b = 0; b < 4; b++) for (int d = 0; d < 4; d++)
            if (lay.size() == 3 && lay[0] == combi[a] && lay[1] == combi[b] && lay[2] == combi[d]) known = true;
        if (lay == "nnn" || !known) lay = "nnb";
        c->layout = lay;
        std::mt19937 mte(seed);
        auto randp = [&](double A, double B) { return A + (B - A) * mte() / (mte.max() - mte.min()); };
        const int Np = n_points;
        c->pts.assign(size_t(Np) * 3, 0);
        auto P = [&](int i, int d) -> int & { return c->pts[size_t(i) * 3 + d]; };
        if (lay == "v") {
            for (int i = 0; i < Np; i++) {
                P(i, 0) = static_cast<int>(randp(s->xs_s, s->xs_e - 1) + 0.5);
                P(i, 1) = static_cast<int>(randp(s->ys_s, s->ys_e - 1) + 0.5);
                P(i, 2) = static_cast<int>(randp(s->zs_s, s->zs_e - 1) + 0.5);
            }
        } else {
            const int Nx = s->Nx, Ny = s->Ny, Nz = s->Nz;
            int n_face[6] = {0, 0, 0, 0, 0, 0};   // xd, xu, yd, yu, zd, zu
            const int area[3] = {Ny * Nz, Nx * Nz, Nx * Ny};
            for (int a = 0; a < 3; a++) {
                if (lay[a] == 'd' || lay[a] == 'b') n_face[2 * a] = area[a];
                if (lay[a] == 'u' || lay[a] == 'b') n_face[2 * a + 1] = area[a];
            }
            const double tot_area = n_face[0] + n_face[1] + n_face[2] + n_face[3] + n_face[4] + n_face[5];
            int N_left = Np;
            for (int f = 0; f < 6; f++) {
                int N_alloc = static_cast<int>(Np * n_face[f] / tot_area + 0.5);
                N_alloc = N_alloc < N_left ? N_alloc : N_left;
                N_left -= N_alloc;
                n_face[f] = N_alloc;
            }
            int off = 0;
            const int lo[3] = {s->xs_s, s->ys_s, s->zs_s}, hi[3] = {s->xs_e - 1, s->ys_e - 1, s->zs_e - 1};
            for (int f = 0; f < 6; f++) {
                const int axis = f / 2;
                for (int i = off; i < off + n_face[f]; i++)
                    for (int d = 0; d < 3; d++)
                        P(i, d) = d == axis ? (f % 2 ? hi[d] : lo[d]) : static_cast<int>(randp(lo[d], hi[d]) + 0.5);
                off += n_face[f];
            }
        }
        c->w.resize(Np);
        for (int i = 0; i < Np; i++) c->w[i] = 2.0 * Pi * c_light / randp(lambda_min, lambda_max);
        const double T = std::max(lambda_min, lambda_max) / c_light;
        c->n_avg = std::max(1, static_cast<int>(T / s->Dt));
        c->step0 = s->tstep;
        try {
            c->dpts.alloc(c->pts.size() * sizeof(int), s->dev_bytes);
            AE_CUDA(cudaMemcpy(c->dpts.p, c->pts.data(), c->pts.size() * sizeof(int), cudaMemcpyHostToDevice));
            c->acc.alloc(size_t(Np) * 3 * 16, s->dev_bytes);
            c->ring.alloc(size_t(6) * Np * c->n_avg * 8, s->dev_bytes);
            c->ctab.alloc(size_t(2) * s->seg_len * Np * 16, s->dev_bytes);
            AE_CUDA(cudaMemsetAsync(c->acc.p, 0, c->acc.n, s->stream));
            AE_CUDA(cudaMemsetAsync(c->ring.p, 0, c->ring.n, s->stream));
            AE_CUDA(cudaStreamSynchronize(s->stream));
        } catch (...) {
            size_t t = 0;
            c->dpts.release(t); c->acc.release(t); c->ring.release(t); c->ctab.release(t);
            s->dev_bytes -= std::min(s->dev_bytes, t);
            delete c;
            throw;
        }
        s->ccft = c;
        s->graphs_dirty = true;
    });
}

aefdtd_status aefdtd_get_completion(aefdtd_sim *s, int32_t *done, int32_t *stop_step, double *ratio) {
    if (!s) return AEFDTD_BAD_ARG;
    if (done) *done = s->cc_done ? 1 : 0;
    if (stop_step) *stop_step = s->cc_stop;
    if (ratio) *ratio = s->ccft ? s->ccft->open_ratio : (s->cc_max > 0 ? s->cc_last / s->cc_max : 0.0);
    return AEFDTD_OK;
}

aefdtd_status aefdtd_get_group_timings(aefdtd_sim *s, double *ms, int64_t *cells, int32_t n) {
    if (!s || n != 2 * kGroups) return AEFDTD_BAD_ARG;
    return guarded(s, [&] {
        for (int half = 0; half < 2; half++)
            for (int g = 0; g < kGroups; g++) {
                const int i = half * kGroups + g;
                if (ms) ms[i] = s->tev_steps > 0 ? s->t_grp[half][g] / s->tev_steps : 0.0;
                if (cells) cells[i] = s->grp_cells[half][g];
            }
    });
}

aefdtd_status aefdtd_get_stream(aefdtd_sim *s, void **stream) {
    if (!s || !stream) return AEFDTD_BAD_ARG;
    *stream = (void *)s->stream;
    return AEFDTD_OK;
}

aefdtd_status aefdtd_get_launch_count(aefdtd_sim *s, uint64_t *launches) {
    if (!s || !launches) return AEFDTD_BAD_ARG;
    *launches = s->launches;
    return AEFDTD_OK;
}

aefdtd_status aefdtd_test_hook(aefdtd_sim *s, int32_t what, int64_t value) {
    if (!s) return AEFDTD_BAD_ARG;
    return guarded(s, [&] {
        if (what == AEFDTD_TEST_DFT_WAIT_CYCLES) {
            if (value < 1) fail(AEFDTD_BAD_ARG, "wait bound must be at least 1 cycle");
            s->tc_wait_cycles = value;
        } else if (what == AEFDTD_TEST_DFT_WITHHOLD_COPY) {
            s->tc_withhold_copy = value ? 1 : 0;
        } else if (what == AEFDTD_TEST_STAGED_WAIT_CYCLES) {
            if (value < 1) fail(AEFDTD_BAD_ARG, "wait bound must be at least 1 cycle");
            s->tma_wait_cycles = value;
            for (auto &p : s->tma_plan) p.wait_cycles = value;
        } else if (what == AEFDTD_TEST_STAGED_WITHHOLD_COPY) {
            s->tma_withhold = value ? 1 : 0;
            for (auto &p : s->tma_plan) p.withhold = s->tma_withhold;
        } else if (what == AEFDTD_TEST_PERSIST_WAIT_CYCLES) {
            if (value < 1) fail(AEFDTD_BAD_ARG, "wait bound must be at least 1 cycle");
            s->ps_wait_cycles = value;
        } else if (what == AEFDTD_TEST_PERSIST_WITHHOLD) {
            s->ps_withhold = value ? 1 : 0;
        } else {
            fail(AEFDTD_BAD_ARG, "unknown test hook");
        }
        s->graphs_dirty = true;   // captured segments hold the old arguments
    });
}

aefdtd_status aefdtd_device_memory(int32_t device, size_t *free_bytes, size_t *total_bytes) {
    if (!free_bytes || !total_bytes) return AEFDTD_BAD_ARG;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return AEFDTD_NO_DEVICE;
    }
    if (device < 0 || device >= n) return AEFDTD_BAD_ARG;
    int prev = 0;
    if (cudaGetDevice(&prev) != cudaSuccess || cudaSetDevice(device) != cudaSuccess) {
        cudaGetLastError();
        return AEFDTD_CUDA_ERROR;
    }
    const cudaError_t e = cudaMemGetInfo(free_bytes, total_bytes);
    cudaSetDevice(prev);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return AEFDTD_CUDA_ERROR;
    }
    return AEFDTD_OK;
}

}  // extern "C"
