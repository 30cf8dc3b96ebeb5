/* Reference-core driver for the oracle build — TEST INFRASTRUCTURE ONLY.
 *
 * Links against the reference's own FDTD core sources, compiled unmodified
 * from the reference tree by oracle/Makefile into oracle/_ref/. This file is
 * project-written: it replays the time loops of the two reference mode
 * drivers without Lua (Lua 5.4 is not installed here), building the FDTD,
 * Material, Spect_Poynting and Oscillator objects directly:
 *   - aeref_run with mode NORMAL replays FDTD_normal_incidence
 *     (src/finite_differences/FDTD/modes/normal_incidence.cpp:161-570,
 *     minus PNG previews and result files);
 *   - mode CUSTOM replays mode_default_fdtd
 *     (src/finite_differences/FDTD/modes/default_fdtd.cpp:24-210).
 * Only tests/, bench.py's reference arm and the golden-fixture script call it;
 * the product library never links or loads it.
 */
#include <fdtd_core.h>
#include <sensors.h>
#include <sources.h>
#include <material.h>

#include <chrono>
#include <cmath>
#include <complex>
#include <filesystem>
#include <fstream>
#include <iostream>
#include <sstream>
#include <vector>

#include "../include/aefdtd.h"

extern const Imdouble Im;

namespace {

// Completion sensor in energy mode (normal mode only), set by
// aeref_set_completion: CompletionSensor(coeff) fed after the planar sensors,
// checked after step t's plane sums when t % every == 0
// (normal_incidence.cpp:284-297, 417-427).
double g_cc_coeff = 0;
int g_cc_every = 500;
// FT mode (CompletionSensor(lmin, lmax, coeff, Np, layout)) when g_cc_np > 0;
// the global generator is reseeded with g_cc_seed (seedp) before the sensor
// draws its probes
int g_cc_np = 0;
double g_cc_lmin = 0, g_cc_lmax = 0;
std::string g_cc_layout;
int g_cc_seed = 0;
int g_cc_stop = -1;
double g_cc_last = 0, g_cc_max = 0;

// One box spectral Poynting sensor (Box_Spect_Poynting, s_spec_power.cpp:
// 124-232), set by aeref_set_box: fed after the planar sensors; its
// rsp_result is kept for aeref_box_result.
bool g_box_on = false;
int g_box[6] = {0, 0, 0, 0, 0, 0};
int g_box_nl = 0, g_box_mask = 0;
double g_box_lmin = 0, g_box_lmax = 0;
std::vector<double> g_box_result;

// Single-wavelength field sensors (FieldMap, FieldBlock, FieldPoint of
// s_fieldmap.cpp), set by aeref_set_fieldmaps: fed after the planar sensors;
// their accumulators (or, for points, FDTD::local_E* at the linked point
// after each feed) are kept for aeref_fieldmap_result.
std::vector<aefdtd_fieldmap_desc> g_maps;
std::vector<std::vector<double>> g_map_results;

int ref_orientation(int o) {
    static const int tbl[6] = {NORMAL_X, NORMAL_XM, NORMAL_Y, NORMAL_YM, NORMAL_Z, NORMAL_ZM};
    return (o >= 0 && o < 6) ? tbl[o] : NORMAL_UNDEF;
}

Material make_material(const aefdtd_material_desc &d) {
    Material m;
    m.eps_inf = d.eps_inf;
    for (int i = 0; i < d.n_debye; i++) { DebyeModel x; x.set(d.debye[i][0], d.debye[i][1]); m.debye.push_back(x); }
    for (int i = 0; i < d.n_drude; i++) { DrudeModel x; x.set(d.drude[i][0], d.drude[i][1]); m.drude.push_back(x); }
    for (int i = 0; i < d.n_lorentz; i++) { LorentzModel x; x.set(d.lorentz[i][0], d.lorentz[i][1], d.lorentz[i][2]); m.lorentz.push_back(x); }
    for (int i = 0; i < d.n_critpoint; i++) {
        CritpointModel x; x.set(d.critpoint[i][0], d.critpoint[i][1], d.critpoint[i][2], d.critpoint[i][3]);
        m.critpoint.push_back(x);
    }
    return m;
}

struct CoutSilencer {
    std::streambuf *old;
    std::ostringstream sink;
    CoutSilencer() : old(std::cout.rdbuf(sink.rdbuf())) {}
    ~CoutSilencer() { std::cout.rdbuf(old); }
};

void copy_fields(FDTD const &f, double *out) {
    size_t n = size_t(f.Nx) * f.Ny * f.Nz;
    Grid3<double> const *g[6] = {&f.Ex, &f.Ey, &f.Ez, &f.Hx, &f.Hy, &f.Hz};
    for (int c = 0; c < 6; c++)
        for (int k = 0; k < f.Nz; k++)
            for (int j = 0; j < f.Ny; j++)
                for (int i = 0; i < f.Nx; i++)
                    out[c * n + i + size_t(j) * f.Nx + size_t(k) * f.Nx * f.Ny] = (*g[c])(i, j, k);
}

}  // namespace

extern "C" {

/* Runs one simulation through the reference core.
 *   map: nx*ny*nz structure material indices, x fastest.
 *   nsteps: time-loop count (the reference's Nt for post-processing).
 * Outputs (each may be NULL):
 *   fields_out: 6 * Ntot doubles, Ex..Hz on the total grid after the loop;
 *   plane_sums_out: 12 * nsteps (normal mode), order of aefdtd_get_plane_sums;
 *   spectra_out: 15 * nl (normal mode), layout of aefdtd_get_normal_spectra;
 *   flux_out: concatenated rsp_result of every sensor;
 *   dims_out: 10 ints Nx Ny Nz xs_s xs_e ys_s ys_e zs_s zs_e Nmat;
 *   loop_seconds: wall time of the time loop alone.
 * Returns 0 on success, nonzero on a bad argument. */
int aeref_run(const aefdtd_grid_desc *g, const uint32_t *map,
              const aefdtd_material_desc *mats, int32_t nmat,
              const aefdtd_normal_desc *nd,
              const aefdtd_source_desc *srcs, int32_t nsrc,
              const aefdtd_sensor_desc *sens, int32_t nsens,
              int32_t nsteps, int32_t quiet,
              double *fields_out, double *plane_sums_out, double *spectra_out,
              double *flux_out, int32_t *dims_out, double *loop_seconds) {
    if (!g || !map || !mats || nmat <= 0 || nsteps < 0) return 1;
    if (g->mode == AEFDTD_MODE_NORMAL && !nd) return 2;
    CoutSilencer *silence = quiet ? new CoutSilencer() : nullptr;

    int Nx = g->nx, Ny = g->ny, Nz = g->nz, Nt = g->nt > 0 ? g->nt : nsteps;
    double Dx = g->dx, Dy = g->dy, Dz = g->dz;

    Grid3<unsigned int> matsgrid(Nx, Ny, Nz, 0);
    for (int k = 0; k < Nz; k++)
        for (int j = 0; j < Ny; j++)
            for (int i = 0; i < Nx; i++)
                matsgrid(i, j, k) = map[i + size_t(j) * Nx + size_t(k) * Nx * Ny];

    double Dt = g->dt;
    if (Dt <= 0) Dt = std::min(std::min(Dx, Dy), Dz) / (std::sqrt(3.0) * c_light) * 0.99 * g->time_mod;

    FDTD *fp = nullptr;
    if (g->mode == AEFDTD_MODE_NORMAL) {
        // normal_incidence.cpp:188-200
        int pad_zm = std::max(5, g->pad[AEFDTD_ZM]);
        int pad_zp = std::max(5, g->pad[AEFDTD_ZP]);
        fp = new FDTD(Nx, Ny, Nz, Nt, Dx, Dy, Dz, Dt, "NORM",
                      0, 0, 0, 0, g->pml[AEFDTD_ZM], g->pml[AEFDTD_ZP],
                      0, 0, 0, 0, pad_zm, pad_zp);
        fp->set_pml_zm(g->pml_kappa[AEFDTD_ZM], g->pml_sigma[AEFDTD_ZM], g->pml_alpha[AEFDTD_ZM]);
        fp->set_pml_zp(g->pml_kappa[AEFDTD_ZP], g->pml_sigma[AEFDTD_ZP], g->pml_alpha[AEFDTD_ZP]);
    } else {
        // default_fdtd.cpp:47-62
        fp = new FDTD(Nx, Ny, Nz, Nt, Dx, Dy, Dz, Dt, "CUSTOM",
                      g->pml[0], g->pml[1], g->pml[2], g->pml[3], g->pml[4], g->pml[5],
                      g->pad[0], g->pad[1], g->pad[2], g->pad[3], g->pad[4], g->pad[5]);
        fp->set_pml_xm(g->pml_kappa[0], g->pml_sigma[0], g->pml_alpha[0]);
        fp->set_pml_xp(g->pml_kappa[1], g->pml_sigma[1], g->pml_alpha[1]);
        fp->set_pml_ym(g->pml_kappa[2], g->pml_sigma[2], g->pml_alpha[2]);
        fp->set_pml_yp(g->pml_kappa[3], g->pml_sigma[3], g->pml_alpha[3]);
        fp->set_pml_zm(g->pml_kappa[4], g->pml_sigma[4], g->pml_alpha[4]);
        fp->set_pml_zp(g->pml_kappa[5], g->pml_sigma[5], g->pml_alpha[5]);
    }
    FDTD &fdtd = *fp;
    fdtd.set_tapering(g->tapering);
    fdtd.set_matsgrid(matsgrid);
    for (int m = 0; m < nmat; m++) fdtd.set_material(m, make_material(mats[m]));
    fdtd.bootstrap();

    Nx = fdtd.Nx; Ny = fdtd.Ny; Nz = fdtd.Nz;
    if (dims_out) {
        int d[10] = {fdtd.Nx, fdtd.Ny, fdtd.Nz, fdtd.xs_s, fdtd.xs_e, fdtd.ys_s, fdtd.ys_e,
                     fdtd.zs_s, fdtd.zs_e, int(fdtd.Nmat)};
        for (int i = 0; i < 10; i++) dims_out[i] = d[i];
    }

    std::vector<Sensor *> sensors;
    for (int s = 0; s < nsens; s++) {
        Spect_Poynting *sp = new Spect_Poynting(ref_orientation(sens[s].orientation),
                                                sens[s].box[0], sens[s].box[1], sens[s].box[2],
                                                sens[s].box[3], sens[s].box[4], sens[s].box[5]);
        sp->set_spectrum(sens[s].nl, sens[s].lambda_min, sens[s].lambda_max);
        sp->name = "aeref_sensor";
        sp->link(fdtd, std::filesystem::path("."));
        sp->set_silent(true);
        sensors.push_back(sp);
    }
    Box_Spect_Poynting *bx = nullptr;
    if (g_box_on) {
        bx = new Box_Spect_Poynting(g_box[0], g_box[1], g_box[2], g_box[3], g_box[4], g_box[5]);
        bx->disable_xm = g_box_mask & 1; bx->disable_xp = g_box_mask & 2;
        bx->disable_ym = g_box_mask & 4; bx->disable_yp = g_box_mask & 8;
        bx->disable_zm = g_box_mask & 16; bx->disable_zp = g_box_mask & 32;
        bx->set_spectrum(g_box_nl, g_box_lmin, g_box_lmax);
        bx->name = "aeref_box";
        bx->set_silent(true);
        bx->link(fdtd, std::filesystem::path("."));
    }
    std::vector<Sensor *> maps;
    g_map_results.assign(g_maps.size(), {});
    for (const aefdtd_fieldmap_desc &d : g_maps) {
        Sensor *m = nullptr;
        if (d.kind == AEFDTD_MAP_PLANE) {
            FieldMap *fm = new FieldMap(ref_orientation(d.orientation), d.box[0], d.box[1], d.box[2], d.box[3],
                                        d.box[4], d.box[5]);
            fm->set_cumulative(d.cumulative != 0);
            fm->set_mag_map(d.magnetic != 0);
            fm->set_spectrum(d.lambda);
            m = fm;
        } else if (d.kind == AEFDTD_MAP_BLOCK) {
            m = new FieldBlock(d.box[0], d.box[1], d.box[2], d.box[3], d.box[4], d.box[5]);
            m->set_spectrum(d.lambda);
        } else {
            m = new FieldPoint(d.box[0], d.box[2], d.box[4]);
            m->set_spectrum(d.lambda > 0 ? d.lambda : 500e-9);
        }
        m->name = "aeref_map";
        m->set_silent(true);
        // FieldPoint::initialize opens its text output under the working directory
        m->link(fdtd, std::filesystem::temp_directory_path());
        maps.push_back(m);
    }
    auto feed_maps = [&] {
        for (size_t i = 0; i < maps.size(); i++) {
            maps[i]->feed(fdtd);
            if (g_maps[i].kind == AEFDTD_MAP_POINT) {
                const Sensor &p = *maps[i];
                g_map_results[i].push_back(fdtd.local_Ex(p.x1, p.y1, p.z1));
                g_map_results[i].push_back(fdtd.local_Ey(p.x1, p.y1, p.z1));
                g_map_results[i].push_back(fdtd.local_Ez(p.x1, p.y1, p.z1));
            }
        }
    };
    std::vector<Source *> sources;
    if (g->mode == AEFDTD_MODE_CUSTOM) {
        for (int s = 0; s < nsrc; s++) {
            Oscillator *o = new Oscillator(ref_orientation(srcs[s].orientation),
                                           srcs[s].box[0], srcs[s].box[1], srcs[s].box[2],
                                           srcs[s].box[3], srcs[s].box[4], srcs[s].box[5]);
            o->set_spectrum(srcs[s].lambda_min, srcs[s].lambda_max);
            o->link(fdtd);
            sources.push_back(o);
        }
    }

    auto t0 = std::chrono::steady_clock::now();

    if (g->mode == AEFDTD_MODE_NORMAL) {
        int zs_s = fdtd.zs_s, zs_e = fdtd.zs_e;
        int Nl = nd->nl;
        std::vector<double> Lambda(Nl), w(Nl);
        for (int l = 0; l < Nl; l++) Lambda[l] = nd->lambda_min + (nd->lambda_max - nd->lambda_min) * l / (Nl - 1.0);
        for (int l = 0; l < Nl; l++) w[l] = 2.0 * Pi * c_light / Lambda[l];
        double pol = nd->polarization == 1 ? 90 : 0;
        double eps_sub = fdtd.mats[fdtd.matsgrid(0, 0, zs_s)].ei;
        double eps_sup = fdtd.mats[fdtd.matsgrid(0, 0, zs_e)].ei;
        double index_sub = std::sqrt(eps_sub);
        double index_sup = std::sqrt(eps_sup);
        ChpIn inj_chp;
        inj_chp.init_pulse(nd->lambda_min, nd->lambda_max, 0, pol, 0, 0, 0, (zs_e - 1) * Dz, index_sup);

        int NtR = nsteps;
        std::vector<double> S[12];
        for (auto &v : S) v.assign(NtR, 0.0);
        CompletionSensor *cpl = nullptr;
        g_cc_stop = -1;
        g_cc_last = g_cc_max = 0;
        if (g_cc_coeff > 0 && g_cc_np > 0) {
            seedp(g_cc_seed);
            cpl = new CompletionSensor(g_cc_lmin, g_cc_lmax, g_cc_coeff, g_cc_np, g_cc_layout);
            cpl->link(fdtd, std::filesystem::path("."));
        } else if (g_cc_coeff > 0) {
            cpl = new CompletionSensor(g_cc_coeff);
            cpl->link(fdtd, std::filesystem::path("."));
        }
        int NtSpec = NtR;
        double tb = 0;
        for (int t = 0; t < NtR; t++) {
            fdtd.update_E();
            tb = t * Dt;
            double inj_Hx = inj_chp.Hx(0, 0, (zs_e - 1 + 0.5) * Dz, tb);
            double inj_Hy = inj_chp.Hy(0, 0, (zs_e - 1 + 0.5) * Dz, tb);
            for (int j = 0; j < Ny; j++)
                for (int i = 0; i < Nx; i++) {
                    fdtd.Ex(i, j, zs_e - 1) -= fdtd.dtdez * inj_Hy / eps_sup;
                    fdtd.Ey(i, j, zs_e - 1) += fdtd.dtdez * inj_Hx / eps_sup;
                }
            fdtd.update_H();
            tb = (t + 0.5) * Dt;
            double inj_Ex = inj_chp.Ex(0, 0, (zs_e - 1) * Dz, tb);
            double inj_Ey = inj_chp.Ey(0, 0, (zs_e - 1) * Dz, tb);
            for (int j = 0; j < Ny; j++)
                for (int i = 0; i < Nx; i++) {
                    fdtd.Hx(i, j, zs_e - 1) += fdtd.dtdmz * inj_Ey;
                    fdtd.Hy(i, j, zs_e - 1) -= fdtd.dtdmz * inj_Ex;
                }
            for (auto *s : sensors) s->feed(fdtd);
            if (bx) bx->feed(fdtd);
            feed_maps();
            if (cpl) cpl->feed(fdtd);   // fed with the sensors, after the planar ones

            tb = (t + 0.5) * Dt;
            double Dx2 = Dx / 2.0, Dy2 = Dy / 2.0, Dz2 = Dz / 2.0;
            double tapering = 1.0;
            if (t >= Nt - g->tapering) tapering = s_curve(t, Nt - 1.0, Nt - g->tapering);
            for (int j = 0; j < Ny; j++) {
                double y = j * Dy;
                for (int i = 0; i < Nx; i++) {
                    double x = i * Dx;
                    double z = (zs_e - 2) * Dz;
                    S[0][t] += inj_chp.Ex(x + Dx2, y, z, tb) * tapering;
                    S[1][t] += inj_chp.Ey(x, y + Dy2, z, tb) * tapering;
                    S[2][t] += inj_chp.Ez(x, y, z + Dz2, tb) * tapering;
                    S[3][t] += (fdtd.Ex(i, j, zs_e - 2) - inj_chp.Ex(x + Dx2, y, z, tb)) * tapering;
                    S[4][t] += (fdtd.Ey(i, j, zs_e - 2) - inj_chp.Ey(x, y + Dy2, z, tb)) * tapering;
                    S[5][t] += (fdtd.Ez(i, j, zs_e - 2) - inj_chp.Ez(x, y, z + Dz2, tb)) * tapering;
                    z = (zs_s)*Dz;
                    S[6][t] += inj_chp.Ex(x + Dx2, y, z, tb) * tapering;
                    S[7][t] += inj_chp.Ey(x, y + Dy2, z, tb) * tapering;
                    S[8][t] += inj_chp.Ez(x, y, z + Dz2, tb) * tapering;
                    S[9][t] += fdtd.Ex(i, j, zs_s) * tapering;
                    S[10][t] += fdtd.Ey(i, j, zs_s) * tapering;
                    S[11][t] += fdtd.Ez(i, j, zs_s) * tapering;
                }
            }
            if (cpl && t % g_cc_every == 0 && cpl->completion_check()) {
                // the driver's Nt = t: spectra from the first t samples
                g_cc_stop = t;
                g_cc_last = cpl->energy_last;
                g_cc_max = cpl->energy_max;
                NtSpec = t;
                break;
            }
            if (cpl) { g_cc_last = cpl->energy_last; g_cc_max = cpl->energy_max; }
        }
        delete cpl;
        if (loop_seconds) loop_seconds[0] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (plane_sums_out)
            for (int c = 0; c < 12; c++)
                for (int t = 0; t < NtR; t++) plane_sums_out[size_t(c) * NtR + t] = S[c][t];

        if (spectra_out) {
            // normal_incidence.cpp:442-570 with Nt = number of steps run
            // (or the completion step).
            int NtP = NtSpec;
            double hsup, hsub, hstruc;
            fdtd.find_slab(zs_s, zs_e - 1, hsub, hstruc, hsup);
            hsup -= Dz / 2.0;
            hsub -= Dz / 2.0;
            for (int l = 0; l < Nl; l++) {
                Imdouble ref1x = 0, ref1y = 0, ref1z = 0, ref2x = 0, ref2y = 0, ref2z = 0;
                Imdouble trans1x = 0, trans1y = 0, trans1z = 0, trans2x = 0, trans2y = 0, trans2z = 0;
                double k0 = -w[l] / c_light;
                double k1 = k0 * index_sup;
                double k3 = k0 * index_sub;
                Imdouble tmp_sup = std::exp(2.0 * k1 * hsup * Im);
                Imdouble tmp_sub = std::exp((k3 * hsub - k0 * (hstruc + hsub)) * Im);
                for (int t = 0; t < NtP; t++) {
                    Imdouble tmp1 = std::exp(t * Dt * w[l] * Im) / (NtP - 1.0);
                    Imdouble tmp2 = tmp1 * tmp_sup;
                    Imdouble tmp3 = tmp1 * tmp_sub;
                    ref1x += S[0][t] * tmp1; ref1y += S[1][t] * tmp1; ref1z += S[2][t] * tmp1;
                    ref2x += S[3][t] * tmp2; ref2y += S[4][t] * tmp2; ref2z += S[5][t] * tmp2;
                    trans1x += S[6][t] * tmp1; trans1y += S[7][t] * tmp1; trans1z += S[8][t] * tmp1;
                    trans2x += S[9][t] * tmp3; trans2y += S[10][t] * tmp3; trans2z += S[11][t] * tmp3;
                }
                double *o = spectra_out + size_t(l) * 15;
                o[0] = Lambda[l];
                double a = std::sqrt(std::norm(ref2x) + std::norm(ref2y) + std::norm(ref2z));
                double b = std::sqrt(std::norm(ref1x) + std::norm(ref1y) + std::norm(ref1z));
                o[1] = a / b;
                a = std::sqrt(std::norm(trans2x) + std::norm(trans2y) + std::norm(trans2z));
                b = std::sqrt(std::norm(trans1x) + std::norm(trans1y) + std::norm(trans1z));
                o[2] = a / b;
                Imdouble ref0 = ref1y, trans0 = trans1y;
                if (nd->polarization == 1) { ref0 = ref1x; trans0 = trans1x; }
                Imdouble refx = ref2x / ref0, refy = ref2y / ref0;
                Imdouble transx = trans2x / trans0, transy = trans2y / trans0;
                o[3] = std::abs(refx); o[4] = std::arg(refx); o[5] = std::norm(refx);
                o[6] = std::abs(refy); o[7] = std::arg(refy); o[8] = std::norm(refy);
                o[9] = std::abs(transx); o[10] = std::arg(transx); o[11] = std::norm(transx) * index_sub / index_sup;
                o[12] = std::abs(transy); o[13] = std::arg(transy); o[14] = std::norm(transy) * index_sub / index_sup;
            }
        }
    } else {
        for (int t = 0; t < nsteps; t++) {
            fdtd.update_E();
            for (auto *s : sources) s->inject_E(fdtd);
            fdtd.update_H();
            for (auto *s : sensors) s->feed(fdtd);
            if (bx) bx->feed(fdtd);
            feed_maps();
            for (auto *s : sources) s->inject_H(fdtd);
        }
        if (loop_seconds) loop_seconds[0] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }

    if (fields_out) copy_fields(fdtd, fields_out);
    size_t off = 0;
    for (size_t s = 0; s < sensors.size(); s++) {
        sensors[s]->treat();
        if (flux_out)
            for (int l = 0; l < sensors[s]->Nl; l++) flux_out[off + l] = sensors[s]->rsp_result[l];
        off += sensors[s]->Nl;
    }
    if (bx) {
        bx->treat();
        g_box_result.assign(bx->Nl, 0.0);
        for (int l = 0; l < bx->Nl; l++) g_box_result[l] = bx->rsp_result[l];
        delete bx;
    }
    for (size_t i = 0; i < maps.size(); i++) {
        std::vector<double> &o = g_map_results[i];
        if (g_maps[i].kind == AEFDTD_MAP_PLANE) {
            FieldMap &fm = *static_cast<FieldMap *>(maps[i]);
            Grid2<Imdouble> *acc[3] = {&fm.acc_Ex, &fm.acc_Ey, &fm.acc_Ez};
            for (int c = 0; c < 3; c++)
                for (int j = 0; j < fm.span2; j++)
                    for (int i = 0; i < fm.span1; i++) {
                        o.push_back((*acc[c])(i, j).real());
                        o.push_back((*acc[c])(i, j).imag());
                    }
        } else if (g_maps[i].kind == AEFDTD_MAP_BLOCK) {
            FieldBlock &fb = *static_cast<FieldBlock *>(maps[i]);
            Grid3<Imdouble> *acc[6] = {&fb.Ex, &fb.Ey, &fb.Ez, &fb.Hx, &fb.Hy, &fb.Hz};
            for (int c = 0; c < 6; c++)
                for (int k = 0; k < fb.span3; k++)
                    for (int j = 0; j < fb.span2; j++)
                        for (int i = 0; i < fb.span1; i++) {
                            o.push_back((*acc[c])(i, j, k).real());
                            o.push_back((*acc[c])(i, j, k).imag());
                        }
        }
        delete maps[i];
    }
    for (auto *s : sensors) delete s;
    for (auto *s : sources) delete s;
    delete fp;
    delete silence;
    return 0;
}

/* Oblique incidence at one in-plane wavevector through the reference core:
 * FDTD_oblique_biphase_comp (oblique_biphase.cpp:29-480) minus the
 * structure discretisation (map is the structure-size material map), the
 * previews, sensors and files. Outputs (each may be NULL): fields_out 12 *
 * Ntot doubles (Ex..Hz of fdtd_r, then of fdtd_i, without the ghost layers);
 * series_out nsteps * 18 (BRsensorX..Z, RsensorX..Z, TsensorX..Z as re, im);
 * spectra_out nl_max * 10 (the obl_ file columns), nl_out the resized Nl;
 * dims_out as for aeref_run. */
int aeref_run_oblique(const aefdtd_grid_desc *g, const uint32_t *map, const aefdtd_material_desc *mats, int32_t nmat,
                      const aefdtd_oblique_desc *od, int32_t nsteps, int32_t quiet, double *fields_out,
                      double *series_out, double *spectra_out, int32_t nl_max, int32_t *nl_out, int32_t *dims_out,
                      double *loop_seconds) {
    if (!g || !map || !mats || nmat <= 0 || nsteps < 0 || !od) return 1;
    CoutSilencer *silence = quiet ? new CoutSilencer() : nullptr;
    int Nx = g->nx, Ny = g->ny, Nz = g->nz, Nt = nsteps;
    double Dx = g->dx, Dy = g->dy, Dz = g->dz;
    Grid3<unsigned int> matsgrid(Nx, Ny, Nz, 0);
    for (int k = 0; k < Nz; k++)
        for (int j = 0; j < Ny; j++)
            for (int i = 0; i < Nx; i++) matsgrid(i, j, k) = map[i + size_t(j) * Nx + size_t(k) * Nx * Ny];
    double Dt = g->dt;
    if (Dt <= 0) Dt = std::min(std::min(Dx, Dy), Dz) / (std::sqrt(3.0) * c_light) * 0.99 * g->time_mod;
    const int pad_zm = std::max(5, g->pad[AEFDTD_ZM]), pad_zp = std::max(5, g->pad[AEFDTD_ZP]);
    FDTD fdtd_r(Nx, Ny, Nz, Nt, Dx, Dy, Dz, Dt, "OBL_PHASE", 0, 0, 0, 0, g->pml[AEFDTD_ZM], g->pml[AEFDTD_ZP],
                0, 0, 0, 0, pad_zm, pad_zp);
    FDTD fdtd_i(Nx, Ny, Nz, Nt, Dx, Dy, Dz, Dt, "OBL_PHASE", 0, 0, 0, 0, g->pml[AEFDTD_ZM], g->pml[AEFDTD_ZP],
                0, 0, 0, 0, pad_zm, pad_zp);
    for (FDTD *f : {&fdtd_r, &fdtd_i}) {
        f->set_pml_zm(g->pml_kappa[AEFDTD_ZM], g->pml_sigma[AEFDTD_ZM], g->pml_alpha[AEFDTD_ZM]);
        f->set_pml_zp(g->pml_kappa[AEFDTD_ZP], g->pml_sigma[AEFDTD_ZP], g->pml_alpha[AEFDTD_ZP]);
        f->set_tapering(g->tapering);
        f->set_matsgrid(matsgrid);
        for (int m = 0; m < nmat; m++) f->set_material(m, make_material(mats[m]));
        f->bootstrap();
    }
    Nx = fdtd_r.Nx; Ny = fdtd_r.Ny; Nz = fdtd_r.Nz;
    const int zs_s = fdtd_r.zs_s, zs_e = fdtd_r.zs_e;
    if (dims_out) {
        int d[10] = {fdtd_r.Nx, fdtd_r.Ny, fdtd_r.Nz, fdtd_r.xs_s, fdtd_r.xs_e, fdtd_r.ys_s, fdtd_r.ys_e,
                     fdtd_r.zs_s, fdtd_r.zs_e, int(fdtd_r.Nmat)};
        for (int i = 0; i < 10; i++) dims_out[i] = d[i];
    }
    double eps_sub = fdtd_r.mats[fdtd_r.matsgrid(0, 0, zs_s)].ei;
    double eps_sup = fdtd_r.mats[fdtd_r.matsgrid(0, 0, zs_e)].ei;
    double index_sub = std::sqrt(eps_sub), index_sup = std::sqrt(eps_sup);
    double kx = od->kx_in * index_sup, ky = od->ky_in * index_sup, kxy = std::sqrt(kx * kx + ky * ky);
    AngleRad pol;
    pol.degree(0);
    if (od->polarization == 1) pol.degree(90);
    Bloch_Wideband inc_field(0, Nx, 0, Ny, 0, fdtd_r.Nz_s, kx, ky, pol);
    inc_field.set_spectrum(od->lambda_min, od->lambda_max);
    inc_field.link(fdtd_r);
    Imdouble dephasE_x = std::exp(kx * Nx * Dx * Im), dephasE_y = std::exp(ky * Ny * Dy * Im);
    Imdouble dephasH_x = std::exp(-kx * Nx * Dx * Im), dephasH_y = std::exp(-ky * Ny * Dy * Im);
    fdtd_r.set_kx(kx); fdtd_r.set_ky(ky);
    fdtd_i.set_kx(kx); fdtd_i.set_ky(ky);
    Grid2<double> inc_Ex(Nx, Ny, 0), inc_Ey(Nx, Ny, 0), inc_Ez(Nx, Ny, 0);
    Grid2<Imdouble> mk_x(Nx, Ny, 0), mk_y(Nx, Ny, 0), mk_z(Nx, Ny, 0);
    for (int i = 0; i < Nx; i++)
        for (int j = 0; j < Ny; j++) {
            mk_x(i, j) = std::exp(-(kx * (i + 0.5) * Dx + ky * j * Dy) * Im);
            mk_y(i, j) = std::exp(-(kx * i * Dx + ky * (j + 0.5) * Dy) * Im);
            mk_z(i, j) = std::exp(-(kx * i * Dx + ky * j * Dy) * Im);
        }
    std::vector<Imdouble> BR[3], R[3], T[3];
    for (int d = 0; d < 3; d++) { BR[d].assign(Nt, 0); R[d].assign(Nt, 0); T[d].assign(Nt, 0); }
    fdtd_r.reset_fields();
    fdtd_i.reset_fields();
    fdtd_r.tstep = 0;
    fdtd_i.tstep = 0;
    auto t0 = std::chrono::steady_clock::now();
    Imdouble i_E, i_H;
    for (int t = 0; t < Nt; t++) {
        for (int k = 0; k < Nz; k++) {   // Bloch conditions, H (:211-240)
            for (int i = 0; i < Nx; i++) {
                i_H = fdtd_r.Hx(i, Ny - 1, k) + fdtd_i.Hx(i, Ny - 1, k) * Im;
                fdtd_r.Hx(i, Ny, k) = std::real(i_H * dephasH_y);
                fdtd_i.Hx(i, Ny, k) = std::imag(i_H * dephasH_y);
                i_H = fdtd_r.Hz(i, Ny - 1, k) + fdtd_i.Hz(i, Ny - 1, k) * Im;
                fdtd_r.Hz(i, Ny, k) = std::real(i_H * dephasH_y);
                fdtd_i.Hz(i, Ny, k) = std::imag(i_H * dephasH_y);
            }
            for (int j = 0; j < Ny; j++) {
                i_H = fdtd_r.Hy(Nx - 1, j, k) + fdtd_i.Hy(Nx - 1, j, k) * Im;
                fdtd_r.Hy(Nx, j, k) = std::real(i_H * dephasH_x);
                fdtd_i.Hy(Nx, j, k) = std::imag(i_H * dephasH_x);
                i_H = fdtd_r.Hz(Nx - 1, j, k) + fdtd_i.Hz(Nx - 1, j, k) * Im;
                fdtd_r.Hz(Nx, j, k) = std::real(i_H * dephasH_x);
                fdtd_i.Hz(Nx, j, k) = std::imag(i_H * dephasH_x);
            }
        }
        fdtd_r.update_E();
        fdtd_i.update_E();
        inc_field.inject_E(fdtd_r, fdtd_i);
        for (int k = 0; k < Nz; k++) {   // Bloch conditions, E (:252-282)
            for (int i = 0; i < Nx; i++) {
                i_E = fdtd_r.Ex(i, 0, k) + fdtd_i.Ex(i, 0, k) * Im;
                fdtd_r.Ex(i, Ny, k) = std::real(i_E * dephasE_y);
                fdtd_i.Ex(i, Ny, k) = std::imag(i_E * dephasE_y);
                i_E = fdtd_r.Ez(i, 0, k) + fdtd_i.Ez(i, 0, k) * Im;
                fdtd_r.Ez(i, Ny, k) = std::real(i_E * dephasE_y);
                fdtd_i.Ez(i, Ny, k) = std::imag(i_E * dephasE_y);
            }
            for (int j = 0; j < Ny; j++) {
                i_E = fdtd_r.Ey(0, j, k) + fdtd_i.Ey(0, j, k) * Im;
                fdtd_r.Ey(Nx, j, k) = std::real(i_E * dephasE_x);
                fdtd_i.Ey(Nx, j, k) = std::imag(i_E * dephasE_x);
                i_E = fdtd_r.Ez(0, j, k) + fdtd_i.Ez(0, j, k) * Im;
                fdtd_r.Ez(Nx, j, k) = std::real(i_E * dephasE_x);
                fdtd_i.Ez(Nx, j, k) = std::imag(i_E * dephasE_x);
            }
        }
        fdtd_r.update_H();
        fdtd_i.update_H();
        inc_field.inject_H(fdtd_r, fdtd_i);
        double tb = (t + 0.5) * Dt;   // R/T sums (:300-327)
        double z = zs_s * Dz;
        inc_field.get_E(inc_Ex, inc_Ey, inc_Ez, z, tb);
        for (int i = 0; i < Nx; i++)
            for (int j = 0; j < Ny; j++) {
                BR[0][t] += inc_Ex(i, j) * mk_x(i, j);
                BR[1][t] += inc_Ey(i, j) * mk_y(i, j);
                BR[2][t] += inc_Ez(i, j) * mk_z(i, j);
                R[0][t] += fdtd_r.Ex(i, j, zs_e + 2) * mk_x(i, j);
                R[1][t] += fdtd_r.Ey(i, j, zs_e + 2) * mk_y(i, j);
                R[2][t] += 0.5 * (fdtd_r.Ez(i, j, zs_e + 1) + fdtd_r.Ez(i, j, zs_e + 2)) * mk_z(i, j);
                T[0][t] += fdtd_r.Ex(i, j, zs_s) * mk_x(i, j);
                T[1][t] += fdtd_r.Ey(i, j, zs_s) * mk_y(i, j);
                T[2][t] += 0.5 * (fdtd_r.Ez(i, j, zs_s) + fdtd_r.Ez(i, j, zs_s - 1)) * mk_z(i, j);
            }
    }
    if (loop_seconds) loop_seconds[0] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (fields_out) {
        const size_t n = size_t(Nx) * Ny * Nz;
        copy_fields(fdtd_r, fields_out);
        copy_fields(fdtd_i, fields_out + 6 * n);
    }
    if (series_out)
        for (int t = 0; t < Nt; t++)
            for (int d = 0; d < 3; d++) {
                double *o = series_out + size_t(t) * 18;
                o[2 * d] = BR[d][t].real(); o[2 * d + 1] = BR[d][t].imag();
                o[6 + 2 * d] = R[d][t].real(); o[7 + 2 * d] = R[d][t].imag();
                o[12 + 2 * d] = T[d][t].real(); o[13 + 2 * d] = T[d][t].imag();
            }
    if (spectra_out && Nt >= 2) {
        // :334-480
        int Nl = od->nl;
        double lambda_min = od->lambda_min, lambda_max = od->lambda_max;
        double lambda_limit_max = lambda_max;
        if (kx != 0 || ky != 0) lambda_limit_max = 2 * Pi * std::sin(89.0 * Pi / 180.0) * index_sup / kxy;
        if (lambda_limit_max < lambda_max) {
            double D_lambda = (lambda_max - lambda_min) / (Nl - 1.0);
            Nl = static_cast<int>((lambda_limit_max - lambda_min) / D_lambda);
            if (Nl < 2) Nl = 2;
            lambda_max = lambda_min + (Nl - 1.0) * D_lambda;
        }
        if (nl_out) *nl_out = Nl;
        double hsup, hsub, hstruc;
        fdtd_r.find_slab(zs_s, zs_e + 2, hsub, hstruc, hsup);
        AngleRad inc_ang, ref_ang, phi(std::atan2(ky, kx));
        phi = std::atan2(ky, kx);
        double cp = std::cos(phi), sp = std::sin(phi);
        for (int l = 0; l < Nl && l < nl_max; l++) {
            double lambda = lambda_min + (lambda_max - lambda_min) * l / (Nl - 1.0);
            double w = 2.0 * Pi * c_light / lambda;
            double kn = 2.0 * Pi * index_sup / lambda;
            inc_ang = std::asin(kxy / kn);
            ref_ang = std::asin(index_sup / index_sub * std::sin(inc_ang));
            double s_k0 = -w / c_light, s_k1 = s_k0 * index_sup, s_k3 = s_k0 * index_sub;
            Imdouble BRS[3] = {0, 0, 0}, RS[3] = {0, 0, 0}, BTS[3] = {0, 0, 0}, TS[3] = {0, 0, 0};
            for (int t = 0; t < Nt; t++) {
                Imdouble coeff = std::exp(w * t * Dt * Im);
                for (int d = 0; d < 3; d++) {
                    BRS[d] += BR[d][t] * coeff;
                    RS[d] += R[d][t] * coeff;
                    BTS[d] += BR[d][t] * coeff;
                    TS[d] += T[d][t] * coeff;
                }
            }
            Imdouble *rot[4] = {BRS, RS, BTS, TS};
            for (Imdouble *v : rot) {
                Imdouble tmp_x = v[0], tmp_y = v[1];
                v[0] = cp * tmp_x + sp * tmp_y;
                v[1] = -sp * tmp_x + cp * tmp_y;
            }
            double s_k1z = s_k1 * std::cos(inc_ang);
            Imdouble tmp_sup = im_exp((2.0 * hsup + 2 * Dz) * s_k1z);
            Imdouble tmp_sub = im_exp(s_k3 * (hsub - Dz / 2.0) * std::cos(ref_ang) + s_k0 * (hsup + Dz / 2.0) * std::cos(inc_ang));
            bool tm = od->polarization == 1;
            Imdouble Rbase = tm ? BRS[0] : BRS[1], Tbase = tm ? BTS[0] : BTS[1];
            double base_norm_ref = std::abs(BRS[1]), base_norm_trans = std::abs(BTS[1]);
            if (tm) {
                base_norm_ref = std::sqrt(std::norm(BRS[0]) + std::norm(BRS[2]));
                base_norm_trans = std::sqrt(std::norm(BTS[0]) + std::norm(BTS[2]));
            }
            double TE_norm_ref = std::abs(RS[1]), TM_norm_ref = std::sqrt(std::norm(RS[0]) + std::norm(RS[2]));
            double TE_norm_trans = std::abs(TS[1]), TM_norm_trans = std::sqrt(std::norm(TS[0]) + std::norm(TS[2]));
            double TE_arg_ref = std::arg(RS[1] / Rbase * tmp_sup), TM_arg_ref = std::arg(RS[0] / Rbase * tmp_sup);
            double TE_arg_trans = std::arg(TS[1] / Tbase * tmp_sub), TM_arg_trans = std::arg(TS[0] / Tbase * tmp_sub);
            Imdouble sp4[4] = {TE_norm_ref / base_norm_ref * std::exp(TE_arg_ref * Im),
                               TM_norm_ref / base_norm_ref * std::exp(TM_arg_ref * Im),
                               TE_norm_trans / base_norm_trans * std::exp(TE_arg_trans * Im),
                               TM_norm_trans / base_norm_trans * std::exp(TM_arg_trans * Im)};
            double *o = spectra_out + size_t(l) * 10;
            o[0] = lambda;
            o[1] = inc_ang.degree();
            for (int q = 0; q < 4; q++) { o[2 + 2 * q] = std::abs(sp4[q]); o[3 + 2 * q] = std::arg(sp4[q]); }
        }
    }
    delete silence;
    return 0;
}

/* Number of worker threads the reference core uses per FDTD object. */
int aeref_threads(void) { return max_threads_number(); }

/* Box spectral Poynting sensor for the following aeref_run calls: box in
 * structure cells, disabled_mask bits xm, xp, ym, yp, zm, zp; nl <= 0 turns
 * it off. */
void aeref_set_box(const int32_t box[6], int32_t nl, double lmin, double lmax, int32_t disabled_mask) {
    g_box_on = nl > 0;
    for (int i = 0; i < 6; i++) g_box[i] = box ? box[i] : 0;
    g_box_nl = nl;
    g_box_lmin = lmin;
    g_box_lmax = lmax;
    g_box_mask = disabled_mask;
}

/* Field sensors for the following aeref_run calls (n = 0: none). */
void aeref_set_fieldmaps(const aefdtd_fieldmap_desc *d, int32_t n) {
    g_maps.assign(d, d + (n > 0 ? n : 0));
}

/* Results of field sensor idx after the last aeref_run: plane maps 3 x span2
 * x span1 and blocks 6 x span3 x span2 x span1 complex as (re, im), i fastest;
 * points steps x 3. Returns the number of doubles, copying at most count. */
int64_t aeref_fieldmap_result(int32_t idx, double *out, int64_t count) {
    if (idx < 0 || idx >= (int)g_map_results.size()) return -1;
    const std::vector<double> &v = g_map_results[idx];
    for (int64_t i = 0; i < count && i < (int64_t)v.size(); i++) out[i] = v[i];
    return (int64_t)v.size();
}

/* rsp_result of the box after the last aeref_run (nl values). */
int aeref_box_result(double *out, int32_t nl) {
    if ((int)g_box_result.size() != nl) return 1;
    for (int l = 0; l < nl; l++) out[l] = g_box_result[l];
    return 0;
}

/* Completion sensor for the following aeref_run calls (normal mode):
 * coeff <= 0 disables; every = the driver's cc_step. */
void aeref_set_completion(double coeff, int32_t every) {
    g_cc_coeff = coeff;
    g_cc_every = every > 0 ? every : 500;
    g_cc_np = 0;
}

/* FT-mode completion sensor for the following aeref_run calls (normal mode). */
void aeref_set_completion_ft(double lmin, double lmax, double coeff, int32_t np, const char *layout, int32_t seed,
                             int32_t every) {
    aeref_set_completion(coeff, every);
    g_cc_np = np;
    g_cc_lmin = lmin;
    g_cc_lmax = lmax;
    g_cc_layout = layout ? layout : "";
    g_cc_seed = seed;
}

/* Result of the last aeref_run with completion: stop step t (-1 if it ran
 * to the end) and the last and largest grid energies. */
void aeref_completion_result(int32_t *stop, double *last, double *max) {
    if (stop) *stop = g_cc_stop;
    if (last) *last = g_cc_last;
    if (max) *max = g_cc_max;
}

}  // extern "C"
