/* fdtd_oracle.cpp — CPU restatement of the reference FDTD path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA library. Only tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg load it; the
 * product library never links or calls it.
 *
 * A single-threaded FP64 restatement, in plain loops, of the reference core
 * (KAHR-Alpha/Aether, src/finite_differences/FDTD). Each function cites the
 * reference lines it follows. Operation order inside every expression is the
 * reference's, and the library is built with -ffp-contract=off like the
 * reference's x86-64 build (SSE2, no FMA), so on the same inputs it is
 * bit-identical to the reference core; tests pin it against the reference
 * compiled from source (oracle/_ref) and against committed golden fixtures.
 * std::complex and <cmath> are used where the reference uses them, so the
 * coefficient generation (complex exp/pow) matches bit for bit.
 *
 * Exported entry: aeoracle_run, same signature and outputs as aeref_run
 * (oracle/ref_driver.cpp).
 */
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <numbers>
#include <vector>

#include "../include/aefdtd.h"

namespace {

typedef std::complex<double> cplx;
const cplx Im(0, 1);
const double Pi = std::numbers::pi_v<double>;
// src/common/phys_constants.h:18-20
const double e0 = 8.854187817e-12;
const double mu0 = 12.566370614e-7;
const double c_light = 299792458.0;

// src/common/mathUT.cpp:1186-1193
double s_curve(double x, double xmin, double xmax) {
    double u = (x - xmin) / (xmax - xmin);
    if (u <= 0) return 0;
    else if (u >= 1.0) return 1.0;
    else return u * u * (3.0 - 2.0 * u);
}

struct Grid {
    int nx = 0, ny = 0, nz = 0;
    std::vector<double> v;
    void init(int a, int b, int c) { nx = a; ny = b; nz = c; v.assign(size_t(a) * b * c, 0.0); }
    double &operator()(int i, int j, int k) { return v[i + size_t(j) * nx + size_t(k) * nx * ny]; }
    double operator()(int i, int j, int k) const { return v[i + size_t(j) * nx + size_t(k) * nx * ny]; }
};

struct Mat {
    // FDTD_Material (src/finite_differences/FDTD/core/fdtd_material.h:38-268)
    bool rc = false;
    int Np = 0;
    double C1 = 1, C2x = 0, C2y = 0, C2z = 0, C3 = 0, C4 = 0, ei = 1, sig = 0;
    std::vector<cplx> Crec, Dchi, chi;
    int x1 = 0, y1 = 0, z1 = 0, xs = 0, ys = 0, zs = 0;
    std::vector<cplx> psi;  // (i-x1, j-y1, k-z1, 3p+d), i fastest (Grid4 order)
    cplx &P(int i, int j, int k, int c) {
        return psi[(i - x1) + size_t(j - y1) * xs + size_t(k - z1) * xs * ys + size_t(c) * xs * ys * zs];
    }
};

struct Osc {
    // Oscillator (src/finite_differences/FDTD/sources/sc_oscillator.cpp)
    int comp, x1, x2, y1, y2, z1, z2, step = 0;
    double w0, dw;
    int tshift;
};

struct PlaneSensor {
    // Spect_Poynting / SensorFieldHolder (sensors.cpp:423-644, s_spec_power.cpp:32-119)
    int type, x1, x2, y1, y2, z1, z2, span1, span2, Nl, step = 0;
    double tapering_E = 1.0, tapering_H = 1.0;
    std::vector<double> lambda;
    std::vector<double> t[6];
    std::vector<cplx> sp[6];
    std::vector<double> rsp;
};

struct Sim {
    int mode;
    int Nx, Ny, Nz, Nt, Ntap, tstep = 0;
    int Nx_s, Ny_s, Nz_s, xs_s, xs_e, ys_s, ys_e, zs_s, zs_e;
    int pml_xm, pml_xp, pml_ym, pml_yp, pml_zm, pml_zp;
    double Dx, Dy, Dz, Dt, dtm, dtdex, dtdey, dtdez, dtdmx, dtdmy, dtdmz;
    double pml_kappa[6] = {1, 1, 1, 1, 1, 1}, pml_sigma[6] = {0}, pml_alpha[6] = {0};
    double pml_m = 4, pml_ma = 2;
    Grid Ex, Ey, Ez, Hx, Hy, Hz;
    std::vector<unsigned> mg;
    unsigned Nmat = 1;
    std::vector<Mat> mats;
    Grid PsiExy, PsiExz, PsiEyx, PsiEyz, PsiEzx, PsiEzy;
    Grid PsiHxy, PsiHxz, PsiHyx, PsiHyz, PsiHzx, PsiHzy;
    std::vector<double> kxE, kyE, kzE, kxH, kyH, kzH, bxE, byE, bzE, bxH, byH, bzH, cxE, cyE, czE, cxH, cyH, czH;

    unsigned &M(int i, int j, int k) { return mg[i + size_t(j) * Nx + size_t(k) * Nx * Ny]; }

    // FDTD::FDTD, 18-argument form (fdtd_core.cpp:158-285) for modes NORM and CUSTOM.
    void construct(const aefdtd_grid_desc *g, int pads[6]) {
        Nx = g->nx; Ny = g->ny; Nz = g->nz;
        Nx_s = Nx; Ny_s = Ny; Nz_s = Nz;
        pml_xm = g->pml[0]; pml_xp = g->pml[1]; pml_ym = g->pml[2];
        pml_yp = g->pml[3]; pml_zm = g->pml[4]; pml_zp = g->pml[5];
        int pad_xm = pads[0], pad_xp = pads[1], pad_ym = pads[2], pad_yp = pads[3], pad_zm = pads[4], pad_zp = pads[5];
        if (pml_xm || pml_xp) { pad_xm = std::max(5, pad_xm); pad_xp = std::max(5, pad_xp); }
        if (pml_ym || pml_yp) { pad_ym = std::max(5, pad_ym); pad_yp = std::max(5, pad_yp); }
        if (pml_zm || pml_zp) { pad_zm = std::max(5, pad_zm); pad_zp = std::max(5, pad_zp); }
        Nx += pml_xm + pad_xm + pad_xp + pml_xp;
        Ny += pml_ym + pad_ym + pad_yp + pml_yp;
        Nz += pml_zm + pad_zm + pad_zp + pml_zp;
        xs_s = pml_xm + pad_xm; xs_e = xs_s + Nx_s;
        ys_s = pml_ym + pad_ym; ys_e = ys_s + Ny_s;
        zs_s = pml_zm + pad_zm; zs_e = zs_s + Nz_s;
        for (Grid *f : {&Ex, &Ey, &Ez, &Hx, &Hy, &Hz}) f->init(Nx, Ny, Nz);
        mg.assign(size_t(Nx) * Ny * Nz, 0);
        // basic_differentials_compute (fdtd_core.cpp:1137-1148)
        dtm = Dt / mu0;
        dtdex = Dt / (Dx * e0); dtdey = Dt / (Dy * e0); dtdez = Dt / (Dz * e0);
        dtdmx = Dt / (Dx * mu0); dtdmy = Dt / (Dy * mu0); dtdmz = Dt / (Dz * mu0);
        // allocate_pml (fdtd_pml.cpp:26-86)
        if (pml_xm || pml_xp) for (Grid *p : {&PsiEyx, &PsiEzx, &PsiHyx, &PsiHzx}) p->init(pml_xm + pml_xp, Ny, Nz);
        if (pml_ym || pml_yp) for (Grid *p : {&PsiExy, &PsiEzy, &PsiHxy, &PsiHzy}) p->init(Nx, pml_ym + pml_yp, Nz);
        if (pml_zm || pml_zp) for (Grid *p : {&PsiExz, &PsiEyz, &PsiHxz, &PsiHyz}) p->init(Nx, Ny, pml_zm + pml_zp);
    }

    // set_pml_* (fdtd_pml.cpp:445-497): sigma is a scale on 0.8(m+1)/(eta0 D).
    void set_pml(int face, double kap, double sig, double alp) {
        double D = face < 2 ? Dx : (face < 4 ? Dy : Dz);
        pml_kappa[face] = kap;
        pml_sigma[face] = 0.8 * (pml_m + 1.0) / (std::sqrt(mu0 / e0) * D) * sig;
        pml_alpha[face] = alp;
    }

    // pml_{x,y,z}_coeffs (fdtd_pml.cpp:345-433)
    void pml_coeffs(double ind, int N, int pm, int pp, double km, double kp, double sm, double sp,
                    double am, double ap, double &kappa, double &b, double &c) {
        kappa = 1.0;
        if (ind < pm) {
            double x = (pm - ind) / static_cast<double>(pm);
            kappa = 1.0 + (km - 1.0) * std::pow(x, pml_m);
            double sig = sm * std::pow(x, pml_m);
            double alp = am * std::pow(1.0 - x, pml_ma);
            b = std::exp(-(sig / kappa + alp) * Dt / e0);
            c = sig / (sig * kappa + kappa * kappa * alp) * (b - 1.0);
        }
        if (ind > N - pp) {
            double x = (ind - (N - pp)) / static_cast<double>(pp);
            kappa = 1.0 + (kp - 1.0) * std::pow(x, pml_m);
            double sig = sp * std::pow(x, pml_m);
            double alp = ap * std::pow(1.0 - x, pml_ma);
            b = std::exp(-(sig / kappa + alp) * Dt / e0);
            c = sig / (sig * kappa + kappa * kappa * alp) * (b - 1.0);
        }
    }

    // pml_coeff_calc (fdtd_pml.cpp:305-343), re-run at tstep 0 (fdtd_core.cpp:1165).
    void pml_coeff_calc() {
        auto axis = [&](int N, int pm, int pp, int f, std::vector<double> &kE, std::vector<double> &bE,
                        std::vector<double> &cE, std::vector<double> &kH, std::vector<double> &bH,
                        std::vector<double> &cH) {
            kE.assign(N, 1.0); kH.assign(N, 1.0);
            bE.assign(N, 0.0); bH.assign(N, 0.0); cE.assign(N, 0.0); cH.assign(N, 0.0);
            if (pm || pp)
                for (int i = 0; i < N; i++) {
                    pml_coeffs(i, N, pm, pp, pml_kappa[f], pml_kappa[f + 1], pml_sigma[f], pml_sigma[f + 1],
                               pml_alpha[f], pml_alpha[f + 1], kE[i], bE[i], cE[i]);
                    pml_coeffs(i + 0.5, N, pm, pp, pml_kappa[f], pml_kappa[f + 1], pml_sigma[f], pml_sigma[f + 1],
                               pml_alpha[f], pml_alpha[f + 1], kH[i], bH[i], cH[i]);
                }
        };
        axis(Nx, pml_xm, pml_xp, 0, kxE, bxE, cxE, kxH, bxH, cxH);
        axis(Ny, pml_ym, pml_yp, 2, kyE, byE, cyE, kyH, byH, cyH);
        axis(Nz, pml_zm, pml_zp, 4, kzE, bzE, czE, kzH, bzH, czH);
    }

    // FDTD::set_matsgrid (fdtd_utils.cpp:572-766), modes NORM/CUSTOM.
    void set_matsgrid(const uint32_t *map) {
        for (int i = xs_s; i < xs_e; i++) for (int j = ys_s; j < ys_e; j++) for (int k = zs_s; k < zs_e; k++)
            M(i, j, k) = map[(i - xs_s) + size_t(j - ys_s) * Nx_s + size_t(k - zs_s) * Nx_s * Ny_s];
        for (int i = 0; i < xs_s; i++) for (int j = ys_s; j < ys_e; j++) for (int k = zs_s; k < zs_e; k++)
            M(i, j, k) = M(xs_s, j, k);
        for (int i = xs_e; i < Nx; i++) for (int j = ys_s; j < ys_e; j++) for (int k = zs_s; k < zs_e; k++)
            M(i, j, k) = M(xs_e - 1, j, k);
        for (int i = 0; i < Nx; i++) for (int j = 0; j < ys_s; j++) for (int k = zs_s; k < zs_e; k++)
            M(i, j, k) = M(i, ys_s, k);
        for (int i = 0; i < Nx; i++) for (int j = ys_e; j < Ny; j++) for (int k = zs_s; k < zs_e; k++)
            M(i, j, k) = M(i, ys_e - 1, k);
        for (int i = 0; i < Nx; i++) for (int j = 0; j < Ny; j++) for (int k = 0; k < zs_s; k++)
            M(i, j, k) = M(i, j, zs_s);
        for (int i = 0; i < Nx; i++) for (int j = 0; j < Ny; j++) for (int k = zs_e; k < Nz; k++)
            M(i, j, k) = M(i, j, zs_e - 1);
        Nmat = 1;
        for (unsigned m : mg) Nmat = std::max(Nmat, m + 1);
        mats.assign(Nmat, Mat());
    }

    // FDTD::set_material (fdtd_utils.cpp:810-820) -> link_grid (mats.cpp:394-443),
    // set_base_mat (mats.cpp:445-464), set_const/const_recalc (mats_const.cpp:18-36,71-80),
    // RC_dielec_treat/RC_recalc (mats_RC.cpp:126-184), Dielec_model::get_time_exp and
    // per-model pole pairs (dielec_models.cpp:71-107,143-153,222-226,281-290,350-358,419-423).
    void set_material(unsigned ind, const aefdtd_material_desc &d) {
        if (ind >= Nmat) return;
        bool present = false;
        for (unsigned m : mg) if (m == ind) { present = true; break; }
        if (!present) return;
        Mat &mt = mats[ind];
        // link_grid: bounding box of the material's cells
        std::vector<char> xc(Nx, 0), yc(Ny, 0), zc(Nz, 0);
        for (int i = 0; i < Nx; i++) for (int j = 0; j < Ny; j++) for (int k = 0; k < Nz; k++)
            if (M(i, j, k) == ind) xc[i] = yc[j] = zc[k] = 1;
        int i = 0; while (!xc[i]) i++; mt.x1 = i;
        i = Nx - 1; while (!xc[i]) i--; int x2 = i;
        int j = 0; while (!yc[j]) j++; mt.y1 = j;
        j = Ny - 1; while (!yc[j]) j--; int y2 = j;
        int k = 0; while (!zc[k]) k++; mt.z1 = k;
        k = Nz - 1; while (!zc[k]) k--; int z2 = k;
        mt.xs = x2 + 1 - mt.x1; mt.ys = y2 + 1 - mt.y1; mt.zs = z2 + 1 - mt.z1;

        int Nmod = d.n_debye + d.n_drude + d.n_lorentz + d.n_critpoint;
        if (Nmod == 0) {
            mt.rc = false; mt.Np = 0;
            mt.ei = d.eps_inf; mt.sig = 0;
            mt.C1 = 1;
            mt.C2x = Dt / (Dx * e0 * mt.ei);
            mt.C2y = Dt / (Dy * e0 * mt.ei);
            mt.C2z = Dt / (Dz * e0 * mt.ei);
            mt.C3 = 0;
            mt.C4 = Dt / (e0 * mt.ei);
            return;
        }
        std::vector<cplx> va, vb;
        double sig = 0;
        for (int n = 0; n < d.n_debye; n++) {
            double ds = d.debye[n][0], t0 = d.debye[n][1];
            va.push_back(ds / t0); vb.push_back(-1.0 / t0);
        }
        for (int n = 0; n < d.n_drude; n++) {
            double wd = d.drude[n][0], g = d.drude[n][1], wd2 = wd * wd;
            va.push_back(-wd2 / g); vb.push_back(-g);
        }
        for (int n = 0; n < d.n_lorentz; n++) {
            double A = d.lorentz[n][0], O = d.lorentz[n][1], G = d.lorentz[n][2];
            double alp = G / 2.0;
            cplx bet = std::sqrt(O * O - alp * alp);
            cplx eta = A * O * O / bet;
            va.push_back(-eta * Im); vb.push_back(-alp + bet * Im);
        }
        for (int n = 0; n < d.n_critpoint; n++) {
            double A = d.critpoint[n][0], O = d.critpoint[n][1], P = d.critpoint[n][2], G = d.critpoint[n][3];
            va.push_back(-2.0 * A * O * std::exp(-P * Im) * Im); vb.push_back(-G + O * Im);
        }
        for (int n = 0; n < d.n_drude; n++) {
            double wd = d.drude[n][0], g = d.drude[n][1], wd2 = wd * wd;
            sig += e0 * wd2 / g;
        }
        mt.rc = true; mt.Np = Nmod;
        mt.ei = d.eps_inf; mt.sig = sig;
        mt.Crec.resize(Nmod); mt.chi.resize(Nmod); mt.Dchi.resize(Nmod);
        for (int n = 0; n < Nmod; n++) {
            cplx &pa = va[n], &pb = vb[n];
            mt.Crec[n] = std::exp(pb * Dt);
            mt.chi[n] = pa / pb * (std::exp(pb * Dt) - 1.0);
            mt.Dchi[n] = -pa / pb * std::pow(1.0 - std::exp(pb * Dt), 2.0);
        }
        double chitmp = 0;
        for (int n = 0; n < Nmod; n++) chitmp += std::real(mt.chi[n]);
        double e_eff = mt.ei + chitmp + mt.sig * Dt / e0;
        mt.C1 = mt.ei / e_eff;
        mt.C2x = Dt / (Dx * e0 * e_eff);
        mt.C2y = Dt / (Dy * e0 * e_eff);
        mt.C2z = Dt / (Dz * e0 * e_eff);
        mt.C3 = 1.0 / e_eff;
        mt.C4 = Dt / (e0 * e_eff);
        mt.psi.assign(size_t(mt.xs) * mt.ys * mt.zs * 3 * Nmod, cplx(0, 0));
    }

    // FDTD::update_E (fdtd_core.cpp:1163-1218) with the six phases of
    // threaded_process_E (fdtd_threads.cpp:32-150), each over the whole grid.
    void update_E() {
        if (tstep == 0) pml_coeff_calc();
        // phase 1: advMats_ante -> RC_ante (fdtd_core.cpp:971-1012, mats_RC.cpp:21-36)
        for (int k = 0; k < Nz; k++) for (int j = 0; j < Ny; j++) for (int i = 0; i < Nx; i++) {
            Mat &mt = mats[M(i, j, k)];
            if (!mt.rc) continue;
            for (int p = 0; p < mt.Np; p++) {
                cplx &px = mt.P(i, j, k, 3 * p + 0), &py = mt.P(i, j, k, 3 * p + 1), &pz = mt.P(i, j, k, 3 * p + 2);
                px = mt.Crec[p] * px + mt.Dchi[p] * Ex(i, j, k);
                py = mt.Crec[p] * py + mt.Dchi[p] * Ey(i, j, k);
                pz = mt.Crec[p] * pz + mt.Dchi[p] * Ez(i, j, k);
            }
        }
        // phase 2: advEx/advEy/advEz (fdtd_core.cpp:363-541). The kappa lookup
        // condition `pml_ym || pml_xp` for y is the reference's (fdtd_core.cpp:397,504).
        bool zk = pml_zm || pml_zp, xk = pml_xm || pml_xp, yk = pml_ym || pml_xp;
        for (int k = 0; k < Nz; k++) {
            int k1 = k == 0 ? Nz - 1 : k - 1;
            double ikz = 1.0 / (zk ? kzE[k] : 1.0);
            for (int j = 0; j < Ny; j++) {
                int j1 = j == 0 ? Ny - 1 : j - 1;
                double iky = 1.0 / (yk ? kyE[j] : 1.0);
                for (int i = 0; i < Nx; i++) {
                    Mat &mt = mats[M(i, j, k)];
                    Ex(i, j, k) = mt.C1 * Ex(i, j, k) + mt.C2y * iky * (Hz(i, j, k) - Hz(i, j1, k))
                                - mt.C2z * ikz * (Hy(i, j, k) - Hy(i, j, k1));
                }
            }
        }
        for (int k = 0; k < Nz; k++) {
            int k1 = k == 0 ? Nz - 1 : k - 1;
            double ikz = 1.0 / (zk ? kzE[k] : 1.0);
            for (int j = 0; j < Ny; j++)
                for (int i = 0; i < Nx; i++) {
                    int i1 = i == 0 ? Nx - 1 : i - 1;
                    double ikx = 1.0 / (xk ? kxE[i] : 1.0);
                    Mat &mt = mats[M(i, j, k)];
                    Ey(i, j, k) = mt.C1 * Ey(i, j, k) + mt.C2z * ikz * (Hx(i, j, k) - Hx(i, j, k1))
                                - mt.C2x * ikx * (Hz(i, j, k) - Hz(i1, j, k));
                }
        }
        for (int k = 0; k < Nz; k++)
            for (int j = 0; j < Ny; j++) {
                int j1 = j == 0 ? Ny - 1 : j - 1;
                double iky = 1.0 / (yk ? kyE[j] : 1.0);
                for (int i = 0; i < Nx; i++) {
                    int i1 = i == 0 ? Nx - 1 : i - 1;
                    double ikx = 1.0 / (xk ? kxE[i] : 1.0);
                    Mat &mt = mats[M(i, j, k)];
                    Ez(i, j, k) = mt.C1 * Ez(i, j, k) + mt.C2x * ikx * (Hy(i, j, k) - Hy(i1, j, k))
                                - mt.C2y * iky * (Hx(i, j, k) - Hx(i, j1, k));
                }
            }
        // phase 3: advMats_simp -> RC_apply_E (fdtd_core.cpp:1014-1033, mats_RC.cpp:38-50)
        for (int k = 0; k < Nz; k++) for (int j = 0; j < Ny; j++) for (int i = 0; i < Nx; i++) {
            Mat &mt = mats[M(i, j, k)];
            if (!mt.rc) continue;
            Grid *E[3] = {&Ex, &Ey, &Ez};
            for (int d = 0; d < 3; d++) {
                double s = 0;
                for (int p = 0; p < mt.Np; p++) s += std::real(mt.P(i, j, k, 3 * p + d));
                (*E[d])(i, j, k) += mt.C3 * s;
            }
        }
        // phases 4-5 (advMats_post/self) are no-ops for constant and RC materials.
        // phase 6: app_pml_Ex/Ey/Ez (fdtd_pml.cpp:504-735)
        pml_E();
    }

    void pml_E() {
        double inv_Dx = 1.0 / Dx, inv_Dy = 1.0 / Dy, inv_Dz = 1.0 / Dz;
        // app_pml_Ex (fdtd_pml.cpp:504-580)
        if (pml_ym || pml_yp) {
            for (int i = 0; i < Nx; i++) for (int k = 0; k < Nz; k++) {
                for (int j = 1; j < pml_ym; j++) {
                    double C4 = mats[M(i, j, k)].C4;
                    PsiExy(i, j, k) = byE[j] * PsiExy(i, j, k) + cyE[j] * inv_Dy * (Hz(i, j, k) - Hz(i, j - 1, k));
                    Ex(i, j, k) += C4 * PsiExy(i, j, k);
                }
                for (int j = Ny - pml_yp + 1; j < Ny; j++) {
                    int n = j - (Ny - pml_yp) + pml_ym;
                    double C4 = mats[M(i, j, k)].C4;
                    PsiExy(i, n, k) = byE[j] * PsiExy(i, n, k) + cyE[j] * inv_Dy * (Hz(i, j, k) - Hz(i, j - 1, k));
                    Ex(i, j, k) += C4 * PsiExy(i, n, k);
                }
            }
            for (int i = 0; i < Nx; i++) for (int k = 0; k < Nz; k++) Ex(i, 0, k) = 0;
        }
        if (pml_zm || pml_zp) {
            for (int k = 1; k < pml_zm; k++) for (int j = 0; j < Ny; j++) for (int i = 0; i < Nx; i++) {
                double C4 = mats[M(i, j, k)].C4;
                PsiExz(i, j, k) = bzE[k] * PsiExz(i, j, k) + czE[k] * inv_Dz * (Hy(i, j, k) - Hy(i, j, k - 1));
                Ex(i, j, k) -= C4 * PsiExz(i, j, k);
            }
            for (int k = Nz - pml_zp + 1; k < Nz; k++) for (int j = 0; j < Ny; j++) for (int i = 0; i < Nx; i++) {
                int n = k - (Nz - pml_zp) + pml_zm;
                double C4 = mats[M(i, j, k)].C4;
                PsiExz(i, j, n) = bzE[k] * PsiExz(i, j, n) + czE[k] * inv_Dz * (Hy(i, j, k) - Hy(i, j, k - 1));
                Ex(i, j, k) -= C4 * PsiExz(i, j, n);
            }
            for (int i = 0; i < Nx; i++) for (int j = 0; j < Ny; j++) Ex(i, j, 0) = 0;
        }
        // app_pml_Ey (fdtd_pml.cpp:582-659)
        if (pml_xm || pml_xp) {
            for (int j = 0; j < Ny; j++) for (int k = 0; k < Nz; k++) {
                for (int i = 1; i < pml_xm; i++) {
                    double C4 = mats[M(i, j, k)].C4;
                    PsiEyx(i, j, k) = bxE[i] * PsiEyx(i, j, k) + cxE[i] * inv_Dx * (Hz(i, j, k) - Hz(i - 1, j, k));
                    Ey(i, j, k) -= C4 * PsiEyx(i, j, k);
                }
                for (int i = Nx - pml_xp + 1; i < Nx; i++) {
                    int n = i - (Nx - pml_xp) + pml_xm;
                    double C4 = mats[M(i, j, k)].C4;
                    PsiEyx(n, j, k) = bxE[i] * PsiEyx(n, j, k) + cxE[i] * inv_Dx * (Hz(i, j, k) - Hz(i - 1, j, k));
                    Ey(i, j, k) -= C4 * PsiEyx(n, j, k);
                }
            }
            for (int j = 0; j < Ny; j++) for (int k = 0; k < Nz; k++) Ey(0, j, k) = 0;
        }
        if (pml_zm || pml_zp) {
            for (int k = 1; k < pml_zm; k++) for (int j = 0; j < Ny; j++) for (int i = 0; i < Nx; i++) {
                double C4 = mats[M(i, j, k)].C4;
                PsiEyz(i, j, k) = bzE[k] * PsiEyz(i, j, k) + czE[k] * inv_Dz * (Hx(i, j, k) - Hx(i, j, k - 1));
                Ey(i, j, k) += C4 * PsiEyz(i, j, k);
            }
            for (int k = Nz - pml_zp + 1; k < Nz; k++) for (int j = 0; j < Ny; j++) for (int i = 0; i < Nx; i++) {
                int n = k - (Nz - pml_zp) + pml_zm;
                double C4 = mats[M(i, j, k)].C4;
                PsiEyz(i, j, n) = bzE[k] * PsiEyz(i, j, n) + czE[k] * inv_Dz * (Hx(i, j, k) - Hx(i, j, k - 1));
                Ey(i, j, k) += C4 * PsiEyz(i, j, n);
            }
            for (int i = 0; i < Nx; i++) for (int j = 0; j < Ny; j++) Ey(i, j, 0) = 0;
        }
        // app_pml_Ez (fdtd_pml.cpp:661-735)
        if (pml_xm || pml_xp) {
            for (int j = 0; j < Ny; j++) for (int k = 0; k < Nz; k++) {
                for (int i = 1; i < pml_xm; i++) {
                    double C4 = mats[M(i, j, k)].C4;
                    PsiEzx(i, j, k) = bxE[i] * PsiEzx(i, j, k) + cxE[i] * inv_Dx * (Hy(i, j, k) - Hy(i - 1, j, k));
                    Ez(i, j, k) += C4 * PsiEzx(i, j, k);
                }
                for (int i = Nx - pml_xp + 1; i < Nx; i++) {
                    int n = i - (Nx - pml_xp) + pml_xm;
                    double C4 = mats[M(i, j, k)].C4;
                    PsiEzx(n, j, k) = bxE[i] * PsiEzx(n, j, k) + cxE[i] * inv_Dx * (Hy(i, j, k) - Hy(i - 1, j, k));
                    Ez(i, j, k) += C4 * PsiEzx(n, j, k);
                }
            }
            for (int j = 0; j < Ny; j++) for (int k = 0; k < Nz; k++) Ez(0, j, k) = 0;
        }
        if (pml_ym || pml_yp) {
            for (int i = 0; i < Nx; i++) for (int k = 0; k < Nz; k++) {
                for (int j = 1; j < pml_ym; j++) {
                    double C4 = mats[M(i, j, k)].C4;
                    PsiEzy(i, j, k) = byE[j] * PsiEzy(i, j, k) + cyE[j] * inv_Dy * (Hx(i, j, k) - Hx(i, j - 1, k));
                    Ez(i, j, k) -= C4 * PsiEzy(i, j, k);
                }
                for (int j = Ny - pml_yp + 1; j < Ny; j++) {
                    int n = j - (Ny - pml_yp) + pml_ym;
                    double C4 = mats[M(i, j, k)].C4;
                    PsiEzy(i, n, k) = byE[j] * PsiEzy(i, n, k) + cyE[j] * inv_Dy * (Hx(i, j, k) - Hx(i, j - 1, k));
                    Ez(i, j, k) -= C4 * PsiEzy(i, n, k);
                }
            }
            for (int i = 0; i < Nx; i++) for (int k = 0; k < Nz; k++) Ez(i, 0, k) = 0;
        }
    }

    // FDTD::update_H (fdtd_core.cpp:1316-1335): advHx/Hy/Hz (fdtd_core.cpp:546-698)
    // then app_pml_Hx/Hy/Hz (fdtd_pml.cpp:737-929); tstep++.
    void update_H() {
        bool zk = pml_zm || pml_zp, xk = pml_xm || pml_xp, yk = pml_ym || pml_xp;
        for (int k = 0; k < Nz; k++) {
            int k2 = k == Nz - 1 ? 0 : k + 1;
            double ikz = 1.0 / (zk ? kzH[k] : 1.0);
            for (int j = 0; j < Ny; j++) {
                int j2 = j == Ny - 1 ? 0 : j + 1;
                double iky = 1.0 / (yk ? kyH[j] : 1.0);
                for (int i = 0; i < Nx; i++)
                    Hx(i, j, k) += dtdmz * ikz * (Ey(i, j, k2) - Ey(i, j, k)) - dtdmy * iky * (Ez(i, j2, k) - Ez(i, j, k));
            }
        }
        for (int k = 0; k < Nz; k++) {
            int k2 = k == Nz - 1 ? 0 : k + 1;
            double ikz = 1.0 / (zk ? kzH[k] : 1.0);
            for (int j = 0; j < Ny; j++)
                for (int i = 0; i < Nx; i++) {
                    int i2 = i == Nx - 1 ? 0 : i + 1;
                    double ikx = 1.0 / (xk ? kxH[i] : 1.0);
                    Hy(i, j, k) += dtdmx * ikx * (Ez(i2, j, k) - Ez(i, j, k)) - dtdmz * ikz * (Ex(i, j, k2) - Ex(i, j, k));
                }
        }
        for (int k = 0; k < Nz; k++)
            for (int j = 0; j < Ny; j++) {
                int j2 = j == Ny - 1 ? 0 : j + 1;
                double iky = 1.0 / (yk ? kyH[j] : 1.0);
                for (int i = 0; i < Nx; i++) {
                    int i2 = i == Nx - 1 ? 0 : i + 1;
                    double ikx = 1.0 / (xk ? kxH[i] : 1.0);
                    Hz(i, j, k) += dtdmy * iky * (Ex(i, j2, k) - Ex(i, j, k)) - dtdmx * ikx * (Ey(i2, j, k) - Ey(i, j, k));
                }
            }
        pml_H();
        tstep += 1;
    }

    void pml_H() {
        double inv_Dx = 1.0 / Dx, inv_Dy = 1.0 / Dy, inv_Dz = 1.0 / Dz;
        // app_pml_Hx (fdtd_pml.cpp:737-802)
        if (pml_ym || pml_yp) {
            for (int i = 0; i < Nx; i++) for (int k = 0; k < Nz; k++) {
                for (int j = 0; j < pml_ym; j++) {
                    PsiHxy(i, j, k) = byH[j] * PsiHxy(i, j, k) + cyH[j] * inv_Dy * (Ez(i, j + 1, k) - Ez(i, j, k));
                    Hx(i, j, k) -= dtm * PsiHxy(i, j, k);
                }
                for (int j = Ny - pml_yp; j < Ny - 1; j++) {
                    int n = j - (Ny - pml_yp) + pml_ym;
                    PsiHxy(i, n, k) = byH[j] * PsiHxy(i, n, k) + cyH[j] * inv_Dy * (Ez(i, j + 1, k) - Ez(i, j, k));
                    Hx(i, j, k) -= dtm * PsiHxy(i, n, k);
                }
            }
            for (int i = 0; i < Nx; i++) for (int k = 0; k < Nz; k++) Hx(i, Ny - 1, k) = 0;
        }
        if (pml_zm || pml_zp) {
            for (int k = 0; k < pml_zm; k++) for (int j = 0; j < Ny; j++) for (int i = 0; i < Nx; i++) {
                PsiHxz(i, j, k) = bzH[k] * PsiHxz(i, j, k) + czH[k] * inv_Dz * (Ey(i, j, k + 1) - Ey(i, j, k));
                Hx(i, j, k) += dtm * PsiHxz(i, j, k);
            }
            for (int k = Nz - pml_zp; k < Nz - 1; k++) for (int j = 0; j < Ny; j++) for (int i = 0; i < Nx; i++) {
                int n = k - (Nz - pml_zp) + pml_zm;
                PsiHxz(i, j, n) = bzH[k] * PsiHxz(i, j, n) + czH[k] * inv_Dz * (Ey(i, j, k + 1) - Ey(i, j, k));
                Hx(i, j, k) += dtm * PsiHxz(i, j, n);
            }
            for (int i = 0; i < Nx; i++) for (int j = 0; j < Ny; j++) Hx(i, j, Nz - 1) = Hy(i, j, Nz - 1) = 0;
        }
        // app_pml_Hy (fdtd_pml.cpp:804-867)
        if (pml_xm || pml_xp) {
            for (int j = 0; j < Ny; j++) for (int k = 0; k < Nz; k++) {
                for (int i = 0; i < pml_xm; i++) {
                    PsiHyx(i, j, k) = bxH[i] * PsiHyx(i, j, k) + cxH[i] * inv_Dx * (Ez(i + 1, j, k) - Ez(i, j, k));
                    Hy(i, j, k) += dtm * PsiHyx(i, j, k);
                }
                for (int i = Nx - pml_xp; i < Nx - 1; i++) {
                    int n = i - (Nx - pml_xp) + pml_xm;
                    PsiHyx(n, j, k) = bxH[i] * PsiHyx(n, j, k) + cxH[i] * inv_Dx * (Ez(i + 1, j, k) - Ez(i, j, k));
                    Hy(i, j, k) += dtm * PsiHyx(n, j, k);
                }
            }
            for (int j = 0; j < Ny; j++) for (int k = 0; k < Nz; k++) Hy(Nx - 1, j, k) = 0;
        }
        if (pml_zm || pml_zp) {
            for (int k = 0; k < pml_zm; k++) for (int j = 0; j < Ny; j++) for (int i = 0; i < Nx; i++) {
                PsiHyz(i, j, k) = bzH[k] * PsiHyz(i, j, k) + czH[k] * inv_Dz * (Ex(i, j, k + 1) - Ex(i, j, k));
                Hy(i, j, k) -= dtm * PsiHyz(i, j, k);
            }
            for (int k = Nz - pml_zp; k < Nz - 1; k++) for (int j = 0; j < Ny; j++) for (int i = 0; i < Nx; i++) {
                int n = k - (Nz - pml_zp) + pml_zm;
                PsiHyz(i, j, n) = bzH[k] * PsiHyz(i, j, n) + czH[k] * inv_Dz * (Ex(i, j, k + 1) - Ex(i, j, k));
                Hy(i, j, k) -= dtm * PsiHyz(i, j, n);
            }
            for (int i = 0; i < Nx; i++) for (int j = 0; j < Ny; j++) Hy(i, j, Nz - 1) = 0;
        }
        // app_pml_Hz (fdtd_pml.cpp:869-929)
        if (pml_xm || pml_xp) {
            for (int j = 0; j < Ny; j++) for (int k = 0; k < Nz; k++) {
                for (int i = 0; i < pml_xm; i++) {
                    PsiHzx(i, j, k) = bxH[i] * PsiHzx(i, j, k) + cxH[i] * inv_Dx * (Ey(i + 1, j, k) - Ey(i, j, k));
                    Hz(i, j, k) -= dtm * PsiHzx(i, j, k);
                }
                for (int i = Nx - pml_xp; i < Nx - 1; i++) {
                    int n = i - (Nx - pml_xp) + pml_xm;
                    PsiHzx(n, j, k) = bxH[i] * PsiHzx(n, j, k) + cxH[i] * inv_Dx * (Ey(i + 1, j, k) - Ey(i, j, k));
                    Hz(i, j, k) -= dtm * PsiHzx(n, j, k);
                }
            }
            for (int j = 0; j < Ny; j++) for (int k = 0; k < Nz; k++) Hz(Nx - 1, j, k) = 0;
        }
        if (pml_ym || pml_yp) {
            for (int i = 0; i < Nx; i++) for (int k = 0; k < Nz; k++) {
                for (int j = 0; j < pml_ym; j++) {
                    PsiHzy(i, j, k) = byH[j] * PsiHzy(i, j, k) + cyH[j] * inv_Dy * (Ex(i, j + 1, k) - Ex(i, j, k));
                    Hz(i, j, k) += dtm * PsiHzy(i, j, k);
                }
                for (int j = Ny - pml_yp; j < Ny - 1; j++) {
                    int n = j - (Ny - pml_yp) + pml_ym;
                    PsiHzy(i, n, k) = byH[j] * PsiHzy(i, n, k) + cyH[j] * inv_Dy * (Ex(i, j + 1, k) - Ex(i, j, k));
                    Hz(i, j, k) += dtm * PsiHzy(i, n, k);
                }
            }
            for (int i = 0; i < Nx; i++) for (int k = 0; k < Nz; k++) Hz(i, Ny - 1, k) = 0;
        }
    }

    // FDTD::local_E*/local_H* (fdtd_utils.cpp:457-507)
    double lEx(int i, int j, int k) const { int jp = j + 1; if (jp == Ny) jp = 0; int kp = k + 1; if (kp == Nz) kp = 0;
        return (Ex(i, j, k) + Ex(i, jp, k) + Ex(i, j, kp) + Ex(i, jp, kp)) / 4.0; }
    double lEy(int i, int j, int k) const { int ip = i + 1; if (ip == Nx) ip = 0; int kp = k + 1; if (kp == Nz) kp = 0;
        return (Ey(i, j, k) + Ey(ip, j, k) + Ey(i, j, kp) + Ey(ip, j, kp)) / 4.0; }
    double lEz(int i, int j, int k) const { int ip = i + 1; if (ip == Nx) ip = 0; int jp = j + 1; if (jp == Ny) jp = 0;
        return (Ez(i, j, k) + Ez(ip, j, k) + Ez(i, jp, k) + Ez(ip, jp, k)) / 4.0; }
    double lHx(int i, int j, int k) const { int ip = i + 1; if (ip == Nx) ip = 0; return (Hx(i, j, k) + Hx(ip, j, k)) / 2.0; }
    double lHy(int i, int j, int k) const { int jp = j + 1; if (jp == Ny) jp = 0; return (Hy(i, j, k) + Hy(i, jp, k)) / 2.0; }
    double lHz(int i, int j, int k) const { int kp = k + 1; if (kp == Nz) kp = 0; return (Hz(i, j, k) + Hz(i, j, kp)) / 2.0; }

    // Sensor::link (sensors.cpp:196-230) + SensorFieldHolder::initialize (sensors.cpp:496-527)
    void add_sensor(PlaneSensor &s, const aefdtd_sensor_desc &d) {
        s.type = d.orientation;
        s.x1 = std::clamp(d.box[0] + xs_s, 0, Nx); s.x2 = std::clamp(d.box[1] + xs_s, 0, Nx);
        s.y1 = std::clamp(d.box[2] + ys_s, 0, Ny); s.y2 = std::clamp(d.box[3] + ys_s, 0, Ny);
        s.z1 = std::clamp(d.box[4] + zs_s, 0, Nz); s.z2 = std::clamp(d.box[5] + zs_s, 0, Nz);
        if (s.type <= AEFDTD_NORMAL_XM) { s.span1 = s.y2 - s.y1; s.span2 = s.z2 - s.z1; }
        else if (s.type <= AEFDTD_NORMAL_YM) { s.span1 = s.x2 - s.x1; s.span2 = s.z2 - s.z1; }
        else { s.span1 = s.x2 - s.x1; s.span2 = s.y2 - s.y1; }
        s.Nl = d.nl;
        s.lambda.resize(s.Nl);
        for (int i = 0; i < s.Nl; i++) s.lambda[i] = d.lambda_min + (d.lambda_max - d.lambda_min) * i / (s.Nl - 1.0);
        for (int c = 0; c < 6; c++) {
            s.t[c].assign(size_t(s.span1) * s.span2, 0.0);
            s.sp[c].assign(size_t(s.span1) * s.span2 * s.Nl, cplx(0, 0));
        }
        s.rsp.assign(s.Nl, 0.0);
    }

    // Sensor::feed (sensors.cpp:232-243) -> update_t_interp (sensors.cpp:601-644)
    // -> FT_comp (sensors.cpp:456-479)
    void feed(PlaneSensor &s) {
        auto put = [&](int a, int b, int i, int j, int k) {
            size_t o = a + size_t(b) * s.span1;
            s.t[0][o] = lEx(i, j, k); s.t[1][o] = lEy(i, j, k); s.t[2][o] = lEz(i, j, k);
            s.t[3][o] = lHx(i, j, k); s.t[4][o] = lHy(i, j, k); s.t[5][o] = lHz(i, j, k);
        };
        if (s.type <= AEFDTD_NORMAL_XM) {
            for (int j = s.y1; j < s.y2; j++) for (int k = s.z1; k < s.z2; k++) put(j - s.y1, k - s.z1, s.x1, j, k);
        } else if (s.type <= AEFDTD_NORMAL_YM) {
            for (int i = s.x1; i < s.x2; i++) for (int k = s.z1; k < s.z2; k++) put(i - s.x1, k - s.z1, i, s.y1, k);
        } else {
            for (int i = s.x1; i < s.x2; i++) for (int j = s.y1; j < s.y2; j++) put(i - s.x1, j - s.y1, i, j, s.z1);
        }
        for (int l = 0; l < s.Nl; l++) {
            double w = 2.0 * Pi * c_light / s.lambda[l];
            cplx coeff_E = s.tapering_E * std::exp(w * s.step * Dt * Im);
            cplx coeff_H = s.tapering_H * std::exp(w * (s.step + 0.5) * Dt * Im);
            for (int j = 0; j < s.span2; j++) for (int i = 0; i < s.span1; i++) {
                size_t o = i + size_t(j) * s.span1, q = o + size_t(l) * s.span1 * s.span2;
                for (int c = 0; c < 3; c++) s.sp[c][q] += coeff_E * s.t[c][o];
                for (int c = 3; c < 6; c++) s.sp[c][q] += coeff_H * s.t[c][o];
            }
        }
        if (s.step >= Nt - Ntap) {
            s.tapering_E = s_curve(s.step, Nt - 1.0, Nt - Ntap);
            s.tapering_H = s_curve(s.step + 0.5, Nt - 1.0, Nt - Ntap);
        }
        s.step += 1;
    }

    // Spect_Poynting::treat (s_spec_power.cpp:44-119)
    void treat(PlaneSensor &s) {
        for (int l = 0; l < s.Nl; l++) {
            double Sx = 0, Sy = 0, Sz = 0;
            for (int i = 0; i < s.span1; i++) for (int j = 0; j < s.span2; j++) {
                size_t q = i + size_t(j) * s.span1 + size_t(l) * s.span1 * s.span2;
                cplx ex = s.sp[0][q], ey = s.sp[1][q], ez = s.sp[2][q], hx = s.sp[3][q], hy = s.sp[4][q], hz = s.sp[5][q];
                Sx += std::real(ey * std::conj(hz) - ez * std::conj(hy));
                Sy += std::real(ez * std::conj(hx) - ex * std::conj(hz));
                Sz += std::real(ex * std::conj(hy) - ey * std::conj(hx));
            }
            double f;
            if (s.type <= AEFDTD_NORMAL_XM) f = Dy * Dz;
            else if (s.type <= AEFDTD_NORMAL_YM) f = Dx * Dz;
            else f = Dx * Dy;
            Sx *= f; Sy *= f; Sz *= f;
            double r = 0;
            switch (s.type) {
                case AEFDTD_NORMAL_X: r = Sx; break;
                case AEFDTD_NORMAL_Y: r = Sy; break;
                case AEFDTD_NORMAL_Z: r = Sz; break;
                case AEFDTD_NORMAL_XM: r = -Sx; break;
                case AEFDTD_NORMAL_YM: r = -Sy; break;
                case AEFDTD_NORMAL_ZM: r = -Sz; break;
            }
            s.rsp[l] = r;
        }
    }

    // Oscillator::initialize/deep_inject_E (sc_oscillator.cpp:34-84), Source::link (sources.cpp:252-283)
    void add_osc(Osc &o, const aefdtd_source_desc &d) {
        int t = d.orientation;
        o.comp = (t <= AEFDTD_NORMAL_XM) ? 0 : (t <= AEFDTD_NORMAL_YM ? 1 : 2);
        o.x1 = std::clamp(d.box[0] + xs_s, 0, Nx); o.x2 = std::clamp(d.box[1] + xs_s, 0, Nx);
        o.y1 = std::clamp(d.box[2] + ys_s, 0, Ny); o.y2 = std::clamp(d.box[3] + ys_s, 0, Ny);
        o.z1 = std::clamp(d.box[4] + zs_s, 0, Nz); o.z2 = std::clamp(d.box[5] + zs_s, 0, Nz);
        double alp = std::sqrt(0.1), bet = 1e-7;
        double w1 = 2.0 * Pi * c_light / d.lambda_max;   // m_to_rad_Hz (phys_tools.cpp:159)
        double w2 = 2.0 * Pi * c_light / d.lambda_min;
        o.w0 = (w1 + w2) / 2.0;
        o.dw = std::abs(w2 - w1) / (2.0 * std::sqrt(-std::log(alp)));
        o.tshift = int(std::sqrt(-4.0 / (o.dw * o.dw) * std::log(bet)) / Dt);
    }
    void inject_E(Osc &o) {
        cplx im_val = std::exp(-o.w0 * o.step * Dt * Im) * std::exp(-std::pow(o.dw / 2.0 * ((o.step - o.tshift) * Dt), 2.0));
        double val = std::real(im_val) * 50;
        Grid *E[3] = {&Ex, &Ey, &Ez};
        for (int i = o.x1; i < o.x2; i++) for (int j = o.y1; j < o.y2; j++) for (int k = o.z1; k < o.z2; k++)
            (*E[o.comp])(i, j, k) += val;
    }

    // FDTD::find_slab (fdtd_utils.cpp:347-392)
    void find_slab(int sub_ref, int sup_ref, double &hsub, double &hstruc, double &hsup) {
        int Nsub = 0, Nsup = 0, IDmoy = 0, IDsup = 0, IDsub = 0, k;
        for (int i = xs_s; i < xs_e; i++) for (int j = ys_s; j < ys_e; j++) { IDsup += M(i, j, zs_e); IDsub += M(i, j, zs_s); }
        IDmoy = IDsub; k = sub_ref;
        while (IDmoy == IDsub && k < sup_ref) {
            IDmoy = 0;
            for (int i = xs_s; i < xs_e; i++) for (int j = ys_s; j < ys_e; j++) IDmoy += M(i, j, k + 1);
            Nsub++; k++;
        }
        IDmoy = IDsup; k = sup_ref;
        while (IDmoy == IDsup && k >= sub_ref) {
            IDmoy = 0;
            for (int i = xs_s; i < xs_e; i++) for (int j = ys_s; j < ys_e; j++) IDmoy += M(i, j, k - 1);
            Nsup++; k--;
        }
        hsup = (Nsup - 1) * Dz; hsub = Nsub * Dz; hstruc = (Nz_s - Nsup - Nsub) * Dz;
    }
};

// ChpIn pulse (chpin.cpp:44-90,479-545) for theta=0, dir=0, start (0,0,startz).
struct Pulse {
    double k, omega, kx, ky, kz, n_ind, dz, C1, Ex0, Ey0, Ez0, Hx0, Hy0, Hz0;
    void init(double li, double lf, double poli, double startz, double n_ind_i) {
        double wi = 2.0 * Pi * c_light / li, wf = 2.0 * Pi * c_light / lf;
        double w0 = (wi + wf) / 2.0;
        double l0 = 2.0 * Pi * c_light / w0;
        double dw = std::abs(0.5 * (wi - w0));
        double lambda = l0;
        n_ind = n_ind_i;
        double inc = 0 * Pi / 180.0, pol = poli * Pi / 180.0, dir = 0 * Pi / 180.0;
        dz = 2.0 * c_light / dw / n_ind;
        // setfields (chpin.cpp:516-545)
        k = 2.0 * Pi / lambda * n_ind;
        omega = 2.0 * Pi * c_light / lambda;
        double incr = Pi / 2.0 - inc;
        double Ca = std::cos(incr), Sa = std::sin(incr), Cb = std::cos(dir), Sb = std::sin(dir);
        double Cc = std::cos(pol), Sc = std::sin(pol);
        kx = k * (Ca * Cb); ky = k * (Ca * Sb); kz = k * (-Sa);
        double amp = 1;
        Ex0 = (Sa * Cb * Sc - Sb * Cc) * amp; Ey0 = (Sa * Sb * Sc + Cb * Cc) * amp; Ez0 = Ca * Sc * amp;
        double tmp = 1.0 / (c_light * mu0) * amp * n_ind;
        Hx0 = tmp * (Sa * Cb * Cc + Sb * Sc); Hy0 = tmp * (Sa * Sb * Cc - Cb * Sc); Hz0 = tmp * (Ca * Cc);
        double bet = 1e-4;
        C1 = -1.0 / k * (kx * 0 + ky * 0 + kz * startz) + dz * std::sqrt(-std::log(bet));
    }
    double f(double A0, double x, double y, double z, double t) const {
        double p = kx * x + ky * y + kz * z;
        double a = p - omega * t;
        double b = (1.0 / k * p - c_light * t / n_ind + C1) / dz;
        return A0 * std::exp(-b * b) * std::cos(a);
    }
};

}  // namespace

extern "C" int aeoracle_run(const aefdtd_grid_desc *g, const uint32_t *map,
                            const aefdtd_material_desc *mats, int32_t nmat,
                            const aefdtd_normal_desc *nd,
                            const aefdtd_source_desc *srcs, int32_t nsrc,
                            const aefdtd_sensor_desc *sens, int32_t nsens,
                            int32_t nsteps, int32_t quiet,
                            double *fields_out, double *plane_sums_out, double *spectra_out,
                            double *flux_out, int32_t *dims_out, double *loop_seconds) {
    (void)quiet;
    if (!g || !map || !mats || nmat <= 0 || nsteps < 0) return 1;
    if (g->mode == AEFDTD_MODE_NORMAL && !nd) return 2;
    Sim S;
    S.mode = g->mode;
    S.Dx = g->dx; S.Dy = g->dy; S.Dz = g->dz;
    S.Nt = g->nt > 0 ? g->nt : nsteps;
    S.Ntap = g->tapering;
    if (g->pml_m > 0) S.pml_m = g->pml_m;
    if (g->pml_ma > 0) S.pml_ma = g->pml_ma;
    S.Dt = g->dt;
    if (S.Dt <= 0) S.Dt = std::min(std::min(S.Dx, S.Dy), S.Dz) / (std::sqrt(3.0) * c_light) * 0.99 * g->time_mod;
    aefdtd_grid_desc gg = *g;
    int pads[6];
    if (g->mode == AEFDTD_MODE_NORMAL) {
        // normal_incidence.cpp:188-195: only z PML, pads max(5, .)
        for (int f = 0; f < 4; f++) { gg.pml[f] = 0; pads[f] = 0; }
        pads[4] = std::max(5, g->pad[4]); pads[5] = std::max(5, g->pad[5]);
    } else {
        for (int f = 0; f < 6; f++) pads[f] = g->pad[f];
    }
    S.construct(&gg, pads);
    if (g->mode == AEFDTD_MODE_NORMAL) {
        S.set_pml(4, g->pml_kappa[4], g->pml_sigma[4], g->pml_alpha[4]);
        S.set_pml(5, g->pml_kappa[5], g->pml_sigma[5], g->pml_alpha[5]);
    } else {
        for (int f = 0; f < 6; f++) S.set_pml(f, g->pml_kappa[f], g->pml_sigma[f], g->pml_alpha[f]);
    }
    S.set_matsgrid(map);
    for (int m = 0; m < nmat; m++) S.set_material(m, mats[m]);
    S.pml_coeff_calc();
    if (dims_out) {
        int d[10] = {S.Nx, S.Ny, S.Nz, S.xs_s, S.xs_e, S.ys_s, S.ys_e, S.zs_s, S.zs_e, int(S.Nmat)};
        for (int i = 0; i < 10; i++) dims_out[i] = d[i];
    }
    std::vector<PlaneSensor> sensors(nsens);
    for (int s = 0; s < nsens; s++) S.add_sensor(sensors[s], sens[s]);
    std::vector<Osc> oscs;
    if (g->mode == AEFDTD_MODE_CUSTOM) {
        oscs.resize(nsrc);
        for (int s = 0; s < nsrc; s++) S.add_osc(oscs[s], srcs[s]);
    }
    double Dt = S.Dt, Dx = S.Dx, Dy = S.Dy, Dz = S.Dz;
    if (loop_seconds) loop_seconds[0] = 0;

    if (g->mode == AEFDTD_MODE_NORMAL) {
        // FDTD_normal_incidence (normal_incidence.cpp:228-436)
        int zs_s = S.zs_s, zs_e = S.zs_e, Nx = S.Nx, Ny = S.Ny;
        int Nl = nd->nl;
        std::vector<double> Lambda(Nl), w(Nl);
        for (int l = 0; l < Nl; l++) Lambda[l] = nd->lambda_min + (nd->lambda_max - nd->lambda_min) * l / (Nl - 1.0);
        for (int l = 0; l < Nl; l++) w[l] = 2.0 * Pi * c_light / Lambda[l];
        double pol = nd->polarization == 1 ? 90 : 0;
        double eps_sub = S.mats[S.M(0, 0, zs_s)].ei;
        double eps_sup = S.mats[S.M(0, 0, zs_e)].ei;
        double index_sub = std::sqrt(eps_sub), index_sup = std::sqrt(eps_sup);
        Pulse P;
        P.init(nd->lambda_min, nd->lambda_max, pol, (zs_e - 1) * Dz, index_sup);
        int Nt = S.Nt;
        std::vector<double> SS[12];
        for (auto &v : SS) v.assign(nsteps, 0.0);
        for (int t = 0; t < nsteps; t++) {
            S.update_E();
            double tb = t * Dt;
            double inj_Hx = P.f(P.Hx0, 0, 0, (zs_e - 1 + 0.5) * Dz, tb);
            double inj_Hy = P.f(P.Hy0, 0, 0, (zs_e - 1 + 0.5) * Dz, tb);
            for (int j = 0; j < Ny; j++) for (int i = 0; i < Nx; i++) {
                S.Ex(i, j, zs_e - 1) -= S.dtdez * inj_Hy / eps_sup;
                S.Ey(i, j, zs_e - 1) += S.dtdez * inj_Hx / eps_sup;
            }
            S.update_H();
            tb = (t + 0.5) * Dt;
            double inj_Ex = P.f(P.Ex0, 0, 0, (zs_e - 1) * Dz, tb);
            double inj_Ey = P.f(P.Ey0, 0, 0, (zs_e - 1) * Dz, tb);
            for (int j = 0; j < Ny; j++) for (int i = 0; i < Nx; i++) {
                S.Hx(i, j, zs_e - 1) += S.dtdmz * inj_Ey;
                S.Hy(i, j, zs_e - 1) -= S.dtdmz * inj_Ex;
            }
            for (auto &s : sensors) S.feed(s);
            tb = (t + 0.5) * Dt;
            double Dx2 = Dx / 2.0, Dy2 = Dy / 2.0, Dz2 = Dz / 2.0;
            double tapering = 1.0;
            if (t >= Nt - S.Ntap) tapering = s_curve(t, Nt - 1.0, Nt - S.Ntap);
            for (int j = 0; j < Ny; j++) {
                double y = j * Dy;
                for (int i = 0; i < Nx; i++) {
                    double x = i * Dx;
                    double z = (zs_e - 2) * Dz;
                    SS[0][t] += P.f(P.Ex0, x + Dx2, y, z, tb) * tapering;
                    SS[1][t] += P.f(P.Ey0, x, y + Dy2, z, tb) * tapering;
                    SS[2][t] += P.f(P.Ez0, x, y, z + Dz2, tb) * tapering;
                    SS[3][t] += (S.Ex(i, j, zs_e - 2) - P.f(P.Ex0, x + Dx2, y, z, tb)) * tapering;
                    SS[4][t] += (S.Ey(i, j, zs_e - 2) - P.f(P.Ey0, x, y + Dy2, z, tb)) * tapering;
                    SS[5][t] += (S.Ez(i, j, zs_e - 2) - P.f(P.Ez0, x, y, z + Dz2, tb)) * tapering;
                    z = (zs_s)*Dz;
                    SS[6][t] += P.f(P.Ex0, x + Dx2, y, z, tb) * tapering;
                    SS[7][t] += P.f(P.Ey0, x, y + Dy2, z, tb) * tapering;
                    SS[8][t] += P.f(P.Ez0, x, y, z + Dz2, tb) * tapering;
                    SS[9][t] += S.Ex(i, j, zs_s) * tapering;
                    SS[10][t] += S.Ey(i, j, zs_s) * tapering;
                    SS[11][t] += S.Ez(i, j, zs_s) * tapering;
                }
            }
        }
        if (plane_sums_out)
            for (int c = 0; c < 12; c++) for (int t = 0; t < nsteps; t++) plane_sums_out[size_t(c) * nsteps + t] = SS[c][t];
        if (spectra_out) {
            // normal_incidence.cpp:442-570
            int NtP = nsteps;
            double hsup, hsub, hstruc;
            S.find_slab(zs_s, zs_e - 1, hsub, hstruc, hsup);
            hsup -= Dz / 2.0; hsub -= Dz / 2.0;
            for (int l = 0; l < Nl; l++) {
                cplx r1x = 0, r1y = 0, r1z = 0, r2x = 0, r2y = 0, r2z = 0, t1x = 0, t1y = 0, t1z = 0, t2x = 0, t2y = 0, t2z = 0;
                double k0 = -w[l] / c_light, k1 = k0 * index_sup, k3 = k0 * index_sub;
                cplx tmp_sup = std::exp(2.0 * k1 * hsup * Im);
                cplx tmp_sub = std::exp((k3 * hsub - k0 * (hstruc + hsub)) * Im);
                for (int t = 0; t < NtP; t++) {
                    cplx tmp1 = std::exp(t * Dt * w[l] * Im) / (NtP - 1.0);
                    cplx tmp2 = tmp1 * tmp_sup, tmp3 = tmp1 * tmp_sub;
                    r1x += SS[0][t] * tmp1; r1y += SS[1][t] * tmp1; r1z += SS[2][t] * tmp1;
                    r2x += SS[3][t] * tmp2; r2y += SS[4][t] * tmp2; r2z += SS[5][t] * tmp2;
                    t1x += SS[6][t] * tmp1; t1y += SS[7][t] * tmp1; t1z += SS[8][t] * tmp1;
                    t2x += SS[9][t] * tmp3; t2y += SS[10][t] * tmp3; t2z += SS[11][t] * tmp3;
                }
                double *o = spectra_out + size_t(l) * 15;
                o[0] = Lambda[l];
                double a = std::sqrt(std::norm(r2x) + std::norm(r2y) + std::norm(r2z));
                double b = std::sqrt(std::norm(r1x) + std::norm(r1y) + std::norm(r1z));
                o[1] = a / b;
                a = std::sqrt(std::norm(t2x) + std::norm(t2y) + std::norm(t2z));
                b = std::sqrt(std::norm(t1x) + std::norm(t1y) + std::norm(t1z));
                o[2] = a / b;
                cplx ref0 = r1y, trans0 = t1y;
                if (nd->polarization == 1) { ref0 = r1x; trans0 = t1x; }
                cplx refx = r2x / ref0, refy = r2y / ref0, transx = t2x / trans0, transy = t2y / trans0;
                o[3] = std::abs(refx); o[4] = std::arg(refx); o[5] = std::norm(refx);
                o[6] = std::abs(refy); o[7] = std::arg(refy); o[8] = std::norm(refy);
                o[9] = std::abs(transx); o[10] = std::arg(transx); o[11] = std::norm(transx) * index_sub / index_sup;
                o[12] = std::abs(transy); o[13] = std::arg(transy); o[14] = std::norm(transy) * index_sub / index_sup;
            }
        }
    } else {
        // mode_default_fdtd loop (default_fdtd.cpp:156-204)
        for (int t = 0; t < nsteps; t++) {
            S.update_E();
            for (auto &o : oscs) S.inject_E(o);
            S.update_H();
            for (auto &s : sensors) S.feed(s);
            for (auto &o : oscs) o.step += 1;   // Source::inject_H (sources.cpp:245-250)
        }
    }
    if (fields_out) {
        size_t n = size_t(S.Nx) * S.Ny * S.Nz;
        Grid *F[6] = {&S.Ex, &S.Ey, &S.Ez, &S.Hx, &S.Hy, &S.Hz};
        for (int c = 0; c < 6; c++) std::memcpy(fields_out + c * n, F[c]->v.data(), n * sizeof(double));
    }
    size_t off = 0;
    for (auto &s : sensors) {
        S.treat(s);
        if (flux_out) for (int l = 0; l < s.Nl; l++) flux_out[off + l] = s.rsp[l];
        off += s.Nl;
    }
    return 0;
}

// ---------------------------------------------------------------------------
// Structure discretisation: Structure::discretize (src/structure/structure.cpp:94-113)
// with Structure::index (structure.cpp:228-258, no flips) and the primitive
// tests Add_Block::index (structure_primitives.cpp:24-39), Add_Layer::index
// (:317-339), Add_Sphere::index (:484-499), Add_Cylinder (:255-285, with
// Vector3::norm/normalize, src/common/vector23.cpp:266-282, and
// scalar_prod, vector23.cpp:702-705).
namespace {
struct OOp {
    int kind, mat;
    double p[8];
    double bx, by, bz, length;
};

int oop_index(const OOp &o, double x, double y, double z) {
    switch (o.kind) {
        case AEFDTD_OP_BLOCK:
            if (x < o.p[0] || x >= o.p[1] || y < o.p[2] || y >= o.p[3] || z < o.p[4] || z >= o.p[5]) return -1;
            return o.mat;
        case AEFDTD_OP_LAYER: {
            int t = (int)o.p[0];
            if (t == 0 && x >= o.p[1] && x < o.p[2]) return o.mat;
            if (t == 1 && y >= o.p[1] && y < o.p[2]) return o.mat;
            if (t == 2 && z >= o.p[1] && z < o.p[2]) return o.mat;
            return -1;
        }
        case AEFDTD_OP_SPHERE: {
            x = x - o.p[0]; y = y - o.p[1]; z = z - o.p[2];
            if (x * x + y * y + z * z <= o.p[3] * o.p[3]) return o.mat;
            return -1;
        }
        case AEFDTD_OP_CYLINDER: {
            double x1 = o.p[0], y1 = o.p[1], z1 = o.p[2], x2 = o.p[3], y2 = o.p[4], z2 = o.p[5], r = o.p[6];
            if (x < std::min(x1, x2) - r || x > std::max(x1, x2) + r || y < std::min(y1, y2) - r ||
                y > std::max(y1, y2) + r || z < std::min(z1, z2) - r || z > std::max(z1, z2) + r)
                return -1;
            double dx = x - x1, dy = y - y1, dz = z - z1;
            double proj = o.bx * dx + o.by * dy + o.bz * dz;
            if (proj >= 0 && proj <= o.length) {
                dx = dx - proj * o.bx; dy = dy - proj * o.by; dz = dz - proj * o.bz;
                double rt = dx * dx + dy * dy + dz * dz;
                if (rt <= r * r) return o.mat;
            }
            return -1;
        }
    }
    return -1;
}
}  // namespace

extern "C" int aeoracle_voxelize(int32_t nx, int32_t ny, int32_t nz, double dx, double dy, double dz,
                                 const aefdtd_structure_op *ops, int32_t n_ops, int32_t def,
                                 const int32_t periodic[3], const double lengths[3], uint32_t *out) {
    std::vector<OOp> v(n_ops);
    for (int q = 0; q < n_ops; q++) {
        OOp &o = v[q];
        o.kind = ops[q].kind; o.mat = ops[q].mat_index;
        for (int t = 0; t < 8; t++) o.p[t] = ops[q].p[t];
        o.bx = o.by = o.bz = o.length = 0;
        if (o.kind == AEFDTD_OP_BLOCK)
            for (int a = 0; a < 3; a++) if (o.p[2 * a] > o.p[2 * a + 1]) std::swap(o.p[2 * a], o.p[2 * a + 1]);
        if (o.kind == AEFDTD_OP_CYLINDER) {
            double vx = o.p[3] - o.p[0], vy = o.p[4] - o.p[1], vz = o.p[5] - o.p[2];
            double n = std::sqrt(vx * vx + vy * vy + vz * vz);
            o.length = n;
            o.bx = vx / n; o.by = vy / n; o.bz = vz / n;
        }
    }
    int per[3] = {periodic ? (periodic[0] ? 1 : 0) : 0, periodic ? (periodic[1] ? 1 : 0) : 0,
                  periodic ? (periodic[2] ? 1 : 0) : 0};
    double L[3] = {lengths ? lengths[0] : 0, lengths ? lengths[1] : 0, lengths ? lengths[2] : 0};
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++)
            for (int k = 0; k < nz; k++) {
                double x = i * dx, y = j * dy, z = k * dz;
                if (per[0]) { while (x < 0) x += L[0]; while (x >= L[0]) x -= L[0]; }
                if (per[1]) { while (y < 0) y += L[1]; while (y >= L[1]) y -= L[1]; }
                if (per[2]) { while (z < 0) z += L[2]; while (z >= L[2]) z -= L[2]; }
                int res = def;
                bool found = false;
                for (int l = n_ops - 1; l >= 0 && !found; l--)
                    for (int a = -per[0]; a <= per[0] && !found; a++)
                        for (int b = -per[1]; b <= per[1] && !found; b++)
                            for (int c = -per[2]; c <= per[2] && !found; c++) {
                                int h = oop_index(v[l], x + a * L[0], y + b * L[1], z + c * L[2]);
                                if (h != -1) { res = h; found = true; }
                            }
                out[i + size_t(j) * nx + size_t(k) * nx * ny] = (uint32_t)res;
            }
    return 0;
}
