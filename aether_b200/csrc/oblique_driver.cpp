// oblique_driver.cpp — the oblique driver "fdtd_oblique_ARS" at one in-plane
// wavevector (FDTD_oblique_biphase_comp, oblique_biphase.cpp:29-480): setup
// of the wideband Bloch source and the phases, the per-step R/T sums, and
// the spectra. The two grids (real and imaginary part) step on the shared
// Yee kernels; their Bloch-wrap cells and the injection planes run in the
// general kernels (yee.cuh, bloch_ghost and the kobl injection).
#include "sim.hpp"

namespace {

using aefdtd::cplx;
using namespace aefdtd::phys;

struct V3 {
    double x, y, z;
};
// Vector3 arithmetic of the reference (vector23.cpp:156-161, 266-283, 447-475)
V3 cross(const V3 &a, const V3 &b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
V3 scale(double s, const V3 &v) { return {s * v.x, s * v.y, s * v.z}; }
V3 plus(const V3 &a, const V3 &b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
double norm3(const V3 &v) { return std::sqrt(v.x * v.x + v.y * v.y + v.z * v.z); }

// dichotomy<...>(a, b, f, params..., eps) (mathUT.h:549-566) on
// value_s_curve(x, 0, 1, v) = s_curve(x, 0, 1) - v (mathUT.cpp:1204-1207)
double dichotomy_s_curve(double a, double b, double v, double eps) {
    double c = (a + b) / 2.0;
    while (2.0 * std::abs((b - a) / (a + b)) > eps) {
        c = (a + b) / 2.0;
        const double fa = s_curve(a, 0, 1) - v, fc = s_curve(c, 0, 1) - v;
        if (fc / fa > 0) a = c;
        else b = c;
    }
    return c;
}

// Bloch_Wideband::initialize (sc_bloch.cpp:85-214): 30001 spectral lines
// between the cut and safe angles' frequencies, s-curve windows, E and H
// bases normalised so that the summed E is 1, and the time offset at which
// the pulse at z2 has decayed below 1e-4.
void bloch_initialize(aefdtd::Oblique &o, double lambda_min, double lambda_max, double polar, double Dt, double Dz) {
    const double safe_angle = 75 * (Pi / 180.0), cut_angle = 85 * (Pi / 180.0);   // Degree(75), Degree(85)
    const double kx = o.kx, ky = o.ky, kxy = o.kxy;
    double w_max = 2.0 * Pi * c_light / lambda_min;
    double w_min = 2.0 * Pi * c_light / lambda_max;
    const double w_cut = kxy * c_light / (std::sqrt(o.eps_inf) * std::sin(cut_angle));
    const double w_safe = kxy * c_light / (std::sqrt(o.eps_inf) * std::sin(safe_angle));
    const double xs = dichotomy_s_curve(0, 1, std::sqrt(0.1), 1e-6);
    w_min = std::max(w_min, w_safe);
    const double w_med = 0.5 * (w_min + w_max);
    double w_out = xs / (1.0 - xs) * (w_med - w_min);
    double w1m, w1p, w2m, w2p;
    if (w_min - w_cut > w_out) {
        w1m = w_min - w_out;
        w1p = w_med;
        w2m = w_med;
        w2p = w_max + w_out;
    } else {
        w_out = w_min - w_cut;
        const double w_tmp = w_out / xs;
        w1m = w_cut;
        w1p = w1m + w_tmp;
        w2p = w_max + w_out;
        w2m = w2p - w_tmp;
    }
    const int Nl = 30001;
    o.nlines = Nl;
    o.w.resize(Nl);
    const double span = w2p - w1m;   // linspace (mathUT.cpp:1011-1018)
    for (int i = 0; i < Nl; i++) o.w[i] = w1m + span * i / (Nl - 1.0);
    o.kz.resize(Nl);
    std::vector<V3> E(Nl), H(Nl);
    double SEx = 0, SEy = 0, SEz = 0;
    for (int l = 0; l < Nl; l++) {
        const double kn = std::sqrt(o.eps_inf) * o.w[l] / c_light;
        o.kz[l] = std::sqrt(kn * kn - kxy * kxy);
        const double Sp = s_curve(o.w[l], w1m, w1p) * s_curve(o.w[l], w2p, w2m);
        const V3 k_vec{kx, ky, -o.kz[l]};
        V3 p_vec{-ky / kxy, kx / kxy, 0};
        if (kx == 0 && ky == 0) p_vec = V3{0, 1, 0};
        const V3 kvp = cross(k_vec, p_vec);
        V3 t_vec = kvp;
        const double n = norm3(t_vec);
        t_vec = V3{t_vec.x / n, t_vec.y / n, t_vec.z / n};
        const V3 kvt = cross(k_vec, t_vec);
        E[l] = scale(Sp, plus(scale(std::cos(polar), p_vec), scale(std::sin(polar), t_vec)));
        H[l] = scale(Sp / (o.w[l] * mu0), plus(scale(std::cos(polar), kvp), scale(std::sin(polar), kvt)));
        SEx += E[l].x;
        SEy += E[l].y;
        SEz += E[l].z;
    }
    double Snorm = std::sqrt(SEx * SEx + SEy * SEy + SEz * SEz);
    for (int l = 0; l < Nl; l++) {
        E[l] = V3{E[l].x / Snorm, E[l].y / Snorm, E[l].z / Snorm};
        H[l] = V3{H[l].x / Snorm, H[l].y / Snorm, H[l].z / Snorm};
    }
    Snorm = 1.0;
    const cplx Im(0, 1);
    o.t_offset = 0;
    while (Snorm >= 1e-4) {
        cplx ex = 0, ey = 0, ez = 0;
        for (int l = 0; l < Nl; l++) {
            const cplx im_arg = std::exp(-(o.kz[l] * o.z2 * Dz + o.w[l] * Dt * o.t_offset) * Im);
            ex += im_arg * E[l].x;
            ey += im_arg * E[l].y;
            ez += im_arg * E[l].z;
        }
        Snorm = std::sqrt(std::real(ex * std::conj(ex) + ey * std::conj(ey) + ez * std::conj(ez)));
        o.t_offset += 100;
    }
    o.t_offset = -2 * o.t_offset;
    o.eb.resize(size_t(Nl) * 3);
    o.hb.resize(size_t(Nl) * 2);
    for (int l = 0; l < Nl; l++) {
        o.eb[3 * l] = E[l].x; o.eb[3 * l + 1] = E[l].y; o.eb[3 * l + 2] = E[l].z;
        o.hb[2 * l] = H[l].x; o.hb[2 * l + 1] = H[l].y;
    }
}

}  // namespace

// FDTD::find_slab (fdtd_utils.cpp:347-392)
void aefdtd_sim::find_slab(int sub_ref, int sup_ref, double &hsub, double &hstruc, double &hsup) const {
    auto M = [&](int i, int j, int k) { return map[i + size_t(j) * Nx + size_t(k) * Nx * Ny]; };
    int Nsub = 0, Nsup = 0, IDmoy = 0, IDsup = 0, IDsub = 0, k;
    for (int i = xs_s; i < xs_e; i++)
        for (int j = ys_s; j < ys_e; j++) { IDsup += M(i, j, zs_e); IDsub += M(i, j, zs_s); }
    IDmoy = IDsub;
    k = sub_ref;
    while (IDmoy == IDsub && k < sup_ref) {
        IDmoy = 0;
        for (int i = xs_s; i < xs_e; i++) for (int j = ys_s; j < ys_e; j++) IDmoy += M(i, j, k + 1);
        Nsub++;
        k++;
    }
    IDmoy = IDsup;
    k = sup_ref;
    while (IDmoy == IDsup && k >= sub_ref) {
        IDmoy = 0;
        for (int i = xs_s; i < xs_e; i++) for (int j = ys_s; j < ys_e; j++) IDmoy += M(i, j, k - 1);
        Nsup++;
        k--;
    }
    hsup = (Nsup - 1) * Dz;
    hsub = Nsub * Dz;
    hstruc = (Nz_s - Nsup - Nsub) * Dz;
}

// Incident sums for steps [0, steps) and the R/T history, grown on demand.
void aefdtd_sim::obl_ensure(int steps) {
    Oblique &o = *obl;
    if (steps <= o.cap) return;
    const int cap = std::max(steps, std::max(2 * o.cap, std::max(Nt, 64)));
    DBuf inc, hist;
    inc.alloc(size_t(cap) * 14 * 8, dev_bytes);
    hist.alloc(size_t(cap) * 18 * 8, dev_bytes);
    AE_CUDA(cudaMemsetAsync(hist.p, 0, hist.n, stream));
    if (o.hist.p) AE_CUDA(cudaMemcpyAsync(hist.p, o.hist.p, size_t(o.cap) * 18 * 8, cudaMemcpyDeviceToDevice, stream));
    OblIncArgs a{};
    a.nl = o.nlines;
    a.w = o.dw.as<double>(); a.kz = o.dkz.as<double>(); a.eb = o.deb.as<double>(); a.hb = o.dhb.as<double>();
    a.Dt = Dt; a.Dz = Dz;
    a.z2 = o.z2; a.zs_s = zs_s; a.t_offset = o.t_offset;
    a.t0 = 0; a.n = cap;
    a.out = inc.as<double>();
    launch_obl_incident(a, stream);
    launches++;
    AE_CUDA(cudaGetLastError());
    AE_CUDA(cudaStreamSynchronize(stream));
    o.inc.release(dev_bytes);
    o.hist.release(dev_bytes);
    o.inc = inc;
    o.hist = hist;
    o.cap = cap;
}

template <typename T> int aefdtd_sim::launch_obl_sums(int q, const StepScalars *tbl, cudaStream_t st) {
    Oblique &o = *obl;
    OblSumArgs<T> a{};
    a.Nx = Nx; a.Ny = Ny; a.NxNy = (long long)Nx * Ny;
    a.Ex = F[0].as<T>(); a.Ey = F[1].as<T>(); a.Ez = F[2].as<T>();
    a.kr = zs_e + 2;
    a.kt = zs_s;
    a.mk = o.mk.as<double2>();
    a.ph = o.ph.as<double2>();
    a.inc = o.inc.as<double>();
    a.sc = tbl;
    a.q = q;
    a.partial = o.part.as<double>() + size_t(q) * o.nb * 18;
    return aefdtd::launch_obl_sums(a, o.nb, st);
}
template int aefdtd_sim::launch_obl_sums<double>(int, const StepScalars *, cudaStream_t);
template int aefdtd_sim::launch_obl_sums<float>(int, const StepScalars *, cudaStream_t);

extern "C" {

aefdtd_status aefdtd_setup_oblique(aefdtd_sim *s, const aefdtd_oblique_desc *od) {
    if (!s || !od) return AEFDTD_BAD_ARG;
    return guarded(s, [&] {
        if (s->g.mode != AEFDTD_MODE_OBLIQUE) fail(AEFDTD_BAD_ARG, "setup_oblique needs mode OBLIQUE");
        if (s->obl) fail(AEFDTD_BAD_ARG, "oblique incidence is already set up");
        if (s->batch) fail(AEFDTD_NOT_READY, "batch members run normal or custom mode only");
        if (!s->map_set) fail(AEFDTD_NOT_READY, "set the material map first");
        if (od->nl < 2 || !(od->lambda_min > 0) || !(od->lambda_max > od->lambda_min))
            fail(AEFDTD_BAD_ARG, "bad spectrum");
        if (s->zs_e + 2 >= s->Nz || s->zs_s < 1) fail(AEFDTD_BAD_ARG, "z pads too thin for the R/T planes");
        s->set_device();
        auto *o = new Oblique();
        o->d = *od;
        s->obl = o;
        try {
            const cplx Im(0, 1);
            auto M = [&](int i, int j, int k) { return s->map[i + size_t(j) * s->Nx + size_t(k) * s->Nx * s->Ny]; };
            // oblique_biphase.cpp:117-131
            o->eps_sub = s->mats[M(0, 0, s->zs_s)].ei;
            o->eps_sup = s->mats[M(0, 0, s->zs_e)].ei;
            o->index_sub = std::sqrt(o->eps_sub);
            o->index_sup = std::sqrt(o->eps_sup);
            o->kx = od->kx_in * o->index_sup;
            o->ky = od->ky_in * o->index_sup;
            o->kxy = std::sqrt(o->kx * o->kx + o->ky * o->ky);
            const double polar = (od->polarization == 1 ? 90 : 0) * Pi / 180.0;   // AngleRad::degree
            // Bloch_Wideband(0, Nx, 0, Ny, 0, Nz_s) linked to the real grid (Source::link, sources.cpp:252-283)
            o->z2 = std::clamp(s->Nz_s + s->zs_s, 0, s->Nz);
            o->eps_inf = s->mats[M(0, 0, o->z2)].ei;
            o->c2z = s->mats[M(0, 0, o->z2)].C2z;   // coeffsX of the injection plane's material
            bloch_initialize(*o, od->lambda_min, od->lambda_max, polar, s->Dt, s->Dz);
            // Bloch phases of the wraps (oblique_biphase.cpp:144-148)
            const double kx = o->kx, ky = o->ky, Dx = s->Dx, Dy = s->Dy;
            const int Nx = s->Nx, Ny = s->Ny;
            o->dE_x = std::exp(kx * Nx * Dx * Im);
            o->dE_y = std::exp(ky * Ny * Dy * Im);
            o->dH_x = std::exp(-kx * Nx * Dx * Im);
            o->dH_y = std::exp(-ky * Ny * Dy * Im);
            // per-column phases: the source's e^{+ik.r} at the Ex, Ey, Ez points
            // (sc_bloch.cpp:72-74, 236-237, 272-273) and the sensors' e^{-ik.r}
            // (oblique_biphase.cpp:158-163)
            const size_t P = size_t(Nx) * Ny;
            std::vector<cplx> ph(3 * P), mk(3 * P);
            for (int i = 0; i < Nx; i++)
                for (int j = 0; j < Ny; j++) {
                    const size_t c = i + size_t(j) * Nx;
                    ph[c] = std::exp(((i + 0.5) * Dx * kx + j * Dy * ky) * Im);
                    ph[P + c] = std::exp((i * Dx * kx + (j + 0.5) * Dy * ky) * Im);
                    ph[2 * P + c] = std::exp((i * Dx * kx + j * Dy * ky) * Im);
                    mk[c] = std::exp(-(kx * (i + 0.5) * Dx + ky * j * Dy) * Im);
                    mk[P + c] = std::exp(-(kx * i * Dx + ky * (j + 0.5) * Dy) * Im);
                    mk[2 * P + c] = std::exp(-(kx * i * Dx + ky * j * Dy) * Im);
                }
            auto up = [&](DBuf &b, const void *src, size_t bytes) {
                b.alloc(bytes, s->dev_bytes);
                AE_CUDA(cudaMemcpy(b.p, src, bytes, cudaMemcpyHostToDevice));
            };
            up(o->ph, ph.data(), ph.size() * sizeof(cplx));
            up(o->mk, mk.data(), mk.size() * sizeof(cplx));
            up(o->dw, o->w.data(), o->w.size() * 8);
            up(o->dkz, o->kz.data(), o->kz.size() * 8);
            up(o->deb, o->eb.data(), o->eb.size() * 8);
            up(o->dhb, o->hb.data(), o->hb.size() * 8);
            // the imaginary grid: fields, CPML psi (z slabs) and dispersive psi
            const size_t es = s->fp64 ? 8 : 4, N = size_t(Nx) * Ny * s->Nz;
            for (int c = 0; c < 6; c++) {
                o->Fi[c].alloc(N * es, s->dev_bytes);
                o->psiEi[c].alloc(s->psiE[c].n, s->dev_bytes);
                o->psiHi[c].alloc(s->psiH[c].n, s->dev_bytes);
                DBuf *b[3] = {&o->Fi[c], &o->psiEi[c], &o->psiHi[c]};
                for (DBuf *x : b) if (x->p) AE_CUDA(cudaMemsetAsync(x->p, 0, x->n, s->stream));
            }
            o->nb = (int)std::max<size_t>(1, std::min<size_t>(2 * 148, (P + 255) / 256));
            o->part.alloc(size_t(s->seg_len) * o->nb * 18 * 8, s->dev_bytes);
            s->obl_ensure(std::max(s->Nt, 64));
            AE_CUDA(cudaStreamSynchronize(s->stream));
        } catch (...) {
            size_t t = 0;
            for (int c = 0; c < 6; c++) { o->Fi[c].release(t); o->psiEi[c].release(t); o->psiHi[c].release(t); }
            DBuf *b[] = {&o->psi_i, &o->ph, &o->mk, &o->inc, &o->part, &o->hist, &o->dw, &o->dkz, &o->deb, &o->dhb};
            for (DBuf *x : b) x->release(t);
            s->dev_bytes -= std::min(s->dev_bytes, t);
            delete o;
            s->obl = nullptr;
            throw;
        }
        s->tables_dirty = true;   // the dispersive psi of the imaginary grid
        s->work_dirty = true;
        s->graphs_dirty = true;
    });
}

aefdtd_status aefdtd_get_oblique_series(aefdtd_sim *s, double *out, size_t count) {
    if (!s || !out) return AEFDTD_BAD_ARG;
    return guarded(s, [&] {
        if (!s->obl) fail(AEFDTD_NOT_READY, "oblique mode is not set up");
        if (count != size_t(s->tstep) * 18) fail(AEFDTD_BAD_ARG, "count must be 18 x the completed steps");
        s->set_device();
        if (count) AE_CUDA(cudaMemcpyAsync(out, s->obl->hist.p, count * 8, cudaMemcpyDeviceToHost, s->stream));
        AE_CUDA(cudaStreamSynchronize(s->stream));
    });
}

// oblique_biphase.cpp:334-480 and the driver's obl_ file columns (:640-652),
// FP64 on the host over the completed steps.
aefdtd_status aefdtd_get_oblique_spectra(aefdtd_sim *s, double *out, int32_t nl_max, int32_t *nl_out) {
    if (!s || !out) return AEFDTD_BAD_ARG;
    return guarded(s, [&] {
        if (!s->obl) fail(AEFDTD_NOT_READY, "oblique mode is not set up");
        const Oblique &o = *s->obl;
        const int Nt = s->tstep;
        if (Nt < 2) fail(AEFDTD_NOT_READY, "run at least two steps");
        std::vector<double> S(size_t(Nt) * 18);
        s->set_device();
        AE_CUDA(cudaMemcpyAsync(S.data(), o.hist.p, S.size() * 8, cudaMemcpyDeviceToHost, s->stream));
        AE_CUDA(cudaStreamSynchronize(s->stream));
        const cplx Im(0, 1);
        const double kx = o.kx, ky = o.ky, kxy = o.kxy, Dz = s->Dz, Dt = s->Dt;
        int Nl = o.d.nl;
        const double lambda_min = o.d.lambda_min;
        double lambda_max = o.d.lambda_max;
        // spectrum resizing to the 89-degree limit (:334-347)
        double lambda_limit_max = lambda_max;
        if (kx != 0 || ky != 0) lambda_limit_max = 2 * Pi * std::sin(89.0 * Pi / 180.0) * o.index_sup / kxy;
        if (lambda_limit_max < lambda_max) {
            const double D_lambda = (lambda_max - lambda_min) / (Nl - 1.0);
            Nl = static_cast<int>((lambda_limit_max - lambda_min) / D_lambda);
            if (Nl < 2) Nl = 2;
            lambda_max = lambda_min + (Nl - 1.0) * D_lambda;
        }
        if (nl_out) *nl_out = Nl;
        double hsup, hsub, hstruc;
        s->find_slab(s->zs_s, s->zs_e + 2, hsub, hstruc, hsup);
        const double phi = std::atan2(ky, kx);
        const double cp = std::cos(phi), sp = std::sin(phi);
        auto series = [&](int c, int t) { return cplx(S[size_t(t) * 18 + c], S[size_t(t) * 18 + c + 1]); };
        // wavelengths are independent; each one's sums run in the driver's order
        parallel_for(std::min(Nl, nl_max), [&](int l) {
            const double lambda = lambda_min + (lambda_max - lambda_min) * l / (Nl - 1.0);
            const double w = 2.0 * Pi * c_light / lambda;
            const double kn = 2.0 * Pi * o.index_sup / lambda;
            const double inc_ang = std::asin(kxy / kn);
            const double ref_ang = std::asin(o.index_sup / o.index_sub * std::sin(inc_ang));
            const double s_k0 = -w / c_light, s_k1 = s_k0 * o.index_sup, s_k3 = s_k0 * o.index_sub;
            // BR, R, T (BT = BR) x, y, z
            cplx BR[3] = {0, 0, 0}, R[3] = {0, 0, 0}, T[3] = {0, 0, 0};
            for (int t = 0; t < Nt; t++) {
                const cplx coeff = std::exp(w * t * Dt * Im);
                for (int d = 0; d < 3; d++) {
                    BR[d] += series(2 * d, t) * coeff;
                    R[d] += series(6 + 2 * d, t) * coeff;
                    T[d] += series(12 + 2 * d, t) * coeff;
                }
            }
            cplx BT[3] = {BR[0], BR[1], BR[2]};
            auto rotate = [&](cplx *v) {
                const cplx tx = v[0], ty = v[1];
                v[0] = cp * tx + sp * ty;
                v[1] = -sp * tx + cp * ty;
            };
            rotate(BR); rotate(R); rotate(BT); rotate(T);
            const double s_k1z = s_k1 * std::cos(inc_ang);
            const cplx tmp_sup = std::exp(((2.0 * hsup + 2 * Dz) * s_k1z) * Im);   // im_exp
            const cplx tmp_sub = std::exp((s_k3 * (hsub - Dz / 2.0) * std::cos(ref_ang) +
                                           s_k0 * (hsup + Dz / 2.0) * std::cos(inc_ang)) * Im);
            const bool tm = o.d.polarization == 1;
            const cplx Rbase = tm ? BR[0] : BR[1], Tbase = tm ? BT[0] : BT[1];
            const double base_norm_ref = tm ? std::sqrt(std::norm(BR[0]) + std::norm(BR[2])) : std::abs(BR[1]);
            const double base_norm_trans = tm ? std::sqrt(std::norm(BT[0]) + std::norm(BT[2])) : std::abs(BT[1]);
            const double TE_norm_ref = std::abs(R[1]);
            const double TM_norm_ref = std::sqrt(std::norm(R[0]) + std::norm(R[2]));
            const double TE_norm_trans = std::abs(T[1]);
            const double TM_norm_trans = std::sqrt(std::norm(T[0]) + std::norm(T[2]));
            const double TE_arg_ref = std::arg(R[1] / Rbase * tmp_sup);
            const double TM_arg_ref = std::arg(R[0] / Rbase * tmp_sup);
            const double TE_arg_trans = std::arg(T[1] / Tbase * tmp_sub);
            const double TM_arg_trans = std::arg(T[0] / Tbase * tmp_sub);
            const cplx te_r = TE_norm_ref / base_norm_ref * std::exp(TE_arg_ref * Im);
            const cplx tm_r = TM_norm_ref / base_norm_ref * std::exp(TM_arg_ref * Im);
            const cplx te_t = TE_norm_trans / base_norm_trans * std::exp(TE_arg_trans * Im);
            const cplx tm_t = TM_norm_trans / base_norm_trans * std::exp(TM_arg_trans * Im);
            double *r = out + size_t(l) * 10;
            r[0] = lambda;
            r[1] = inc_ang * 180.0 / Pi;   // AngleRad::degree
            r[2] = std::abs(te_r); r[3] = std::arg(te_r);
            r[4] = std::abs(tm_r); r[5] = std::arg(tm_r);
            r[6] = std::abs(te_t); r[7] = std::arg(te_t);
            r[8] = std::abs(tm_t); r[9] = std::arg(tm_t);
        });
    });
}

}  // extern "C"
