/* aefdtd.hpp — header-only C++ shim over the C ABI (aefdtd.h) with the
 * method names of the reference's FDTD class (src/finite_differences/FDTD/
 * core/fdtd_core.h:26-285), for mode drivers written against that class.
 *
 *   aefdtd::FDTD f(Nx, Ny, Nz, Nt, Dx, Dy, Dz, Dt, "NORMAL", pml..., pad...);
 *   f.set_pml_zm(kappa, sigma, alpha); ...   // before the first use, as in the reference
 *   f.set_matsgrid(map);                      // FDTD::set_matsgrid
 *   f.set_material(i, mat);                   // FDTD::set_material
 *   f.bootstrap();
 *   f.setup_normal(nd);                       // normal_incidence.cpp:161-436 setup
 *   for (...) f.update(1);                    // update_E + injection + update_H + injection + sensors
 *
 * Differences a caller sees: the grid lives on the GPU, so fields are read
 * and written with get_field/set_field (x-fastest, the Grid3 order) instead
 * of through public Grid3 members; errors throw aefdtd::Error (the reference
 * prints and exits). One host thread owns an object, as in the reference. */
#ifndef AEFDTD_HPP
#define AEFDTD_HPP

#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "aefdtd.h"

namespace aefdtd {

struct Error : std::runtime_error {
    aefdtd_status status;
    Error(aefdtd_status s, const std::string &m) : std::runtime_error(m), status(s) {}
};

inline void check(aefdtd_status s, const aefdtd_sim *h) {
    if (s != AEFDTD_OK)
        throw Error(s, std::string(aefdtd_status_string(s)) + ": " + (aefdtd_last_error(h) ? aefdtd_last_error(h) : ""));
}

class FDTD {
  public:
    /* FDTD::FDTD(Nx, Ny, Nz, Nt, Dx, Dy, Dz, Dt, mode, pml x6, pad x6)
     * (fdtd_core.cpp:158-285). mode: "NORMAL" (normal incidence) or
     * "CUSTOM". Dt <= 0 selects the drivers' Courant rule with time_mod. */
    FDTD(int Nx, int Ny, int Nz, int Nt, double Dx, double Dy, double Dz, double Dt, const std::string &mode,
         int pml_xm, int pml_xp, int pml_ym, int pml_yp, int pml_zm, int pml_zp, int pad_xm, int pad_xp,
         int pad_ym, int pad_yp, int pad_zm, int pad_zp, aefdtd_precision precision = AEFDTD_FP64, int device = 0) {
        std::memset(&d_, 0, sizeof(d_));
        d_.abi_version = AEFDTD_ABI_VERSION;
        if (mode == "NORMAL" || mode == "NORM") d_.mode = AEFDTD_MODE_NORMAL;
        else if (mode == "CUSTOM") d_.mode = AEFDTD_MODE_CUSTOM;
        else throw Error(AEFDTD_BAD_ARG, "unknown FDTD mode " + mode);
        d_.precision = precision;
        d_.nx = Nx; d_.ny = Ny; d_.nz = Nz; d_.nt = Nt;
        d_.dx = Dx; d_.dy = Dy; d_.dz = Dz; d_.dt = Dt; d_.time_mod = 1.0;
        const int p[6] = {pml_xm, pml_xp, pml_ym, pml_yp, pml_zm, pml_zp};
        const int q[6] = {pad_xm, pad_xp, pad_ym, pad_yp, pad_zm, pad_zp};
        for (int i = 0; i < 6; i++) { d_.pml[i] = p[i]; d_.pad[i] = q[i]; d_.pml_kappa[i] = 1.0; }
        d_.device = device;
    }
    FDTD(const FDTD &) = delete;
    FDTD &operator=(const FDTD &) = delete;
    ~FDTD() { if (h_) aefdtd_destroy(h_); }

    /* FDTD::set_pml_{xm..zp}(kappa, sigma, alpha) (fdtd_pml.cpp): before the first use */
    void set_pml_xm(double k, double s, double a) { pml(0, k, s, a); }
    void set_pml_xp(double k, double s, double a) { pml(1, k, s, a); }
    void set_pml_ym(double k, double s, double a) { pml(2, k, s, a); }
    void set_pml_yp(double k, double s, double a) { pml(3, k, s, a); }
    void set_pml_zm(double k, double s, double a) { pml(4, k, s, a); }
    void set_pml_zp(double k, double s, double a) { pml(5, k, s, a); }
    void set_tapering(int Ntap) { before_create(); d_.tapering = Ntap; }
    void set_time_mod(double m) { before_create(); d_.time_mod = m; }
    void set_dft_block(int K) { before_create(); d_.dft_block = K; }

    /* FDTD::set_matsgrid (fdtd_utils.cpp:572-800): structure-size map, x fastest */
    void set_matsgrid(const std::vector<uint32_t> &map) {
        check(aefdtd_set_material_map(h(), map.data(), map.size()), h_);
    }
    /* FDTD::set_material (fdtd_utils.cpp:810-820) */
    void set_material(unsigned idx, const aefdtd_material_desc &m) { check(aefdtd_set_material(h(), idx, &m), h_); }
    /* FDTD::bootstrap (fdtd_core.cpp:1137-1148): fields are created zeroed */
    void bootstrap() { h(); }

    void setup_normal(const aefdtd_normal_desc &nd) { check(aefdtd_setup_normal(h(), &nd), h_); }
    int add_oscillator(const aefdtd_source_desc &s) {
        int32_t id = -1;
        check(aefdtd_add_oscillator(h(), &s, &id), h_);
        return id;
    }
    int add_planar_sensor(const aefdtd_sensor_desc &s) {
        int32_t id = -1;
        check(aefdtd_add_planar_sensor(h(), &s, &id), h_);
        return id;
    }

    /* n full steps: update_E, E injection, update_H, H injection, sensor feed */
    void update(int n = 1) { check(aefdtd_step(h(), n), h_); }
    void synchronize() { check(aefdtd_synchronize(h()), h_); }
    void reset() { check(aefdtd_reset(h()), h_); }

    /* the public Grid3 members Ex..Hz: component 0..5 = Ex, Ey, Ez, Hx, Hy, Hz */
    std::vector<double> get_field(int comp) {
        aefdtd_dims dm = dims();
        std::vector<double> v(size_t(dm.nx) * dm.ny * dm.nz);
        check(aefdtd_get_field(h(), comp, v.data(), v.size()), h_);
        return v;
    }
    void set_field(int comp, const std::vector<double> &v) { check(aefdtd_set_field(h(), comp, v.data(), v.size()), h_); }

    aefdtd_dims dims() {
        aefdtd_dims dm{};
        check(aefdtd_get_dims(h(), &dm), h_);
        return dm;
    }
    /* the FDTD scalars callers read: total sizes, structure range, tstep, Dt */
    int Nx() { return dims().nx; }
    int Ny() { return dims().ny; }
    int Nz() { return dims().nz; }
    int zs_s() { return dims().zs_s; }
    int zs_e() { return dims().zs_e; }
    int tstep() { return dims().step; }
    double Dt() { return dims().dt; }

    std::vector<double> normal_spectra(int nl) {
        std::vector<double> v(size_t(15) * nl);
        check(aefdtd_get_normal_spectra(h(), v.data(), nl), h_);
        return v;
    }
    std::vector<double> sensor_flux(int id, int nl) {
        std::vector<double> v(nl);
        check(aefdtd_get_sensor_flux(h(), id, v.data(), nl), h_);
        return v;
    }
    aefdtd_sim *handle() { return h(); }

  private:
    aefdtd_grid_desc d_;
    aefdtd_sim *h_ = nullptr;
    void before_create() const {
        if (h_) throw Error(AEFDTD_BAD_ARG, "PML, tapering and time settings must precede the first use");
    }
    void pml(int f, double k, double s, double a) {
        before_create();
        d_.pml_kappa[f] = k; d_.pml_sigma[f] = s; d_.pml_alpha[f] = a;
    }
    aefdtd_sim *h() {
        if (!h_) check(aefdtd_create(&d_, &h_), nullptr);
        return h_;
    }
};

}  // namespace aefdtd

#endif /* AEFDTD_HPP */
