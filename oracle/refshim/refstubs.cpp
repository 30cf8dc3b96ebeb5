/* Link stubs for the oracle build of the reference FDTD core.
 *
 * Test infrastructure only. The reference's FDTD sources are compiled
 * unmodified; these definitions satisfy symbols that the FDTD time loop never
 * reaches: PNG previews (libpng is absent here), cubic splines (Eigen is
 * absent; splines are excluded from FDTD by Material::fdtd_compatible), the
 * FFT Poynting sensor (FFTW is absent), and the guided-mode source (needs the
 * FDFD solver). Each unreachable entry aborts so that a stray call cannot pass
 * silently; the Bitmap entries are no-ops because FDTD::set_matsgrid always
 * writes a debug preview of the material map. */
#include <bitmap3.h>
#include <math_approx.h>
#include <sources.h>
#include <fftw3.h>

#include <cstdio>
#include <cstdlib>

[[noreturn]] static void aeoracle_unreachable(const char *what) {
    std::fprintf(stderr, "aeoracle: unreachable reference path called: %s\n", what);
    std::abort();
}

// Bitmap: previews are not produced by the oracle build.
Bitmap::Bitmap() : width(0), height(0) {}
Bitmap::Bitmap(int x, int y) : width(x), height(y) {}
void Bitmap::degra(int, int, double, double, double) {}
void Bitmap::degra_circ(int, int, double, double, double) {}
void Bitmap::G2degra(Grid2<double> &, std::string) {}
void Bitmap::G2degraM(Grid2<double> &, std::string, int, std::string, double, double) {}
void Bitmap::set_full(double, double, double) {}
void Bitmap::set_size(int w, int h) { width = w; height = h; }
void Bitmap::write(std::string const &) {}

// Cspline: only tabulated (non-FDTD) materials use it.
Cspline::Cspline() {}
Cspline::Cspline(Cspline const &) {}
std::size_t Cspline::get_N() const { aeoracle_unreachable("Cspline::get_N"); }
double Cspline::get_x_base(std::size_t const &) const { aeoracle_unreachable("Cspline::get_x_base"); }
double Cspline::get_y_base(std::size_t const &) const { aeoracle_unreachable("Cspline::get_y_base"); }
void Cspline::init(std::vector<double> const &, std::vector<double> const &, int) { aeoracle_unreachable("Cspline::init"); }
double Cspline::operator()(double const &) const { aeoracle_unreachable("Cspline::operator()"); }
void Cspline::operator=(Cspline const &) {}
bool Cspline::operator==(Cspline const &) const { return true; }

// FFTW: only the FFT Poynting sensor uses it.
void *fftw_malloc(unsigned long) { aeoracle_unreachable("fftw_malloc"); }
void fftw_free(void *) { aeoracle_unreachable("fftw_free"); }
fftw_plan fftw_plan_dft_1d(int, fftw_complex *, fftw_complex *, int, unsigned) { aeoracle_unreachable("fftw_plan_dft_1d"); }
void fftw_execute(const fftw_plan) { aeoracle_unreachable("fftw_execute"); }
void fftw_destroy_plan(fftw_plan) { aeoracle_unreachable("fftw_destroy_plan"); }

// Guided planar source: needs the FDFD mode solver.
Guided_planar::Guided_planar(int type_, int x1_, int x2_, int y1_, int y2_, int z1_, int z2_,
                             int, double, double, double)
    : Source(x1_, x2_, y1_, y2_, z1_, z2_) {
    (void)type_;
    aeoracle_unreachable("Guided_planar");
}
Guided_planar::~Guided_planar() {}
void Guided_planar::deep_inject_E(FDTD &) { aeoracle_unreachable("Guided_planar::deep_inject_E"); }
void Guided_planar::deep_inject_H(FDTD &) { aeoracle_unreachable("Guided_planar::deep_inject_H"); }
void Guided_planar::deep_link(FDTD const &) { aeoracle_unreachable("Guided_planar::deep_link"); }
void Guided_planar::initialize() { aeoracle_unreachable("Guided_planar::initialize"); }
