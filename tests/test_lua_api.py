"""The scripting front end with the reference's Lua method names
(aether_b200.lua_api): parameters and sizes as in the reference's
tests/fdtd/parametric_structure.lua, FDTD_Mode::finalize's pad rules, the
sensors' real-to-cell rounding, and (GPU) a mode run through compute()
against the reference core on the scene the front end builds."""
import numpy as np
import pytest

import oracle_lib
from aether_b200 import _abi as A
from aether_b200 import lua_api as L


def basic_parametric(st):
    """The sample structure the reference's parametric test loads: three
    declared sizes and a vacuum default."""
    st.lx = st.declare_parameter("px", 200e-9)
    st.ly = st.declare_parameter("py", 300e-9)
    st.lz = st.declare_parameter("pz", 400e-9)
    st.default_material(0)


def test_parametric_structure_sizes():
    structure = L.Structure(basic_parametric)
    fdtd = L.MODE("fdtd_normal")
    fdtd.structure(structure)
    assert (fdtd.Lx(), fdtd.Ly(), fdtd.Lz()) == (200e-9, 300e-9, 400e-9)
    assert (fdtd.Nx(), fdtd.Ny(), fdtd.Nz()) == (40, 60, 80)

    structure.parameter("px", 220e-9)
    structure.parameter("py", 330e-9)
    structure.parameter("pz", 440e-9)
    # a recorded parameter takes effect when a mode takes the structure
    assert fdtd.Lx() == 200e-9
    fdtd = L.MODE("fdtd_normal")
    fdtd.structure(structure)
    assert (fdtd.Lx(), fdtd.Ly(), fdtd.Lz()) == (220e-9, 330e-9, 440e-9)


def test_discretisation_rounds_to_nearest_cell():
    st = L.Structure(lambda s: s.size(101e-9, 12e-9, 1e-9))
    f = L.MODE("fdtd")
    f.structure(st)
    f.Dx(5e-9)
    f.Dy(5e-9)
    f.Dz(5e-9)
    # 20.2 -> 20, 2.4 -> 2, 0.2 -> 0 -> at least one cell
    assert (f.Nx(), f.Ny(), f.Nz()) == (20, 2, 1)
    f.Dxyz(4e-9)
    assert (f.Nx(), f.Ny(), f.Nz()) == (25, 3, 1)


def test_sensor_and_source_locations():
    s = L.create_sensor("planar_spectral_poynting")
    s.location(12.4e-9, 12.6e-9, -8e-9, 30e-9, 10e-9, 10e-9)
    # nearest_integer (negative values round down from -x.5); empty ranges get one cell
    assert s.to_discrete(5e-9, 5e-9, 5e-9) == (2, 3, -2, 6, 2, 3)
    s.location_grid(1, 4, 2, 5, 7, 8)
    assert s.to_discrete(5e-9, 5e-9, 5e-9) == (1, 4, 2, 5, 7, 8)
    p = L.create_sensor("fieldpoint")
    p.location(10e-9, 20e-9, 30e-9)
    assert p.to_discrete(5e-9, 5e-9, 5e-9) == (2, 3, 4, 5, 6, 7)
    o = L.create_source("oscillator")
    o.location_grid(3, 4, 5)
    assert o.to_discrete(5e-9, 5e-9, 5e-9) == (3, 4, 4, 5, 5, 6)
    o.location(10e-9, 20e-9, 30e-9)
    assert o.to_discrete(5e-9, 5e-9, 5e-9) == (2, 3, 4, 5, 6, 7)
    for txt, want in (("X", A.NORMAL_X), ("x+", A.NORMAL_X), ("-y", A.NORMAL_YM), ("Z-", A.NORMAL_ZM),
                      ("+Z", A.NORMAL_Z)):
        s.orientation(txt)
        assert s.orient == want
    b = L.create_sensor("box_spectral_poynting")
    b.disable("-z")
    b.disable("X")
    assert b.disabled == (1 << 4) | (1 << 1)
    with pytest.raises(ValueError):
        L.create_sensor("farfield")


def test_finalize_pads_custom_mode():
    """FDTD_Mode::finalize: a face with PML gets at least 5 pad cells, 5 more
    than any sensor reaches past the structure and 50 around an oscillator;
    a face without PML gets none."""
    st = L.Structure(lambda s: s.size(200e-9, 200e-9, 300e-9))
    f = L.MODE("fdtd")
    f.structure(st)
    f.pml_xm(10, 25, 1, 0.2)
    f.pml_xp(10, 25, 1, 0.2)
    f.pml_zm(12, 25, 1, 0.2)
    f.pml_zp(12, 25, 1, 0.2)
    f.padding(7, 0, 9, 9, 0, 0)
    s = L.create_sensor("box_spectral_poynting")
    s.location_grid(-3, 45, 5, 10, 20, 70)
    f.register_sensor(s)
    o = L.create_source("oscillator")
    o.location_grid(20, 21, 20, 21, 30, 31)
    f.register_source(o)
    n = [f.Nx(), f.Ny(), f.Nz()]
    assert n == [40, 40, 60]
    pml, pad = f._finalize(n)
    assert pml == [10, 10, 0, 0, 12, 12]
    assert pad[0] == max(7, 5, 5 + 3, 50 - 20)
    assert pad[1] == max(0, 5, 5 + 45 - 40, 50 + 21 - 40)
    assert pad[2:4] == [0, 0]
    assert pad[4] == max(5, 5 - 20, 50 - 30)
    assert pad[5] == max(5, 5 + 70 - 60, 50 + 31 - 60)


def test_finalize_pads_normal_mode():
    st = L.Structure(lambda s: s.size(40e-9, 40e-9, 200e-9))
    f = L.MODE("fdtd_normal")
    f.structure(st)
    f.pml_xm(10, 25, 1, 0.2)
    f.padding(3, 3, 3, 3, 2, 8)
    pml, pad = f._finalize([f.Nx(), f.Ny(), f.Nz()])
    assert pml == [0, 0, 0, 0, 25, 25]
    assert pad == [0, 0, 0, 0, 5, 8]


def test_mode_settings():
    f = L.MODE("fdtd_normal")
    assert (f.Nt, f.Nl, f.lmin, f.lmax) == (5000, 481, 370e-9, 850e-9)
    f.spectrum(400e-9, 900e-9)
    assert f.Nl == 481
    f.spectrum(400e-9, 900e-9, 51)
    assert (f.lmin, f.lmax, f.Nl) == (400e-9, 900e-9, 51)
    f.polarization("tm")
    assert f.pol == 1
    f.polarization(30)             # an angle runs as TE in both drivers
    assert f.pol == 0
    f.auto_tsteps(20000, 400, 1e-4)
    assert f.cc == ("energy", 400, 1e-4)
    f.auto_tsteps(20000, 400, 500e-9, 800e-9, 1e-3, 200)
    assert f.cc == ("ft", 400, 500e-9, 800e-9, 1e-3, 200, "nnb")
    f.N_tsteps(3000)
    assert f.cc is None and f.Nt == 3000
    m = L.Material()
    m.refractive_index(2.0)
    m.add_lorentz(1.0, 3e15, 1e14)
    d = m.desc()
    assert d.eps_inf == 4.0 and d.n_lorentz == 1 and d.lorentz[0][1] == 3e15
    with pytest.raises(FileNotFoundError):   # a material file is located, then read (tests/test_matlib.py)
        f.material(1, "no_such_material_file.lua")
    with pytest.raises(ValueError):
        L.MODE("fdtd_lab")


def test_loop_sets_periodic_flags():
    st = L.Structure(lambda s: (s.size(1e-7, 1e-7, 1e-7), s.loop(2, 0, -1)))
    assert st.periodic == [1, 0, 1]


# ---- GPU ------------------------------------------------------------------------

def slab(st):
    st.lx, st.ly = 40e-9, 40e-9
    st.lz = st.declare_parameter("h", 200e-9)
    st.default_material(0)
    st.add_layer("Z", 80e-9, 120e-9, 1)


def _slab_mode(precision=A.FP64):
    f = L.MODE("fdtd_normal", precision=precision)
    f.structure(L.Structure(slab))
    f.Dxyz(5e-9)
    f.N_tsteps(900)
    f.time_mod(0.9)
    f.spectrum(450e-9, 900e-9, 31)
    f.polarization("TM")
    f.pml_zm(20, 25, 1, 0.2)
    f.pml_zp(20, 25, 1, 0.2)
    m = L.Material()
    m.refractive_index(1.6)
    f.material(0, L.Material())
    f.material(1, m)
    s = L.create_sensor("planar_spectral_poynting")
    s.location(0, 40e-9, 0, 40e-9, 150e-9, 150e-9)
    s.orientation("Z")
    s.spectrum(450e-9, 900e-9, 31)
    s.name("top")
    f.register_sensor(s)
    return f


@pytest.mark.gpu
def test_normal_mode_compute_matches_reference_core():
    f = _slab_mode()
    sc = f.scene()
    # the layer holds the cell corners z = k*5 nm with 80 nm <= z < 120 nm
    k = np.arange(40) * 5e-9
    want = ((k >= 80e-9) & (k < 120e-9)).astype(np.uint32)
    assert np.array_equal(sc.map[:, 0, 0], want)
    assert list(sc.grid.pad) == [0, 0, 0, 0, 5, 5] and list(sc.grid.pml) == [0, 0, 0, 0, 20, 20]
    out = f.compute()
    which = "ref" if oracle_lib.available("ref") else "port"
    ref = oracle_lib.run(sc, which=which, want_fields=False)
    assert out["steps"] == 900
    rel = np.linalg.norm(out["spectra"] - ref["spectra"]) / np.linalg.norm(ref["spectra"])
    assert rel <= 1e-12
    name, flux = out["sensors"][0]
    assert name == "top"
    assert np.linalg.norm(flux - ref["flux"][0]) <= 1e-12 * np.linalg.norm(ref["flux"][0])


@pytest.mark.gpu
def test_custom_mode_sensors_through_the_front_end():
    """A custom-mode run with an oscillator, a box sensor and a field point:
    compute() returns what the direct API gives on the same scene."""
    from aether_b200 import fdtd as FD

    def cell(st):
        st.size(60e-9, 60e-9, 60e-9)
        st.default_material(0)
        st.add_sphere(30e-9, 30e-9, 30e-9, 12e-9, 1)

    f = L.MODE("fdtd")
    f.structure(L.Structure(cell))
    f.Dxyz(5e-9)
    f.N_tsteps(300)
    for face in (f.pml_xm, f.pml_xp, f.pml_ym, f.pml_yp, f.pml_zm, f.pml_zp):
        face(8, 25, 1, 0.2)
    m = L.Material()
    m.refractive_index(2.0)
    f.material(1, m)
    o = L.create_source("oscillator")
    o.location(30e-9, 30e-9, 10e-9)
    o.orientation("X")
    o.spectrum(400e-9, 800e-9)
    f.register_source(o)
    b = L.create_sensor("box_spectral_poynting")
    b.location(15e-9, 45e-9, 15e-9, 45e-9, 15e-9, 45e-9)
    b.spectrum(400e-9, 800e-9, 11)
    b.name("box")
    f.register_sensor(b)
    p = L.create_sensor("fieldpoint")
    p.location(30e-9, 30e-9, 50e-9)
    p.wavelength(600e-9)
    f.register_sensor(p)
    sc = f.scene()
    # the oscillator sits 2 cells above the structure bottom: 48 pad cells below
    assert sc.grid.pad[4] == 48
    out = f.compute()
    with FD.build_simulation(sc) as sim:
        bid = sim.add_box_sensor(b.to_discrete(5e-9, 5e-9, 5e-9), 11, 400e-9, 800e-9)
        mid = sim.add_fieldmap(A.MAP_POINT, p.to_discrete(5e-9, 5e-9, 5e-9), 600e-9)
        sim.step(300)
        sim.synchronize()
        assert np.array_equal(out["sensors"][0][1], sim.box_flux(bid))
        assert np.array_equal(out["sensors"][1][1], sim.fieldmap(mid))
    assert [n for n, _ in out["sensors"]] == ["box", "sensor"]


@pytest.mark.gpu
def test_oblique_mode_compute_runs_the_kp_sweep():
    from aether_b200 import oblique as OBL

    def film(st):
        st.size(100e-9, 80e-9, 100e-9)
        st.default_material(0)
        st.add_layer("Z", 40e-9, 60e-9, 1)

    f = L.MODE("fdtd_oblique_ARS")
    f.structure(L.Structure(film))
    f.Dxyz(5e-9)
    f.N_tsteps(400)
    f.spectrum(500e-9, 900e-9, 11)
    f.pml_zm(12, 25, 1, 0.2)
    f.pml_zp(12, 25, 1, 0.2)
    m = L.Material()
    m.refractive_index(1.5)
    f.material(1, m)
    f.kp_target(600e-9, 20)
    f.incident_plane(30)
    out = f.compute()
    kp = 2 * np.pi / 600e-9 * np.sin(np.deg2rad(20))
    assert np.isclose(out["kp"][0], kp, rtol=1e-15)
    direct = OBL.sweep(f.scene(), [kp], phi_deg=30)
    assert np.array_equal(out["obl"][0], direct[0])


@pytest.mark.gpu
@pytest.mark.skipif(not oracle_lib.available("ref"), reason="reference build absent")
def test_structure_script_with_every_kind_matches_reference():
    """A structure script using the primitives, coatings, loop and flip
    through the front end, against the reference's own Structure."""
    def script(st):
        st.size(80e-9, 60e-9, 70e-9)
        st.default_material(0)
        st.loop(1, 0, 0)
        st.flip(0, 1, 0)
        st.add_layer("Z", 0, 15e-9, 1)
        st.add_cone(40e-9, 30e-9, 15e-9, 0, 0, 40e-9, 20e-9, 2)
        st.add_ellipsoid(10e-9, 45e-9, 30e-9, 12e-9, 8e-9, 10e-9, 3)
        st.add_sin_layer(50e-9, 4e-9, 58e-9, -3e-9, 40e-9, 0.1, 0, 0, 4)
        st.add_vect_tri(55e-9, 5e-9, 20e-9, 20e-9, 0, 0, 0, 20e-9, 0, 0, 0, 25e-9, 0.3, 5)
        st.add_conformal_coating(5e-9, 2.5e-9, 0, 6)

    st = L.Structure(script)
    d = (2.5e-9,) * 3
    gpu = st.discretize(32, 24, 28, *d)
    desc = A.structure_desc(st.default, st.periodic, st.flips, (st.lx, st.ly, st.lz))
    ref = oracle_lib.ref_discretize(32, 24, 28, d, st.ops, desc)
    assert np.array_equal(gpu, ref)
    assert set(np.unique(ref)) >= {0, 1, 2, 3, 6}


@pytest.mark.skipif(not oracle_lib.available("ref"), reason="reference build absent")
@pytest.mark.parametrize("case", [(200e-9, 200e-9, 20e-9, 12, 5), (300e-9, 250e-9, 15e-9, 30, 9)])
def test_random_packing_matches_reference(case):
    """The structure scripts' random_packing against the reference's own
    (phys_tools.cpp) compiled in the oracle build: same seeded draws, same
    relaxation, bit-identical positions."""
    import ctypes as C
    x_max, y_max, r, n, seed = case
    lib = C.CDLL(oracle_lib.REF_PATH)
    f = lib.aeref_random_packing
    f.argtypes = [C.c_double] * 3 + [C.c_int32] * 2 + [C.POINTER(C.c_double)] * 2
    x, y = np.zeros(n), np.zeros(n)
    assert f(x_max, y_max, r, n, seed, x.ctypes.data_as(C.POINTER(C.c_double)),
             y.ctypes.data_as(C.POINTER(C.c_double))) == 0
    px, py = L.random_packing(x_max, y_max, r, n, seed)
    assert np.array_equal(x, px) and np.array_equal(y, py)
    # the discs end up apart: no pair (with periodic images) closer than 1.5 r
    for i in range(n):
        for j in range(i + 1, n):
            ddx = min(abs(px[i] - px[j]), x_max - abs(px[i] - px[j]))
            ddy = min(abs(py[i] - py[j]), y_max - abs(py[i] - py[j]))
            assert (ddx * ddx + ddy * ddy) ** 0.5 > 1.5 * r


def test_mersenne_twister_known_answer():
    # std::mt19937 with the default seed 5489: its 10000th output is 4123659995 (C++ [rand.predef])
    g = L._MT19937(5489)
    for _ in range(9999):
        g()
    assert g() == 4123659995
