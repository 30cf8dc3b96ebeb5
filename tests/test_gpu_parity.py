"""GPU parity: the CUDA library (through its C ABI) against the reference.

FP64 path: fields bit-identical to the reference core (SHA-256 of the golden
fixtures, which come from the reference compiled from source) and to the CPU
restatement; plane sums, R/T spectra and flux spectra within the relative
tolerances below (they differ only by device reduction order and 1-ulp
phasors). FP32 path: R/T and flux spectra within 1e-4 absolute of the FP64
reference (relative for flux), fields within relative L2 1e-3."""
import hashlib
import os

import numpy as np
import pytest

import oracle_lib
import scenes
from aether_b200 import _abi as A
from aether_b200 import configs as CF
from aether_b200 import fdtd

pytestmark = pytest.mark.gpu

GOLDEN_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
GOLDEN = ["slab_tm", "slab_te", "gold_sphere", "debye_lorentz_sphere", "custom_box", "thin_column"]

RTOL_PLANE = 1e-12      # plane sums: reduction order only
RTOL_SPECTRA = 1e-10    # R/T spectra (ratios of DFTs of the plane sums)
RTOL_FLUX = 1e-10       # flux spectra: DFT block sums + reduction order
FP32_ABS_RT = 1e-4      # FP32 R/T vs FP64 oracle, absolute
FP32_REL_FIELD = 1e-3   # FP32 fields, relative L2


def sha(fields):
    f = np.ascontiguousarray(fields, dtype=np.float64)
    return [hashlib.sha256(f[c].tobytes()).hexdigest() for c in range(6)]


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("name", GOLDEN)
def test_fp64_bit_identical_to_reference_golden(name):
    g = np.load(os.path.join(GOLDEN_DIR, f"{name}.npz"))
    r = fdtd.run(scenes.ALL[name]())
    assert np.array_equal(r["dims"], g["dims"])
    assert sha(r["fields"]) == list(g["field_sha256"]), "FP64 fields differ from the reference core"
    if "plane_sums" in g:
        assert rel(r["plane_sums"], g["plane_sums"]) < RTOL_PLANE
        assert rel(r["spectra"], g["spectra"]) < RTOL_SPECTRA
    for i, f in enumerate(r["flux"]):
        assert rel(f, g[f"flux{i}"]) < RTOL_FLUX, (i, f, g[f"flux{i}"])
    assert r["launches"] > 0


def test_fp64_many_materials_uint16_ids():
    sc = scenes.custom_many_materials(nsteps=60)
    assert sc.map.max() > 255
    a = oracle_lib.run(sc, "port")
    b = fdtd.run(sc)
    assert np.array_equal(a["fields"], b["fields"])


def test_fp64_exact_dft_with_one_step_blocks():
    sc = scenes.gold_sphere(nsteps=200)
    sc.grid.dft_block = 1
    a = oracle_lib.run(sc, "port")
    b = fdtd.run(sc)
    for fa, fb in zip(a["flux"], b["flux"]):
        assert rel(fb, fa) < 1e-12


@pytest.mark.parametrize("block", [7, 64])
def test_fp64_dft_block_sizes_agree(block):
    sc = scenes.slab_tm(nsteps=150)
    sc.grid.dft_block = block
    a = oracle_lib.run(sc, "port")
    b = fdtd.run(sc)
    for fa, fb in zip(a["flux"], b["flux"]):
        assert rel(fb, fa) < RTOL_FLUX


def test_fp64_step_in_pieces_equals_one_call():
    sc = scenes.gold_sphere(nsteps=90)
    with fdtd.build_simulation(sc) as s1, fdtd.build_simulation(sc) as s2:
        s1.step(90)
        for n in (1, 10, 33, 46):
            s2.step(n)
        assert np.array_equal(s1.fields(), s2.fields())
        assert np.array_equal(s1.plane_sums(), s2.plane_sums())
        for i in range(2):
            assert np.array_equal(s1.sensor_flux(i), s2.sensor_flux(i))


@pytest.mark.parametrize("prec", [A.FP64, A.FP32])
def test_reading_sensors_mid_run_then_continuing(prec):
    """Flux read after 150 of 330 steps (accumulating the pending and partial
    DFT blocks), then 180 more steps: the final flux equals an uninterrupted
    run up to the regrouping of the block sums (1e-10 relative in FP64, 1e-6
    in FP32), and the fields are unchanged bit for bit."""
    sc = scenes.gold_sphere(precision=prec, nsteps=330)
    with fdtd.build_simulation(sc) as s1, fdtd.build_simulation(sc) as s2:
        s1.step(330)
        s2.step(150)
        mid = [s2.sensor_flux(i) for i in range(2)]
        s2.step(180)
        assert np.array_equal(s1.fields(), s2.fields())
        tol = RTOL_FLUX if prec == A.FP64 else 1e-6
        for i in range(2):
            assert rel(s2.sensor_flux(i), s1.sensor_flux(i)) < tol
            assert np.all(np.isfinite(mid[i]))


def test_reset_restarts_bitwise():
    sc = scenes.slab_te(nsteps=60)
    with fdtd.build_simulation(sc) as s:
        s.step(60)
        f1 = s.fields()
        s.reset()
        s.step(60)
        assert np.array_equal(f1, s.fields())


@pytest.mark.parametrize("name", ["slab_tm", "gold_sphere", "debye_lorentz_sphere"])
def test_fp32_spectra_close_to_fp64_oracle(name):
    sc64 = scenes.ALL[name](nsteps=400)
    sc32 = scenes.ALL[name](precision=A.FP32, nsteps=400)
    a = oracle_lib.run(sc64, "port")
    b = fdtd.run(sc32)
    assert rel(b["fields"], a["fields"]) < FP32_REL_FIELD
    # columns 1, 2: |r|, |t| amplitude ratios (spectdata_norm)
    assert np.max(np.abs(b["spectra"][:, 1:3] - a["spectra"][:, 1:3])) < FP32_ABS_RT
    for fa, fb in zip(a["flux"], b["flux"]):
        assert np.max(np.abs(fb - fa)) <= 1e-3 * np.max(np.abs(fa)) + 1e-300


def test_fp32_custom_mode_close_to_fp64_oracle():
    a = oracle_lib.run(scenes.custom_box(nsteps=100), "port")
    b = fdtd.run(scenes.custom_box(precision=A.FP32, nsteps=100))
    assert rel(b["fields"], a["fields"]) < FP32_REL_FIELD


@pytest.mark.parametrize("prec", [A.FP64, A.FP32])
def test_interior_and_boundary_kernels_agree(prec, monkeypatch):
    """Items run by the curl-only interior kernels give the same cells as the
    full kernels: bit-identical in FP64, 1e-6 relative in FP32."""
    monkeypatch.setenv("AEFDTD_FUSED", "0")   # the split half-step kernels (the fused ones: test_fused.py)
    sc = scenes.gold_sphere(precision=prec, nsteps=80)
    a = fdtd.run(sc)
    monkeypatch.setenv("AEFDTD_ALL_BOUNDARY", "1")
    b = fdtd.run(sc)
    if prec == A.FP64:
        assert np.array_equal(a["fields"], b["fields"])
    else:
        assert rel(a["fields"], b["fields"]) < 1e-6


@pytest.mark.parametrize("name", ["gold_sphere", "custom_box"])
def test_concurrent_groups_match_serial_groups(name, monkeypatch):
    """Boundary groups on side streams (parallel graph branches) against all
    groups launched in order on one stream: bit-identical."""
    sc = getattr(scenes, name)(nsteps=90)
    a = fdtd.run(sc)
    monkeypatch.setenv("AEFDTD_SERIAL_GROUPS", "1")
    b = fdtd.run(sc)
    assert np.array_equal(a["fields"], b["fields"])
    for fa, fb in zip(a["flux"], b["flux"]):
        assert np.array_equal(fa, fb)


@pytest.mark.parametrize("kchunk,zunroll", [("1", "2"), ("3", "2"), ("3", "1"), ("1000", "1"), ("1000", "2")])
def test_z_chunking_does_not_change_results(kchunk, zunroll, monkeypatch):
    """Planes per work item and planes per interior-kernel iteration (odd
    chunks leave a one-plane tail in the two-plane loop) change no bit."""
    monkeypatch.setenv("AEFDTD_FUSED", "0")   # the split half-step kernels' items
    sc = scenes.custom_box(nsteps=40)
    a = fdtd.run(sc)
    monkeypatch.setenv("AEFDTD_KCHUNK", kchunk)
    monkeypatch.setenv("AEFDTD_ZUNROLL", zunroll)
    b = fdtd.run(sc)
    assert np.array_equal(a["fields"], b["fields"])


def _wide_cell(n, precision, nsteps=120):
    """A periodic nanodisk cell n x n (ragged against 64-column items when n
    is not a multiple of 64) with z CPML and, by the seed, a Drude-Lorentz disk."""
    rng = np.random.default_rng(5)
    return CF.metasurface_cell(rng, nz_total=64, pml=8, nsteps=nsteps, nl=9, precision=precision,
                               period_range=(n * 5e-9, n * 5e-9))


@pytest.mark.parametrize("name,mask", [("slab_tm", "3"), ("gold_sphere", "3"), ("custom_box", "3"),
                                       ("wide130", "3"), ("wide130", "1"), ("wide130", "2"), ("wide192", "3"),
                                       ("wide129", "3")])
def test_two_cells_per_thread_bit_identical(name, mask, monkeypatch):
    """Interior and z-CPML kernels moving two x cells per thread (64-column
    items, pair loads, lane shuffles for the x neighbour, 32-column half items
    beside other groups) against one cell per thread: FP64 fields, plane sums
    and flux bit-identical, including the periodic x wrap, ragged last items
    and odd Nx (which keeps one cell per thread)."""
    sc = _wide_cell(int(name[4:]), A.FP64) if name.startswith("wide") else getattr(scenes, name)(nsteps=120)
    monkeypatch.setenv("AEFDTD_FUSED", "0")   # the split half-step kernels
    monkeypatch.setenv("AEFDTD_PAIR", "0")
    a = fdtd.run(sc)
    monkeypatch.setenv("AEFDTD_PAIR", mask)
    b = fdtd.run(sc)
    assert np.array_equal(a["fields"], b["fields"])
    assert np.array_equal(a["plane_sums"], b["plane_sums"])
    for fa, fb in zip(a["flux"], b["flux"]):
        assert np.array_equal(fa, fb)


def test_two_cells_per_thread_fp32_and_cell_cover(monkeypatch):
    """FP32 pair kernels within 1e-6 relative of one cell per thread, and the
    64- and 32-column items of each half-step still cover every cell once."""
    sc = _wide_cell(130, A.FP32, nsteps=100)
    monkeypatch.setenv("AEFDTD_FUSED", "0")   # the split half-step kernels
    monkeypatch.setenv("AEFDTD_PAIR", "0")
    a = fdtd.run(sc)
    monkeypatch.setenv("AEFDTD_PAIR", "3")
    with fdtd.build_simulation(sc) as s:
        s.enable_timing(True, mode=2)
        s.step(100)
        assert rel(s.fields(), a["fields"]) < 1e-6
        g = s.group_timings()
        d = s.dims()
        for half in "EH":
            assert sum(c for (h, _), (ms, c) in g.items() if h == half) == d.nx * d.ny * d.nz
        assert g[("E", "interior")][1] > 0 and g[("E", "pml_z")][1] > 0


def test_graph_replay_matches_direct_launches(monkeypatch):
    """Whole 64-step segments replayed from CUDA graphs (default) against the
    same steps launched one by one."""
    sc = scenes.gold_sphere(nsteps=200)
    a = fdtd.run(sc)
    monkeypatch.setenv("AEFDTD_NO_GRAPHS", "1")
    b = fdtd.run(sc)
    assert np.array_equal(a["fields"], b["fields"])
    assert np.array_equal(a["plane_sums"], b["plane_sums"])
    for fa, fb in zip(a["flux"], b["flux"]):
        assert np.array_equal(fa, fb)
    assert a["launches"] == b["launches"]


def test_timing_mode_does_not_change_results():
    sc = scenes.slab_tm(nsteps=100)
    with fdtd.build_simulation(sc) as s1, fdtd.build_simulation(sc) as s2:
        s1.step(100)
        s2.enable_timing(True)
        s2.step(100)
        e, h, s = s2.timings()
        assert e > 0 and h > 0 and s >= 0
        assert np.array_equal(s1.fields(), s2.fields())


def test_group_timing_mode_covers_every_cell_once(monkeypatch):
    """Mode-2 timing runs each group alone between events: same fields, and
    the groups of each half-step cover every cell of the grid once (split
    half-step kernels; the fused groups: test_fused.py)."""
    monkeypatch.setenv("AEFDTD_FUSED", "0")
    sc = scenes.gold_sphere(nsteps=70)
    with fdtd.build_simulation(sc) as s1, fdtd.build_simulation(sc) as s2:
        s1.step(70)
        s2.enable_timing(True, mode=2)
        s2.step(70)
        assert np.array_equal(s1.fields(), s2.fields())
        g = s2.group_timings()
        d = s2.dims()
        for half in "EH":
            cells = sum(c for (h, _), (ms, c) in g.items() if h == half)
            assert cells == d.nx * d.ny * d.nz
        assert g[("E", "interior")][0] > 0 and g[("E", "dispersive")][1] > 0


def test_fp32_tensor_core_dft_matches_simt_dft(monkeypatch):
    """FP32 path: the DFT blocks on the tensor cores (tcgen05, 3xTF32) against
    the FP64 SIMT accumulation of the same samples."""
    sc = scenes.gold_sphere(precision=A.FP32, nsteps=192)
    a = fdtd.run(sc, want_fields=False)
    monkeypatch.setenv("AEFDTD_NO_TC", "1")
    b = fdtd.run(sc, want_fields=False)
    for fa, fb in zip(a["flux"], b["flux"]):
        assert np.max(np.abs(fa - fb)) <= 1e-5 * np.max(np.abs(fb))


def test_fp64_mma_dft_matches_fma_dft(monkeypatch):
    """FP64 path: DFT blocks on the FP64 tensor path (mma.sync f64, the
    default) against the FMA kernel on the same samples: accumulators within
    1e-13 of their magnitude (only the order of the sums within four steps
    differs); 201 wavelengths (a partial last wavelength tile) and 150 steps
    (a partial last block)."""
    sc = scenes.slab_tm(nsteps=150)
    for s in sc.sensors:
        s.nl = 201

    def dft(env):
        monkeypatch.setenv("AEFDTD_DFT_MMA", env)
        with fdtd.build_simulation(sc) as sim:
            sim.step(150)
            sim.synchronize()
            return [sim.sensor_dft(i) for i in range(len(sc.sensors))], [sim.sensor_flux(i) for i in range(len(sc.sensors))]

    (da, fa), (db, fb) = dft("1"), dft("0")
    for x, y in zip(da, db):
        assert np.count_nonzero(y) > 0
        assert np.max(np.abs(x - y)) <= 1e-13 * np.max(np.abs(y))
    for x, y in zip(fa, fb):
        assert np.max(np.abs(x - y)) <= 1e-12 * np.max(np.abs(y))


def test_fp32_tensor_core_dft_many_wavelengths():
    """Two N tiles (2 nl > 256 columns) and a partial last block."""
    sc64 = scenes.slab_tm(nsteps=150)
    sc32 = scenes.slab_tm(precision=A.FP32, nsteps=150)
    for s in sc64.sensors + sc32.sensors:
        s.nl = 201
    a = oracle_lib.run(sc64, "port", want_fields=False)
    b = fdtd.run(sc32, want_fields=False)
    for fa, fb in zip(a["flux"], b["flux"]):
        assert np.max(np.abs(fb - fa)) <= 2e-3 * np.max(np.abs(fa))


def test_cpp_shim_matches_python_path():
    """The FDTD-named C++ shim (include/aefdtd.hpp) and the ctypes path give
    the same fields bit for bit (sequential sum of Ex^2 after 60 steps)."""
    import subprocess
    import tempfile
    import test_abi
    with tempfile.TemporaryDirectory() as d:
        exe = test_abi.build_shim_program(d)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()
    assert out[0] == "ok" and int(out[1]) == 60, out
    r = fdtd.run(test_abi.shim_scene(), 60)
    s = 0.0
    for v in r["fields"][0].ravel():
        s += float(v) * float(v)
    assert s == float(out[2]) and s > 0
