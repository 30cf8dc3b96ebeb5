"""Parity at the benchmark configurations' own sizes and shapes.

Each case runs the FP64 GPU path through the C ABI and the reference's own
FDTD core compiled from source (oracle/_ref) on the same seeded scene:
fields must be bit-identical (SHA-256 per component), plane sums within
1e-12 and flux spectra within 1e-10 relative (device reduction order only).

  * the dispersive unit cell at its full 128 x 128 x 256 size (gold-like
    Drude + 2 critical-point sphere, 24-cell CPML, two 201-wavelength DFT
    planes), 200 steps;
  * the large random grid's scene at 256 x 256 x 128 (32-cell CPML on all six
    faces, dielectric spheres with their own indices, Lorentz spheres sharing
    one index, a point oscillator), 128 steps: the field front reaches every
    CPML face and most spheres;
  * two nanodisk metasurface cells at their real size (one gold, one
    dielectric), alone with flux planes, then both inside one batch;
  * CPML grading order 3 (the slab workload's stated grading): outside what
    the reference can run (it fixes m = 4, fdtd_pml.cpp:309-310), so checked
    against the CPU restatement, which takes the order as a parameter."""
import hashlib

import numpy as np
import pytest

import oracle_lib
from aether_b200 import _abi as A
from aether_b200 import configs as CF
from aether_b200 import fdtd

pytestmark = pytest.mark.gpu

RTOL_PLANE = 1e-12
RTOL_FLUX = 1e-10
NM = 1e-9


def sha(f):
    f = np.ascontiguousarray(f, dtype=np.float64)
    return [hashlib.sha256(f[c].tobytes()).hexdigest() for c in range(f.shape[0])]


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def need_ref():
    if not oracle_lib.available("ref"):
        pytest.skip("reference core not built (oracle/Makefile ref)")


def check(got, ref):
    assert np.array_equal(got["dims"], ref["dims"])
    assert sha(got["fields"]) == sha(ref["fields"]), "FP64 fields differ from the reference core"
    assert np.count_nonzero(ref["fields"]) > 0
    if ref["plane_sums"] is not None:
        assert rel(got["plane_sums"], ref["plane_sums"]) < RTOL_PLANE
    for a, b in zip(got["flux"], ref["flux"]):
        assert rel(a, b) < RTOL_FLUX


def test_dispersive_cell_full_size_200_steps():
    need_ref()
    sc = CF.sphere_scene(nx=128, ny=128, nz_total=256, dx=2.5 * NM, pml=24, radius=40 * NM, nsteps=20000,
                         nl=201, precision=A.FP64)
    ref = oracle_lib.run(sc, "ref", nsteps=200)
    got = fdtd.run(sc, nsteps=200)
    check(got, ref)


def test_large_grid_scene_256x256x128_128_steps():
    need_ref()
    # the large grid's densities (500 + 50 spheres in 1024 x 1024 x 512) scaled
    # to a 64x smaller grid, rounded up so that several spheres of each kind
    # exist and the Lorentz spheres share one material index and bounding box
    sc = CF.random_spheres_scene(n_total=(256, 256, 128), n_dielectric=12, n_lorentz=3, nsteps=5000,
                                 seed=1234, precision=A.FP64)
    assert sc.total_dims() == (256, 256, 128)
    ref = oracle_lib.run(sc, "ref", nsteps=128)
    got = fdtd.run(sc, nsteps=128)
    check(got, ref)
    # the front has reached every CPML face
    f = np.abs(ref["fields"]).sum(axis=0)
    assert f[:, :, :32].any() and f[:, :, -32:].any() and f[:, :32].any() and f[:, -32:].any()
    assert f[:32].any() and f[-32:].any()


def nanodisk_pair(flux_planes, nsteps):
    """The first gold and the first dielectric cell of a seeded draw from the
    metasurface distribution (period U(200, 600) nm at 5 nm, z = 200, 16-cell
    CPML), periods capped at 90 cells to bound the reference's time."""
    rng = np.random.default_rng(4242)
    got = {}
    while len(got) < 2:
        state = rng.bit_generator.state
        sc = CF.metasurface_cell(rng, precision=A.FP64, nsteps=nsteps, nl=51, flux_planes=flux_planes)
        gold = sc.materials[1].n_drude > 0
        if sc.grid.nx <= 90 and gold not in got:
            got[gold] = state
    out = []
    for gold in (True, False):
        r = np.random.default_rng()
        r.bit_generator.state = got[gold]
        out.append(CF.metasurface_cell(r, precision=A.FP64, nsteps=nsteps, nl=51, flux_planes=flux_planes))
    return out


def test_nanodisk_cells_alone_and_batched():
    need_ref()
    steps = 400
    with_planes = nanodisk_pair(True, steps)
    without = nanodisk_pair(False, steps)
    refs = []
    for sc in with_planes:
        ref = oracle_lib.run(sc, "ref", nsteps=steps)
        got = fdtd.run(sc, nsteps=steps)
        check(got, ref)
        refs.append(ref)
    # the same cells (without DFT planes, which batch members do not carry) in one batch
    sims = [fdtd.build_simulation(sc) for sc in without]
    try:
        with fdtd.Batch() as b:
            for s in sims:
                b.add(s, steps)
            assert b.run(10 ** 6) == steps
            for s, ref in zip(sims, refs):
                assert sha(s.fields()) == sha(ref["fields"])
                assert rel(s.plane_sums(), ref["plane_sums"]) < RTOL_PLANE
    finally:
        for s in sims:
            s.close()


def test_cpml_grading_order_3_against_restatement():
    sc = CF.slab_scene(precision=A.FP64, nsteps=600)
    sc.grid.pml_m = 3
    port = oracle_lib.run(sc, "port")
    got = fdtd.run(sc)
    assert sha(got["fields"]) == sha(port["fields"])
    assert rel(got["plane_sums"], port["plane_sums"]) < RTOL_PLANE
    for a, b in zip(got["flux"], port["flux"]):
        assert rel(a, b) < RTOL_FLUX
    # the order took effect: order 4 gives other fields
    sc.grid.pml_m = 4
    port4 = oracle_lib.run(sc, "port")
    assert sha(port4["fields"]) != sha(port["fields"])
