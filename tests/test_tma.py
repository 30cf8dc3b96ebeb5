"""Staged interior half-steps (AEFDTD_TMA=1): curl-only and z-CPML 64 x 8
tiles whose planes reach shared memory through tensor copies
(interior_tma.cuh); every scene below has z-CPML planes in its staged tiles.

FP64: fields, plane sums and flux bit-identical to the one-cell kernels
(AEFDTD_TMA=0) on every tile situation the staged kernels meet: both periodic
wraps inside one tile (64 x 8 grid), the x wrap of the first tile (E) and of
the last (H), grids whose width or height leaves columns and rows to the
other kernels, CPML on every face, dispersive spheres, 16-bit material ids,
unit lengths from one plane to whole runs, steps in pieces (captured graphs
and direct launches); and SHA-identical to the reference core compiled from
source on the dispersive unit cell at its full 128 x 128 x 256 size.
FP32: fields within 1e-5 relative of the one-cell kernels (contraction may
differ)."""
import hashlib
import os

import numpy as np
import pytest

import oracle_lib
from aether_b200 import _abi as A
from aether_b200 import _lib
from aether_b200 import configs as CF
from aether_b200 import fdtd
from aether_b200._lib import AefdtdError

pytestmark = pytest.mark.gpu

NM = 1e-9


def sha(f):
    f = np.ascontiguousarray(f, dtype=np.float64)
    return [hashlib.sha256(f[c].tobytes()).hexdigest() for c in range(f.shape[0])]


def run(scene, pieces, tma, env=None):
    env = dict(env or {})
    env["AEFDTD_TMA"] = "1" if tma else "0"
    env.setdefault("AEFDTD_FUSED", "0")
    saved = {k: os.environ.get(k) for k in env}
    os.environ.update(env)
    try:
        with fdtd.build_simulation(scene) as s:
            for n in pieces:
                s.step(n)
            s.synchronize()
            out = {"fields": s.fields(), "flux": [s.sensor_flux(i) for i in range(len(scene.sensors))],
                   "groups": s.group_timings(), "dims": s.dims()}
            if scene.grid.mode == A.MODE_NORMAL:
                out["plane_sums"] = s.plane_sums()
            return out
    finally:
        for k, v in saved.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v


SCENES = {
    # one 64 x 8 tile: E and H x wraps and both y wraps in the same tile
    "single_tile": lambda p: CF.sphere_scene(nx=64, ny=8, nz_total=80, dx=2.5e-9, pml=8, radius=3e-9, nsteps=120,
                                             nl=5, sensor_gap=4, precision=p),
    # two tiles across: E wraps in the first, H in the second
    "cell128": lambda p: CF.sphere_scene(nx=128, ny=32, nz_total=96, dx=2.5e-9, pml=8, radius=25e-9, nsteps=120,
                                         nl=5, sensor_gap=4, precision=p),
    # columns 128, 129 and rows 64..69 outside every staged tile
    "wide_sphere": lambda p: CF.sphere_scene(nx=130, ny=70, nz_total=96, dx=2.5e-9, pml=8, radius=30e-9, nsteps=120,
                                             nl=5, sensor_gap=4, precision=p),
    # width not a multiple of 64, custom mode, CPML on all six faces
    "custom_pml6": lambda p: CF.random_spheres_scene(n_total=(150, 40, 48), pml=8, n_dielectric=10, n_lorentz=3,
                                                     r_range=(8e-9, 20e-9), nsteps=80, nl=5, precision=p, seed=11),
    # more than 256 materials: 16-bit material ids (x tiles 64..191 clear of the CPML)
    "ids16": lambda p: CF.random_spheres_scene(n_total=(200, 48, 40), pml=6, n_dielectric=300, n_lorentz=2,
                                               r_range=(3e-9, 8e-9), nsteps=60, nl=5, precision=p, seed=3),
}


def test_scenes_reach_the_staged_kernels():
    """Every scene has tiles for the staged kernels, the interior group then
    holds whole 64 x 8 tile-planes, and every cell is updated by exactly one
    group in each half-step (so the checks below are not vacuous)."""
    for name, make in SCENES.items():
        sc = make(A.FP64)
        nx, ny, _ = sc.total_dims()
        assert nx >= 64 and ny >= 8 and nx % 2 == 0, name
        out = run(sc, [2], tma=True)
        d = out["dims"]
        for h in "EH":
            cells = {g: c for (hh, g), (_, c) in out["groups"].items() if hh == h}
            assert sum(cells.values()) == d.nx * d.ny * d.nz, (name, h, cells)
            assert cells["interior"] > 0 and cells["interior"] % (64 * 8) == 0, (name, h, cells)
    assert max(m.n_drude for m in SCENES["cell128"](A.FP64).materials) > 0
    assert len(SCENES["ids16"](A.FP64).materials) > 256


@pytest.mark.parametrize("name", sorted(SCENES))
def test_tma_fp64_bit_identical(name):
    sc = SCENES[name](A.FP64)
    pieces = [37, 64, 19]
    a = run(sc, pieces, tma=True)
    b = run(sc, pieces, tma=False)
    assert sha(a["fields"]) == sha(b["fields"])
    assert np.count_nonzero(b["fields"]) > 0
    if "plane_sums" in b:
        assert np.array_equal(a["plane_sums"], b["plane_sums"])
    for x, y in zip(a["flux"], b["flux"]):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("env", [{"AEFDTD_TMA_UNIT": "1"}, {"AEFDTD_TMA_UNIT": "3"}, {"AEFDTD_TMA_UNIT": "4096"},
                                 {"AEFDTD_NO_GRAPHS": "1"}, {"AEFDTD_SERIAL_GROUPS": "1"}, {"AEFDTD_TILE_Y": "2"},
                                 {"AEFDTD_TILE_Y": "8"}])
def test_tma_layouts_no_bit(env):
    """Unit lengths, direct launches, serial groups and tile heights: same bits."""
    sc = SCENES["cell128"](A.FP64)
    a = run(sc, [sc.nsteps], tma=True, env=env)
    b = run(sc, [sc.nsteps], tma=False)
    assert sha(a["fields"]) == sha(b["fields"])


@pytest.mark.parametrize("name", ["cell128", "custom_pml6"])
def test_tma_fp32_close(name):
    sc = SCENES[name](A.FP32)
    a = run(sc, [sc.nsteps], tma=True)
    b = run(sc, [sc.nsteps], tma=False)
    d = np.linalg.norm(a["fields"] - b["fields"]) / np.linalg.norm(b["fields"])
    assert d < 1e-5, d


def test_tma_fp64_full_cell_matches_reference_core():
    """The dispersive unit cell at 128 x 128 x 256 (gold Drude + 2 critical
    points, 24-cell CPML, two 201-wavelength planes), 200 steps."""
    if not oracle_lib.available("ref"):
        pytest.skip("reference core not built")
    sc = CF.sphere_scene(nx=128, ny=128, nz_total=256, dx=2.5 * NM, pml=24, radius=40 * NM, nsteps=20000, nl=201,
                         precision=A.FP64)
    ref = oracle_lib.run(sc, "ref", nsteps=200)
    got = run(sc, [200], tma=True)
    assert sha(got["fields"]) == sha(ref["fields"])


STAGED_WAIT, STAGED_WITHHOLD = 3, 4   # AEFDTD_TEST_STAGED_WAIT_CYCLES, AEFDTD_TEST_STAGED_WITHHOLD_COPY
TIMEOUT = 3


def test_staged_wait_runs_out_then_handle_recovers():
    """Bounded waits of the staged kernels: the test hook withholds every
    tensor copy (and the stage arrives), so the consumers' first wait runs
    out after 2^20 cycles; each CTA raises its abort flag and the error flag,
    and the step's synchronising call returns AEFDTD_TIMEOUT with no GPU
    fault. After the hook is cleared and the handle reset, a run gives the
    fields of a fresh handle bit for bit (the unit counters were cleared)."""
    sc = SCENES["cell128"](A.FP64)
    want = run(sc, [64], tma=True)
    lib = _lib.load()
    saved = {k: os.environ.get(k) for k in ("AEFDTD_TMA", "AEFDTD_FUSED")}
    os.environ.update({"AEFDTD_TMA": "1", "AEFDTD_FUSED": "0"})
    try:
        s = fdtd.build_simulation(sc)
    finally:
        for k, v in saved.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    with s:
        _lib.check(lib.aefdtd_test_hook(s._h, STAGED_WAIT, 1 << 20))
        _lib.check(lib.aefdtd_test_hook(s._h, STAGED_WITHHOLD, 1))
        with pytest.raises(AefdtdError) as e:
            s.step(64)
            s.synchronize()
        assert e.value.status == TIMEOUT
        s.synchronize()   # the flag was read and cleared
        _lib.check(lib.aefdtd_test_hook(s._h, STAGED_WITHHOLD, 0))
        _lib.check(lib.aefdtd_test_hook(s._h, STAGED_WAIT, 1 << 32))
        s.reset()
        s.step(64)
        s.synchronize()
        assert sha(s.fields()) == sha(want["fields"])
