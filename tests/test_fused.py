"""The fused time step (one launch per step and feature group, ping-pong
buffers) against the split half-step kernels and the reference.

FP64: fields, plane sums and flux bit-identical to the split path on every
scene shape (normal and custom mode, CPML on z or on all faces, dispersive
spheres, 16-bit material ids, grids narrower than a fused tile, odd Nx down
to a single column, odd step counts that leave the current state in the
second buffer set, steps in pieces); and fields SHA-identical to the reference core compiled from source.
FP32: fields within 1e-5 relative of the split path (contraction may differ)."""
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


def sha(f):
    f = np.ascontiguousarray(f, dtype=np.float64)
    return [hashlib.sha256(f[c].tobytes()).hexdigest() for c in range(f.shape[0])]


def run(scene, pieces, fused):
    old = os.environ.get("AEFDTD_FUSED")
    os.environ["AEFDTD_FUSED"] = "1" if fused else "0"
    try:
        with fdtd.build_simulation(scene) as s:
            for n in pieces:
                s.step(n)
            s.synchronize()
            out = {"fields": s.fields(), "flux": [s.sensor_flux(i) for i in range(len(scene.sensors))]}
            if scene.grid.mode == A.MODE_NORMAL:
                out["plane_sums"] = s.plane_sums()
            return out
    finally:
        if old is None:
            os.environ.pop("AEFDTD_FUSED", None)
        else:
            os.environ["AEFDTD_FUSED"] = old


SCENES = {
    "slab_tm": lambda p: scenes.slab_tm(precision=p, nsteps=150),
    "gold_sphere": lambda p: scenes.gold_sphere(precision=p, nsteps=150),
    "debye_lorentz_sphere": lambda p: scenes.debye_lorentz_sphere(precision=p, nsteps=150),
    "custom_box": lambda p: scenes.custom_box(precision=p, nsteps=90),
    "custom_many_materials": lambda p: scenes.custom_many_materials(precision=p, nsteps=60),
    "wide_sphere": lambda p: CF.sphere_scene(nx=130, ny=70, nz_total=96, dx=2.5e-9, pml=8, radius=30e-9, nsteps=120,
                                             nl=5, sensor_gap=4, precision=p),
    # odd Nx: per-cell loads, and the last tile's odd width (recomputed next column in its last lane)
    "odd_sphere": lambda p: CF.sphere_scene(nx=67, ny=21, nz_total=80, dx=2.5e-9, pml=8, radius=20e-9, nsteps=100,
                                            nl=5, sensor_gap=4, precision=p),
    "odd_custom": lambda p: CF.random_spheres_scene(n_total=(71, 40, 44), pml=6, n_dielectric=8, n_lorentz=3,
                                                    r_range=(10e-9, 30e-9), nsteps=70, nl=5, precision=p, seed=9),
    "thin_column": lambda p: scenes.thin_column(precision=p, nsteps=120),
}


@pytest.mark.parametrize("name", sorted(SCENES))
def test_fused_fp64_bit_identical_to_split(name):
    sc = SCENES[name](A.FP64)
    pieces = [37, 64, 19]   # odd pieces: the current set moves between the two buffer sets
    a = run(sc, pieces, fused=True)
    b = run(sc, pieces, fused=False)
    assert sha(a["fields"]) == sha(b["fields"])
    if "plane_sums" in b:
        assert np.array_equal(a["plane_sums"], b["plane_sums"])
    for x, y in zip(a["flux"], b["flux"]):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("name", ["gold_sphere", "custom_box", "odd_custom"])
def test_fused_fp32_close_to_split(name):
    sc = SCENES[name](A.FP32)
    a = run(sc, [sc.nsteps], fused=True)
    b = run(sc, [sc.nsteps], fused=False)
    d = np.linalg.norm(a["fields"] - b["fields"]) / np.linalg.norm(b["fields"])
    assert d < 1e-5, d


def test_fused_fp64_matches_reference_core():
    if not oracle_lib.available("ref"):
        pytest.skip("reference core not built")
    sc = CF.random_spheres_scene(n_total=(70, 66, 60), pml=8, n_dielectric=20, n_lorentz=4, r_range=(8e-9, 25e-9),
                                 nsteps=75, nl=5, precision=A.FP64, seed=5)
    ref = oracle_lib.run(sc, "ref")
    got = run(sc, [sc.nsteps], fused=True)
    assert sha(got["fields"]) == sha(ref["fields"])


def _env_run(scene, env):
    saved = {k: os.environ.get(k) for k in env}
    os.environ.update(env)
    try:
        return run(scene, [scene.nsteps], fused=True)
    finally:
        for k, v in saved.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v


@pytest.mark.parametrize("env", [{"AEFDTD_ALL_BOUNDARY": "1"}, {"AEFDTD_FUSED_KCHUNK": "5"},
                                 {"AEFDTD_FUSED_KCHUNK": "1000"}, {"AEFDTD_FUSED_TY": "3"},
                                 {"AEFDTD_FUSED_TY": "1"}, {"AEFDTD_SERIAL_GROUPS": "1"}])
def test_fused_layout_changes_no_bit(env):
    """Every item on the kernel with every phase, other z-chunk depths and tile
    heights, serial groups: FP64 fields and flux bit-identical to the default."""
    sc = SCENES["debye_lorentz_sphere"](A.FP64)
    a = run(sc, [sc.nsteps], fused=True)
    b = _env_run(sc, env)
    assert sha(a["fields"]) == sha(b["fields"])
    for x, y in zip(a["flux"], b["flux"]):
        assert np.array_equal(x, y)


def test_fused_group_timings_cover_every_cell_once():
    """With group timing on, the fused groups report their owned cells in the
    E-side slots: together every cell once per step, nothing on the H side."""
    sc = SCENES["wide_sphere"](A.FP32)
    os.environ["AEFDTD_FUSED"] = "1"
    try:
        s = fdtd.build_simulation(sc)
    finally:
        os.environ.pop("AEFDTD_FUSED", None)
    with s:
        s.enable_timing(True, mode=2)
        s.step(20)
        g = s.group_timings()
        d = s.dims()
        assert sum(c for (h, _), (ms, c) in g.items() if h == "E") == d.nx * d.ny * d.nz
        assert sum(c for (h, _), (ms, c) in g.items() if h == "H") == 0
        assert g[("E", "interior")][1] > 0 and g[("E", "interior")][0] > 0
