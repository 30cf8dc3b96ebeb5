"""Single-wavelength field sensors (aefdtd_add_fieldmap) against the
reference's own FieldMap, FieldBlock and FieldPoint run in the compiled
reference core, in both drivers. FP64: accumulators and point series within
1e-12 of the largest magnitude (the phases are the reference's expressions
evaluated on the host; the kernels use round-to-nearest FP64 products and
sums in the reference's order). FP32: within 1e-4 of the largest magnitude
of the FP64 reference.

FieldBlock::threaded_computation (s_fieldmap.cpp:214) lets worker threads
with ID >= span1 write past its grids when the block's x span is at most the
reference's thread count, so the blocks compared here are wider than that."""
import numpy as np
import pytest

import oracle_lib
import scenes
from aether_b200 import _abi as A
from aether_b200 import configs as CF
from aether_b200 import fdtd

pytestmark = pytest.mark.gpu

RTOL64 = 1e-12
RTOL32 = 1e-4


def md(kind, box, lam=600e-9, ori=A.NORMAL_Z, cum=False, mag=False):
    d = A.FieldMapDesc()
    d.kind, d.orientation = kind, ori
    for k in range(6):
        d.box[k] = box[k]
    d.cumulative, d.magnetic, d.lambda_ = int(cum), int(mag), lam
    return d


def flat(kind, v):
    """A Simulation.fieldmap result in the reference driver's flat layout."""
    if kind == A.MAP_POINT:
        return np.asarray(v, dtype=np.float64).ravel()
    z = np.asarray(v)
    return np.stack([z.real, z.imag], axis=-1).ravel()


def gpu_maps(sc, maps, steps):
    with fdtd.build_simulation(sc) as s:
        ids = [s.add_fieldmap(d.kind, list(d.box), d.lambda_, d.orientation, d.cumulative, d.magnetic)
               for d in maps]
        s.step(steps)
        return [flat(d.kind, s.fieldmap(i)) for d, i in zip(maps, ids)]


def close(got, want, rtol):
    scale = max(np.max(np.abs(want)), 1e-300)
    return got.shape == want.shape and np.max(np.abs(got - want)) <= rtol * scale


def wide_box(precision=A.FP64, nsteps=100):
    """Custom-mode scene with spheres and an oscillator, 58 structure cells
    across x (room for a block wider than the reference's thread count)."""
    return CF.random_spheres_scene(n_total=(80, 30, 40), pml=6, n_dielectric=4, n_lorentz=2,
                                   r_range=(10e-9, 30e-9), nsteps=nsteps, nl=5, precision=precision, seed=3)


def need_ref():
    if not oracle_lib.available("ref"):
        pytest.skip("reference core not built")


def normal_maps():
    return [md(A.MAP_PLANE, (0, 12, 0, 10, 5, 9)),
            md(A.MAP_PLANE, (2, 6, 0, 10, 0, 20), ori=A.NORMAL_XM, cum=True),
            md(A.MAP_PLANE, (0, 12, 3, 4, 0, 20), ori=A.NORMAL_Y, mag=True),
            md(A.MAP_PLANE, (0, 12, 0, 10, 2, 12), ori=A.NORMAL_Z, cum=True, mag=True, lam=800e-9),
            md(A.MAP_POINT, (3, 0, 4, 0, 7, 0))]


@pytest.mark.parametrize("prec", [A.FP64, A.FP32])
def test_plane_maps_and_point_match_reference_normal_mode(prec):
    need_ref()
    steps = 150
    maps = normal_maps()
    ref = oracle_lib.run_ref_fieldmaps(scenes.gold_sphere(nsteps=steps), maps, nsteps=steps)["maps"]
    got = gpu_maps(scenes.gold_sphere(precision=prec, nsteps=steps), maps, steps)
    for d, g, r in zip(maps, got, ref):
        assert np.any(r != 0)
        assert close(g, r, RTOL64 if prec == A.FP64 else RTOL32), (d.kind, d.orientation, d.cumulative)


@pytest.mark.parametrize("prec", [A.FP64, A.FP32])
def test_block_and_maps_match_reference_custom_mode(prec):
    need_ref()
    steps = 100
    sc = wide_box(nsteps=steps)
    g = sc.grid
    w = oracle_lib.ref_threads() + 2
    if w + 2 > g.nx:
        pytest.skip(f"grid too narrow for a block wider than the reference's {w - 2} threads")
    src = sc.sources[0]
    lam = 0.5 * (src.lambda_min + src.lambda_max)
    maps = [md(A.MAP_BLOCK, (1, 1 + w, 3, 9, 10, 16), lam=lam),
            md(A.MAP_PLANE, (0, g.nx, 0, g.ny, g.nz // 2, g.nz // 2 + 1), lam=lam),
            md(A.MAP_PLANE, (0, g.nx, g.ny // 2, g.ny // 2 + 4, 0, g.nz), ori=A.NORMAL_YM, cum=True, mag=True,
               lam=lam),
            md(A.MAP_POINT, (g.nx // 2, 0, g.ny // 2, 0, g.nz // 2, 0))]
    ref = oracle_lib.run_ref_fieldmaps(sc, maps, nsteps=steps)["maps"]
    got = gpu_maps(wide_box(precision=prec, nsteps=steps), maps, steps)
    for d, gm, r in zip(maps, got, ref):
        assert np.any(r != 0)
        assert close(gm, r, RTOL64 if prec == A.FP64 else RTOL32), d.kind


def test_maps_do_not_change_fields_and_survive_reset():
    sc = scenes.gold_sphere(nsteps=90)
    with fdtd.build_simulation(sc) as a, fdtd.build_simulation(sc) as b:
        a.step(90)
        ids = [b.add_fieldmap(d.kind, list(d.box), d.lambda_, d.orientation, d.cumulative, d.magnetic)
               for d in normal_maps()]
        b.step(90)
        assert np.array_equal(a.fields(), b.fields())
        first = [b.fieldmap(i) for i in ids]
        assert b.fieldmap(ids[-1]).shape == (90, 3)
        b.reset()
        assert b.fieldmap(ids[-1]).shape == (0, 3)
        assert not np.any(b.fieldmap(ids[0]))
        b.step(90)
        for i, f in zip(ids, first):
            assert np.array_equal(b.fieldmap(i), f)


def test_step_pieces_and_graphs_agree(monkeypatch):
    """Maps fed through captured 64-step segments equal maps fed by direct
    launches in uneven pieces, bit for bit (FP64)."""
    sc = scenes.gold_sphere(nsteps=200)
    maps = normal_maps()
    a = gpu_maps(sc, maps, 200)
    monkeypatch.setenv("AEFDTD_NO_GRAPHS", "1")
    with fdtd.build_simulation(sc) as s:
        ids = [s.add_fieldmap(d.kind, list(d.box), d.lambda_, d.orientation, d.cumulative, d.magnetic)
               for d in maps]
        for n in (1, 63, 70, 66):
            s.step(n)
        b = [flat(d.kind, s.fieldmap(i)) for d, i in zip(maps, ids)]
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_fieldmap_argument_checks():
    sc = scenes.slab_tm(nsteps=10)
    with fdtd.build_simulation(sc) as s:
        with pytest.raises(Exception):
            s.add_fieldmap(A.MAP_PLANE, (0, 4, 0, 4, 0, 1), 0.0)          # lambda must be positive
        with pytest.raises(Exception):
            s.add_fieldmap(7, (0, 4, 0, 4, 0, 1), 500e-9)                # unknown kind
        with pytest.raises(Exception):
            s.add_fieldmap(A.MAP_BLOCK, (3, 3, 0, 4, 0, 1), 500e-9)      # empty box
        for _ in range(8):
            s.add_fieldmap(A.MAP_POINT, (0, 0, 0, 0, 0, 0))
        with pytest.raises(Exception):
            s.add_fieldmap(A.MAP_POINT, (0, 0, 0, 0, 0, 0))               # at most 8
