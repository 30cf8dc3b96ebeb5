"""The persistent batch launch (aefdtd_batch_opts.persistent): each chunk of a
subset's steps is one cooperative launch whose CTAs own bands x z-chunks of
the members and wait only on their neighbours' progress counters.

FP64 fields must be bit-identical to each member stepped alone (the cells are
updated by the same kernel bodies); the plane sums are added per row band
instead of per block, so they agree to 1e-12 relative. FP32 members agree
with the split batch path to 1e-5. A wait that is made to run out (test hook:
the first unit never reports its progress, short bound) returns
AEFDTD_TIMEOUT, and after a reset the same members run correctly again."""
import numpy as np
import pytest

from aether_b200 import _abi as A
from aether_b200 import _lib
from aether_b200 import configs as CF
from aether_b200 import fdtd
from aether_b200._lib import AefdtdError

pytestmark = pytest.mark.gpu

NM = 1e-9
PERSIST_WAIT, PERSIST_WITHHOLD = 5, 6   # AEFDTD_TEST_PERSIST_WAIT_CYCLES, AEFDTD_TEST_PERSIST_WITHHOLD


def cells(seed, n=4, precision=A.FP64, nsteps=400, nz=64, pml=8, period=(80 * NM, 180 * NM)):
    """Nanodisk unit cells of uneven sizes (16-36 cells across for the default period)."""
    rng = np.random.default_rng(seed)
    return [CF.metasurface_cell(rng, nz_total=nz, pml=pml, nsteps=nsteps, nl=11, precision=precision,
                                period_range=period, flux_planes=False) for _ in range(n)]


def alone(scene, steps):
    with fdtd.build_simulation(scene) as s:
        s.step(steps)
        return s.fields(), (s.plane_sums() if scene.normal is not None else None)


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-300)


def run_batch(scenes, steps, **opts):
    sims = [fdtd.build_simulation(sc) for sc in scenes]
    try:
        with fdtd.Batch(persistent=True, **opts) as b:
            for s in sims:
                b.add(s, steps)
            first = b.advance(min(steps, 32))
            info = b.info()
            done = first + b.run(10 ** 6)
            assert done == steps
            return [(s.fields(), s.plane_sums() if sc.normal is not None else None)
                    for s, sc in zip(sims, scenes)], info
    finally:
        for s in sims:
            s.close()


@pytest.mark.parametrize("opts", [dict(), dict(l2_budget_bytes=1), dict(l2_budget_bytes=-1),
                                  dict(tile_y=2, kchunk=4), dict(tile_y=8, kchunk=16), dict(use_graphs=False),
                                  dict(graph_steps=7), dict(lanes=3, l2_budget_bytes=1)])
def test_fp64_persistent_members_bit_identical_to_alone(opts):
    scenes = cells(3)
    steps = 150
    want = [alone(sc, steps) for sc in scenes]
    got, info = run_batch(scenes, steps, **opts)
    assert info["n_persistent"] == info["n_subsets"] > 0
    for (f, p), (wf, wp) in zip(got, want):
        assert np.array_equal(f, wf)
        assert rel(p, wp) < 1e-12


def test_fp64_persistent_real_size_nanodisk_cells():
    """Two cells of the bench's distribution at their real size (z = 200,
    16-cell CPML), one subset each and both in one subset."""
    scenes = cells(11, n=2, nz=200, pml=16, period=(200 * NM, 320 * NM))
    steps = 96
    want = [alone(sc, steps) for sc in scenes]
    for budget in (0, -1):
        got, info = run_batch(scenes, steps, l2_budget_bytes=budget)
        assert info["n_persistent"] > 0
        for (f, p), (wf, wp) in zip(got, want):
            assert np.array_equal(f, wf)
            assert rel(p, wp) < 1e-12


def test_fp64_persistent_custom_mode_oscillator():
    """A custom-mode member (CPML on every face, a point oscillator, no plane
    sums) with odd sizes: units cut ragged bands and z-chunks."""
    sc = CF.random_spheres_scene(n_total=(37, 29, 45), dx=5 * NM, pml=6, n_dielectric=3, n_lorentz=1, seed=4,
                                 r_range=(5 * NM, 15 * NM), nsteps=120, precision=A.FP64)
    steps = 90
    want = alone(sc, steps)
    got, info = run_batch([sc], steps, kchunk=4)
    assert info["n_persistent"] == 1
    assert np.array_equal(got[0][0], want[0])


def test_fp32_persistent_close_to_split_batch():
    scenes = cells(7, precision=A.FP32)
    steps = 200
    sims = [fdtd.build_simulation(sc) for sc in scenes]
    with fdtd.Batch() as b:
        for s in sims:
            b.add(s, steps)
        b.run(10 ** 6)
        want = [(s.fields(), s.plane_sums()) for s in sims]
    for s in sims:
        s.close()
    got, info = run_batch(scenes, steps)
    assert info["n_persistent"] > 0
    for (f, p), (wf, wp) in zip(got, want):
        assert rel(f, wf) < 1e-5
        assert rel(p, wp) < 1e-5


def test_persistent_wait_runs_out_then_members_recover():
    """The first unit withholds its progress reports: the neighbours'
    waits run out (2^20-cycle bound), the advance returns AEFDTD_TIMEOUT, and
    after the hook is cleared and the members reset, a new batch gives the
    fields of the members stepped alone."""
    scenes = cells(9, n=2)
    steps = 64
    want = [alone(sc, steps) for sc in scenes]
    lib = _lib.load()
    sims = [fdtd.build_simulation(sc) for sc in scenes]
    try:
        for s in sims:
            _lib.check(lib.aefdtd_test_hook(s._h, PERSIST_WAIT, 1 << 20))
            _lib.check(lib.aefdtd_test_hook(s._h, PERSIST_WITHHOLD, 1))
        with fdtd.Batch(persistent=True, l2_budget_bytes=-1) as b:
            for s in sims:
                b.add(s, steps)
            with pytest.raises(AefdtdError) as e:
                b.advance(steps)
            assert e.value.status == 3   # AEFDTD_TIMEOUT
        for s in sims:
            _lib.check(lib.aefdtd_test_hook(s._h, PERSIST_WITHHOLD, 0))
            _lib.check(lib.aefdtd_test_hook(s._h, PERSIST_WAIT, 1 << 31))
            s.reset()
        with fdtd.Batch(persistent=True, l2_budget_bytes=-1) as b:
            for s in sims:
                b.add(s, steps)
            assert b.run(10 ** 6) == steps
            for s, (f, p) in zip(sims, want):
                assert np.array_equal(s.fields(), f)
                assert rel(s.plane_sums(), p) < 1e-12
    finally:
        for s in sims:
            s.close()



def test_fp64_persistent_16bit_material_ids():
    """300 materials (16-bit ids) on the persistent launch: fields equal the run alone."""
    sc = CF.random_spheres_scene(n_total=(70, 40, 44), dx=5 * NM, pml=6, n_dielectric=300, n_lorentz=2, seed=3,
                                 r_range=(3 * NM, 8 * NM), nsteps=80, precision=A.FP64)
    steps = 80
    want = alone(sc, steps)
    got, info = run_batch([sc], steps)
    assert info["n_persistent"] == 1
    assert np.array_equal(got[0][0], want[0])


def test_fp64_oblique_member_keeps_split_launches():
    """An oblique member (two coupled grids) keeps the split launches in its
    own subset of a persistent batch; the normal-mode member beside it takes
    the persistent launch. Both members' fields equal their runs alone."""
    scenes = [cells(13, n=1)[0], CF.oblique_scene(nsteps=80)]
    steps = 80
    want = [alone(sc, steps)[0] for sc in scenes]
    sims = [fdtd.build_simulation(sc) for sc in scenes]
    try:
        with fdtd.Batch(persistent=True) as b:
            for s in sims:
                b.add(s, steps)
            first = b.advance(32)
            info = b.info()
            assert first + b.run(10 ** 6) == steps
            assert info["n_subsets"] == 2 and info["n_persistent"] == 1
            for s, w in zip(sims, want):
                assert np.array_equal(s.fields(), w)
    finally:
        for s in sims:
            s.close()
