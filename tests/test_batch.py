"""Batches (aefdtd_batch_*): many simulations advanced together.

A member's results must not depend on the batch. In FP64, fields and plane
sums of every member are bit-identical to the same simulation stepped alone,
whatever the subset budget, tile height, planes per item, step budgets or
autotuning. In FP32 they agree to 1e-5 relative: the batched kernels are
separate instantiations and may contract multiply-adds differently."""
import numpy as np
import pytest

from aether_b200 import _abi as A
from aether_b200 import configs as CF
from aether_b200 import fdtd
from aether_b200._lib import AefdtdError

pytestmark = pytest.mark.gpu

NM = 1e-9


def cells(seed, n=4, precision=A.FP64, nsteps=400):
    """Small nanodisk unit cells of uneven sizes (16-36 cells across)."""
    rng = np.random.default_rng(seed)
    return [CF.metasurface_cell(rng, nz_total=64, pml=8, nsteps=nsteps, nl=11, precision=precision,
                                period_range=(80 * NM, 180 * NM), flux_planes=False) for _ in range(n)]


def alone(scene, steps):
    with fdtd.build_simulation(scene) as s:
        s.step(steps)
        return s.fields(), s.plane_sums()


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-300)


@pytest.mark.parametrize("opts", [dict(), dict(l2_budget_bytes=1), dict(l2_budget_bytes=-1),
                                  dict(tile_y=2, kchunk=16), dict(tile_y=8, kchunk=4), dict(use_graphs=False),
                                  dict(graph_steps=7), dict(graph_steps=64), dict(l2_budget_bytes=1, lanes=3),
                                  dict(l2_budget_bytes=1, lanes=8)])
def test_fp64_batch_members_bit_identical_to_alone(opts):
    scenes = cells(3)
    steps = 150
    want = [alone(sc, steps) for sc in scenes]
    sims = [fdtd.build_simulation(sc) for sc in scenes]
    with fdtd.Batch(**opts) as b:
        for s in sims:
            b.add(s, steps)
        assert b.run(10 ** 6) == steps
        assert len(b.finished()) == len(sims)
        for s, (f, p) in zip(sims, want):
            assert np.array_equal(s.fields(), f)
            assert np.array_equal(s.plane_sums(), p)
    for s in sims:
        s.close()


def test_uneven_budgets_finish_exactly():
    """Members with different budgets (one subset and several): each stops at
    exactly its budget, and its results equal its run alone."""
    scenes = cells(5, n=3)
    budgets = [70, 130, 200]
    want = [alone(sc, n) for sc, n in zip(scenes, budgets)]
    for budget in (-1, 1):
        sims = [fdtd.build_simulation(sc) for sc in scenes]
        with fdtd.Batch(l2_budget_bytes=budget) as b:
            for s, n in zip(sims, budgets):
                b.add(s, n)
            while b.advance(64) > 0:
                pass
            assert len(b.finished()) == 3
            for s, n, (f, p) in zip(sims, budgets, want):
                assert s.dims().step == n
                assert np.array_equal(s.fields(), f)
                assert np.array_equal(s.plane_sums(), p)
        for s in sims:
            s.close()


def test_members_join_and_leave_between_segments():
    """Continuous batching: a member retires when done, another joins later;
    each result equals its run alone."""
    scenes = cells(11, n=3)
    want = [alone(sc, 100) for sc in scenes]
    s0, s1, s2 = (fdtd.build_simulation(sc) for sc in scenes)
    with fdtd.Batch() as b:
        b.add(s0, 100)
        b.add(s1, 100)
        assert b.advance(40) == 40
        b.add(s2, 100)              # joins while the others are mid-run
        done = []
        while len(done) < 3:
            n = b.advance(10 ** 6)
            assert n > 0
            for s in b.finished():
                done.append(s)
                b.remove(s)
        for s, (f, p) in zip((s0, s1, s2), want):
            assert np.array_equal(s.fields(), f)
            assert np.array_equal(s.plane_sums(), p)
    for s in (s0, s1, s2):
        s.close()


def test_autotune_then_run_matches_alone():
    scenes = cells(21, n=4)
    steps = 128
    want = [alone(sc, steps) for sc in scenes]
    sims = [fdtd.build_simulation(sc) for sc in scenes]
    with fdtd.Batch() as b:
        for s in sims:
            b.add(s, steps)
        b.autotune()
        info = b.info()
        assert len(info["classes"]) >= 1
        for c in info["classes"]:
            assert c["tile_y"] in (2, 4, 8) and c["kchunk"] in (4, 8)
        assert all(s.dims().step == 0 for s in sims)
        first = b.advance(64)
        # the persistent launch adds the plane sums per row band (last bits differ)
        persistent = b.info()["n_persistent"] > 0
        assert first + b.run(10 ** 6) == steps
        for s, (f, p) in zip(sims, want):
            assert np.array_equal(s.fields(), f)
            if persistent:
                assert rel(s.plane_sums(), p) < 1e-12
            else:
                assert np.array_equal(s.plane_sums(), p)
    for s in sims:
        s.close()


def test_fp32_batch_close_to_alone():
    scenes = cells(7, n=3, precision=A.FP32)
    steps = 200
    want = [alone(sc, steps) for sc in scenes]
    sims = [fdtd.build_simulation(sc) for sc in scenes]
    with fdtd.Batch() as b:
        for s in sims:
            b.add(s, steps)
        b.run(10 ** 6)
        for s, (f, p) in zip(sims, want):
            assert rel(s.fields(), f) < 1e-5
            assert rel(s.plane_sums(), p) < 1e-5
    for s in sims:
        s.close()


def test_member_refuses_direct_steps_and_leaves_on_destroy():
    scenes = cells(2, n=2)
    s0, s1 = (fdtd.build_simulation(sc) for sc in scenes)
    with fdtd.Batch() as b:
        b.add(s0, 64)
        b.add(s1, 64)
        with pytest.raises(AefdtdError):
            s0.step(1)
        h1 = s1._h.value
        s1.close()                  # destroying a member detaches it
        b.members.pop(h1, None)
        assert b.info()["n_members"] == 1
        assert b.run(10 ** 6) == 64
    s0.close()


def alone_completion(scene, budget, coeff, every):
    with fdtd.build_simulation(scene) as s:
        s.set_completion(coeff, every)
        s.step(budget)
        return s.completion(), s.normal_spectra()


@pytest.mark.parametrize("opts", [dict(), dict(l2_budget_bytes=-1), dict(graph_steps=7)])
def test_completion_inside_a_batch_stops_where_alone_stops(opts):
    """Members with the energy-mode completion sensor: each completes at the
    same step as alone (checks every 40 steps, not aligned with the batch's
    segments) and its spectra, read up to that step, are bit-identical; a
    member without the sensor runs its whole budget beside them."""
    scenes = cells(11, n=3, nsteps=3000)
    budget, coeff, every = 3000, 5e-2, 40
    want = [alone_completion(sc, budget, coeff, every) for sc in scenes]
    assert all(w[0][0] for w in want), "the cells must complete inside the budget"
    plain = cells(12, n=1, nsteps=700)[0]
    sims = [fdtd.build_simulation(sc) for sc in scenes]
    for s in sims:
        s.set_completion(coeff, every)
    ps = fdtd.build_simulation(plain)
    with fdtd.Batch(**opts) as b:
        for s in sims:
            b.add(s, budget)
        b.add(ps, 700)
        b.run(10 ** 6)
        assert len(b.finished()) == len(sims) + 1
        for s, ((done, stop, ratio), spec) in zip(sims, want):
            got = s.completion()
            assert got[0] and got[1] == stop and got[2] == ratio
            assert s.dims().step > stop and s.dims().step <= stop + 1 + 64
            assert np.array_equal(s.normal_spectra(), spec)
        assert ps.dims().step == 700
        assert np.array_equal(ps.plane_sums(), alone(plain, 700)[1])
    for s in sims + [ps]:
        s.close()


@pytest.mark.parametrize("coeff,layout,npts,seed", [(2e-2, "nnb", 40, 7), (5e-2, "bnn", 24, 11)])
def test_ft_completion_inside_a_batch_stops_where_alone_stops(coeff, layout, npts, seed):
    """FT-mode completion sensor (probes drawn from the seeded generator) on
    batch members: the check reads the probe ring as it stood after each
    check step, so a member completes at the step it completes alone, with
    bit-identical spectra, although it runs on past it within its segment."""
    import scenes
    scs = [scenes.slab_tm(nsteps=6000), scenes.slab_tm(nsteps=6000, n_slab=2.0)]
    for sc in scs:
        sc.sensors = []            # batch members carry plane sums only
    want = []
    for sc in scs:
        with fdtd.build_simulation(sc) as s:
            s.set_completion_ft(400e-9, 1000e-9, coeff, npts, layout, seed, 50)
            s.step(6000)
            want.append((s.completion(), s.normal_spectra()))
    assert all(w[0][0] for w in want), "the runs must complete inside the budget"
    sims = [fdtd.build_simulation(sc) for sc in scs]
    for s in sims:
        s.set_completion_ft(400e-9, 1000e-9, coeff, npts, layout, seed, 50)
    with fdtd.Batch(graph_steps=16) as b:
        for s in sims:
            b.add(s, 6000)
        b.run(10 ** 6)
        for s, ((done, stop, ratio), spec) in zip(sims, want):
            got = s.completion()
            assert got[0] and got[1] == stop and got[2] == ratio
            assert np.array_equal(s.normal_spectra(), spec)
    for s in sims:
        s.close()
