"""The serving loop (aefdtd_server_*): continuous batching with admission by
device-memory footprint.

Each job's spectra must be the same in the mix as served alone (bit-identical:
a member's arithmetic does not depend on its neighbours), and in FP64 the same
as the single-simulation path. Jobs arrive while others run, memory budgets
are respected, and a job larger than the budget fails without stopping the
server."""
import numpy as np
import pytest

from aether_b200 import _abi as A
from aether_b200 import configs as CF
from aether_b200 import fdtd

pytestmark = pytest.mark.gpu

NM = 1e-9


def jobs(seed, n, precision):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        sc = CF.metasurface_cell(rng, nz_total=64, pml=8, nsteps=400, nl=21, precision=precision,
                                 period_range=(80 * NM, 180 * NM), flux_planes=False)
        out.append((sc, int(rng.integers(90, 260))))
    return out


def serve_alone(sc, steps):
    with fdtd.Server() as v:
        j = v.submit(sc, steps)
        v.drain()
        assert v.info(j)["state"] == A.JOB_DONE
        return v.spectra(j)


@pytest.mark.parametrize("precision", [A.FP64, A.FP32])
def test_results_same_alone_and_in_the_mix(precision):
    js = jobs(5, 6, precision)
    with fdtd.Server() as v:
        ids = []
        # arrivals while others run: two at a time, one poll in between
        for k in range(0, len(js), 2):
            for sc, steps in js[k:k + 2]:
                ids.append(v.submit(sc, steps))
            v.poll()
        v.drain()
        st = v.stats()
        assert st["done"] == len(js) and st["failed"] == 0
        assert st["p99_s"] >= st["p50_s"] > 0
        admits = [v.info(j)["t_admit"] for j in ids]
        dones = [v.info(j)["t_done"] for j in ids]
        assert any(a < d for a, d in zip(admits[2:], dones[:2]))   # later arrivals ran beside earlier jobs
        mix = [v.spectra(j) for j in ids]
    for (sc, steps), got in zip(js, mix):
        assert np.array_equal(got, serve_alone(sc, steps))
    if precision == A.FP64:
        for (sc, steps), got in zip(js[:3], mix[:3]):
            with fdtd.build_simulation(sc) as s:
                s.step(steps)
                assert np.array_equal(got, s.normal_spectra())


def test_memory_budget_limits_running_jobs():
    """A budget of 60% of the jobs' summed footprint estimates: fewer than all
    run at once, actual device bytes never exceed the budget (the estimate is
    an upper bound), and every job completes."""
    js = jobs(9, 5, A.FP32)
    with fdtd.Server() as probe:
        ests = [probe.info(probe.submit(sc, steps))["est_bytes"] for sc, steps in js]
    budget = int(0.6 * sum(ests))
    with fdtd.Server(budget_bytes=budget) as v:
        ids = [v.submit(sc, steps) for sc, steps in js]
        peak_running = 0
        for _ in range(100000):
            st = v.stats()
            peak_running = max(peak_running, st["running"])
            assert st["in_use_bytes"] <= st["budget_bytes"]
            if st["queued"] == 0 and st["running"] == 0:
                break
            v.poll()
        st = v.stats()
        assert st["done"] == len(js)
        assert st["peak_bytes"] <= st["budget_bytes"]
        assert peak_running < len(js)


def test_job_above_budget_fails_alone():
    js = jobs(13, 2, A.FP32)
    with fdtd.Server(budget_bytes=1 << 20) as v:   # 1 MiB: nothing fits
        ids = [v.submit(sc, steps) for sc, steps in js]
        v.poll()
        assert all(v.info(j)["state"] == A.JOB_FAILED for j in ids)
        with pytest.raises(Exception):
            v.spectra(ids[0])


def test_jobs_with_completion_end_at_their_completion_step():
    """auto_tsteps for served jobs: each job stops at the step its completion
    sensor gives alone, and its spectra are the ones of that run."""
    # cells that complete inside the budget at this coefficient
    rng = np.random.default_rng(11)
    scs = [CF.metasurface_cell(rng, nz_total=64, pml=8, nsteps=3000, nl=11, precision=A.FP64,
                               period_range=(80 * NM, 180 * NM), flux_planes=False) for _ in range(3)]
    budget, coeff, every = 3000, 5e-2, 40
    with fdtd.Server() as v:
        ids = [v.submit(sc, budget, completion=(coeff, every)) for sc in scs]
        v.drain()
        got = [(v.info(j), v.spectra(j)) for j in ids]
    for sc, (info, spec) in zip(scs, got):
        assert info["state"] == A.JOB_DONE
        with fdtd.build_simulation(sc) as s:
            s.set_completion(coeff, every)
            s.step(budget)
            done, stop, _ = s.completion()
            assert done and info["stop_step"] == stop
            assert np.array_equal(spec, s.normal_spectra())
