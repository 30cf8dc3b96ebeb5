"""Benchmark of the FDTD time-stepping core on one B200.

Workload (the headline): the dispersive unit cell -- 128x128x256 total cells
at 2.5 nm, periodic x/y, 24-cell CPML on z, a 40 nm gold-like sphere (Drude +
2 critical points) on an n=1.45 substrate, normal-incidence 400-1000 nm pulse,
two planar flux sensors at 201 wavelengths with K=64 buffered steps per DFT
block (seeded synthetic geometry; no dataset). The headline value is the FP64
path, the reference's own arithmetic (fields bit-identical to the reference
core); the FP32 path, the large random grid (1024x1024x512), the batch of
nanodisk cells and the serving loop are reported in sub-objects. One bench
step = 64 FDTD time steps (one DFT block), inputs resident in HBM.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Metric: Gcell-updates/s = total cells x time steps / s / 1e9."""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

STEPS_PER_BENCH_STEP = 64
METRIC = "Gcell-updates/s"


def log(*a):
    print(*a, file=sys.stderr, flush=True)


WORKLOAD = ("dispersive unit cell 128x128x256 @2.5nm, gold Drude+2CP sphere r=40nm on n=1.45 substrate, "
            "24-cell CPML z, normal incidence 400-1000nm, 2 DFT planes x 201 lambda, K=64")


def config_dict(ws):
    """The workload description both arms print, identical by construction."""
    return {"workload": WORKLOAD, "precision": "FP64 (the reference's arithmetic)",
            "l2": "inputs exceed L2 (201 MB of FP64 fields, 632 MB of DFT accumulators); a 256 MiB buffer "
                  "is also written between timed GPU steps",
            "parallelism": f"replicas x{ws}"}


def workload(precision):
    from aether_b200 import configs as CF
    return CF.sphere_scene(nx=128, ny=128, nz_total=256, dx=2.5e-9, pml=24, radius=40e-9, nsteps=20000,
                           nl=201, precision=precision)


def rta(spec):
    """R, T, A per wavelength from the spectdata_norm2 columns: |r|^2 and
    |t|^2 n_sub/n_sup of both polarisation components."""
    r = spec[:, 5] + spec[:, 8]
    t = spec[:, 11] + spec[:, 14]
    return r, t, 1.0 - r - t


def spectrum_error_sample():
    """FP32 against FP64 (the FP64 path is bit-identical to the reference
    core) on complete runs of the n=1.5 slab (64x64x128, 4000 steps, 61
    wavelengths) and of the bench's gold-sphere cell (20000 steps, 201
    wavelengths): the largest absolute R, T and A differences."""
    import numpy as np
    from aether_b200 import _abi as A
    from aether_b200 import configs as CF
    from aether_b200 import fdtd
    out = {}
    for name, make in (("slab_64x64x128_4000_steps", lambda p: CF.slab_scene(precision=p)),
                       ("gold_sphere_128x128x256_20000_steps", workload)):
        res = {}
        for prec in (A.FP32, A.FP64):
            res[prec] = rta(fdtd.run(make(prec), want_fields=False)["spectra"])
        d = [float(np.max(np.abs(res[A.FP32][q] - res[A.FP64][q]))) for q in range(3)]
        out[name] = {"max_abs_dR": d[0], "max_abs_dT": d[1], "max_abs_dA": d[2]}
        log(f"[accuracy] {name}: |dR| {d[0]:.2e} |dT| {d[1]:.2e} |dA| {d[2]:.2e}")
    out["source"] = "FP32 vs FP64 spectra of complete runs; FP64 fields are bit-identical to the reference core"
    return out


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def max_over_ranks(ms, device="cuda"):
    """The slowest rank's timed duration: the job ends when its last replica
    ends. `device` is where the reduction tensor lives: "cuda" under NCCL,
    "cpu" under gloo. Without an initialised group of two or more ranks, `ms`
    comes back as given."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() < 2:
        return ms
    t = torch.tensor([ms], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_gcells(cells, steps, ms, ws):
    """Whole-job Gcell-updates/s of `ws` replicas that each advance `cells`
    cells by `steps` time steps, over the slowest rank's `ms`."""
    from aether_b200 import metrics as MT
    return MT.gcells(cells, steps, ms / 1e3) * ws


class ClockSampler:
    """nvidia-smi samples during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.25)
        return self

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.15)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                p = [x.strip() for x in line.split(",")]
                if len(p) >= 9:
                    rows.append(p)
        except Exception:
            pass
        finally:
            try:
                os.unlink(self.path)
            except Exception:
                pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic(kernel, precision):
    """DRAM bytes per launch from the committed ncu summary, if present."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.txt")
    try:
        for line in open(path):
            p = line.split()
            if len(p) >= 3 and not line.startswith("#") and p[0] == kernel and p[1] == precision:
                return float(p[2])
    except Exception:
        pass
    return None


def run_gpu_arm(args):
    import torch
    from aether_b200 import _abi as A
    from aether_b200 import fdtd
    from aether_b200 import metrics as MT

    ws, rank, local = dist_env()
    if ws > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()

    # Replicas only: every rank advances its own copy of the workload; no
    # data-path collective exists on this path.
    results = {}
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MiB > L2
    for prec_name, prec in (("fp32", A.FP32), ("fp64", A.FP64)):
        scene = workload(prec)
        scene.grid.device = dev
        sim = fdtd.build_simulation(scene)
        ext = torch.cuda.ExternalStream(sim.stream_ptr())
        cells = scene.cells
        kb = MT.kernel_bytes(scene)
        for _ in range(args.warmup):
            sim.step(STEPS_PER_BENCH_STEP)
        sim.synchronize()
        launches0 = sim.launch_count()
        times = []
        with ClockSampler(dev) as cs:
            if ws > 1:
                torch.distributed.barrier()
            torch.cuda.synchronize()
            for _ in range(args.steps):
                with torch.cuda.stream(ext):
                    flush.zero_()   # L2 flush between timed steps
                    ev0 = torch.cuda.Event(enable_timing=True)
                    ev1 = torch.cuda.Event(enable_timing=True)
                    ev0.record(ext)
                sim.step(STEPS_PER_BENCH_STEP)   # one CUDA-graph replay of 64 steps
                with torch.cuda.stream(ext):
                    ev1.record(ext)
                times.append((ev0, ev1))
            torch.cuda.synchronize()
            if ws > 1:
                torch.distributed.barrier()
        launches = sim.launch_count() - launches0
        per = [a.elapsed_time(b) for a, b in times]
        ms = sum(per)
        log(f"[{prec_name}] bench-step ms: min {min(per):.3f} median {statistics.median(per):.3f} "
            f"max {max(per):.3f}")
        # per-kernel split: the same steps launched one by one with CUDA events
        # around each half-step and the sensor launch (timing pass after the
        # timed region)
        sim.enable_timing(True)
        e_ms = h_ms = s_ms = 0.0
        tsteps = 2 * STEPS_PER_BENCH_STEP
        for _ in range(2):
            with torch.cuda.stream(ext):
                flush.zero_()
            sim.step(STEPS_PER_BENCH_STEP)
            a, b, c = sim.timings()
            e_ms += a; h_ms += b; s_ms += c
        # per-group pass: each work-item group alone between CUDA events on the
        # simulation's stream (the launch durations behind the roofline)
        sim.enable_timing(True, mode=2)
        with torch.cuda.stream(ext):
            flush.zero_()
        sim.step(STEPS_PER_BENCH_STEP)
        groups = sim.group_timings()
        sim.enable_timing(False)
        sim.synchronize()
        ms = max_over_ranks(ms, device="cuda")
        nsteps = args.steps * STEPS_PER_BENCH_STEP
        # the fused path reports its groups in the E-side slots and none in the H side
        fused = groups.get(("H", "interior"), (0.0, 0))[1] == 0
        results[prec_name] = {
            "gcells": whole_job_gcells(cells, nsteps, ms, ws),
            "ms_per_step": ms / args.steps,
            "e_ms": e_ms / tsteps, "h_ms": h_ms / tsteps, "s_ms": s_ms / tsteps,
            "bytes": kb, "launches": launches, "clocks": cs.summary(), "cells": cells,
            "groups": groups, "step_bytes": MT.step_bytes(scene, fused=fused), "fused": fused,
            "staged": not fused and os.environ.get("AEFDTD_TMA", "0") != "0",
        }
        sim.close()
        log(f"[{prec_name}] {results[prec_name]['gcells']:.2f} Gcell/s  E {e_ms / tsteps * 1e3:.1f} us  "
            f"H {h_ms / tsteps * 1e3:.1f} us  sensors {s_ms / tsteps * 1e3:.1f} us per time step (timing pass)")
    if ws > 1:
        # the run's last collective is done: all ranks leave the group together
        # (no CUDA graph holds an NCCL call); rank 0's later samples are local
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return results, ws, rank


def e2e_job(precision, nsteps):
    """One complete job through the public API from host buffers: geometry and
    materials uploaded, all steps run, spectra read back."""
    from aether_b200 import fdtd
    scene = workload(precision)
    t0 = time.perf_counter()
    with fdtd.build_simulation(scene) as sim:
        sim.step(nsteps)
        spec = sim.normal_spectra()
        flux = [sim.sensor_flux(i) for i in range(len(scene.sensors))]
    dt = time.perf_counter() - t0
    h2d = scene.map.nbytes + sum(len(bytes(m)) for m in scene.materials)
    d2h = spec.nbytes + sum(f.nbytes for f in flux) + 12 * 8 * nsteps
    return dt, h2d, d2h, scene.cells


def cpu_baseline(scene_fn, seconds_budget=20.0):
    """The reference's own FDTD core (oracle/_ref, compiled from source) on a
    bounded sample of the workload on the host cores."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib
    if not oracle_lib.available("ref"):
        which, kind = "port", "port"
    else:
        which, kind = "ref", "reference"
    from aether_b200 import _abi as A
    scene = scene_fn(A.FP64)
    nsteps = 4
    r = oracle_lib.run(scene, which, nsteps=nsteps, want_fields=False)
    per_step = r["seconds"] / nsteps
    n2 = max(4, min(64, int(seconds_budget / max(per_step, 1e-6))))
    r = oracle_lib.run(scene, which, nsteps=n2, want_fields=False)
    cores = 1
    if kind == "reference":
        import ctypes as C
        lib = C.CDLL(oracle_lib.REF_PATH)
        cores = int(lib.aeref_threads())
    val = scene.cells * n2 / r["seconds"] / 1e9
    return {"value": val, "unit": METRIC, "cores": cores, "kind": kind,
            "sample": f"{n2} time steps of the full 128x128x256 FP64 workload incl. 2x201-lambda DFT sensors "
                      f"(time loop only, {r['seconds']:.2f} s)"}


def reference_arm(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib
    from aether_b200 import _abi as A
    which = "ref" if oracle_lib.available("ref") else "port"
    kind = "reference" if which == "ref" else "port"
    scene = workload(A.FP64)
    sample_steps = 4
    for _ in range(args.warmup):
        oracle_lib.run(scene, which, nsteps=1, want_fields=False)
    secs = 0.0
    for _ in range(args.steps):
        r = oracle_lib.run(scene, which, nsteps=sample_steps, want_fields=False)
        secs += r["seconds"]
    nsteps = args.steps * sample_steps
    val = scene.cells * nsteps / secs / 1e9
    cores = 1
    if which == "ref":
        import ctypes as C
        cores = int(C.CDLL(oracle_lib.REF_PATH).aeref_threads())
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": METRIC, "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": secs / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": config_dict(ws),
        "step": f"{sample_steps} FDTD time steps per bench step (bounded CPU sample of the same workload)",
        "cpu_baseline": {"value": val, "unit": METRIC, "cores": cores, "kind": kind,
                         "sample": f"{sample_steps} time steps per bench step, reference time loop"},
        "e2e": {"value": val, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def batch_sample(n_cells=512, steps=256, seed=2024):
    """Batch: n_cells seeded nanodisk unit cells (period U(200, 600) nm at
    5 nm, z = 200 cells with 16-cell CPML, gold or n U(1.8, 3.5) disk on
    n = 1.45, 101 wavelengths) advanced as one FP32 batch. Fixed batch settings
    (tile 32 x 4, 8 planes per item, 48 MiB subsets, two at a time, 32-step graphs); a bounded sample of
    `steps` steps after a one-segment warm-up, timed on the host around the
    synchronous advance calls, extrapolated to the 8000-step job."""
    import numpy as np
    from aether_b200 import _abi as A
    from aether_b200 import configs as CF
    from aether_b200 import fdtd
    rng = np.random.default_rng(seed)
    scenes = [CF.metasurface_cell(rng, precision=A.FP32, nsteps=8000, nl=101, flux_planes=False)
              for _ in range(n_cells)]
    t0 = time.perf_counter()
    sims = [fdtd.build_simulation(sc) for sc in scenes]
    setup = time.perf_counter() - t0
    cells = sum(sc.cells for sc in scenes)
    with fdtd.Batch(l2_budget_bytes=48 << 20, tile_y=4, kchunk=8, lanes=2, graph_steps=32) as b:
        for s in sims:
            b.add(s, steps + STEPS_PER_BENCH_STEP)
        b.advance(STEPS_PER_BENCH_STEP)            # warm-up: captures every subset's graph
        t0 = time.perf_counter()
        done = 0
        while done < steps:
            done += b.advance(steps - done)
        dt = time.perf_counter() - t0
        info = b.info()
    for s in sims:
        s.close()
    g = cells * done / dt / 1e9
    # algorithmic bytes per step over all members (fused steps) against the L2
    # copy ceiling: the subsets are sized to stay in L2
    from aether_b200 import metrics as MT
    fused_ok = os.environ.get("AEFDTD_FUSED", "0") != "0"
    step_b = sum(MT.step_bytes(sc, A.FP32, fused=fused_ok) for sc in scenes)
    l2 = fdtd.copy_bandwidth(64 << 20, 50)
    l2_frac = step_b * done / dt / 1e9 / l2
    # the plain FP64 single-simulation path on the same cells: a seeded sample
    # of 8 cells, each stepped alone (its own graphs), timed on the device
    import torch
    single_cells = single_s = 0.0
    for sc in scenes[:: max(1, n_cells // 8)][:8]:
        sc.grid.precision = A.FP64
        with fdtd.build_simulation(sc) as s1:
            s1.step(3 * STEPS_PER_BENCH_STEP)      # warm-up: every graph of the run captured
            s1.synchronize()
            ext = torch.cuda.ExternalStream(s1.stream_ptr())
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(ext)
            s1.step(steps)
            e1.record(ext)
            e1.synchronize()
            single_s += e0.elapsed_time(e1) * 1e-3
            single_cells += sc.cells * steps
        sc.grid.precision = A.FP32
    g64 = single_cells / single_s / 1e9
    return {"workload": f"batch: {n_cells} nanodisk unit cells, FP32, {cells / 1e6:.1f} M cells in total",
            "gcells": g, "sims_per_s": n_cells / (dt * 8000.0 / done), "sample_steps": done, "seconds": dt,
            "subsets": info["n_subsets"], "setup_seconds": setup,
            "fp64_single_gcells": g64, "over_fp64_single_same_cells": g / g64,
            "bytes_per_step": step_b, "l2_copy_gbs": l2, "l2_frac": l2_frac,
            "l2_source": "aefdtd_probe_copy_bandwidth over a 64 MiB buffer (read + written bytes), this run",
            "note": "sims/s extrapolated from the timed sample to 8000 steps per cell; fp64_single_gcells: "
                    "8 of the cells stepped one at a time as plain FP64 simulations, device-timed"}


def serving_sample(n_jobs=32, rate=1.5, seed=77, fp64_check=8, **server_opts):
    """Serving: a seeded Poisson stream (rate jobs/s) of the batch sample's unit cells
    plus 10% large cells (period U(640, 1280) nm -> up to 256 x 256 cells,
    z = 384), step budgets U(4000, 20000), 101 wavelengths, FP32, served with
    continuous batching under an 80%-of-HBM budget. Jobs are submitted when
    their arrival time passes; the loop polls the server in between. A seeded
    sample of fp64_check jobs is re-run alone in FP64 (the path bit-identical
    to the reference core) for the R/T error."""
    import numpy as np
    from aether_b200 import _abi as A
    from aether_b200 import configs as CF
    from aether_b200 import fdtd
    rng = np.random.default_rng(seed)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, n_jobs))
    reqs = []
    for _ in range(n_jobs):
        large = rng.uniform() < 0.1
        steps = int(rng.integers(4000, 20001))
        if large:
            sc = CF.metasurface_cell(rng, precision=A.FP32, nsteps=steps, nl=101, nz_total=384,
                                     period_range=(640e-9, 1280e-9), flux_planes=False)
        else:
            sc = CF.metasurface_cell(rng, precision=A.FP32, nsteps=steps, nl=101, flux_planes=False)
        reqs.append((sc, steps, large))
    with fdtd.Server(**server_opts) as v:
        ids = [None] * n_jobs
        nxt = 0
        t0 = time.perf_counter()
        while True:
            now = time.perf_counter() - t0
            while nxt < n_jobs and arrivals[nxt] <= now:
                ids[nxt] = v.submit(reqs[nxt][0], reqs[nxt][1])
                nxt += 1
            st = v.stats()
            if nxt == n_jobs and st["queued"] == 0 and st["running"] == 0:
                break
            if st["queued"] == 0 and st["running"] == 0:
                time.sleep(max(0.0, min(0.05, arrivals[nxt] - now)))
                continue
            v.poll()
        st = v.stats()
        spectra = [v.spectra(j) for j in ids]
    # FP64 check on a seeded sample
    pick = sorted(np.random.default_rng(seed + 1).choice(n_jobs, size=min(fp64_check, n_jobs), replace=False))
    err = 0.0
    for k in pick:
        sc, steps, _ = reqs[k]
        sc.grid.precision = A.FP64
        with fdtd.build_simulation(sc) as s:
            s.step(steps)
            ref = s.normal_spectra()
        err = max(err, float(np.max(np.abs(spectra[k][:, 1:3] - ref[:, 1:3]))))
    cu = sum(sc.cells * steps for sc, steps, _ in reqs)
    return {"workload": f"serving: {n_jobs} Poisson arrivals at {rate}/s, 10% large cells, steps U(4000, 20000), "
                        "FP32, 80% HBM budget",
            "p50_s": st["p50_s"], "p99_s": st["p99_s"], "mean_s": st["mean_s"], "sims_per_s": st["sims_per_s"],
            "gcells": st["gcells_per_s"], "elapsed_s": st["elapsed_s"], "peak_bytes": st["peak_bytes"],
            "budget_bytes": st["budget_bytes"], "cell_updates": cu, "large_jobs": int(sum(r[2] for r in reqs)),
            "rt_abs_err_vs_fp64": err, "fp64_sample_jobs": [int(k) for k in pick]}


def large_grid_sample(steps=128, seed=1234):
    """Large grid: 1024 x 1024 x 512 cells at 5 nm, 32-cell CPML on all six
    faces, 500 seeded dielectric spheres (r U(20, 80) nm, eps U(2, 12)) plus 50
    Lorentz spheres sharing one material, an oscillator at the centre (600 nm,
    300 nm band), custom mode. FP32 and FP64: `steps` steps after a 64-step
    warm-up, timed with CUDA events on the simulation's stream (inputs far
    larger than L2)."""
    import torch
    from aether_b200 import _abi as A
    from aether_b200 import configs as CF
    from aether_b200 import fdtd
    from aether_b200 import metrics as MT
    peak, _ = measured_peaks()
    sc = CF.random_spheres_scene(seed=seed, precision=A.FP32)
    out = {"workload": "large grid: 1024x1024x512 @5nm, 32-cell CPML x6, 500 dielectric + 50 Lorentz spheres, "
                       "oscillator source"}
    for name, prec in (("fp32", A.FP32), ("fp64", A.FP64)):
        sc.grid.precision = prec
        t0 = time.perf_counter()
        sim = fdtd.build_simulation(sc)
        setup = time.perf_counter() - t0
        sim.step(STEPS_PER_BENCH_STEP)
        sim.synchronize()
        ext = torch.cuda.ExternalStream(sim.stream_ptr())
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(ext)
        sim.step(steps)
        e1.record(ext)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / steps
        sb = MT.step_bytes(sc, prec, fused=os.environ.get("AEFDTD_FUSED", "0") != "0")
        out[name] = {"gcells": sc.cells / (ms * 1e-3) / 1e9, "ms_per_step": ms,
                     "step_frac": sb / (ms * 1e-3) / 1e9 / peak, "bytes_per_step": sb,
                     "device_gb": sim.dims().device_bytes / 1e9, "setup_seconds": setup}
        sim.close()
        log(f"[large {name}] {out[name]['gcells']:.1f} Gcell/s, {out[name]['step_frac']:.2f} of HBM peak, "
            f"{out[name]['device_gb']:.1f} GB on the device")
    return out


def large_grid_cpu_crop(steps=8, seed=1234):
    """The reference core on a 256 x 256 x 128 crop of the large grid's scene
    (the same densities scaled to a 64x smaller grid: 12 dielectric spheres
    with their own indices, 3 Lorentz spheres sharing one, an oscillator,
    32-cell CPML on all six faces), FP64, `steps` steps timed on the host
    cores. The full 1024 x 1024 x 512 grid is out of reach for the reference:
    its setup scans the whole grid once per material index
    (FDTD_Material::link_grid, mats.cpp:394-443), 552 scans of 537 M cells."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import ctypes as C
    import oracle_lib
    from aether_b200 import _abi as A
    from aether_b200 import configs as CF
    which = "ref" if oracle_lib.available("ref") else "port"
    sc = CF.random_spheres_scene(n_total=(256, 256, 128), n_dielectric=12, n_lorentz=3, nsteps=5000, seed=seed,
                                 precision=A.FP64)
    r = oracle_lib.run(sc, which, nsteps=steps, want_fields=False)
    cores = int(C.CDLL(oracle_lib.REF_PATH).aeref_threads()) if which == "ref" else 1
    return {"value": sc.cells * steps / r["seconds"] / 1e9, "unit": METRIC, "cores": cores,
            "kind": "reference" if which == "ref" else "port",
            "sample": f"{steps} time steps of a 256x256x128 crop of the large grid's scene (same densities), "
                      f"time loop only, {r['seconds']:.2f} s"}


def profile_run(args):
    """The bench workload with every kernel launched directly (no CUDA graphs),
    for ncu launch lists and captures: `--segments` DFT blocks of 64 steps at
    precision `--profile`. Prints nothing on stdout."""
    os.environ["AEFDTD_NO_GRAPHS"] = "1"
    from aether_b200 import _abi as A
    from aether_b200 import configs as CF
    from aether_b200 import fdtd
    prec = A.FP32 if args.profile == "fp32" else A.FP64
    if args.profile_grid in ("batch", "batch-persistent"):
        # 8 of the batch sample's nanodisk cells, one subset each, 64 steps in one chunk of
        # direct launches (split groups, or one persistent launch per subset)
        import numpy as np
        rng = np.random.default_rng(2024)
        scenes = [CF.metasurface_cell(rng, precision=prec, nsteps=8000, nl=101, flux_planes=False)
                  for _ in range(8)]
        sims = [fdtd.build_simulation(sc) for sc in scenes]
        with fdtd.Batch(l2_budget_bytes=48 << 20, tile_y=4, kchunk=8, lanes=1, use_graphs=False,
                        persistent=args.profile_grid == "batch-persistent") as b:
            for s in sims:
                b.add(s, STEPS_PER_BENCH_STEP * args.segments)
            b.run(STEPS_PER_BENCH_STEP * args.segments)
            log(f"profile run: batch of 8 cells, {args.profile}, {b.info()['launches']} launches")
        for s in sims:
            s.close()
        return
    if args.profile_grid == "large":
        # the large grid's scene at 384 x 384 x 192 (CPML on six faces, spheres, oscillator)
        sc = CF.random_spheres_scene(n_total=(384, 384, 192), n_dielectric=60, n_lorentz=6, seed=1234,
                                     precision=prec)
    else:
        sc = workload(prec)
    sim = fdtd.build_simulation(sc)
    sim.step(STEPS_PER_BENCH_STEP * args.segments)
    sim.synchronize()
    log(f"profile run: {args.profile}, {STEPS_PER_BENCH_STEP * args.segments} steps, {sim.launch_count()} launches")
    sim.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="aefdtd")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the batch sample (512 nanodisk unit cells)")
    ap.add_argument("--no-large", action="store_true", help="skip the 1024x1024x512 large-grid sample")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving sample (Poisson stream of unit cells)")
    ap.add_argument("--no-accuracy", action="store_true", help="skip the FP32-vs-FP64 spectrum error runs")
    ap.add_argument("--profile", choices=["fp32", "fp64"], help="direct-launch run for ncu (no timing)")
    ap.add_argument("--segments", type=int, default=2)
    ap.add_argument("--profile-grid", choices=["bench", "large", "batch", "batch-persistent"], default="bench",
                    help="--profile on the bench grid, on the large grid's scene at 384 x 384 x 192, or on a "
                         "batch of 8 nanodisk cells (split or persistent launches)")
    args = ap.parse_args()
    if args.profile:
        profile_run(args)
        return
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        reference_arm(args)
        return

    res, ws, rank = run_gpu_arm(args)
    if rank != 0:
        return
    from aether_b200 import _abi as A
    r32, r64 = res["fp32"], res["fp64"]
    peak, peak_kind = measured_peaks()

    def interior_roofline(r, s, kernel, traffic_key):
        # dominant kernel: the interior group (fused step, or the E half-step's curl update)
        ms, cells = r["groups"][("E", "interior")]
        per = (12 if r["fused"] else 9) * s + r["bytes"]["detail"]["id_bytes"]
        b = cells * per
        ach = b / (ms * 1e-3) / 1e9
        if r["fused"]:
            kernel = f"yee_fused<{'double' if s == 8 else 'float'}, uint8, 0>"
            traffic_key = ("yee_fused", "fp64" if s == 8 else "fp32")
        elif r["staged"]:
            kernel = f"interior_tma<{'double' if s == 8 else 'float'}, uint8, E>"
            traffic_key = ("interior_tma", "fp64" if s == 8 else "fp32")
        return {"bound": "hbm", "kernel": kernel, "achieved": ach, "peak": peak, "unit": "GB/s",
                "frac": ach / peak, "peak_source": peak_kind, "traffic": profiled_traffic(*traffic_key),
                "algorithmic_bytes_per_launch": b, "launch_us": ms * 1e3, "cells_per_launch": cells,
                "source": "CUDA events around each launch on the simulation's stream in a 64-step "
                          f"group-timing pass after the timed region; bytes = cells x "
                          + (f"(12 x {s} + id bytes): six fields read and six written once per fused step"
                             if r["fused"] else f"(9 x {s} + id bytes)")}

    def step_roofline(r):
        a = r["step_bytes"] / (r["ms_per_step"] * 1e-3 / STEPS_PER_BENCH_STEP) / 1e9
        return {"achieved": a, "peak": peak, "unit": "GB/s", "frac": a / peak, "bytes_per_step": r["step_bytes"],
                "note": "algorithmic bytes of a whole time step (E, H, sensor samples, 1/64 of each DFT block) "
                        "over the graph-replay step time of the timed region"}

    def kernel_split(r):
        return {"e": r["e_ms"] * 1e3, "h": r["h_ms"] * 1e3, "sensors": r["s_ms"] * 1e3,
                "groups": {f"{h}/{g}": round(v[0] * 1e3, 2) for (h, g), v in r["groups"].items() if v[1] > 0},
                "source": "phases: CUDA events between the joined branches of each phase in a 128-step timing "
                          "pass; groups: each group alone between events in a 64-step pass"}

    line = {
        "metric": METRIC, "value": r64["gcells"], "unit": METRIC, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": r64["ms_per_step"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_dict(ws),
        "step": f"{STEPS_PER_BENCH_STEP} FDTD time steps (one DFT block) per bench step",
        "roofline": interior_roofline(r64, 8, "e_interior<double, uint8, 2>", ("e_interior", "fp64")),
        "step_roofline": step_roofline(r64),
        "kernel_us_per_time_step": kernel_split(r64),
        "gpu_launches": r64["launches"],
        "clocks": r64["clocks"],
        "fp32": {"value": r32["gcells"], "unit": METRIC, "ms_per_step": r32["ms_per_step"], "dtype": "f32",
                 "over_fp64": r32["gcells"] / r64["gcells"],
                 "roofline": interior_roofline(r32, 4, "e_interior_v2<float, uint8, false>", ("e_interior_v2", "fp32")),
                 "step_roofline": step_roofline(r32), "kernel_us_per_time_step": kernel_split(r32),
                 "gpu_launches": r32["launches"], "clocks": r32["clocks"]},
    }
    if not args.no_e2e:
        for prec, where in ((A.FP64, line), (A.FP32, line["fp32"])):
            e2e_job(prec, 2 * STEPS_PER_BENCH_STEP)        # warm-up: module load, first captures
            dt, h2d, d2h, cells = e2e_job(prec, 20000)
            where["e2e"] = {"value": cells * 20000 / dt / 1e9, "unit": METRIC, "h2d_bytes_per_step": h2d,
                            "d2h_bytes_per_step": d2h,
                            "step": "one complete 20000-step job through the public API from host buffers "
                                    "(geometry and materials uploaded, all steps, spectra and flux read back)",
                            "seconds": dt}
    if not args.no_accuracy:
        line["fp32"]["spectrum_error"] = spectrum_error_sample()
    if not args.no_large:
        line["large_grid"] = large_grid_sample()
        if not args.no_cpu:
            try:
                line["large_grid"]["cpu_reference_crop"] = large_grid_cpu_crop()
                c = line["large_grid"]["cpu_reference_crop"]
                line["large_grid"]["fp64"]["over_cpu_reference"] = line["large_grid"]["fp64"]["gcells"] / c["value"]
            except Exception as e:  # pragma: no cover
                line["large_grid"]["cpu_reference_crop"] = {"value": None, "error": str(e)}
    if not args.no_batch:
        line["batch"] = batch_sample()
        line["batch"]["over_fp64_single"] = line["batch"]["gcells"] / r64["gcells"]
        log(f"[batch] {line['batch']['gcells']:.2f} Gcell/s, {line['batch']['sims_per_s']:.2f} sims/s, "
            f"{line['batch']['over_fp64_single_same_cells']:.2f}x the plain FP64 single simulations of the same cells")
    if not args.no_serving:
        line["serving"] = serving_sample()
        sv = line["serving"]
        log(f"[serving] p50 {sv['p50_s']:.2f} s p99 {sv['p99_s']:.2f} s, {sv['sims_per_s']:.2f} sims/s, "
            f"{sv['gcells']:.1f} Gcell/s, R/T err {sv['rt_abs_err_vs_fp64']:.2e}")
    if not args.no_cpu:
        try:
            line["cpu_baseline"] = cpu_baseline(workload)
        except Exception as e:  # pragma: no cover
            line["cpu_baseline"] = {"value": None, "error": str(e)}
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
