"""Simulation handle over the C ABI, and `run(scene)` — the counterpart of the
reference mode drivers FDTD_normal_incidence / mode_default_fdtd
(src/finite_differences/FDTD/modes/normal_incidence.cpp:161-607,
default_fdtd.cpp:24-210) for a Scene."""
from __future__ import annotations

import ctypes as C
import time

import numpy as np

from . import _abi as A
from ._lib import AefdtdError, check, load

_P = C.POINTER


class Simulation:
    """One FDTD grid on one GPU (the reference's `FDTD` object plus its mode
    driver's sensors and sources)."""

    def __init__(self, grid: A.GridDesc):
        self._lib = load()
        self._h = C.c_void_p()
        st = self._lib.aefdtd_create(C.byref(grid), C.byref(self._h))
        check(st, None)
        self.grid = grid
        self.sensor_nl = []

    # -- lifecycle
    def close(self):
        if self._h:
            self._lib.aefdtd_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _c(self, st):
        check(st, self._h)

    # -- setup
    def dims(self) -> A.Dims:
        d = A.Dims()
        self._c(self._lib.aefdtd_get_dims(self._h, C.byref(d)))
        return d

    def set_material_map(self, m: np.ndarray):
        m = np.ascontiguousarray(m, dtype=np.uint32)
        self._c(self._lib.aefdtd_set_material_map(self._h, m.ctypes.data_as(_P(C.c_uint32)), m.size))

    def set_material(self, idx: int, mat: A.MaterialDesc):
        self._c(self._lib.aefdtd_set_material(self._h, idx, C.byref(mat)))

    def setup_normal(self, nd: A.NormalDesc):
        self._c(self._lib.aefdtd_setup_normal(self._h, C.byref(nd)))
        self.normal_nl = nd.nl

    def add_oscillator(self, src: A.SourceDesc) -> int:
        i = C.c_int32()
        self._c(self._lib.aefdtd_add_oscillator(self._h, C.byref(src), C.byref(i)))
        return i.value

    def add_planar_sensor(self, s: A.SensorDesc) -> int:
        i = C.c_int32()
        self._c(self._lib.aefdtd_add_planar_sensor(self._h, C.byref(s), C.byref(i)))
        self.sensor_nl.append(s.nl)
        return i.value

    # -- stepping
    def step(self, n: int):
        self._c(self._lib.aefdtd_step(self._h, int(n)))

    def synchronize(self):
        self._c(self._lib.aefdtd_synchronize(self._h))

    def reset(self):
        self._c(self._lib.aefdtd_reset(self._h))

    def add_box_sensor(self, box, nl, lambda_min, lambda_max, disabled=0) -> int:
        """Box spectral Poynting sensor: six planar faces (bits of `disabled`:
        xm, xp, ym, yp, zm, zp); returns the box id."""
        d = A.BoxSensorDesc()
        for k in range(6):
            d.box[k] = int(box[k])
        d.nl, d.disabled = int(nl), int(disabled)
        d.lambda_min, d.lambda_max = float(lambda_min), float(lambda_max)
        bid = C.c_int32(-1)
        self._c(self._lib.aefdtd_add_box_sensor(self._h, C.byref(d), C.byref(bid)))
        self.box_nl = getattr(self, "box_nl", {})
        self.box_nl[bid.value] = int(nl)
        return bid.value

    def box_flux(self, bid: int) -> np.ndarray:
        nl = self.box_nl[bid]
        out = np.empty(nl)
        self._c(self._lib.aefdtd_get_box_flux(self._h, int(bid), out.ctypes.data_as(C.POINTER(C.c_double)), nl))
        return out

    def add_fieldmap(self, kind, box, lambda_=0.0, orientation=A.NORMAL_Z, cumulative=False,
                     magnetic=False) -> int:
        """Single-wavelength field sensor (include/aefdtd.h, aefdtd_add_fieldmap):
        kind MAP_PLANE (FieldMap), MAP_BLOCK (FieldBlock) or MAP_POINT
        (FieldPoint); box in structure cells; returns the map id."""
        d = A.FieldMapDesc()
        d.kind, d.orientation = int(kind), int(orientation)
        for k in range(6):
            d.box[k] = int(box[k])
        d.cumulative, d.magnetic, d.lambda_ = int(bool(cumulative)), int(bool(magnetic)), float(lambda_)
        mid = C.c_int32(-1)
        self._c(self._lib.aefdtd_add_fieldmap(self._h, C.byref(d), C.byref(mid)))
        self._map_kinds = getattr(self, "_map_kinds", {})
        self._map_kinds[mid.value] = int(kind)
        return mid.value

    def fieldmap(self, mid: int) -> np.ndarray:
        """Plane maps: complex (3, span2, span1); blocks: complex (6, span3,
        span2, span1); points: (steps, 3) real E."""
        sh = (C.c_int32 * 4)()
        self._c(self._lib.aefdtd_get_fieldmap_shape(self._h, int(mid), sh))
        s1, s2, s3, nc = sh[0], sh[1], sh[2], sh[3]
        kind = getattr(self, "_map_kinds", {}).get(int(mid), A.MAP_PLANE)
        shape = (s1, 3) if kind == A.MAP_POINT else (nc, s3, s2, s1, 2)
        out = np.empty(shape)
        self._c(self._lib.aefdtd_get_fieldmap(self._h, int(mid), out.ctypes.data_as(C.POINTER(C.c_double)),
                                              out.size))
        if kind == A.MAP_POINT:
            return out
        z = out[..., 0] + 1j * out[..., 1]
        return z[:, 0] if kind == A.MAP_PLANE else z

    def set_completion(self, coeff=1e-3, check_every=500):
        """Energy-mode completion sensor (coeff <= 0: off)."""
        self._c(self._lib.aefdtd_set_completion(self._h, float(coeff), int(check_every)))

    def set_completion_ft(self, lambda_min, lambda_max, coeff=1e-3, n_points=500, layout="nnb", seed=0,
                          check_every=500):
        """FT-mode completion sensor: probes on the faces named by layout, std::mt19937(seed) draws."""
        self._c(self._lib.aefdtd_set_completion_ft(self._h, float(lambda_min), float(lambda_max), float(coeff),
                                                   int(n_points), layout.encode(), int(seed), int(check_every)))

    def completion(self):
        """(done, stop step t or -1, last/max energy at the last check)."""
        d, t, r = C.c_int32(), C.c_int32(), C.c_double()
        self._c(self._lib.aefdtd_get_completion(self._h, C.byref(d), C.byref(t), C.byref(r)))
        return bool(d.value), t.value, r.value

    def group_timings(self):
        """Mode-2 timing: {(half, group): (ms per step, cells)}; half 'E'/'H',
        group 'interior'/'pml_z'/'dispersive'/'general'/'pml_xy'."""
        names = ["interior", "pml_z", "dispersive", "general", "pml_xy"]
        G = len(names)
        ms = (C.c_double * (2 * G))()
        cells = (C.c_int64 * (2 * G))()
        self._c(self._lib.aefdtd_get_group_timings(self._h, ms, cells, 2 * G))
        return {(h, names[g]): (ms[i * G + g], cells[i * G + g]) for i, h in enumerate("EH") for g in range(G)}

    def enable_timing(self, on=True, mode=1):
        """mode 1: per phase; mode 2: per work-item group (groups in order)."""
        self._c(self._lib.aefdtd_enable_timing(self._h, int(mode) if on else 0))

    def timings(self):
        e, h, s = C.c_double(), C.c_double(), C.c_double()
        self._c(self._lib.aefdtd_get_timings(self._h, C.byref(e), C.byref(h), C.byref(s)))
        return e.value, h.value, s.value

    def stream_ptr(self) -> int:
        p = C.c_void_p()
        self._c(self._lib.aefdtd_get_stream(self._h, C.byref(p)))
        return p.value or 0

    def launch_count(self) -> int:
        n = C.c_uint64()
        self._c(self._lib.aefdtd_get_launch_count(self._h, C.byref(n)))
        return n.value

    # -- results
    def field(self, comp: int) -> np.ndarray:
        d = self.dims()
        out = np.empty(d.nx * d.ny * d.nz)
        self._c(self._lib.aefdtd_get_field(self._h, comp, out.ctypes.data_as(_P(C.c_double)), out.size))
        return out.reshape(d.nz, d.ny, d.nx)

    def fields(self, grid: int = 0) -> np.ndarray:
        """Ex..Hz; grid 1: the imaginary grid of the oblique driver."""
        return np.stack([self.field(6 * grid + c) for c in range(6)])

    def setup_oblique(self, od):
        self._c(self._lib.aefdtd_setup_oblique(self._h, C.byref(od)))
        self._obl_nl = int(od.nl)

    def oblique_spectra(self) -> np.ndarray:
        """(nl', 10): lambda, angle (deg), |r_TE|, arg, |r_TM|, arg, |t_TE|, arg, |t_TM|, arg."""
        out = np.empty((self._obl_nl, 10))
        n = C.c_int32(0)
        self._c(self._lib.aefdtd_get_oblique_spectra(self._h, out.ctypes.data_as(_P(C.c_double)), self._obl_nl,
                                                     C.byref(n)))
        return out[:n.value]

    def oblique_series(self) -> np.ndarray:
        """(steps, 18): BR, R, T sums (x, y, z as re, im) per step."""
        n = self.dims().step
        out = np.empty((n, 18))
        self._c(self._lib.aefdtd_get_oblique_series(self._h, out.ctypes.data_as(_P(C.c_double)), out.size))
        return out

    def set_field(self, comp: int, values: np.ndarray):
        v = np.ascontiguousarray(values, dtype=np.float64).ravel()
        self._c(self._lib.aefdtd_set_field(self._h, comp, v.ctypes.data_as(_P(C.c_double)), v.size))

    def plane_sums(self) -> np.ndarray:
        n = self.dims().step
        out = np.empty(12 * n)
        self._c(self._lib.aefdtd_get_plane_sums(self._h, out.ctypes.data_as(_P(C.c_double)), n))
        return out.reshape(12, n)

    def normal_spectra(self) -> np.ndarray:
        out = np.empty(15 * self.normal_nl)
        self._c(self._lib.aefdtd_get_normal_spectra(self._h, out.ctypes.data_as(_P(C.c_double)), self.normal_nl))
        return out.reshape(self.normal_nl, 15)

    def sensor_flux(self, sid: int) -> np.ndarray:
        nl = self.sensor_nl[sid]
        out = np.empty(nl)
        self._c(self._lib.aefdtd_get_sensor_flux(self._h, sid, out.ctypes.data_as(_P(C.c_double)), nl))
        return out

    def sensor_dft(self, sid: int) -> np.ndarray:
        s1, s2, nl = C.c_int32(), C.c_int32(), C.c_int32()
        self._c(self._lib.aefdtd_get_sensor_shape(self._h, sid, C.byref(s1), C.byref(s2), C.byref(nl)))
        out = np.empty(6 * s1.value * s2.value * nl.value * 2)
        self._c(self._lib.aefdtd_get_sensor_dft(self._h, sid, out.ctypes.data_as(_P(C.c_double)), out.size))
        z = out.view(np.complex128)
        return z.reshape(6, nl.value, s2.value, s1.value)


def device_memory(device: int = 0):
    """(free, total) bytes of a device (aefdtd_device_memory)."""
    lib = load()
    fr, tot = C.c_size_t(), C.c_size_t()
    check(lib.aefdtd_device_memory(device, C.byref(fr), C.byref(tot)))
    return fr.value, tot.value


def copy_bandwidth(nbytes=64 << 20, reps=50, device=0) -> float:
    """Copy bandwidth (read + written GB/s) of a device over an nbytes buffer
    (aefdtd_probe_copy_bandwidth): below the L2 size, the L2 ceiling."""
    lib = load()
    v = C.c_double()
    check(lib.aefdtd_probe_copy_bandwidth(device, nbytes, reps, C.byref(v)))
    return v.value


def build_simulation(scene) -> Simulation:
    """Creates the device simulation of a Scene (grid, map, materials,
    excitation, sensors), in the order of the reference drivers."""
    sim = Simulation(scene.grid)
    try:
        sim.set_material_map(scene.map)
        for i, m in enumerate(scene.materials):
            sim.set_material(i, m)
        if scene.grid.mode == A.MODE_NORMAL:
            sim.setup_normal(scene.normal)
        if scene.grid.mode == A.MODE_OBLIQUE:
            sim.setup_oblique(scene.oblique)
        for s in scene.sources:
            sim.add_oscillator(s)
        for s in scene.sensors:
            sim.add_planar_sensor(s)
    except Exception:
        sim.close()
        raise
    return sim


def run(scene, nsteps=None, want_fields=True):
    """Runs a Scene on the GPU and returns the same dict as the oracle
    runner: fields (6, nz, ny, nx) as float64, plane_sums, spectra, flux,
    dims, seconds (device time of the steps, host clock)."""
    nsteps = scene.nsteps if nsteps is None else nsteps
    with build_simulation(scene) as sim:
        t0 = time.perf_counter()
        sim.step(nsteps)
        sim.synchronize()
        secs = time.perf_counter() - t0
        d = sim.dims()
        out = {"dims": np.array([d.nx, d.ny, d.nz, d.xs_s, d.xs_e, d.ys_s, d.ys_e, d.zs_s, d.zs_e, d.n_materials]),
               "seconds": secs}
        out["fields"] = sim.fields() if want_fields else None
        if scene.grid.mode == A.MODE_NORMAL:
            out["plane_sums"] = sim.plane_sums()
            out["spectra"] = sim.normal_spectra() if nsteps >= 2 else None
        elif scene.grid.mode == A.MODE_OBLIQUE:
            out["fields_imag"] = sim.fields(1) if want_fields else None
            out["plane_sums"] = sim.oblique_series()
            out["spectra"] = sim.oblique_spectra() if nsteps >= 2 else None
        else:
            out["plane_sums"] = None
            out["spectra"] = None
        out["flux"] = [sim.sensor_flux(i) for i in range(len(scene.sensors))]
        out["launches"] = sim.launch_count()
        return out


class Batch:
    """Many simulations advanced together (include/aefdtd.h, aefdtd_batch_*):
    merged launches per work-item group over all members of an L2-sized
    subset, one captured graph per subset and segment; with persistent=True
    each chunk of a subset is one persistent cooperative launch instead. Members are ordinary
    Simulations (normal, custom or oblique mode; a completion sensor, set
    before they join, ends them at their completion step); the batch keeps
    references to them while they are members."""

    def __init__(self, l2_budget_bytes=0, tile_y=0, kchunk=0, use_graphs=True, device=0, graph_steps=0, lanes=0,
                 persistent=False):
        self._lib = load()
        o = A.BatchOpts()
        o.abi_version = A.ABI_VERSION
        o.device = device
        o.l2_budget_bytes = int(l2_budget_bytes)
        o.tile_y, o.kchunk = int(tile_y), int(kchunk)
        o.use_graphs = 0 if use_graphs else -1
        o.graph_steps = int(graph_steps)
        o.lanes = int(lanes)
        o.persistent = 1 if persistent else 0
        self._h = C.c_void_p()
        st = self._lib.aefdtd_batch_create(C.byref(o), C.byref(self._h))
        if st != 0:
            raise AefdtdError(st, "aefdtd_batch_create failed")
        self.members = {}

    def _c(self, st):
        if st != 0:
            msg = self._lib.aefdtd_batch_last_error(self._h)
            raise AefdtdError(st, msg.decode() if msg else "")

    def close(self):
        if self._h:
            self._lib.aefdtd_batch_destroy(self._h)
            self._h = C.c_void_p()
        self.members = {}

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def add(self, sim: Simulation, steps: int):
        self._c(self._lib.aefdtd_batch_add(self._h, sim._h, int(steps)))
        self.members[sim._h.value] = sim

    def remove(self, sim: Simulation):
        self._c(self._lib.aefdtd_batch_remove(self._h, sim._h))
        self.members.pop(sim._h.value, None)

    def set_budget(self, sim: Simulation, steps: int):
        self._c(self._lib.aefdtd_batch_set_budget(self._h, sim._h, int(steps)))

    def autotune(self):
        self._c(self._lib.aefdtd_batch_autotune(self._h))

    def advance(self, max_steps: int) -> int:
        done = C.c_int32(0)
        self._c(self._lib.aefdtd_batch_advance(self._h, int(max_steps), C.byref(done)))
        return done.value

    def run(self, max_steps: int) -> int:
        """Advances until every member used its budget (or max_steps)."""
        total = 0
        while total < max_steps:
            n = self.advance(max_steps - total)
            if n == 0:
                break
            total += n
        return total

    def finished(self):
        n = C.c_int32(0)
        self._c(self._lib.aefdtd_batch_finished(self._h, None, 0, C.byref(n)))
        if n.value == 0:
            return []
        arr = (C.c_void_p * n.value)()
        self._c(self._lib.aefdtd_batch_finished(self._h, arr, n.value, C.byref(n)))
        return [self.members[p] for p in arr[:n.value] if p in self.members]

    def info(self) -> dict:
        i = A.BatchInfo()
        self._c(self._lib.aefdtd_batch_get_info(self._h, C.byref(i)))
        k = min(i.n_classes, A.BATCH_MAX_CLASSES)
        return {"n_members": i.n_members, "n_active": i.n_active, "n_subsets": i.n_subsets, "n_lanes": i.n_lanes,
                "n_persistent": i.n_persistent,
                "cells": i.cells,
                "member_bytes": i.member_bytes, "batch_bytes": i.batch_bytes,
                "l2_budget_bytes": i.l2_budget_bytes, "launches": i.launches,
                "classes": [{"key": i.class_key[c], "tile_y": i.class_tile_y[c], "kchunk": i.class_kchunk[c]}
                            for c in range(k)]}


class Server:
    """The serving loop (include/aefdtd.h, aefdtd_server_*): jobs queue on the
    host, are admitted by device-memory footprint against a budget (80% of
    HBM by default), run as members of one batch and retire when done."""

    def __init__(self, hbm_fraction=0.0, budget_bytes=0, max_active=0, segment_steps=0, lookahead=0,
                 l2_budget_bytes=0, tile_y=0, kchunk=0, device=0):
        self._lib = load()
        o = A.ServerOpts()
        o.abi_version = A.ABI_VERSION
        o.device = device
        o.hbm_fraction = float(hbm_fraction)
        o.budget_bytes = int(budget_bytes)
        o.max_active, o.segment_steps, o.lookahead = int(max_active), int(segment_steps), int(lookahead)
        o.batch.l2_budget_bytes = int(l2_budget_bytes)
        o.batch.tile_y, o.batch.kchunk = int(tile_y), int(kchunk)
        self._h = C.c_void_p()
        st = self._lib.aefdtd_server_create(C.byref(o), C.byref(self._h))
        if st != 0:
            raise AefdtdError(st, "aefdtd_server_create failed")
        self.nl = {}

    def _c(self, st):
        if st != 0:
            msg = self._lib.aefdtd_server_last_error(self._h)
            raise AefdtdError(st, msg.decode() if msg else "")

    def close(self):
        if self._h:
            self._lib.aefdtd_server_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def submit(self, scene, steps=None, completion=None) -> int:
        """Queues a normal-incidence Scene for `steps` steps (default its own).
        completion=(coeff, check_every): energy-mode completion sensor; the
        job then ends at its completion step (info()['stop_step'])."""
        m = np.ascontiguousarray(scene.map, dtype=np.uint32).ravel()
        mats = (A.MaterialDesc * len(scene.materials))(*scene.materials)
        g = scene.grid
        nd = scene.normal
        jd = A.JobDesc()
        jd.grid = C.pointer(g)
        jd.map = m.ctypes.data_as(C.POINTER(C.c_uint32))
        jd.map_count = m.size
        jd.materials = mats
        jd.n_materials = len(scene.materials)
        jd.normal = C.pointer(nd)
        jd.steps = int(steps if steps is not None else scene.nsteps)
        if completion is not None:
            jd.cc_coeff, jd.cc_step = float(completion[0]), int(completion[1])
        jid = C.c_int32(-1)
        self._c(self._lib.aefdtd_server_submit(self._h, C.byref(jd), C.byref(jid)))
        self.nl[jid.value] = nd.nl
        return jid.value

    def poll(self) -> int:
        n = C.c_int32(0)
        self._c(self._lib.aefdtd_server_poll(self._h, C.byref(n)))
        return n.value

    def info(self, job: int) -> dict:
        i = A.JobInfo()
        self._c(self._lib.aefdtd_server_job_info(self._h, int(job), C.byref(i)))
        return {k: getattr(i, k) for k, _ in A.JobInfo._fields_}

    def spectra(self, job: int) -> np.ndarray:
        nl = self.nl[job]
        out = np.empty(15 * nl)
        self._c(self._lib.aefdtd_server_job_spectra(self._h, int(job), out.ctypes.data_as(C.POINTER(C.c_double)), nl))
        return out.reshape(nl, 15)

    def stats(self) -> dict:
        s = A.ServerStats()
        self._c(self._lib.aefdtd_server_get_stats(self._h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in A.ServerStats._fields_}

    def drain(self, max_polls=10 ** 7):
        """Polls until no job is queued or running."""
        for _ in range(max_polls):
            st = self.stats()
            if st["queued"] == 0 and st["running"] == 0:
                return
            self.poll()
