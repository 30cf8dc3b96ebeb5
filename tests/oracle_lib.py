"""Loads the oracle libraries (test infrastructure) and runs a Scene through
them.

  port: oracle/liboracle_fdtd.so — the CPU restatement (oracle/fdtd_oracle.cpp)
  ref:  oracle/_ref/libaeref.so — the reference's own FDTD core compiled from
        source by oracle/Makefile (only where it was built)
Both export the same entry point signature, so results are directly
comparable."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from aether_b200 import _abi as A

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PORT_PATH = os.path.join(ROOT, "oracle", "liboracle_fdtd.so")
REF_PATH = os.path.join(ROOT, "oracle", "_ref", "libaeref.so")

_P = C.POINTER
_libs = {}


def _bind(path, sym):
    lib = C.CDLL(path)
    fn = getattr(lib, sym)
    fn.argtypes = [_P(A.GridDesc), _P(C.c_uint32), _P(A.MaterialDesc), C.c_int32, _P(A.NormalDesc),
                   _P(A.SourceDesc), C.c_int32, _P(A.SensorDesc), C.c_int32, C.c_int32, C.c_int32,
                   _P(C.c_double), _P(C.c_double), _P(C.c_double), _P(C.c_double), _P(C.c_int32),
                   _P(C.c_double)]
    fn.restype = C.c_int
    return lib, fn


def available(which: str) -> bool:
    return os.path.exists(PORT_PATH if which == "port" else REF_PATH)


def get(which: str):
    if which not in _libs:
        if which == "port":
            _libs[which] = _bind(PORT_PATH, "aeoracle_run")
        elif which == "ref":
            _libs[which] = _bind(REF_PATH, "aeref_run")
        else:
            raise ValueError(which)
    return _libs[which][1]


def _dptr(a):
    return None if a is None else a.ctypes.data_as(_P(C.c_double))


def run(scene, which="port", nsteps=None, want_fields=True):
    """Runs the scene for nsteps (default scene.nsteps) and returns a dict with
    fields (6, nz, ny, nx), plane_sums (12, nsteps), spectra (nl, 15), flux
    (list per sensor), dims (10,), seconds."""
    fn = get(which)
    nsteps = scene.nsteps if nsteps is None else nsteps
    nx, ny, nz = scene.total_dims()
    ntot = nx * ny * nz
    fields = np.zeros(6 * ntot) if want_fields else None
    ps = np.zeros(12 * max(nsteps, 1)) if scene.normal is not None else None
    nl = scene.normal.nl if scene.normal is not None else 0
    spectra = np.zeros(15 * nl) if scene.normal is not None else None
    nflux = sum(s.nl for s in scene.sensors)
    flux = np.zeros(max(nflux, 1))
    dims = (C.c_int32 * 10)()
    secs = C.c_double(0)
    mats = (A.MaterialDesc * len(scene.materials))(*scene.materials)
    sens = (A.SensorDesc * max(len(scene.sensors), 1))(*scene.sensors) if scene.sensors else None
    srcs = (A.SourceDesc * max(len(scene.sources), 1))(*scene.sources) if scene.sources else None
    rc = fn(C.byref(scene.grid), scene.map.ctypes.data_as(_P(C.c_uint32)), mats, len(scene.materials),
            C.byref(scene.normal) if scene.normal is not None else None,
            srcs, len(scene.sources), sens, len(scene.sensors), nsteps, 1,
            _dptr(fields), _dptr(ps), _dptr(spectra), _dptr(flux), dims, C.byref(secs))
    if rc != 0:
        raise RuntimeError(f"{which} oracle run failed with code {rc}")
    d = list(dims)
    assert (d[0], d[1], d[2]) == (nx, ny, nz), (d, (nx, ny, nz))
    out = {"dims": np.array(d), "seconds": secs.value}
    out["fields"] = fields.reshape(6, nz, ny, nx) if want_fields else None
    out["plane_sums"] = ps.reshape(12, nsteps) if ps is not None else None
    out["spectra"] = spectra.reshape(nl, 15) if spectra is not None else None
    fl, off = [], 0
    for s in scene.sensors:
        fl.append(flux[off:off + s.nl].copy())
        off += s.nl
    out["flux"] = fl
    return out


def run_ref_completion(scene, coeff, every, nsteps=None):
    """The reference core with its energy-mode CompletionSensor(coeff), checked
    every `every` steps (normal mode): the run dict of `run` plus 'stop' (the
    completion step t, or -1) and the last and largest grid energies."""
    lib = C.CDLL(REF_PATH)
    lib.aeref_set_completion.argtypes = [C.c_double, C.c_int32]
    lib.aeref_completion_result.argtypes = [_P(C.c_int32), _P(C.c_double), _P(C.c_double)]
    lib.aeref_set_completion(coeff, every)
    try:
        out = run(scene, "ref", nsteps=nsteps, want_fields=True)
        stop, last, mx = C.c_int32(), C.c_double(), C.c_double()
        lib.aeref_completion_result(C.byref(stop), C.byref(last), C.byref(mx))
    finally:
        lib.aeref_set_completion(0.0, 500)
    out.update(stop=stop.value, energy_last=last.value, energy_max=mx.value)
    return out


def run_ref_completion_ft(scene, lmin, lmax, coeff, n_points, layout, seed, every, nsteps=None):
    """As run_ref_completion with the FT-mode CompletionSensor(lmin, lmax,
    coeff, n_points, layout), the reference's generator reseeded with seed."""
    lib = C.CDLL(REF_PATH)
    lib.aeref_set_completion_ft.argtypes = [C.c_double, C.c_double, C.c_double, C.c_int32, C.c_char_p, C.c_int32,
                                            C.c_int32]
    lib.aeref_set_completion.argtypes = [C.c_double, C.c_int32]
    lib.aeref_completion_result.argtypes = [_P(C.c_int32), _P(C.c_double), _P(C.c_double)]
    lib.aeref_set_completion_ft(lmin, lmax, coeff, n_points, layout.encode(), seed, every)
    try:
        out = run(scene, "ref", nsteps=nsteps, want_fields=True)
        stop, last, mx = C.c_int32(), C.c_double(), C.c_double()
        lib.aeref_completion_result(C.byref(stop), C.byref(last), C.byref(mx))
    finally:
        lib.aeref_set_completion(0.0, 500)
    out.update(stop=stop.value)
    return out


def run_ref_box(scene, box, nl, lambda_min, lambda_max, disabled=0, nsteps=None):
    """The reference core with one Box_Spect_Poynting sensor: the run dict of
    `run` plus 'box_flux' (its rsp_result, nl values)."""
    lib = C.CDLL(REF_PATH)
    lib.aeref_set_box.argtypes = [_P(C.c_int32), C.c_int32, C.c_double, C.c_double, C.c_int32]
    lib.aeref_box_result.argtypes = [_P(C.c_double), C.c_int32]
    b = (C.c_int32 * 6)(*box)
    lib.aeref_set_box(b, nl, lambda_min, lambda_max, disabled)
    try:
        out = run(scene, "ref", nsteps=nsteps, want_fields=False)
        res = np.zeros(nl)
        assert lib.aeref_box_result(res.ctypes.data_as(_P(C.c_double)), nl) == 0
    finally:
        lib.aeref_set_box(None, 0, 0.0, 0.0, 0)
    out["box_flux"] = res
    return out


def run_ref_fieldmaps(scene, maps, nsteps=None):
    """The reference core with FieldMap / FieldBlock / FieldPoint sensors
    (maps: list of aefdtd FieldMapDesc): the run dict of `run` plus 'maps',
    one flat float64 array per sensor in the aefdtd_get_fieldmap layout."""
    lib = C.CDLL(REF_PATH)
    lib.aeref_set_fieldmaps.argtypes = [_P(A.FieldMapDesc), C.c_int32]
    lib.aeref_fieldmap_result.argtypes = [C.c_int32, _P(C.c_double), C.c_int64]
    lib.aeref_fieldmap_result.restype = C.c_int64
    arr = (A.FieldMapDesc * max(1, len(maps)))(*maps)
    lib.aeref_set_fieldmaps(arr, len(maps))
    try:
        out = run(scene, "ref", nsteps=nsteps, want_fields=False)
        res = []
        for i in range(len(maps)):
            n = lib.aeref_fieldmap_result(i, None, 0)
            v = np.zeros(max(n, 0))
            lib.aeref_fieldmap_result(i, v.ctypes.data_as(_P(C.c_double)), n)
            res.append(v)
    finally:
        lib.aeref_set_fieldmaps(arr, 0)
    out["maps"] = res
    return out


def ref_threads():
    """Worker threads per sensor and FDTD object in the reference core."""
    lib = C.CDLL(REF_PATH)
    lib.aeref_threads.restype = C.c_int
    return int(lib.aeref_threads())


def run_ref_oblique(scene, nsteps=None, want_fields=True):
    """The reference's oblique driver (two OBL_PHASE grids, Bloch_Wideband)
    on an oblique Scene: dict with fields (6, nz, ny, nx) of the real grid,
    fields_imag, series (nsteps, 18), spectra (nl', 10), dims, seconds."""
    lib = C.CDLL(REF_PATH)
    fn = lib.aeref_run_oblique
    fn.argtypes = [_P(A.GridDesc), _P(C.c_uint32), _P(A.MaterialDesc), C.c_int32, _P(A.ObliqueDesc), C.c_int32,
                   C.c_int32, _P(C.c_double), _P(C.c_double), _P(C.c_double), C.c_int32, _P(C.c_int32),
                   _P(C.c_int32), _P(C.c_double)]
    fn.restype = C.c_int
    nsteps = scene.nsteps if nsteps is None else nsteps
    nx, ny, nz = scene.total_dims()
    ntot = nx * ny * nz
    fields = np.zeros(12 * ntot) if want_fields else None
    series = np.zeros(18 * max(nsteps, 1))
    nl = scene.oblique.nl
    spectra = np.zeros(10 * nl)
    nl_out = C.c_int32(0)
    dims = (C.c_int32 * 10)()
    secs = C.c_double(0)
    mats = (A.MaterialDesc * len(scene.materials))(*scene.materials)
    rc = fn(C.byref(scene.grid), scene.map.ctypes.data_as(_P(C.c_uint32)), mats, len(scene.materials),
            C.byref(scene.oblique), nsteps, 1, _dptr(fields), _dptr(series), _dptr(spectra), nl, C.byref(nl_out),
            dims, C.byref(secs))
    if rc != 0:
        raise RuntimeError(f"reference oblique run failed with code {rc}")
    out = {"dims": np.array(list(dims)), "seconds": secs.value}
    if want_fields:
        f = fields.reshape(2, 6, nz, ny, nx)
        out["fields"], out["fields_imag"] = f[0], f[1]
    out["series"] = series[:18 * nsteps].reshape(nsteps, 18)
    out["spectra"] = spectra.reshape(nl, 10)[:nl_out.value]
    return out


def ref_discretize(nx, ny, nz, d, ops, desc):
    """The reference's own Structure::discretize (oracle/_ref) on the given
    operations and structure settings; (nz, ny, nx) uint32 map."""
    lib = C.CDLL(REF_PATH)
    fn = lib.aeref_discretize
    fn.argtypes = [C.c_int32] * 3 + [C.c_double] * 3 + [_P(A.StructureOp), C.c_int32, _P(A.StructureDesc),
                                                      _P(C.c_uint32)]
    out = np.zeros(nx * ny * nz, np.uint32)
    arr = (A.StructureOp * max(len(ops), 1))(*ops)
    rc = fn(nx, ny, nz, d[0], d[1], d[2], arr, len(ops), C.byref(desc), out.ctypes.data_as(_P(C.c_uint32)))
    if rc != 0:
        raise RuntimeError(f"reference discretize failed with code {rc}")
    return out.reshape(nz, ny, nx)
