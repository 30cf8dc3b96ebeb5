"""ctypes binding of the CUDA library aether_b200/libaefdtd.so (include/aefdtd.h).

The library is the only compute path: if it is missing, loading fails with an
error naming the build command; if no CUDA device is visible, its calls return
AEFDTD_NO_DEVICE and the wrappers raise."""
from __future__ import annotations

import ctypes as C
import os

from . import _abi as A

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libaefdtd.so")

_P = C.POINTER
_lib = None

# name -> (restype, argtypes)
_SIGS = {
    "aefdtd_create": (C.c_int, [_P(A.GridDesc), _P(C.c_void_p)]),
    "aefdtd_destroy": (C.c_int, [C.c_void_p]),
    "aefdtd_get_dims": (C.c_int, [C.c_void_p, _P(A.Dims)]),
    "aefdtd_last_error": (C.c_char_p, [C.c_void_p]),
    "aefdtd_status_string": (C.c_char_p, [C.c_int]),
    "aefdtd_set_material_map": (C.c_int, [C.c_void_p, _P(C.c_uint32), C.c_size_t]),
    "aefdtd_set_material": (C.c_int, [C.c_void_p, C.c_uint32, _P(A.MaterialDesc)]),
    "aefdtd_voxelize": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_double, C.c_double,
                                  C.c_double, _P(A.StructureOp), C.c_int32, C.c_int32, _P(C.c_int32),
                                  _P(C.c_double), _P(C.c_uint32), C.c_int32]),
    "aefdtd_discretize": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_double, C.c_double,
                                    C.c_double, _P(A.StructureOp), C.c_int32, _P(A.StructureDesc),
                                    _P(C.c_uint32), C.c_int32]),
    "aefdtd_setup_normal": (C.c_int, [C.c_void_p, _P(A.NormalDesc)]),
    "aefdtd_add_oscillator": (C.c_int, [C.c_void_p, _P(A.SourceDesc), _P(C.c_int32)]),
    "aefdtd_add_planar_sensor": (C.c_int, [C.c_void_p, _P(A.SensorDesc), _P(C.c_int32)]),
    "aefdtd_step": (C.c_int, [C.c_void_p, C.c_int32]),
    "aefdtd_synchronize": (C.c_int, [C.c_void_p]),
    "aefdtd_reset": (C.c_int, [C.c_void_p]),
    "aefdtd_get_field": (C.c_int, [C.c_void_p, C.c_int32, _P(C.c_double), C.c_size_t]),
    "aefdtd_set_field": (C.c_int, [C.c_void_p, C.c_int32, _P(C.c_double), C.c_size_t]),
    "aefdtd_field_device_ptr": (C.c_int, [C.c_void_p, C.c_int32, _P(C.c_void_p)]),
    "aefdtd_get_plane_sums": (C.c_int, [C.c_void_p, _P(C.c_double), C.c_int32]),
    "aefdtd_get_normal_spectra": (C.c_int, [C.c_void_p, _P(C.c_double), C.c_int32]),
    "aefdtd_get_sensor_flux": (C.c_int, [C.c_void_p, C.c_int32, _P(C.c_double), C.c_int32]),
    "aefdtd_get_sensor_dft": (C.c_int, [C.c_void_p, C.c_int32, _P(C.c_double), C.c_size_t]),
    "aefdtd_get_sensor_shape": (C.c_int, [C.c_void_p, C.c_int32, _P(C.c_int32), _P(C.c_int32), _P(C.c_int32)]),
    "aefdtd_get_timings": (C.c_int, [C.c_void_p, _P(C.c_double), _P(C.c_double), _P(C.c_double)]),
    "aefdtd_enable_timing": (C.c_int, [C.c_void_p, C.c_int32]),
    "aefdtd_get_stream": (C.c_int, [C.c_void_p, _P(C.c_void_p)]),
    "aefdtd_get_group_timings": (C.c_int, [C.c_void_p, _P(C.c_double), _P(C.c_int64), C.c_int32]),
    "aefdtd_set_completion": (C.c_int, [C.c_void_p, C.c_double, C.c_int32]),
    "aefdtd_add_box_sensor": (C.c_int, [C.c_void_p, _P(A.BoxSensorDesc), _P(C.c_int32)]),
    "aefdtd_get_box_flux": (C.c_int, [C.c_void_p, C.c_int32, _P(C.c_double), C.c_int32]),
    "aefdtd_add_fieldmap": (C.c_int, [C.c_void_p, _P(A.FieldMapDesc), _P(C.c_int32)]),
    "aefdtd_setup_oblique": (C.c_int, [C.c_void_p, _P(A.ObliqueDesc)]),
    "aefdtd_set_completion_ft": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_int32, C.c_char_p,
                                           C.c_uint32, C.c_int32]),
    "aefdtd_get_oblique_spectra": (C.c_int, [C.c_void_p, _P(C.c_double), C.c_int32, _P(C.c_int32)]),
    "aefdtd_get_oblique_series": (C.c_int, [C.c_void_p, _P(C.c_double), C.c_size_t]),
    "aefdtd_get_fieldmap_shape": (C.c_int, [C.c_void_p, C.c_int32, _P(C.c_int32)]),
    "aefdtd_get_fieldmap": (C.c_int, [C.c_void_p, C.c_int32, _P(C.c_double), C.c_size_t]),
    "aefdtd_get_completion": (C.c_int, [C.c_void_p, _P(C.c_int32), _P(C.c_int32), _P(C.c_double)]),
    "aefdtd_get_launch_count": (C.c_int, [C.c_void_p, _P(C.c_uint64)]),
    "aefdtd_device_memory": (C.c_int, [C.c_int32, _P(C.c_size_t), _P(C.c_size_t)]),
    "aefdtd_test_hook": (C.c_int, [C.c_void_p, C.c_int32, C.c_int64]),
    "aefdtd_probe_copy_bandwidth": (C.c_int, [C.c_int32, C.c_size_t, C.c_int32, _P(C.c_double)]),
    "aefdtd_plane_sums_static": (C.c_int, [_P(C.c_void_p), C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                           _P(C.c_int32), C.c_int32, C.c_double, C.c_void_p, C.c_void_p,
                                           C.c_char_p, C.c_size_t]),
    "aefdtd_batch_create": (C.c_int, [_P(A.BatchOpts), _P(C.c_void_p)]),
    "aefdtd_batch_destroy": (C.c_int, [C.c_void_p]),
    "aefdtd_batch_last_error": (C.c_char_p, [C.c_void_p]),
    "aefdtd_batch_add": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32]),
    "aefdtd_batch_remove": (C.c_int, [C.c_void_p, C.c_void_p]),
    "aefdtd_batch_set_budget": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32]),
    "aefdtd_batch_autotune": (C.c_int, [C.c_void_p]),
    "aefdtd_batch_advance": (C.c_int, [C.c_void_p, C.c_int32, _P(C.c_int32)]),
    "aefdtd_batch_finished": (C.c_int, [C.c_void_p, _P(C.c_void_p), C.c_int32, _P(C.c_int32)]),
    "aefdtd_batch_get_info": (C.c_int, [C.c_void_p, _P(A.BatchInfo)]),
    "aefdtd_server_create": (C.c_int, [_P(A.ServerOpts), _P(C.c_void_p)]),
    "aefdtd_server_destroy": (C.c_int, [C.c_void_p]),
    "aefdtd_server_last_error": (C.c_char_p, [C.c_void_p]),
    "aefdtd_server_submit": (C.c_int, [C.c_void_p, _P(A.JobDesc), _P(C.c_int32)]),
    "aefdtd_server_poll": (C.c_int, [C.c_void_p, _P(C.c_int32)]),
    "aefdtd_server_job_info": (C.c_int, [C.c_void_p, C.c_int32, _P(A.JobInfo)]),
    "aefdtd_server_job_spectra": (C.c_int, [C.c_void_p, C.c_int32, _P(C.c_double), C.c_int32]),
    "aefdtd_server_get_stats": (C.c_int, [C.c_void_p, _P(A.ServerStats)]),
}


class AefdtdError(RuntimeError):
    def __init__(self, status, msg):
        self.status = status
        super().__init__(f"{A.STATUS.get(status, status)}: {msg}")


def load():
    """Loads libaefdtd.so (once) and declares every exported signature."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing; build it with `python -m aether_b200.build` "
                          "(there is no CPU fallback)")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def exported_symbols():
    return list(_SIGS)


def check(status, handle=None):
    if status != 0:
        lib = load()
        msg = lib.aefdtd_last_error(handle)
        raise AefdtdError(status, msg.decode() if msg else "")
