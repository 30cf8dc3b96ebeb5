"""ctypes mirror of the C ABI structures declared in include/aefdtd.h.

Kept field-for-field identical to the header; tests check the struct sizes
against the compiled library (aefdtd_abi_sizes)."""
import ctypes as C

import numpy as np

ABI_VERSION = 2
MAX_TERMS = 8

MODE_NORMAL, MODE_CUSTOM, MODE_OBLIQUE = 0, 1, 2
FP64, FP32 = 0, 1
EX, EY, EZ, HX, HY, HZ = range(6)
NORMAL_X, NORMAL_XM, NORMAL_Y, NORMAL_YM, NORMAL_Z, NORMAL_ZM = range(6)
XM, XP, YM, YP, ZM, ZP = range(6)
(OP_BLOCK, OP_LAYER, OP_SPHERE, OP_CYLINDER, OP_CONE, OP_ELLIPSOID, OP_SIN_LAYER, OP_VECT_BLOCK, OP_VECT_TRI,
 OP_COATING, OP_CONF_COATING, OP_MESH) = range(12)

STATUS = {
    0: "OK", 1: "BAD_ARG", 2: "OOM", 3: "TIMEOUT", 4: "CUDA_ERROR",
    5: "NOT_READY", 6: "NO_DEVICE",
}


class GridDesc(C.Structure):
    _fields_ = [
        ("abi_version", C.c_int32), ("mode", C.c_int32), ("precision", C.c_int32),
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
        ("nt", C.c_int32), ("tapering", C.c_int32),
        ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
        ("dt", C.c_double), ("time_mod", C.c_double),
        ("pml", C.c_int32 * 6), ("pad", C.c_int32 * 6),
        ("pml_kappa", C.c_double * 6), ("pml_sigma", C.c_double * 6),
        ("pml_alpha", C.c_double * 6),
        ("pml_m", C.c_int32), ("pml_ma", C.c_int32),
        ("device", C.c_int32), ("dft_block", C.c_int32),
    ]


class MaterialDesc(C.Structure):
    _fields_ = [
        ("eps_inf", C.c_double),
        ("n_debye", C.c_int32), ("n_drude", C.c_int32),
        ("n_lorentz", C.c_int32), ("n_critpoint", C.c_int32),
        ("debye", (C.c_double * 2) * MAX_TERMS),
        ("drude", (C.c_double * 2) * MAX_TERMS),
        ("lorentz", (C.c_double * 3) * MAX_TERMS),
        ("critpoint", (C.c_double * 4) * MAX_TERMS),
    ]


class NormalDesc(C.Structure):
    _fields_ = [
        ("polarization", C.c_int32), ("nl", C.c_int32),
        ("lambda_min", C.c_double), ("lambda_max", C.c_double),
    ]


class SensorDesc(C.Structure):
    _fields_ = [
        ("orientation", C.c_int32), ("box", C.c_int32 * 6), ("nl", C.c_int32),
        ("lambda_min", C.c_double), ("lambda_max", C.c_double),
    ]


class SourceDesc(C.Structure):
    _fields_ = [
        ("orientation", C.c_int32), ("box", C.c_int32 * 6),
        ("lambda_min", C.c_double), ("lambda_max", C.c_double),
    ]


class Dims(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
        ("xs_s", C.c_int32), ("xs_e", C.c_int32), ("ys_s", C.c_int32),
        ("ys_e", C.c_int32), ("zs_s", C.c_int32), ("zs_e", C.c_int32),
        ("n_materials", C.c_int32), ("step", C.c_int32),
        ("dt", C.c_double), ("device_bytes", C.c_size_t),
    ]


class BatchOpts(C.Structure):
    _fields_ = [
        ("abi_version", C.c_int32), ("device", C.c_int32), ("l2_budget_bytes", C.c_int64),
        ("tile_y", C.c_int32), ("kchunk", C.c_int32), ("use_graphs", C.c_int32), ("graph_steps", C.c_int32),
        ("lanes", C.c_int32), ("persistent", C.c_int32),
    ]


BATCH_MAX_CLASSES = 32


class BatchInfo(C.Structure):
    _fields_ = [
        ("n_members", C.c_int32), ("n_active", C.c_int32), ("n_subsets", C.c_int32), ("n_classes", C.c_int32),
        ("n_lanes", C.c_int32), ("n_persistent", C.c_int32),
        ("cells", C.c_int64), ("member_bytes", C.c_int64), ("batch_bytes", C.c_int64),
        ("l2_budget_bytes", C.c_int64), ("launches", C.c_uint64),
        ("class_key", C.c_int32 * BATCH_MAX_CLASSES), ("class_tile_y", C.c_int32 * BATCH_MAX_CLASSES),
        ("class_kchunk", C.c_int32 * BATCH_MAX_CLASSES),
    ]


JOB_QUEUED, JOB_RUNNING, JOB_DONE, JOB_FAILED = 0, 1, 2, 3


class ServerOpts(C.Structure):
    _fields_ = [
        ("abi_version", C.c_int32), ("device", C.c_int32), ("hbm_fraction", C.c_double),
        ("budget_bytes", C.c_int64), ("max_active", C.c_int32), ("segment_steps", C.c_int32),
        ("lookahead", C.c_int32), ("reserved", C.c_int32), ("batch", BatchOpts),
    ]


class JobDesc(C.Structure):
    _fields_ = [
        ("grid", C.POINTER(GridDesc)), ("map", C.POINTER(C.c_uint32)), ("map_count", C.c_size_t),
        ("materials", C.POINTER(MaterialDesc)), ("n_materials", C.c_int32),
        ("normal", C.POINTER(NormalDesc)), ("steps", C.c_int32), ("cc_step", C.c_int32), ("cc_coeff", C.c_double),
    ]


class JobInfo(C.Structure):
    _fields_ = [
        ("state", C.c_int32), ("steps", C.c_int32), ("cells", C.c_int64), ("est_bytes", C.c_int64),
        ("bytes", C.c_int64), ("t_submit", C.c_double), ("t_admit", C.c_double), ("t_done", C.c_double),
        ("stop_step", C.c_int32), ("reserved", C.c_int32),
    ]


class ServerStats(C.Structure):
    _fields_ = [
        ("submitted", C.c_int32), ("queued", C.c_int32), ("running", C.c_int32), ("done", C.c_int32),
        ("failed", C.c_int32), ("reserved", C.c_int32),
        ("budget_bytes", C.c_int64), ("in_use_bytes", C.c_int64), ("peak_bytes", C.c_int64),
        ("p50_s", C.c_double), ("p99_s", C.c_double), ("mean_s", C.c_double), ("elapsed_s", C.c_double),
        ("sims_per_s", C.c_double), ("gcells_per_s", C.c_double),
    ]


class BoxSensorDesc(C.Structure):
    _fields_ = [("box", C.c_int32 * 6), ("nl", C.c_int32), ("disabled", C.c_int32),
                ("lambda_min", C.c_double), ("lambda_max", C.c_double)]


class ObliqueDesc(C.Structure):
    _fields_ = [("polarization", C.c_int32), ("nl", C.c_int32), ("lambda_min", C.c_double),
                ("lambda_max", C.c_double), ("kx_in", C.c_double), ("ky_in", C.c_double)]


MAP_PLANE, MAP_BLOCK, MAP_POINT = range(3)


class FieldMapDesc(C.Structure):
    _fields_ = [("kind", C.c_int32), ("orientation", C.c_int32), ("box", C.c_int32 * 6),
                ("cumulative", C.c_int32), ("magnetic", C.c_int32), ("lambda_", C.c_double)]


class StructureOp(C.Structure):
    _fields_ = [("kind", C.c_int32), ("mat_index", C.c_int32), ("p", C.c_double * 16)]


class Mesh(C.Structure):
    _fields_ = [("vertices", C.POINTER(C.c_double)), ("faces", C.POINTER(C.c_int32)), ("n_vertices", C.c_int32),
                ("n_faces", C.c_int32)]


class StructureDesc(C.Structure):
    _fields_ = [("default_material", C.c_int32), ("periodic", C.c_int32 * 3), ("flip", C.c_int32 * 3),
                ("n_meshes", C.c_int32), ("lengths", C.c_double * 3), ("meshes", C.POINTER(Mesh))]


def structure_op(kind, mat, *p):
    o = StructureOp()
    o.kind, o.mat_index = int(kind), int(mat)
    for i, v in enumerate(p):
        o.p[i] = float(v)
    return o


def structure_desc(default=0, periodic=(0, 0, 0), flip=(0, 0, 0), lengths=(0.0, 0.0, 0.0), meshes=()):
    """meshes: (vertices (nv, 3) float64, faces (nf, 3) int32) pairs; the
    returned struct keeps them alive."""
    d = StructureDesc()
    d.default_material = int(default)
    for a in range(3):
        d.periodic[a], d.flip[a], d.lengths[a] = int(periodic[a]), int(flip[a]), float(lengths[a])
    keep = []
    if meshes:
        arr = (Mesh * len(meshes))()
        for i, (v, f) in enumerate(meshes):
            v = np.ascontiguousarray(v, dtype=np.float64).reshape(-1, 3)
            f = np.ascontiguousarray(f, dtype=np.int32).reshape(-1, 3)
            keep += [v, f]
            arr[i].vertices = v.ctypes.data_as(C.POINTER(C.c_double))
            arr[i].faces = f.ctypes.data_as(C.POINTER(C.c_int32))
            arr[i].n_vertices, arr[i].n_faces = len(v), len(f)
        d.meshes = arr
        d.n_meshes = len(meshes)
        keep.append(arr)
    d._keep = keep
    return d


def material_desc(eps_inf=1.0, debye=(), drude=(), lorentz=(), critpoint=()):
    """Builds a MaterialDesc from term lists (same parameter order as the
    reference's add_debye/add_drude/add_lorentz/add_crit_point)."""
    m = MaterialDesc()
    m.eps_inf = float(eps_inf)
    for name, terms, width in (("debye", debye, 2), ("drude", drude, 2),
                               ("lorentz", lorentz, 3), ("critpoint", critpoint, 4)):
        terms = list(terms)
        if len(terms) > MAX_TERMS:
            raise ValueError(f"at most {MAX_TERMS} {name} terms per material")
        setattr(m, "n_" + name, len(terms))
        arr = getattr(m, name)
        for i, t in enumerate(terms):
            if len(t) != width:
                raise ValueError(f"{name} term needs {width} parameters")
            for j, v in enumerate(t):
                arr[i][j] = float(v)
    return m


def grid_desc(nx, ny, nz, dx, dy=None, dz=None, *, mode=MODE_NORMAL, precision=FP64,
              nt=0, tapering=0, dt=0.0, time_mod=1.0, pml=(0,) * 6, pad=(0,) * 6,
              kappa=(1.0,) * 6, sigma=(1.0,) * 6, alpha=(0.0,) * 6, pml_m=0, pml_ma=0,
              device=0, dft_block=0):
    g = GridDesc()
    g.abi_version = ABI_VERSION
    g.mode, g.precision = mode, precision
    g.nx, g.ny, g.nz = nx, ny, nz
    g.nt, g.tapering = nt, tapering
    g.dx = dx
    g.dy = dx if dy is None else dy
    g.dz = dx if dz is None else dz
    g.dt, g.time_mod = dt, time_mod
    for i in range(6):
        g.pml[i] = int(pml[i])
        g.pad[i] = int(pad[i])
        g.pml_kappa[i] = float(kappa[i])
        g.pml_sigma[i] = float(sigma[i])
        g.pml_alpha[i] = float(alpha[i])
    g.pml_m, g.pml_ma = pml_m, pml_ma
    g.device, g.dft_block = device, dft_block
    return g
